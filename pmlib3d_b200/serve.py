"""Serving loop for unbounded vector Poisson solves (continuous batching).

Requests (a patch, its boundary types and a vorticity field) arrive over time.  The
server keeps plans resident on the GPU -- Green's spectra are shared per grid by the
library's cache -- and admits a waiting request as soon as a slot (a CUDA stream) is
free and the HBM budget has room for its plan and buffers.  Admitted solves run
concurrently on their streams, so requests that arrive while others are on the GPU
overlap with them.  Idle plans are evicted least-recently-used when a new grid needs
room.  Every request records arrival, start and completion times; the report gives
solves/s and p50 / p99 latency (arrival to completion).

The results do not depend on the mix: a request is solved by a plan of its own grid
with the same kernels and tiles as when it is alone.
"""
from __future__ import annotations

import time
from collections import OrderedDict, deque
from dataclasses import dataclass

import numpy as np

from . import pmlib as P


@dataclass
class Request:
    rid: int
    arrival: float            # seconds, on the server clock
    xmin: tuple
    xmax: tuple
    dx: tuple
    bound_cond: tuple
    vort: object = None       # device tensor (nz', ny', nx', 3) of the plan's precision
    vel: object = None        # filled by the server
    start: float = None
    done: float = None
    topo: object = None
    key: tuple = None
    nbytes: int = 0


def grid_key(r: Request):
    return (tuple(float(v) for v in r.xmin), tuple(float(v) for v in r.xmax), tuple(float(v) for v in r.dx),
            tuple(int(b) for b in r.bound_cond))


def plan_bytes(topo, precision: int, kernel: int = 1) -> int:
    """Device bytes a plan holds for one velocity solve: the work spectra X and Y
    (3 components, half spectrum along x padded to a multiple of 8) and the Green
    octant (three octants and three planes for kernel 2; shared, counted once per
    plan as an upper bound)."""
    w = 4 if precision == P.FP32 else 8
    P_ = [topo.ncell[d] + topo.nghost[2 * d] + topo.nghost[2 * d + 1] for d in range(3)]
    per = [topo.bound_cond[2 * d] != 0 for d in range(3)]
    Pp = [topo.ncell[d] if per[d] else P_[d] for d in range(3)]
    M = [Pp[d] if per[d] else 2 * Pp[d] for d in range(3)]
    H = M[0] // 2 + 1
    Hp = (H + 7) // 8 * 8
    X = 3 * Hp * Pp[1] * Pp[2] * 2 * w
    Y = 3 * Hp * M[1] * Pp[2] * 2 * w
    gM1, gM2 = M[1] // 2 + 1, M[2] // 2 + 1
    G = gM2 * gM1 * H * w
    if kernel == 2:
        G = 3 * G + (gM2 * gM1 + gM2 * H + gM1 * H) * w
    return X + Y + G


def field_bytes(topo, precision: int) -> int:
    w = 4 if precision == P.FP32 else 8
    n = 1
    for d in range(3):
        n *= topo.ncell[d] + topo.nghost[2 * d] + topo.nghost[2 * d + 1]
    return 2 * 3 * n * w  # vorticity in, velocity out


@dataclass
class _Slot:
    stream: object
    req: Request = None
    plan: object = None
    event: object = None


class Server:
    """Admission-controlled request loop over `slots` CUDA streams within `budget`
    bytes of device memory (plans + request buffers)."""

    def __init__(self, params, precision: int = P.FP32, slots: int = 8, budget: int = 16 << 30, nghost: int = 4):
        import torch
        self.torch = torch
        self.params = params
        self.precision = precision
        self.nghost = nghost
        self.budget = int(budget)
        self.slots = [_Slot(torch.cuda.Stream()) for _ in range(slots)]
        self.idle = OrderedDict()   # key -> list of idle plans (LRU order of keys)
        self.held = 0               # bytes of all live plans
        self.plan_size = {}         # id(plan) -> bytes
        self.inflight_io = 0
        self.queue = deque()
        self.finished = []

    # -------------------------------------------------------------- plans
    def _topo(self, r: Request):
        pa = P.make_patch(r.xmin, r.xmax, r.dx, bound_cond=r.bound_cond, nghost=self.nghost)
        ierr, t = P.pmlib_topology_cuboid(pa, self.params.interpolation_order)
        if ierr != 0:
            raise RuntimeError(P.last_error())
        return pa, t

    def _evict_one(self) -> bool:
        for key in list(self.idle.keys()):
            plans = self.idle[key]
            if plans:
                plan = plans.pop()
                self.held -= self.plan_size.pop(id(plan))
                plan.close()
                if not plans:
                    del self.idle[key]
                return True
        return False

    def _acquire_plan(self, r: Request):
        """An idle plan of the request's grid, or a new one if the budget allows
        (evicting idle plans of other grids first); None if it must wait."""
        plans = self.idle.get(r.key)
        if plans:
            self.idle.move_to_end(r.key)
            return plans.pop()
        need = plan_bytes(r.topo, self.precision, self.params.poisson_kernel)
        while self.held + self.inflight_io + r.nbytes + need > self.budget:
            if not self._evict_one():
                return None
        pa, t = self._topo(r)
        ierr, plan = P.pmlib_poisson_setup(pa, t, self.params, self.precision)
        if ierr != 0:
            raise RuntimeError(P.last_error())
        self.plan_size[id(plan)] = need
        self.held += need
        return plan

    def _release_plan(self, key, plan):
        self.idle.setdefault(key, []).append(plan)
        self.idle.move_to_end(key)

    # -------------------------------------------------------------- loop
    def submit(self, r: Request):
        pa, t = self._topo(r)
        r.topo = t
        r.key = grid_key(r)
        r.nbytes = field_bytes(t, self.precision)
        self.queue.append(r)

    def _start(self, slot: _Slot, r: Request, plan, now: float):
        torch = self.torch
        with torch.cuda.stream(slot.stream):
            r.vel = torch.empty_like(r.vort)
            rc = P.pmlib_poisson_solve_dev(plan, r.vort.data_ptr(), r.vel.data_ptr(), stream=slot.stream.cuda_stream)
            if rc != 0:
                raise RuntimeError(P.last_error())
            ev = torch.cuda.Event()
            ev.record(slot.stream)
        slot.req, slot.plan, slot.event = r, plan, ev
        r.start = now
        self.inflight_io += r.nbytes

    def poll(self, now: float):
        """Retire finished solves, then admit waiting requests in arrival order."""
        for slot in self.slots:
            if slot.req is not None and slot.event.query():
                r = slot.req
                r.done = now
                self.inflight_io -= r.nbytes
                self._release_plan(r.key, slot.plan)
                self.finished.append(r)
                slot.req = slot.plan = slot.event = None
        for slot in self.slots:
            if slot.req is not None or not self.queue:
                continue
            r = self.queue[0]
            if r.arrival > now:
                break
            plan = self._acquire_plan(r)
            if plan is None:
                if not any(s.req is not None for s in self.slots):
                    raise RuntimeError(f"request {r.rid} needs more device memory than the budget "
                                       f"({self.budget / 1e9:.2f} GB)")
                break  # wait for memory: keep arrival order
            self.queue.popleft()
            self._start(slot, r, plan, now)

    def busy(self) -> bool:
        return bool(self.queue) or any(s.req is not None for s in self.slots)

    def run(self, requests, clock=time.perf_counter):
        """Serve requests whose `arrival` is relative to the start of the run."""
        t0 = clock()
        for r in sorted(requests, key=lambda q: q.arrival):
            self.submit(r)
        while self.busy():
            now = clock() - t0
            self.poll(now)
            if self.queue and all(s.req is not None for s in self.slots):
                time.sleep(0)  # all slots busy: yield
        return self.report(clock() - t0)

    def report(self, wall: float) -> dict:
        lat = np.array([(r.done - r.arrival) * 1e3 for r in self.finished])
        return {"solves": len(self.finished), "seconds": wall,
                "solves_per_s": len(self.finished) / wall if wall > 0 else None,
                "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
                "budget_gb": self.budget / 1e9, "slots": len(self.slots)}

    def close(self):
        while self._evict_one():
            pass


def request_stream(count: int, rate: float, seed: int = 7, nmin: int = 32, nmax: int = 256, h: float = 1.0 / 64,
                   precision: int = P.FP32, device_fields: bool = True):
    """The served workload: Poisson arrivals at `rate` per second, cells per axis
    log-uniform in [nmin, nmax], boundary types from {fff, ppf, pff}, random-axis
    Gaussian blob or vortex-ring vorticity.  Fields are built on the GPU."""
    from . import workloads as Wl
    import torch
    rng = np.random.Generator(np.random.Philox(Wl.SEED + 100 + seed))
    t = 0.0
    reqs = []
    dt = torch.float32 if precision == P.FP32 else torch.float64
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), 3))
        bcn = ("fff", "ppf", "pff")[int(rng.integers(0, 3))]
        bc = Wl.BC_TYPES[bcn]
        cells = [int(round(n[d])) + (int(round(n[d])) % 2 if bc[d] else 0) for d in range(3)]
        L = np.array(cells, dtype=np.float64) * h
        r = Request(rid=i, arrival=t, xmin=tuple(-0.5 * L), xmax=tuple(0.5 * L), dx=(h, h, h), bound_cond=bc)
        pa = P.make_patch(r.xmin, r.xmax, r.dx, bound_cond=bc, nghost=4)
        ierr, topo = P.pmlib_topology_cuboid(pa, 3)
        axis = int(rng.integers(0, 3))
        if device_fields:
            if rng.uniform() < 0.5:
                f = Wl.blob_field(topo, axis, xp=torch)
            else:
                f = _ring_field(topo, axis)
            r.vort = f.to(dt).contiguous()
        reqs.append(r)
    return reqs


def _ring_field(topo, axis: int):
    """A vortex ring around `axis` through the patch centre (radius 0.25 L, core 0.08 L)."""
    import torch
    axes = []
    for d in range(3):
        lo, hi = 1 - topo.nghost[2 * d], topo.ncell[d] + topo.nghost[2 * d + 1]
        i = torch.arange(lo, hi + 1, dtype=torch.float64, device="cuda")
        axes.append(topo.xmin[d] + (i - 0.5) * topo.dx[d])
    c = [0.5 * (topo.xmin[d] + topo.xmax[d]) for d in range(3)]
    L = min(topo.xmax[d] - topo.xmin[d] for d in range(3))
    z, y, x = torch.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    X = [x - c[0], y - c[1], z - c[2]]
    a, b, e = axis, (axis + 1) % 3, (axis + 2) % 3
    rho = torch.sqrt(X[b] ** 2 + X[e] ** 2)
    d = torch.sqrt((rho - 0.25 * L) ** 2 + X[a] ** 2)
    wth = torch.exp(-(d / (0.08 * L)) ** 2)
    rs = torch.where(rho > 0, rho, torch.ones_like(rho))
    out = torch.zeros(x.shape + (3,), dtype=torch.float64, device="cuda")
    out[..., b] = -wth * X[e] / rs
    out[..., e] = wth * X[b] / rs
    return out
