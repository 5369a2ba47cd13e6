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
with the same kernels and tiles as when it is alone.  The report splits each
request's latency into queueing (arrival to set-up), plan set-up, waiting for a
slot and service, and gives the most solves that ran on the device at one time.
"""
from __future__ import annotations

import threading
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
    setup_start: float = None  # the set-up thread took the request
    setup_end: float = None    # its plan was ready (reused or new)
    new_plan: bool = False
    start: float = None        # its solve was queued on a slot
    done: float = None         # the server saw the solve finished
    dev_start_ms: float = None  # device clock (CUDA events) of the solve, from the run's start
    dev_end_ms: float = None
    topo: object = None
    key: tuple = None
    nbytes: int = 0
    plan: object = None
    need: int = 0


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
    ev0: object = None
    ev1: object = None


class Server:
    """Admission-controlled request loop over `slots` CUDA streams within `budget`
    bytes of device memory (plans + request buffers).

    Two host threads: a set-up thread takes the arrived requests in arrival order and
    gets each a plan (an idle plan of its grid, or a new one once the budget has room,
    evicting idle plans of other grids first), at most `ahead` requests ahead of the
    solves; the serving thread queues the solves of prepared requests on free slots
    (arrival order), retires finished ones and returns their plans and memory.  The
    library serialises plan set-up on its own lock, so a new grid's set-up runs while
    solves of other requests are queued and run.  Neither thread spins: each waits on
    a condition variable (the serving thread with a 0.2 ms limit, to look at the
    slots' events)."""

    def __init__(self, params, precision: int = P.FP32, slots: int = 8, budget: int = 16 << 30, nghost: int = 4,
                 ahead: int = None):
        import torch
        self.torch = torch
        self.params = params
        self.precision = precision
        self.nghost = nghost
        self.budget = int(budget)
        # high-priority streams: the blocks of queued solves are dispatched before those
        # of a plan set-up running at the same time (its FP64 Green's function and
        # transform run at the default priority)
        self.slots = [_Slot(torch.cuda.Stream(priority=-1)) for _ in range(slots)]
        self.ahead = ahead if ahead is not None else 2 * slots
        self.idle = OrderedDict()   # key -> list of idle plans (LRU order of keys)
        self.held = 0               # bytes of all live plans and of the admitted requests' buffers
        self.plan_size = {}         # id(plan) -> bytes
        self.cv = threading.Condition()
        self.pending = deque()      # submitted, not yet taken by the set-up thread
        self.prepared = deque()     # plans ready, waiting for a slot
        self.finished = []
        self.inflight = 0
        self.max_inflight = 0
        self.max_held = 0
        self.error = None
        self.stop = False

    # -------------------------------------------------------------- plans (set-up thread)
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

    def _prepare(self, r: Request, clock, t0) -> None:
        """Gets r a plan and reserves its memory; waits (without spinning) for memory
        held by running requests.  Called with self.cv held; releases it while a new
        plan is set up."""
        plans = self.idle.get(r.key)
        if plans:
            self.idle.move_to_end(r.key)
            r.plan = plans.pop()
            self.held += r.nbytes
            self.max_held = max(self.max_held, self.held)
            return
        need = plan_bytes(r.topo, self.precision, self.params.poisson_kernel)
        while self.held + r.nbytes + need > self.budget:
            if self._evict_one():
                continue
            if self.inflight == 0 and not self.prepared:
                raise RuntimeError(f"request {r.rid} needs more device memory than the budget "
                                   f"({self.budget / 1e9:.2f} GB)")
            self.cv.wait()
            if self.stop:
                return
        self.held += need + r.nbytes
        self.max_held = max(self.max_held, self.held)
        r.need = need
        r.new_plan = True
        self.cv.release()
        try:
            pa, t = self._topo(r)
            ierr, plan = P.pmlib_poisson_setup(pa, t, self.params, self.precision)
        finally:
            self.cv.acquire()
        if ierr != 0:
            raise RuntimeError(P.last_error())
        self.plan_size[id(plan)] = need
        r.plan = plan

    def _setup_loop(self, clock, t0):
        try:
            with self.cv:
                while not self.stop:
                    if not self.pending or len(self.prepared) >= self.ahead:
                        if not self.pending and self.submitted_all:
                            return
                        self.cv.wait()
                        continue
                    r = self.pending[0]
                    now = clock() - t0
                    if r.arrival > now:
                        self.cv.wait(timeout=r.arrival - now)
                        continue
                    self.pending.popleft()
                    r.setup_start = clock() - t0
                    self._prepare(r, clock, t0)
                    if self.stop:
                        return
                    r.setup_end = clock() - t0
                    self.prepared.append(r)
                    self.cv.notify_all()
        except BaseException as e:  # handed to the serving thread
            with self.cv:
                self.error = e
                self.cv.notify_all()

    # -------------------------------------------------------------- solves (serving thread)
    def submit(self, r: Request):
        pa, t = self._topo(r)
        r.topo = t
        r.key = grid_key(r)
        r.nbytes = field_bytes(t, self.precision)
        self.pending.append(r)

    def _start(self, slot: _Slot, r: Request, now: float, ref):
        torch = self.torch
        with torch.cuda.stream(slot.stream):
            r.vel = torch.empty_like(r.vort)
            slot.ev0 = torch.cuda.Event(enable_timing=True)
            slot.ev1 = torch.cuda.Event(enable_timing=True)
            slot.ev0.record(slot.stream)
            rc = P.pmlib_poisson_solve_dev(r.plan, r.vort.data_ptr(), r.vel.data_ptr(),
                                           stream=slot.stream.cuda_stream)
            if rc != 0:
                raise RuntimeError(P.last_error())
            slot.ev1.record(slot.stream)
        slot.req = r
        r.start = now
        self.inflight += 1
        self.max_inflight = max(self.max_inflight, self.inflight)

    def _retire(self, now: float, ref) -> bool:
        """Finished solves return their plan and memory; True if any did."""
        any_done = False
        for slot in self.slots:
            if slot.req is not None and slot.ev1.query():
                r = slot.req
                r.done = now
                r.dev_start_ms = ref.elapsed_time(slot.ev0)
                r.dev_end_ms = ref.elapsed_time(slot.ev1)
                self.held -= r.nbytes
                self.idle.setdefault(r.key, []).append(r.plan)
                self.idle.move_to_end(r.key)
                r.plan = None
                self.finished.append(r)
                slot.req = slot.ev0 = slot.ev1 = None
                self.inflight -= 1
                any_done = True
        return any_done

    def run(self, requests, clock=time.perf_counter):
        """Serve requests whose `arrival` is relative to the start of the run.  Plans
        stay resident between runs (idle, evicted as memory is needed)."""
        torch = self.torch
        self.finished = []
        self.pending.clear()
        self.prepared.clear()
        self.max_inflight = 0
        self.error = None
        self.stop = False
        for r in sorted(requests, key=lambda q: q.arrival):
            self.submit(r)
        self.submitted_all = True
        n = len(self.pending)
        ref = torch.cuda.Event(enable_timing=True)
        ref.record()
        t0 = clock()
        worker = threading.Thread(target=self._setup_loop, args=(clock, t0), daemon=True)
        worker.start()
        try:
            with self.cv:
                while len(self.finished) < n:
                    if self.error is not None:
                        raise self.error
                    now = clock() - t0
                    if self._retire(now, ref):
                        self.cv.notify_all()  # memory and plans returned
                    while self.prepared and any(s.req is None for s in self.slots):
                        slot = next(s for s in self.slots if s.req is None)
                        self._start(slot, self.prepared.popleft(), clock() - t0, ref)
                        self.cv.notify_all()  # room to prepare further ahead
                    if len(self.finished) < n:
                        self.cv.wait(timeout=2e-4)
        finally:
            with self.cv:
                self.stop = True
                self.cv.notify_all()
            worker.join()
        return self.report(clock() - t0)

    def report(self, wall: float) -> dict:
        fin = self.finished

        def pct(vals, q):
            return float(np.percentile(vals, q)) if len(vals) else None

        lat = [(r.done - r.arrival) * 1e3 for r in fin]
        queue = [(r.setup_start - r.arrival) * 1e3 for r in fin]
        setup = [(r.setup_end - r.setup_start) * 1e3 for r in fin]
        wait = [(r.start - r.setup_end) * 1e3 for r in fin]
        serv = [(r.done - r.start) * 1e3 for r in fin]
        dev = [r.dev_end_ms - r.dev_start_ms for r in fin]
        # most solves running on the device at one time (CUDA event intervals)
        ev = sorted([(r.dev_start_ms, 1) for r in fin] + [(r.dev_end_ms, -1) for r in fin])
        cur = peak = 0
        for _, d in ev:
            cur += d
            peak = max(peak, cur)
        split = {}
        for name, v in (("queue", queue), ("setup", setup), ("wait_slot", wait), ("service", serv),
                        ("device", dev)):
            split[name] = {"p50_ms": pct(v, 50), "p99_ms": pct(v, 99), "mean_ms": float(np.mean(v)) if v else None}
        return {"solves": len(fin), "seconds": wall,
                "solves_per_s": len(fin) / wall if wall > 0 else None,
                "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                "split": split, "new_plans": sum(1 for r in fin if r.new_plan),
                "max_inflight": self.max_inflight, "max_on_device": peak,
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
