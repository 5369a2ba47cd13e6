"""The oracle's particle map and vorticity right-hand side against hand-worked
cases of the reference's rules (source/particles/pmlib_particles_map.f:63-127, the
communication order of one rank, part_deriv_vorticity.f:57-193).  CPU only."""
import numpy as np

from oracle import oracle as O
from tests.helpers import setup_pair


def _box(bc):
    po, to, _, _, _, _ = setup_pair((0, 0, 0), (1, 1, 1), (0.125,) * 3, bc, 4)
    return po, to


def test_map_order_drop_and_wrap():
    """x periodic, y and z free: low-side leavers first, then high-side leavers, then
    the rest (each in the old order); free-side leavers dropped."""
    po, to = _box((1, 0, 0))
    pos = np.array([[0.5, 0.5, 0.5],    # 0 stays
                    [1.2, 0.5, 0.5],    # 1 leaves high in x -> 0.2
                    [-0.3, 0.5, 0.5],   # 2 leaves low in x -> 0.7
                    [0.5, 1.5, 0.5],    # 3 leaves a free face in y: dropped
                    [-0.1, 0.2, 0.3],   # 4 leaves low in x -> 0.9
                    [0.4, 0.4, 0.4]])   # 5 stays
    n = len(pos)
    vort = np.arange(3 * n, dtype=np.float64).reshape(n, 3)
    z = np.zeros((n, 3))
    ierr, m = O.particles_advance(po, to, 1, 1, 0.0, pos, vort, z.copy(), z.copy(), z.copy(), z.copy())
    assert ierr == 0 and m == 5 and to.npart == 5
    order = [2, 4, 1, 0, 5]
    assert np.array_equal(vort[:m], np.arange(3 * n, dtype=np.float64).reshape(n, 3)[order])
    assert np.allclose(pos[:m, 0], [0.7, 0.9, 0.2, 0.5, 0.4])


def test_map_two_passes_and_axis_order():
    """A particle two patch lengths out is a leaver in two passes; the y pass reorders
    after the x pass."""
    po, to = _box((1, 1, 0))
    pos = np.array([[0.5, 0.5, 0.5],    # 0
                    [-1.5, 0.5, 0.5],   # 1 two low passes in x -> 0.5
                    [-0.5, 0.5, 0.5],   # 2 one low pass in x
                    [2.5, 0.5, 0.5],    # 3 two high passes in x
                    [0.5, -0.2, 0.5],   # 4 low in y
                    [1.5, 1.5, 0.5]])   # 5 high in x, high in y
    n = len(pos)
    ids = np.repeat(np.arange(n, dtype=np.float64)[:, None], 3, axis=1)
    z = np.zeros((n, 3))
    ierr, m = O.particles_advance(po, to, 1, 1, 0.0, pos, ids, z.copy(), z.copy(), z.copy(), z.copy())
    assert ierr == 0 and m == 6
    # x pass 1: L = [1, 2], R = [3, 5], S = [0, 4] -> 1 2 3 5 0 4; pass 2: L = [1],
    # R = [3], S = [2 5 0 4] -> 1 3 2 5 0 4; y pass: L = [4], R = [5], S = [1 3 2 0]
    assert ids[:m, 0].tolist() == [4, 5, 1, 3, 2, 0]
    assert np.all((pos[:m] >= 0) & (pos[:m] < 1))


def test_rk_stages():
    """Third-order scheme over three stages with constant rates moves a particle by
    dt * u (c-weights of the low-storage scheme sum to the full step)."""
    po, to = _box((1, 1, 1))
    pos = np.array([[0.5, 0.5, 0.5]])
    vort = np.array([[1.0, 2.0, 3.0]])
    vel = np.array([[0.1, -0.2, 0.05]])
    dv = np.array([[1.0, 0.0, -1.0]])
    vr, dr = np.zeros((1, 3)), np.zeros((1, 3))
    for s in (1, 2, 3):
        ierr, m = O.particles_advance(po, to, 3, s, 0.1, pos, vort, vel, dv, vr, dr)
        assert ierr == 0 and m == 1
    assert np.allclose(pos[0], [0.5 + 0.01, 0.5 - 0.02, 0.5 + 0.005], atol=1e-14)
    assert np.allclose(vort[0], [1.1, 2.0, 2.9], atol=1e-14)


def test_advance_errors(capfd):
    po, to = _box((0, 0, 0))
    a = np.zeros((1, 3))
    assert O.particles_advance(po, to, 4, 1, 0.1, a, a.copy(), a.copy(), a.copy(), a.copy(), a.copy())[0] == -1
    assert "pmlib_interpolation_order is incorrectly set." in capfd.readouterr().out
    assert O.particles_advance(po, to, 2, 3, 0.1, a, a.copy(), a.copy(), a.copy(), a.copy(), a.copy())[0] == -1


def test_deriv_vorticity_linear_fields():
    """For vel linear in x and vort constant, dvort = (w . grad) u exactly, with no
    diffusion; periodic ghosts copy the far interior."""
    po, to = _box((1, 1, 0))
    shape = O.topo_shape(to, 3)
    ext = [to.ncell[d] + to.nghost[2 * d] + to.nghost[2 * d + 1] for d in range(3)]
    x = to.xmin[0] + (np.arange(ext[0]) - to.nghost[0] + 0.5) * to.dx[0]
    vel = np.zeros(shape)
    vel[..., 1] = 2.0 * x[None, None, :]          # du_y/dx = 2
    vort = np.zeros(shape)
    vort[..., 0] = 3.0                            # w_x = 3
    dvort = np.full(shape, 5.0)
    for fd in (2, 4):
        d = dvort.copy()
        assert O.deriv_vorticity(to, fd, 0.01, vort, vel, d) == 0
        gz = slice(to.nghost[4], to.nghost[4] + to.ncell[2])
        inner = d[gz, to.nghost[2]:to.nghost[2] + to.ncell[1], to.nghost[0]:to.nghost[0] + to.ncell[0]]
        assert np.allclose(inner[..., 1], 6.0) and np.allclose(inner[..., 0], 0.0)
        # free z ghosts keep their values; periodic x ghosts copy the interior
        assert np.all(d[0] == 5.0)
        assert np.array_equal(d[gz, :, 0], d[gz, :, to.ncell[0]])
