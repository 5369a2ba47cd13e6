"""Seeded workload generators (CPU): lattice placement, ring fields and the
algorithmic byte model of the periodic-periodic-free step."""
import numpy as np

from pmlib3d_b200 import workloads as Wl


def test_box_lattice_matches_cubic_lattice():
    a = Wl._lattice(6, -1.0, 1 / 3, np.random.Generator(np.random.Philox(5)))
    b = Wl._lattice_box((6, 6, 6), (-1.0,) * 3, 1 / 3, np.random.Generator(np.random.Philox(5)))
    assert np.array_equal(a, b)


def test_box_lattice_order_and_jitter():
    h = 0.25
    p = Wl._lattice_box((4, 3, 2), (0.0, -1.0, 2.0), h, np.random.Generator(np.random.Philox(9)))
    assert p.shape == (24, 3)
    k, j, i = np.meshgrid(np.arange(2), np.arange(3), np.arange(4), indexing="ij")  # x fastest
    centre = np.stack([(i.ravel() + 0.5) * h, -1.0 + (j.ravel() + 0.5) * h, 2.0 + (k.ravel() + 0.5) * h], -1)
    assert np.all(np.abs(p - centre) <= 0.1 * h)


def test_ring_about_z_is_azimuthal_and_truncated():
    rng = np.random.Generator(np.random.Philox(3))
    pos = rng.uniform(-1, 1, (4000, 3)) * np.array([1.0, 1.0, 0.5])
    w = Wl._ring_vorticity_z(pos, 0.1, 0.5, 0.08, -1.0)
    assert np.all(w[:, 2] == 0)
    radial = w[:, 0] * pos[:, 0] + w[:, 1] * pos[:, 1]
    assert np.max(np.abs(radial)) < 1e-12
    d = np.hypot(np.hypot(pos[:, 0], pos[:, 1]) - 0.5, pos[:, 2] - 0.1)
    assert np.all(w[d >= 0.32] == 0) and np.any(w[d < 0.32] != 0)
    # circulation sign: theta component is -exp(-(d/sigma)^2)
    rho = np.hypot(pos[:, 0], pos[:, 1])
    wt = (-w[:, 0] * pos[:, 1] + w[:, 1] * pos[:, 0]) / rho
    assert np.allclose(wt[d < 0.32], -np.exp(-(d[d < 0.32] / 0.08) ** 2))


def test_ppf_step_model_bytes():
    # 512 x 512 x 256 ppf, FP32: transform input extents (512, 512, 264), lengths (512, 512, 528)
    assert Wl.solve_bytes((512, 512, 528), (512, 512, 264), 4) == 8_608_579_584
    # the cubic model agrees with the general one on a free grid
    mb = Wl.model_bytes(256, 4, 4)
    assert mb["solve"] == Wl.solve_bytes((528, 528, 528), (264, 264, 264), 4)
