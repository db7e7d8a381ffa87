"""The seeded synthetic inputs of the benchmarks (workload.py) have the
shapes and physical properties their docstrings and the benchmark
configurations state: 192- and 12,288-atom water boxes of rigid molecules,
water at 1.0 g/cm^3, FCC Cu with vacancies, and the 512-frame uneven batch.
numpy only (the module is loaded on its own, as the reference arm loads it)."""

import numpy as np
import pytest

import bench

wl = bench._workload_module()


def _min_image(d, L):
    return d - L * np.round(d / L)


@pytest.mark.parametrize("n_side,natoms,box", [(4, 192, 12.4172), (16, 12288, 49.6688)])
def test_water_frame_shape_and_geometry(n_side, natoms, box):
    c, t, b = wl.water_frame(n_side, seed=3)
    assert c.shape == (natoms, 3) and t.shape == (natoms,) and t.dtype == np.int32
    np.testing.assert_array_equal(t, np.tile([0, 1, 1], natoms // 3))
    np.testing.assert_allclose(b, np.diag([box] * 3).reshape(9), rtol=0, atol=1e-12)
    assert (c >= 0).all() and (c < box).all()
    m = c.reshape(-1, 3, 3)
    oh1 = _min_image(m[:, 1] - m[:, 0], box)
    oh2 = _min_image(m[:, 2] - m[:, 0], box)
    np.testing.assert_allclose(np.linalg.norm(oh1, axis=1), wl.OH, atol=1e-12)
    np.testing.assert_allclose(np.linalg.norm(oh2, axis=1), wl.OH, atol=1e-12)
    cosang = (oh1 * oh2).sum(1) / wl.OH ** 2
    np.testing.assert_allclose(np.arccos(np.clip(cosang, -1, 1)), wl.HOH, atol=1e-9)
    # O on the 3.104 A grid within the +-0.3 A jitter
    g = np.arange(n_side) * wl.SPACING
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    assert np.abs(_min_image(m[:, 0] - grid, box)).max() <= 0.3 + 1e-12


def test_water_frame_is_seeded():
    a = wl.water_frame(4, seed=5)
    b = wl.water_frame(4, seed=5)
    c = wl.water_frame(4, seed=6)
    np.testing.assert_array_equal(a[0], b[0])
    assert not np.array_equal(a[0], c[0])


def test_random_rotations_are_proper():
    R = wl.random_rotations(np.random.default_rng(0), 500)
    np.testing.assert_allclose(np.einsum("nij,nkj->nik", R, R),
                               np.broadcast_to(np.eye(3), R.shape), atol=1e-12)
    np.testing.assert_allclose(np.linalg.det(R), 1.0, atol=1e-12)
    # uniform on SO(3): the mean rotation vanishes
    assert np.abs(R.mean(0)).max() < 0.1


@pytest.mark.parametrize("n", [24, 100, 1000, 2958])
def test_water_density_frame(n):
    c, t, b = wl.water_frame_density(n, np.random.default_rng(n))
    nm = max(1, round(n / 3))
    assert c.shape == (3 * nm, 3)
    L = b[0]
    grams = nm * 18.015 / 6.0221408e23
    assert grams / (L * 1e-8) ** 3 == pytest.approx(1.0, rel=1e-9)
    assert (c >= 0).all() and (c < L).all()
    m = c.reshape(-1, 3, 3)
    d = np.linalg.norm(_min_image(m[:, 1:] - m[:, :1], L), axis=2)
    np.testing.assert_allclose(d, wl.OH, atol=1e-12)


@pytest.mark.parametrize("n", [24, 31, 500, 2999])
def test_cu_frame_vacancies(n):
    rng = np.random.default_rng(n)
    c, t, b = wl.cu_frame(n, rng)
    assert c.shape == (n, 3) and (t == 2).all()
    L = b[0]
    k = round(L / wl.CU_A)
    assert k >= 2 and 4 * k ** 3 >= n and (k == 2 or 4 * (k - 1) ** 3 < n)
    assert L > 6.0  # every edge above the cutoff
    assert (c >= 0).all() and (c < L).all()
    # every atom within a few sigma of an FCC site; no two atoms on one site
    frac = c / wl.CU_A
    sites = np.round(frac * 2) / 2
    assert np.abs(_min_image((frac - sites) * wl.CU_A, L)).max() < 6 * 0.05
    key = np.mod(np.round(sites * 2).astype(int), 2 * k)
    assert len({tuple(x) for x in key}) == n


def test_batched_frames_of_the_benchmark():
    fr = wl.batched_frames(512, seed=0)
    counts = np.array([a.size for _, a, _ in fr])
    assert len(fr) == 512 and counts.sum() == 355449
    assert counts.min() >= 24 and counts.max() <= 3000
    for f, (c, a, b) in enumerate(fr[:20]):
        if f % 2 == 0:
            assert set(np.unique(a)) <= {0, 1}
        else:
            assert (a == 2).all()
        assert min(b[0], b[4], b[8]) >= 6.0
    # log-uniform sizes: the median near the geometric mean of the range
    assert 150 < np.median(counts) < 400
