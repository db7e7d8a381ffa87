"""Pins the CPU checkers against the reference's own golden vectors.

The C restatement (``port``) is checked against every golden vector the
reference's unit tests hold for this path, and -- where the reference CPU
library could be compiled from its sources -- bit-for-bit against it on
seeded random inputs. Tolerances are the reference tests' own.
"""

import numpy as np
import pytest

F = "test_env_mat_a.cc:TestEnvMatA:"


def _six_atoms(fx):
    posi = fx[F + "posi"]
    atype = fx[F + "atype"].astype(np.int32)
    box = np.diag([13.0, 13.0, 13.0]).reshape(9)
    return posi, atype, box


def _env_pipeline(lib, posi, atype, box, sec, rc=6.0, rc_smth=0.8, dtype=np.float64):
    c, t, _ = lib.copy_coord(posi, atype, rc, box)
    nloc = atype.size
    ret, il, nn, rb, _ = lib.build_nlist(c.astype(dtype), nloc, rc, atype=t)
    assert ret == 0
    nnei = sec[-1]
    avg = np.zeros((2, nnei * 4), dtype)
    std = np.ones((2, nnei * 4), dtype)
    return c, t, lib.prod_env_mat_a(c.astype(dtype), t, il, nn, rb, avg, std, nloc,
                                    rc, rc_smth, sec)


@pytest.mark.parametrize("cls", ["TestEnvMatA", "TestEnvMatAShortSel"])
def test_env_mat_golden(port, ref_fixtures, cls):
    fx = ref_fixtures
    key = f"test_env_mat_a.cc:{cls}:"
    posi, atype, box = fx[key + "posi"], fx[key + "atype"].astype(np.int32), np.diag([13.0] * 3).reshape(9)
    sec = fx[key + "sec_a"].astype(np.int32)
    _, _, (em, emd, rij, nlist) = _env_pipeline(port, posi, atype, box, sec,
                                                float(fx[key + "rc"]), float(fx[key + "rc_smth"]))
    np.testing.assert_allclose(em.reshape(-1), fx[key + "expected_env"], atol=1e-5, rtol=0)


def test_env_mat_numerical_derivative(port, ref_fixtures):
    """em_deriv is d(em)/d(r_center) (env_mat.cc:146) = -d(em)/d(r_neighbor);
    checked against central differences (test_env_mat_a.cc:281-324)."""
    posi, atype, box = _six_atoms(ref_fixtures)
    sec = np.array([0, 10, 20], np.int32)
    c, t, (em, emd, rij, nlist) = _env_pipeline(port, posi, atype, box, sec)
    nloc, nnei, h = 6, 20, 1e-7
    for i in range(nloc):
        for jj in range(nnei):
            j = nlist[i, jj]
            if j < 0:
                continue
            for d in range(3):
                out = []
                for s in (+1, -1):
                    cc = c.copy()
                    cc[j, d] += s * h
                    r = cc[j] - cc[i]
                    r2 = r @ r
                    nr = np.sqrt(r2)
                    u = (nr - 0.8) / (6.0 - 0.8)
                    sw = 1.0 if nr < 0.8 else (u**3 * (-6 * u * u + 15 * u - 10) + 1 if nr < 6 else 0)
                    out.append(np.array([1 / nr, r[0] / r2, r[1] / r2, r[2] / r2]) * sw)
                num = (out[0] - out[1]) / (2 * h)
                ana = emd[i, jj * 12:(jj + 1) * 12].reshape(4, 3)[:, d]
                np.testing.assert_allclose(ana, -num, atol=1e-5)


def test_prod_force_golden(port, ref_fixtures):
    fx = ref_fixtures
    key = "test_prod_force_a.cc:TestProdForceA:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    box = np.diag([13.0] * 3).reshape(9)
    sec = fx[key + "sec_a"].astype(np.int32)
    c, t, (em, emd, rij, nlist) = _env_pipeline(port, posi, atype, box, sec)
    nloc, nall, nnei = 6, c.shape[0], int(sec[-1])
    nd = 10 - np.arange(nloc * nnei * 4) * 0.01
    # the gtest doubles every array to run two identical frames
    force = port.prod_force_a(np.tile(nd, 2), np.tile(emd.reshape(-1), 2),
                              np.tile(nlist.reshape(-1), 2), nloc, nall, nframes=2)
    exp = np.tile(fx[key + "expected_force"], 2)
    np.testing.assert_allclose(force.reshape(-1), exp, atol=1e-5, rtol=0)


def test_prod_virial_golden(port, ref_fixtures):
    fx = ref_fixtures
    key = "test_prod_virial_a.cc:TestProdVirialA:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    box = np.diag([13.0] * 3).reshape(9)
    sec = fx[key + "sec_a"].astype(np.int32)
    c, t, (em, emd, rij, nlist) = _env_pipeline(port, posi, atype, box, sec)
    nloc, nall, nnei = 6, c.shape[0], int(sec[-1])
    nd = 10 - np.arange(nloc * nnei * 4) * 0.01
    v, av = port.prod_virial_a(nd, emd, rij, nlist, nloc, nall)
    np.testing.assert_allclose(v, fx[key + "expected_virial"], atol=1e-5, rtol=0)
    np.testing.assert_allclose(av.reshape(-1), fx[key + "expected_atom_virial"], atol=1e-5, rtol=0)


def test_prod_force_grad_golden(port, ref_fixtures):
    """test_prod_force_grad_a.cc: grad[i] = 10 - 0.1 i, two identical frames."""
    fx = ref_fixtures
    key = "test_prod_force_grad_a.cc:TestProdForceGradA:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    box = np.diag([13.0] * 3).reshape(9)
    sec = fx[key + "sec_a"].astype(np.int32)
    c, t, (em, emd, rij, nlist) = _env_pipeline(port, posi, atype, box, sec)
    nloc = 6
    grad = 10 - np.arange(nloc * 3) * 0.1
    g = port.prod_force_grad_a(np.tile(grad, 2), np.tile(emd.reshape(-1), 2),
                               np.tile(nlist.reshape(-1), 2), nloc, nframes=2)
    exp = np.tile(fx[key + "expected_grad_net"], 2)
    np.testing.assert_allclose(g.reshape(-1), exp, atol=1e-5, rtol=0)


def test_prod_virial_grad_golden(port, ref_fixtures):
    """test_prod_virial_grad_a.cc: grad[k] = 10 - k."""
    fx = ref_fixtures
    key = "test_prod_virial_grad_a.cc:TestProdVirialGradA:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    box = np.diag([13.0] * 3).reshape(9)
    sec = fx[key + "sec_a"].astype(np.int32)
    c, t, (em, emd, rij, nlist) = _env_pipeline(port, posi, atype, box, sec)
    grad = 10 - np.arange(9) * 1.0
    g = port.prod_virial_grad_a(grad, emd, rij, nlist, 6)
    np.testing.assert_allclose(g.reshape(-1), fx[key + "expected_grad_net"], atol=1e-5, rtol=0)


def _sorted_ghosts(c, t, m, nloc):
    rows = sorted(zip(map(tuple, c[nloc:].tolist()), t[nloc:].tolist(), m[nloc:].tolist()))
    return rows


@pytest.mark.parametrize("cls", ["TestCopyCoord", "TestCopyCoordMoreCell"])
def test_copy_coord_golden(port, ref_fixtures, cls):
    fx = ref_fixtures
    key = f"test_coord.cc:{cls}:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    c, t, m = port.copy_coord(posi, atype, float(fx[key + "rc"]), fx[key + "boxt"])
    ec = fx[key + "_expected_posi_cpy"].reshape(-1, 3)
    et = fx[key + "_expected_atype_cpy"]
    em = fx[key + "_expected_mapping"]
    assert c.shape == ec.shape
    # the gtest compares after sorting the ghost block (test_coord.cc:131-165)
    got, exp = _sorted_ghosts(c, t, m, 6), _sorted_ghosts(ec, et, em, 6)
    for (gc, gt, gm), (xc, xt, xm) in zip(got, exp):
        assert gt == xt and gm == xm
        np.testing.assert_allclose(gc, xc, atol=1e-10)
    np.testing.assert_array_equal(c[:6], ec[:6])


def test_normalize_golden(port, ref_fixtures):
    fx = ref_fixtures
    key = "test_coord.cc:TestNormCoord:"
    for r in ("r0", "r1", "r2"):
        out = port.normalize_coord(fx[key + r], fx[key + "boxt"])
        np.testing.assert_allclose(out, fx[key + "posi"], atol=1e-12, rtol=0)


def test_tabulate_golden_cc(port, ref_fixtures):
    fx = ref_fixtures
    key = "test_tabulate_se_a.cc:TestTabulateSeA:"
    nloc, nnei, M = (int(fx[key + n]) for n in ("nloc", "nnei", "last_layer_size"))
    table, info = fx[key + "table"], fx[key + "info"]
    em_x = fx[key + "em_x"].reshape(nloc, nnei)
    em = fx[key + "em"].reshape(nloc, nnei, 4)
    out = port.tabulate(table, info, em_x, em, M)
    np.testing.assert_allclose(out.reshape(-1), fx[key + "expected_xyz_scatter"], atol=1e-5)
    dy = np.ones((nloc, 4, M))
    dx, de = port.tabulate_grad(table, info, em_x, em, dy, M)
    np.testing.assert_allclose(dx.reshape(-1), fx[key + "expected_dy_dem_x"], atol=1e-5)
    np.testing.assert_allclose(de.reshape(-1), fx[key + "expected_dy_dem"], atol=1e-5)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-10), (np.float32, 1e-5)])
def test_tabulate_golden_py(port, ref_fixtures, dtype, tol):
    fx = ref_fixtures
    key = "test_tabulate_fusion_se_a.py:"
    table = fx[key + "table_tensor"].astype(dtype).reshape(-1)
    info = fx[key + "table_info_tensor"].astype(dtype)
    em_x = fx[key + "em_x_tensor"].astype(dtype)
    em = fx[key + "em_tensor"].astype(dtype)
    M = int(fx[key + "last_layer_size"])
    out = port.tabulate(table, info, em_x, em, M)
    np.testing.assert_allclose(out, fx[key + "expected_descriptor_tensor"], atol=tol, rtol=tol)
    dx, de = port.tabulate_grad(table, info, em_x, em, np.ones_like(out), M)
    np.testing.assert_allclose(dx, fx[key + "expected_dy_dem_x"], atol=tol, rtol=tol)
    np.testing.assert_allclose(de, fx[key + "expected_dy_dem"], atol=tol, rtol=tol)


def test_tabulate_grad_grad_is_adjoint(port, ref_fixtures):
    """grad is linear in dy, so grad_grad must be its adjoint:
    <dz_dy, dy> == <dz_dem_x, dy_dem_x(dy)> + <dz_dem, dy_dem(dy)>."""
    fx = ref_fixtures
    key = "test_tabulate_fusion_se_a.py:"
    table = fx[key + "table_tensor"].reshape(-1)
    info = fx[key + "table_info_tensor"]
    em_x, em = fx[key + "em_x_tensor"], fx[key + "em_tensor"]
    M = 8
    rng = np.random.default_rng(0)
    dy = rng.normal(size=(4, 4, M))
    zx, ze = rng.normal(size=em_x.shape), rng.normal(size=em.shape)
    dx, de = port.tabulate_grad(table, info, em_x, em, dy, M)
    dz = port.tabulate_grad_grad(table, info, em_x, em, zx, ze, M)
    lhs = (dz * dy).sum()
    rhs = (zx * dx).sum() + (ze * de).sum()
    assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs))


# ------------------------------------------------------------------ random parity
def _random_water(rng, nmol=24, box=9.0):
    """Loose random water-like frame: O uniform in the box, two H at ~1 A."""
    o = rng.uniform(0, box, size=(nmol, 3))
    h1 = o + rng.normal(size=(nmol, 3)) * 0.55
    h2 = o + rng.normal(size=(nmol, 3)) * 0.55
    coord = np.stack([o, h1, h2], 1).reshape(-1, 3) % box
    atype = np.tile([0, 1, 1], nmol).astype(np.int32)
    return coord, atype, np.diag([box] * 3).reshape(9)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_port_equals_reference_random(port, ref_lib, dtype):
    rng = np.random.default_rng(7)
    coord, atype, box = _random_water(rng)
    sec = np.array([0, 12, 30], np.int32)
    rc, rs = 4.0, 0.5
    outs = []
    for lib in (port, ref_lib):
        c, t, m = lib.copy_coord(coord, atype, rc, box)
        nloc = atype.size
        ret, il, nn, rb, _ = lib.build_nlist(c.astype(dtype), nloc, rc, atype=t)
        avg = rng.normal(size=(2, sec[-1] * 4)).astype(dtype) * 0 + 0.1
        std = np.full((2, sec[-1] * 4), 0.7, dtype)
        env = lib.prod_env_mat_a(c.astype(dtype), t, il, nn, rb, avg, std, nloc, rc, rs, sec)
        outs.append((c, t, m, nn, rb, env))
    (c0, t0, m0, nn0, rb0, e0), (c1, t1, m1, nn1, rb1, e1) = outs
    np.testing.assert_array_equal(c0, c1)
    np.testing.assert_array_equal(m0, m1)
    np.testing.assert_array_equal(nn0, nn1)
    for a, b in zip(e0, e1):
        np.testing.assert_array_equal(a, b)
    # tabulate / force / virial on these shapes
    em, emd, rij, nlist = e1
    nloc, nnei, M = atype.size, int(sec[-1]), 16
    table = rng.normal(size=(40, 6 * M)).astype(dtype)
    info = np.array([-2.0, 1.0, 2.0, 0.1, 0.2, -1], dtype)
    emv = em.reshape(nloc, nnei, 4)
    ex = emv[:, :, 0].copy()
    o0 = port.tabulate(table, info, ex, emv, M)
    o1 = ref_lib.tabulate(table, info, ex, emv, M)
    np.testing.assert_array_equal(o0, o1)
    dy = rng.normal(size=o0.shape).astype(dtype)
    for a, b in zip(port.tabulate_grad(table, info, ex, emv, dy, M),
                    ref_lib.tabulate_grad(table, info, ex, emv, dy, M)):
        np.testing.assert_array_equal(a, b)
    zx = rng.normal(size=ex.shape).astype(dtype)
    ze = rng.normal(size=emv.shape).astype(dtype)
    np.testing.assert_array_equal(port.tabulate_grad_grad(table, info, ex, emv, zx, ze, M),
                                  ref_lib.tabulate_grad_grad(table, info, ex, emv, zx, ze, M))
    nd = rng.normal(size=(nloc, nnei * 4)).astype(dtype)
    nall = c1.shape[0]
    np.testing.assert_array_equal(port.prod_force_a(nd, emd, nlist, nloc, nall),
                                  ref_lib.prod_force_a(nd, emd, nlist, nloc, nall))
    v0, a0 = port.prod_virial_a(nd, emd, rij, nlist, nloc, nall)
    v1, a1 = ref_lib.prod_virial_a(nd, emd, rij, nlist, nloc, nall)
    # the reference accumulates the virial under an OpenMP atomic in thread
    # order, so FP32 sums of a few hundred terms differ run to run in the
    # last digits
    tol = 1e-12 if dtype == np.float64 else 1e-4
    np.testing.assert_allclose(v0, v1, rtol=tol, atol=tol)
    np.testing.assert_allclose(a0, a1, rtol=tol, atol=tol)
    # second derivatives (prod_force_grad_a / prod_virial_grad_a), neighbor
    # indices of ghosts folded modulo nloc as the reference does
    gf = rng.normal(size=(nloc, 3)).astype(dtype)
    np.testing.assert_array_equal(port.prod_force_grad_a(gf, emd, nlist, nloc),
                                  ref_lib.prod_force_grad_a(gf, emd, nlist, nloc))
    gv = rng.normal(size=9).astype(dtype)
    np.testing.assert_array_equal(port.prod_virial_grad_a(gv, emd, rij, nlist, nloc),
                                  ref_lib.prod_virial_grad_a(gv, emd, rij, nlist, nloc))


def test_format_nlist_ties_break_by_index(port):
    """Equal float r^2 sorts by neighbor index (fmt_nlist.cc:14-26)."""
    posi = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0]], np.float64)
    atype = np.zeros(5, np.int32)
    r, fmt = port_format(port, posi, atype, [4, 3, 2, 1])
    assert r == -1
    np.testing.assert_array_equal(fmt, [1, 2, 3, 4, -1])


def port_format(port, posi, atype, cand):
    from oracle import oracle

    return oracle.format_nlist_i(posi, atype, 0, np.array(cand, np.int32), 6.0,
                                 np.array([0, 5], np.int32))


def test_format_nlist_overflow_reports_type(port):
    posi = np.array([[0, 0, 0], [1, 0, 0], [0, 1.1, 0], [0, 0, 1.2]], np.float64)
    atype = np.array([0, 1, 1, 1], np.int32)
    from oracle import oracle

    r, fmt = oracle.format_nlist_i(posi, atype, 0, np.array([1, 2, 3], np.int32), 6.0,
                                   np.array([0, 1, 3], np.int32))
    assert r == 1  # three type-1 neighbors into two slots: farthest dropped
    np.testing.assert_array_equal(fmt, [-1, 1, 2])


# --------------------------------------------- neighbor-list golden vectors
def _pbc_shift(idx: int, n: int) -> int:
    """compute_pbc_shift (source/lib/src/neighbor_list.cc:731-745)."""
    s = 0
    if idx < 0:
        s = 1
        while idx + s * n < 0:
            s += 1
    elif idx >= n:
        s = -1
        while idx + s * n >= n:
            s -= 1
    return s


def _legacy_copy_coord(posi, atype, rc, box):
    """Ghosts in the order of the reference's older std::vector copy_coord
    (source/lib/src/neighbor_list.cc:747-830 with the cell list of build_clist,
    :43-113), the order behind the ghost indices of the golden lists in
    test_fmt_nlist.cc and test_neighbor_list.cc. Orthorhombic boxes only (the
    fixtures use a 13 A cube): internal coordinates are x / L, a ghost is
    its owner minus the cell-image shift times L, and ghost cells are walked
    x-major over [-ngcell, ncell + ngcell) with the local cells skipped."""
    L = np.diag(np.asarray(box, np.float64).reshape(3, 3))
    ncell = [max(int(L[d] / rc), 1) for d in range(3)]
    ngcell = [int(rc / (L[d] / ncell[d])) + 1 for d in range(3)]
    p = np.asarray(posi, np.float64).reshape(-1, 3)
    nloc = p.shape[0]
    clist: dict[tuple, list] = {}
    for i in range(nloc):
        idx = []
        for d in range(3):
            u = p[i, d] / L[d]
            k = int(u / (1.0 / ncell[d]))
            if u < 0.0:
                k -= 1
            idx.append(min(max(k, 0), ncell[d] - 1))
        clist.setdefault(tuple(idx), []).append(i)
    out_c, out_t, mapping = [x for x in p], list(atype), list(range(nloc))
    rng = [range(-ngcell[d], ncell[d] + ngcell[d]) for d in range(3)]
    for i0 in rng[0]:
        for i1 in rng[1]:
            for i2 in rng[2]:
                ii = (i0, i1, i2)
                if all(0 <= ii[d] < ncell[d] for d in range(3)):
                    continue
                sh = [_pbc_shift(ii[d], ncell[d]) for d in range(3)]
                jj = tuple(ii[d] + sh[d] * ncell[d] for d in range(3))
                shift_v = np.array(sh, np.float64) * L
                for q in clist.get(jj, []):
                    out_c.append(p[q] - shift_v)
                    out_t.append(atype[q])
                    mapping.append(q)
    return (np.array(out_c, np.float64), np.array(out_t, np.int32),
            np.array(mapping, np.int32))


def test_legacy_ghosts_equal_copy_coord_cpu(port, ref_fixtures):
    """On the golden lists' fixture the older ghost order and the oracle's
    copy_coord_cpu order are the same array (owners, types, coordinates), so
    the golden indices below refer to the oracle's own ghosts."""
    fx, key = ref_fixtures, "test_fmt_nlist.cc:TestFormatNlist:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    box = np.diag([13.0] * 3).reshape(9)
    c0, t0, m0 = _legacy_copy_coord(posi, atype, float(fx[key + "rc"]), box)
    c1, t1, m1 = port.copy_coord(posi, atype, float(fx[key + "rc"]), box)
    np.testing.assert_array_equal(m0, m1)
    np.testing.assert_array_equal(t0, t1)
    np.testing.assert_array_equal(c0, c1.reshape(-1, 3))


@pytest.mark.parametrize("which", ["port", "ref_lib"])
@pytest.mark.parametrize("cls", ["TestFormatNlist", "TestFormatNlistShortSel"])
def test_format_nlist_golden(request, ref_fixtures, cls, which):
    """test_fmt_nlist.cc (cpu): ghost copy, raw list and the list formatted
    into the sel slots (type, float r^2, index order) give expect_nlist_cpy
    index for index (the oracle, and the reference library as the harness's
    own check)."""
    port = request.getfixturevalue(which)
    fx, key = ref_fixtures, f"test_fmt_nlist.cc:{cls}:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    rc, sec = float(fx[key + "rc"]), fx[key + "sec_a"].astype(np.int32)
    c, t, _ = port.copy_coord(posi, atype, rc, np.diag([13.0] * 3).reshape(9))
    c = c.reshape(-1, 3)
    nloc, nnei = atype.size, int(sec[-1])
    ret, il, nn, rb, _ = port.build_nlist(c, nloc, rc, atype=t)
    assert ret == 0
    avg = np.zeros((2, nnei * 4))
    std = np.ones((2, nnei * 4))
    nlist = port.prod_env_mat_a(c, t, il, nn, rb, avg, std, nloc, rc, 0.5, sec)[3]
    np.testing.assert_array_equal(nlist.reshape(-1), fx[key + "expect_nlist_cpy"])


@pytest.mark.parametrize("which", ["port", "ref_lib"])
def test_build_nlist_golden(request, ref_fixtures, which):
    """test_neighbor_list.cc (cpu): every extended atom within rc of each
    local atom (strict r^2 < rc^2), compared as sorted rows, and the longest
    row (max_list_size 5)."""
    port = request.getfixturevalue(which)
    fx, key = ref_fixtures, "test_neighbor_list.cc:TestNeighborList:"
    posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
    rc = float(fx[key + "rc"])
    c, t, _ = port.copy_coord(posi, atype, rc, fx[key + "boxt"])
    nloc = atype.size
    ret, il, nn, rb, mx = port.build_nlist(c.reshape(-1, 3), nloc, rc, mem_size=10)
    assert ret == 0 and mx == 5
    np.testing.assert_array_equal(il, np.arange(nloc))
    flat, lens = fx[key + "expect_nlist_cpy"], fx[key + "expect_nlist_cpy_len"]
    np.testing.assert_array_equal(nn, lens)
    o = 0
    for i in range(nloc):
        np.testing.assert_array_equal(np.sort(rb[i, :nn[i]]), np.sort(flat[o:o + lens[i]]))
        o += lens[i]


# ------------------------------------- tabulate extrapolation known answers
def _kat_locate(xx, info):
    """Interval, offset and extrapolation distance of x on a two-stride
    table, as test_tabulate_extrapolate.cc's se_a lookup states it: below
    lower the first interval at offset 0 with distance x - lower; at or above
    max the interval holding nextafter(max, lower) at the offset of max with
    distance x - max."""
    lower, upper, mx, s0, s1 = info[:5]
    if xx < lower:
        return 0, 0.0, xx - lower
    if xx < upper:
        k = int((xx - lower) / s0)
        return k, xx - (k * s0 + lower), 0.0
    first = int((upper - lower) / s0)
    if xx < mx:
        k = first + int((xx - upper) / s1)
        return k, xx - ((k - first) * s1 + upper), 0.0
    k = first + int((np.nextafter(mx, lower) - upper) / s1)
    return k, mx - ((k - first) * s1 + upper), xx - mx


def _poly(c, x):
    return c[0] + (c[1] + (c[2] + (c[3] + (c[4] + c[5] * x) * x) * x) * x) * x


def _dpoly(c, x):
    return c[1] + (2 * c[2] + (3 * c[3] + (4 * c[4] + 5 * c[5] * x) * x) * x) * x


@pytest.mark.parametrize("which", ["port", "ref_lib"])
@pytest.mark.parametrize("info_key,points", [
    ("kTableInfo", ("below", "max", "above")),
    ("kOffGridTableInfo", ("max", "above")),
])
def test_tabulate_extrapolation_known_answers(request, ref_fixtures, info_key, points, which):
    """test_tabulate_extrapolate.cc (SeAUsesC1LinearTails and the off-grid
    max case of the shared lookup): outside [lower, max) the value is the
    boundary polynomial continued linearly with its slope (C1 tails) and
    dy/dx is that slope; one neighbor, em = (1, 0, 0, 0), M = 1."""
    port = request.getfixturevalue(which)
    fx, k = ref_fixtures, "test_tabulate_extrapolate.cc:"
    table, info = fx[k + "kTable"], fx[k + info_key]
    tol = float(fx[k + "kTolerance"])
    lower, mx = float(fx[k + "kLower"]), float(info[2])
    xs = {"below": lower - 0.25, "max": mx, "above": mx + 0.25}
    em = np.array([[[1.0, 0.0, 0.0, 0.0]]])
    for name in points:
        xx = xs[name]
        idx, off, delta = _kat_locate(xx, info)
        c = table[6 * idx:6 * idx + 6]
        want_v = _poly(c, off) + _dpoly(c, off) * delta
        want_g = _dpoly(c, off)
        ex = np.array([[xx]])
        out = port.tabulate(table, info, ex, em, 1)
        assert abs(out.reshape(-1)[0] - want_v) <= tol, (name, out.reshape(-1)[0], want_v)
        dy = np.zeros((1, 4, 1))
        dy[0, 0, 0] = 1.0
        dx, de = port.tabulate_grad(table, info, ex, em, dy, 1)
        assert abs(dx.reshape(-1)[0] - want_g) <= tol, (name, dx.reshape(-1)[0], want_g)
        assert abs(de.reshape(-1)[0] - want_v) <= tol


def test_tabulate_grad_grad_in_tails(port, ref_fixtures):
    """test_tabulate_extrapolate.cc (GradGradKernelsMatchDyFiniteDifferenceInTails,
    se_a): in both tails, the second-derivative op applied to the fixed
    (dz_dem_x, dz_dem) equals the central difference, over dy, of the
    projection <dz_dem_x, dy_dem_x(dy)> + <dz_dem, dy_dem(dy)>."""
    fx, k = ref_fixtures, "test_tabulate_extrapolate.cc:"
    table, info = fx[k + "kTable"], fx[k + "kTableInfo"]
    h = float(fx[k + "kFiniteDiffStep"])
    em = np.array([[[0.7, -0.3, 0.2, 0.5]]])
    zx, ze = np.array([[0.4]]), np.array([[[0.1, -0.2, 0.3, -0.4]]])
    for xx in (float(fx[k + "kLower"]) - 0.25, float(fx[k + "kMax"]) + 0.25):
        ex = np.array([[xx]])
        dz = port.tabulate_grad_grad(table, info, ex, em, zx, ze, 1).reshape(-1)

        def proj(dy):
            dx, de = port.tabulate_grad(table, info, ex, em, dy.reshape(1, 4, 1), 1)
            return float((zx * dx).sum() + (ze * de).sum())

        for i in range(4):
            e = np.zeros(4)
            e[i] = h
            fd = (proj(np.full(4, 0.3) + e) - proj(np.full(4, 0.3) - e)) / (2 * h)
            assert abs(dz[i] - fd) <= 1e-8, (xx, i, dz[i], fd)
