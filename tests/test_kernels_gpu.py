"""Parity of the sm_100a kernels with the CPU oracle (run through the C-ABI).

Bars (the reference tests' own): neighbor lists and ghost arrays bit-exact;
FP64 results within 1e-10 absolute; FP32 results within 1e-5 (relative to
the value scale) -- test_env_mat_a.cc:1015-1029, test_tabulate_fusion_se_a.py:
22-31.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _t(x, dtype=None):
    return torch.tensor(np.asarray(x), device=DEV, dtype=dtype)


@pytest.fixture(scope="module")
def ops(dpb):
    return dpb.ops


@pytest.fixture(scope="module")
def wl(dpb):
    import importlib

    return importlib.import_module("deepmd_kit_lr_pt_b200.workload")


def _fp_tol(dtype):
    return 1e-10 if dtype == np.float64 else 1e-5


def _close(a, b, dtype, what):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    tol = _fp_tol(dtype)
    scale = max(1.0, float(np.abs(b).max())) if dtype == np.float32 else 1.0
    err = float(np.abs(a - b).max()) if a.size else 0.0
    assert err <= tol * scale, f"{what}: max abs error {err:.3e} > {tol * scale:.1e}"


# ------------------------------------------------------------------ coords
@pytest.mark.parametrize("n_side", [2, 4, 6])
def test_copy_coord_bit_exact(ops, port, wl, n_side):
    coord, atype, box = wl.water_frame(n_side, seed=3)
    for rc in (6.0, 4.5):
        c, t, m = ops.copy_coord(_t(coord), _t(atype), rc, box)
        c0, t0, m0 = port.copy_coord(coord, atype, rc, box)
        np.testing.assert_array_equal(c.cpu().numpy(), c0)
        np.testing.assert_array_equal(t.cpu().numpy(), t0)
        np.testing.assert_array_equal(m.cpu().numpy(), m0)


def test_copy_coord_golden(ops, ref_fixtures):
    key = "test_coord.cc:TestCopyCoord:"
    posi, atype = ref_fixtures[key + "posi"], ref_fixtures[key + "atype"].astype(np.int32)
    c, t, m = ops.copy_coord(_t(posi).view(-1, 3), _t(atype), 6.0, ref_fixtures[key + "boxt"])
    exp = ref_fixtures[key + "_expected_posi_cpy"].reshape(-1, 3)
    assert c.shape[0] == exp.shape[0]
    got = sorted(map(tuple, np.round(c.cpu().numpy()[6:], 8).tolist()))
    want = sorted(map(tuple, np.round(exp[6:], 8).tolist()))
    assert got == want


def test_copy_coord_capacity_code(ops, wl):
    coord, atype, box = wl.water_frame(2, seed=1)
    from deepmd_kit_lr_pt_b200 import _capi

    with pytest.raises(_capi.DPBCapacityError):
        ops.copy_coord(_t(coord), _t(atype), 6.0, box, mem_nall=30)


def test_normalize_golden(ops, ref_fixtures):
    key = "test_coord.cc:TestNormCoord:"
    for r in ("r0", "r1", "r2"):
        out = ops.normalize_coord(_t(ref_fixtures[key + r]).view(-1, 3), ref_fixtures[key + "boxt"])
        np.testing.assert_allclose(out.cpu().numpy().reshape(-1), ref_fixtures[key + "posi"],
                                   atol=1e-12, rtol=0)


# ------------------------------------------------------------- nlist build
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_build_nlist_equals_oracle(ops, port, wl, dtype):
    coord, atype, box = wl.water_frame(4, seed=5)
    c0, t0, _ = port.copy_coord(coord, atype, 6.0, box)
    nloc = atype.size
    ret, il0, nn0, rb0, mx0 = port.build_nlist(c0.astype(dtype), nloc, 6.0, atype=t0,
                                               mem_size=512)
    assert ret == 0
    il, nn, rows, mx = ops.build_nlist(_t(c0.astype(dtype)), nloc, 6.0, atype=_t(t0),
                                       mem_size=512)
    np.testing.assert_array_equal(il.cpu().numpy(), il0)
    np.testing.assert_array_equal(nn.cpu().numpy(), nn0)
    assert mx == mx0
    r = rows.cpu().numpy()
    for i in range(nloc):
        np.testing.assert_array_equal(r[i, : nn0[i]], rb0[i, : nn0[i]])


def test_build_nlist_capacity_retry(ops, port, wl):
    coord, atype, box = wl.water_frame(4, seed=2)
    c0, t0, _ = port.copy_coord(coord, atype, 6.0, box)
    nloc = atype.size
    from deepmd_kit_lr_pt_b200 import _capi

    with pytest.raises(_capi.DPBCapacityError):
        ops.build_nlist(_t(c0), nloc, 6.0, atype=_t(t0), mem_size=16)
    # without a fixed size the wrapper doubles until it fits (reference retry loop)
    il, nn, rows, mx = ops.build_nlist(_t(c0), nloc, 6.0, atype=_t(t0))
    assert rows.shape[1] >= mx


# ----------------------------------------------------------------- env mat
def _oracle_env(port, c0, t0, nloc, avg, std, rc, rs, sec, dtype):
    ret, il, nn, rb, _ = port.build_nlist(c0.astype(dtype), nloc, rc, atype=t0,
                                          mem_size=c0.shape[0])
    assert ret == 0
    return port.prod_env_mat_a(c0.astype(dtype), t0, il, nn, rb, avg.astype(dtype),
                               std.astype(dtype), nloc, rc, rs, sec), (il, nn, rb)


def _stats(rng, nnei, ntypes=2):
    avg = np.zeros((ntypes, nnei, 4))
    avg[:, :, 0] = rng.uniform(0.05, 0.2, size=(ntypes, 1))
    std = np.ones((ntypes, nnei, 4))
    std[:, :, 0] = rng.uniform(0.1, 0.3, size=(ntypes, 1))
    std[:, :, 1:] = rng.uniform(0.1, 0.3, size=(ntypes, 1, 1))
    return avg.reshape(ntypes, -1), std.reshape(ntypes, -1)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("sec", [[0, 46, 138], [0, 10, 20]])
def test_prod_env_mat_a_inlist(ops, port, wl, dtype, sec):
    coord, atype, box = wl.water_frame(4, seed=11)
    rc, rs = 6.0, 0.5
    c0, t0, _ = port.copy_coord(coord, atype, rc, box)
    nloc, nnei = atype.size, sec[-1]
    rng = np.random.default_rng(0)
    avg, std = _stats(rng, nnei)
    (e0, ed0, r0, n0), (il, nn, rb) = _oracle_env(port, c0, t0, nloc, avg, std, rc, rs,
                                                  np.array(sec), dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    em, emd, rij, nlist = ops.prod_env_mat_a(
        _t(c0.astype(dtype)), _t(t0), _t(il), _t(nn), _t(rb), _t(avg, tdt), _t(std, tdt),
        nloc, rc, rs, sec)
    np.testing.assert_array_equal(nlist.cpu().numpy(), n0)
    _close(em.cpu().numpy(), e0, dtype, "em")
    _close(emd.cpu().numpy(), ed0, dtype, "em_deriv")
    _close(rij.cpu().numpy(), r0, dtype, "rij")


@pytest.mark.parametrize("mode", ["f64", "f32", "mixed"])
@pytest.mark.parametrize("n_side,sec", [(4, [0, 46, 138]), (6, [0, 46, 138]), (3, [0, 8, 16])])
def test_env_mat_a_cells(ops, port, wl, mode, n_side, sec):
    """Fused neighbor search + format + env mat vs build_nlist_cpu -> prod_env_mat_a_cpu."""
    coord, atype, box = wl.water_frame(n_side, seed=17 + n_side)
    rc, rs = 6.0, 0.5
    c0, t0, _ = port.copy_coord(coord, atype, rc, box)
    nloc, nnei = atype.size, sec[-1]
    rng = np.random.default_rng(1)
    avg, std = _stats(rng, nnei)
    cdt = np.float32 if mode == "f32" else np.float64
    odt = np.float64 if mode == "f64" else np.float32
    (e0, ed0, r0, n0), _ = _oracle_env(port, c0, t0, nloc, avg, std, rc, rs, np.array(sec), cdt)
    tod = torch.float64 if odt == np.float64 else torch.float32
    em, emd, rij, nlist = ops.env_mat_a_cells(_t(c0.astype(cdt)), _t(t0), nloc, _t(avg, tod),
                                              _t(std, tod), rc, rs, sec, out_dtype=tod)
    np.testing.assert_array_equal(nlist.cpu().numpy(), n0)
    _close(em.cpu().numpy(), e0, odt, "em")
    _close(emd.cpu().numpy(), ed0, odt, "em_deriv")
    _close(rij.cpu().numpy(), r0, odt, "rij")


def test_env_mat_golden(ops, port, ref_fixtures):
    for cls in ("TestEnvMatA", "TestEnvMatAShortSel"):
        key = f"test_env_mat_a.cc:{cls}:"
        posi = ref_fixtures[key + "posi"]
        atype = ref_fixtures[key + "atype"].astype(np.int32)
        sec = ref_fixtures[key + "sec_a"].astype(np.int32)
        box = np.diag([13.0] * 3).reshape(9)
        cx, tx, _ = ops.copy_coord(_t(posi).view(-1, 3), _t(atype), 6.0, box)
        nnei = int(sec[-1])
        avg = torch.zeros((2, nnei * 4), dtype=torch.float64, device=DEV)
        std = torch.ones((2, nnei * 4), dtype=torch.float64, device=DEV)
        em, _, _, _ = ops.env_mat_a_cells(cx, tx, 6, avg, std, 6.0, 0.8, sec)
        np.testing.assert_allclose(em.cpu().numpy().reshape(-1), ref_fixtures[key + "expected_env"],
                                   atol=1e-5, rtol=0)


def test_sel_overflow_drops_farthest(ops, port, wl):
    """sel smaller than the neighbor count: the farthest of the type are dropped
    exactly as format_nlist_i_cpu does (fmt_nlist.cc:132-141)."""
    coord, atype, box = wl.water_frame(4, seed=23)
    rc, rs, sec = 6.0, 0.5, [0, 12, 20]
    c0, t0, _ = port.copy_coord(coord, atype, rc, box)
    nloc = atype.size
    avg = np.zeros((2, 80))
    std = np.ones((2, 80))
    (e0, _, _, n0), _ = _oracle_env(port, c0, t0, nloc, avg, std, rc, rs, np.array(sec),
                                    np.float64)
    em, _, _, nlist = ops.env_mat_a_cells(_t(c0), _t(t0), nloc, _t(avg), _t(std), rc, rs, sec)
    np.testing.assert_array_equal(nlist.cpu().numpy(), n0)


def test_env_mat_cpu_tensor_rejected(ops):
    from deepmd_kit_lr_pt_b200 import _capi

    with pytest.raises(_capi.DPBInvalidArgument):
        ops.env_mat_a_cells(torch.zeros((4, 3), dtype=torch.float64),
                            torch.zeros(4, dtype=torch.int32), 4, torch.zeros((1, 4)),
                            torch.ones((1, 4)), 6.0, 0.5, [0, 1])


# ---------------------------------------------------------------- tabulate
def _py_fix(fx, dtype):
    key = "test_tabulate_fusion_se_a.py:"
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    table = _t(fx[key + "table_tensor"], tdt)
    info = torch.tensor(fx[key + "table_info_tensor"], dtype=tdt)
    em_x = _t(fx[key + "em_x_tensor"], tdt)
    em = _t(fx[key + "em_tensor"], tdt)
    return key, table, info, em_x, em


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_tabulate_golden(dpb, ref_fixtures, dtype):
    key, table, info, em_x, em = _py_fix(ref_fixtures, dtype)
    tol = _fp_tol(dtype)
    em_x.requires_grad_(True)
    em.requires_grad_(True)
    out = torch.ops.deepmd.tabulate_fusion_se_a(table, info, em_x, em, 8)[0]
    np.testing.assert_allclose(out.detach().cpu().numpy(),
                               ref_fixtures[key + "expected_descriptor_tensor"], atol=tol, rtol=tol)
    out.sum().backward()
    np.testing.assert_allclose(em_x.grad.cpu().numpy(), ref_fixtures[key + "expected_dy_dem_x"],
                               atol=tol, rtol=tol)
    np.testing.assert_allclose(em.grad.cpu().numpy(), ref_fixtures[key + "expected_dy_dem"],
                               atol=tol, rtol=tol)


def test_tabulate_golden_cc(dpb, ref_fixtures):
    key = "test_tabulate_se_a.cc:TestTabulateSeA:"
    table = _t(ref_fixtures[key + "table"]).view(-1, 48)
    info = torch.tensor(ref_fixtures[key + "info"])
    em_x = _t(ref_fixtures[key + "em_x"]).view(4, 4)
    em = _t(ref_fixtures[key + "em"]).view(4, 4, 4)
    out = torch.ops.deepmd.tabulate_fusion_se_a(table, info, em_x, em, 8)[0]
    np.testing.assert_allclose(out.cpu().numpy().reshape(-1),
                               ref_fixtures[key + "expected_xyz_scatter"], atol=1e-5)
    dx, de = torch.ops.deepmd.tabulate_fusion_se_a_grad(table, info, em_x, em,
                                                        torch.ones_like(out), out)
    np.testing.assert_allclose(dx.cpu().numpy().reshape(-1), ref_fixtures[key + "expected_dy_dem_x"],
                               atol=1e-5)
    np.testing.assert_allclose(de.cpu().numpy().reshape(-1), ref_fixtures[key + "expected_dy_dem"],
                               atol=1e-5)


def _rand_tab_case(rng, nloc, nnei, M, pad, dtype):
    """Random table/em with sorted padding tails and some extrapolated x."""
    info = np.array([-1.0, 2.0, 4.0, 0.05, 0.2, -1.0])
    first = int((info[1] - info[0]) / info[3])
    nspline = first + int((np.nextafter(info[2], info[0]) - info[1]) / info[4]) + 1
    table = rng.normal(size=(nspline, 6 * M)) * 0.3
    em = rng.normal(size=(nloc, nnei, 4))
    em_x = rng.uniform(-1.5, 5.0, size=(nloc, nnei))  # below lower / above max too
    for i in range(nloc):
        npad = pad[i % len(pad)]
        if npad:
            em[i, nnei - npad:, 0] = -0.7
            em[i, nnei - npad:, 1:] = 0.0
            em_x[i, nnei - npad:] = -0.7
    em[:, :, 0] = em_x
    return (table.astype(dtype), info.astype(dtype), em_x.astype(dtype), em.astype(dtype))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("M", [8, 100, 200])
def test_tabulate_random(dpb, port, dtype, M):
    rng = np.random.default_rng(M)
    nloc, nnei = 37, 46
    table, info, em_x, em = _rand_tab_case(rng, nloc, nnei, M, [0, 5, 20, 46, 1], dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    tt, ti, tx, te = _t(table, tdt), torch.tensor(info), _t(em_x, tdt), _t(em, tdt)
    out = torch.ops.deepmd.tabulate_fusion_se_a(tt, ti, tx, te, M)[0]
    _close(out.cpu().numpy(), port.tabulate(table, info, em_x, em, M), dtype, "forward")
    dy = rng.normal(size=(nloc, 4, M)).astype(dtype)
    dx, de = torch.ops.deepmd.tabulate_fusion_se_a_grad(tt, ti, tx, te, _t(dy, tdt), out)
    rx, re = port.tabulate_grad(table, info, em_x, em, dy, M)
    _close(dx.cpu().numpy(), rx, dtype, "dy_dem_x")
    _close(de.cpu().numpy(), re, dtype, "dy_dem")
    zx = rng.normal(size=em_x.shape).astype(dtype)
    ze = rng.normal(size=em.shape).astype(dtype)
    dz = torch.ops.deepmd.tabulate_fusion_se_a_grad_grad(tt, ti, tx, te, _t(zx, tdt),
                                                         _t(ze, tdt), out, True)[0]
    _close(dz.cpu().numpy(), port.tabulate_grad_grad(table, info, em_x, em, zx, ze, M), dtype,
           "grad_grad")


def test_tabulate_empty_neighbors(dpb):
    table = torch.zeros((4, 48), dtype=torch.float64, device=DEV)
    info = torch.tensor([0, 0.2, 0.4, 0.01, 0.1, -1], dtype=torch.float64)
    em_x = torch.zeros((4, 0), dtype=torch.float64, device=DEV)
    em = torch.zeros((4, 0, 4), dtype=torch.float64, device=DEV)
    out = torch.ops.deepmd.tabulate_fusion_se_a(table, info, em_x, em, 8)[0]
    assert out.shape == (4, 4, 8) and float(out.abs().max()) == 0.0


def test_tabulate_second_order_fd(dpb, ref_fixtures):
    """Double backward against central differences of the first backward,
    as test_tabulate_fusion_se_a.py:1495-1508 does (FP64, eps 1e-6)."""
    key, table, info, em_x, em = _py_fix(ref_fixtures, np.float64)
    em_x = em_x.clone().requires_grad_(True)
    em = em.clone().requires_grad_(True)
    torch.manual_seed(0)

    def first(dyv):
        out = torch.ops.deepmd.tabulate_fusion_se_a(table, info, em_x, em, 8)[0]
        gx, ge = torch.autograd.grad((out * dyv).sum(), (em_x, em), create_graph=True)
        return gx, ge

    dy = torch.randn((4, 4, 8), dtype=torch.float64, device=DEV).requires_grad_(True)
    gx, ge = first(dy)
    zx, ze = torch.randn_like(gx), torch.randn_like(ge)
    (ana,) = torch.autograd.grad((gx * zx).sum() + (ge * ze).sum(), dy)
    eps = 1e-6
    num = torch.zeros_like(dy)
    flat = dy.detach().clone().view(-1)
    for k in range(flat.numel()):
        vals = []
        for s in (1.0, -1.0):
            d2 = flat.clone()
            d2[k] += s * eps
            a, b = first(d2.view_as(dy))
            vals.append(float(((a * zx).sum() + (b * ze).sum()).detach()))
        num.view(-1)[k] = (vals[0] - vals[1]) / (2 * eps)
    np.testing.assert_allclose(ana.cpu().numpy(), num.cpu().numpy(), atol=1e-6, rtol=1e-6)


def test_tabulate_device_errors(dpb):
    from deepmd_kit_lr_pt_b200 import _capi

    table = torch.zeros((4, 48), dtype=torch.float64, device=DEV)
    em_x = torch.zeros((4, 4), dtype=torch.float64, device=DEV)
    em = torch.zeros((4, 4, 4), dtype=torch.float64, device=DEV)
    with pytest.raises(Exception, match="table_info must be on the CPU"):
        torch.ops.deepmd.tabulate_fusion_se_a(table, torch.zeros(6, dtype=torch.float64, device=DEV),
                                              em_x, em, 8)
    info = torch.tensor([0, 0.2, 0.4, 0.01, 0.1, -1], dtype=torch.float64)
    with pytest.raises(Exception, match="between 1 and 1024"):
        torch.ops.deepmd.tabulate_fusion_se_a(table, info, em_x, em, 2048)
    with pytest.raises(Exception, match="same device"):
        torch.ops.deepmd.tabulate_fusion_se_a(table, info, em_x.cpu(), em, 8)
    with pytest.raises(Exception):
        torch.ops.deepmd.tabulate_fusion_se_a(table.cpu(), info, em_x.cpu(), em.cpu(), 8)
    del _capi


# ----------------------------------------------------------- force/virial
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_prod_force_virial_random(ops, port, wl, dtype):
    coord, atype, box = wl.water_frame(4, seed=31)
    rc, rs, sec = 6.0, 0.5, np.array([0, 46, 138])
    c0, t0, _ = port.copy_coord(coord, atype, rc, box)
    nloc, nall, nnei = atype.size, c0.shape[0], 138
    avg, std = _stats(np.random.default_rng(3), nnei)
    (e0, ed0, r0, n0), _ = _oracle_env(port, c0, t0, nloc, avg, std, rc, rs, sec, dtype)
    nd = np.random.default_rng(4).normal(size=(nloc, nnei * 4)).astype(dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    f = ops.prod_force_a(_t(nd, tdt), _t(ed0, tdt), _t(n0), nloc, nall)
    _close(f.cpu().numpy(), port.prod_force_a(nd, ed0, n0, nloc, nall), dtype, "force")
    v, av = ops.prod_virial_a(_t(nd, tdt), _t(ed0, tdt), _t(r0, tdt), _t(n0), nloc, nall)
    v0, av0 = port.prod_virial_a(nd, ed0, r0, n0, nloc, nall)
    _close(v.cpu().numpy(), v0, dtype, "virial")
    _close(av.cpu().numpy(), av0, dtype, "atom_virial")


def test_prod_force_virial_golden(ops, port, ref_fixtures):
    kf = "test_prod_force_a.cc:TestProdForceA:"
    kv = "test_prod_virial_a.cc:TestProdVirialA:"
    posi, atype = ref_fixtures[kf + "posi"], ref_fixtures[kf + "atype"].astype(np.int32)
    box = np.diag([13.0] * 3).reshape(9)
    sec = ref_fixtures[kf + "sec_a"].astype(np.int32)
    c0, t0, _ = port.copy_coord(posi, atype, 6.0, box)
    nloc, nall, nnei = 6, c0.shape[0], int(sec[-1])
    avg, std = np.zeros((2, nnei * 4)), np.ones((2, nnei * 4))
    (e0, ed0, r0, n0), _ = _oracle_env(port, c0, t0, nloc, avg, std, 6.0, 0.8, sec, np.float64)
    nd = 10 - np.arange(nloc * nnei * 4) * 0.01
    f = ops.prod_force_a(_t(np.tile(nd, 2)), _t(np.tile(ed0.reshape(-1), 2)),
                         _t(np.tile(n0.reshape(-1), 2)), nloc, nall, nframes=2)
    np.testing.assert_allclose(f.cpu().numpy().reshape(-1),
                               np.tile(ref_fixtures[kf + "expected_force"], 2), atol=1e-5)
    v, av = ops.prod_virial_a(_t(nd), _t(ed0), _t(r0), _t(n0), nloc, nall)
    np.testing.assert_allclose(v.cpu().numpy(), ref_fixtures[kv + "expected_virial"], atol=1e-5)
    np.testing.assert_allclose(av.cpu().numpy().reshape(-1),
                               ref_fixtures[kv + "expected_atom_virial"], atol=1e-5)


# ------------------------------------------ force / virial second derivatives
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_prod_force_virial_grad(ops, port, wl, dtype):
    coord, atype, box = wl.water_frame(4, seed=37)
    rc, rs, sec = 6.0, 0.5, np.array([0, 46, 138])
    c0, t0, _ = port.copy_coord(coord, atype, rc, box)
    nloc, nnei = atype.size, 138
    avg, std = _stats(np.random.default_rng(5), nnei)
    (e0, ed0, r0, n0), _ = _oracle_env(port, c0, t0, nloc, avg, std, rc, rs, sec, dtype)
    rng = np.random.default_rng(6)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    for nframes in (1, 2):
        gf = rng.normal(size=(nframes * nloc, 3)).astype(dtype)
        edn = np.tile(ed0.reshape(-1), nframes)
        nln = np.tile(n0.reshape(-1), nframes)
        g = ops.prod_force_grad_a(_t(gf, tdt), _t(edn, tdt), _t(nln), nloc, nframes)
        _close(g.cpu().numpy(), port.prod_force_grad_a(gf, edn, nln, nloc, nframes), dtype,
               "force_grad")
    gv = rng.normal(size=9).astype(dtype)
    g = ops.prod_virial_grad_a(_t(gv, tdt), _t(ed0, tdt), _t(r0, tdt), _t(n0), nloc)
    _close(g.cpu().numpy(), port.prod_virial_grad_a(gv, ed0, r0, n0, nloc), dtype, "virial_grad")


def test_prod_force_virial_grad_golden(ops, port, ref_fixtures):
    fx = ref_fixtures
    for key, kind in (("test_prod_force_grad_a.cc:TestProdForceGradA:", "force"),
                      ("test_prod_virial_grad_a.cc:TestProdVirialGradA:", "virial")):
        posi, atype = fx[key + "posi"], fx[key + "atype"].astype(np.int32)
        box = np.diag([13.0] * 3).reshape(9)
        sec = fx[key + "sec_a"].astype(np.int32)
        c0, t0, _ = port.copy_coord(posi, atype, 6.0, box)
        nnei = int(sec[-1])
        avg = np.zeros((2, nnei * 4))
        std = np.ones((2, nnei * 4))
        (e0, ed0, r0, n0), _ = _oracle_env(port, c0, t0, 6, avg, std, 6.0, 0.8, sec, np.float64)
        if kind == "force":
            grad = 10 - np.arange(18) * 0.1
            g = ops.prod_force_grad_a(_t(grad), _t(ed0), _t(n0), 6)
        else:
            grad = 10 - np.arange(9) * 1.0
            g = ops.prod_virial_grad_a(_t(grad), _t(ed0), _t(r0), _t(n0), 6)
        np.testing.assert_allclose(g.cpu().numpy().reshape(-1), fx[key + "expected_grad_net"],
                                   atol=1e-5, rtol=0)
