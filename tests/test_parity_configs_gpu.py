"""Parity of the benchmark configurations with the CPU oracle.

* FCC Cu neighbor lists (sel [46, 92, 60]: about 78 Cu neighbors inside 6 A
  against 60 slots, so the truncation order decides which neighbors stay):
  bit-exact against build_nlist_cpu -> format_nlist_i_cpu (fmt_nlist.cc:
  98-143) on the same ghost coordinates, for the single-frame fused env pass
  and for the batched env pass (whose neighbor index is atom * 27 + image
  code; it is mapped back to ghost coordinates for the oracle). Rows whose
  order differs only between exactly tied float r^2 keys are counted apart.
* Batched frames (water and Cu, 3-species model): energy, force and virial
  against the FP64 oracle of the same compressed model and against the FP64
  plain model.
* The 12,288-atom water frame: the compressed FP32 path against the FP64
  oracle of the compressed model over every atom, and the FP64 plain GPU path
  against the FP64 plain oracle.

Tolerances: neighbor lists bit-exact; env rows FP32 1e-5 relative (the
reference tests' FP32 bar); E/F/V |dE|/N <= 1e-6 eV/atom and force RMSE <=
1e-5 eV/A for the mixed-precision path (the target accuracy of this path),
1e-10 for the FP64 plain path.
"""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
SEL3 = (46, 92, 60)


def _t(x, dtype=None):
    return torch.tensor(np.asarray(x), device=DEV, dtype=dtype)


@pytest.fixture(scope="module")
def checker():
    """The reference CPU library compiled from its sources where present,
    else the C restatement (both are pinned to each other by the CPU tests)."""
    from oracle import oracle

    return oracle.ref() or oracle.port()


@pytest.fixture(scope="module")
def mods(dpb):
    imp = importlib.import_module
    return (imp("deepmd_kit_lr_pt_b200.workload"), imp("deepmd_kit_lr_pt_b200.model"),
            imp("deepmd_kit_lr_pt_b200.batch"))


def _stats3(rng, nnei):
    avg = np.zeros((3, nnei, 4))
    avg[:, :, 0] = rng.uniform(0.05, 0.2, size=(3, 1))
    std = np.ones((3, nnei, 4))
    std[:, :, 0] = rng.uniform(0.1, 0.3, size=(3, 1))
    std[:, :, 1:] = rng.uniform(0.1, 0.3, size=(3, 1, 1))
    return avg.reshape(3, -1), std.reshape(3, -1)


def _r2f(ci, cj):
    """format_nlist_i_cpu's key distance: float32 differences, float32 r^2
    summed left to right without contraction."""
    d = cj.astype(np.float32) - ci.astype(np.float32)
    return (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]


def _compare_rows(got, want, r2_of, nloc):
    """Bit-exact comparison of two formatted lists; a row may differ only in
    the order of entries whose float r^2 keys tie exactly. Returns the number
    of such tied rows."""
    ties = 0
    for i in np.nonzero(np.any(got != want, axis=1))[0]:
        g, w = got[i], want[i]
        assert np.array_equal(g >= 0, w >= 0), f"row {i}: different slot occupancy"
        pos = np.nonzero(g != w)[0]
        assert np.array_equal(r2_of(i, g[pos]), r2_of(i, w[pos])), \
            f"row {i}: slots {pos.tolist()} differ and their float r^2 keys do not tie"
        ties += 1
    return ties


# --------------------------------------------------- Cu neighbor lists ---
@pytest.mark.parametrize("n_atoms,seed", [(32, 1), (256, 2), (400, 3), (1500, 4)])
def test_cu_nlist_single_frame_bit_exact(dpb, checker, mods, n_atoms, seed):
    """Fused neighbor search + format (k_env) on FCC Cu frames with vacancies
    against build_nlist_cpu -> prod_env_mat_a_cpu on copy_coord_cpu ghosts."""
    wl = mods[0]
    rng = np.random.default_rng(seed)
    coord, atype, box = wl.cu_frame(n_atoms, rng)
    rc, rs = 6.0, 0.5
    sec = np.concatenate([[0], np.cumsum(SEL3)]).astype(np.int32)
    nnei = int(sec[-1])
    cn = checker.normalize_coord(coord.reshape(-1), box).reshape(-1, 3)
    c0, t0, _ = checker.copy_coord(cn, atype, rc, box)
    avg, std = _stats3(np.random.default_rng(seed + 10), nnei)
    ret, il, nn, rb, _ = checker.build_nlist(c0, n_atoms, rc, atype=t0, mem_size=c0.shape[0])
    assert ret == 0
    # the truncation is exercised: Cu atoms with more than 60 Cu neighbors
    # (all of them in a full lattice; fewer where vacancies thin the shells)
    assert np.mean(nn > SEL3[2]) > 0.1, "the frame does not overflow sel"
    e0, _, _, n0 = checker.prod_env_mat_a(c0, t0, il, nn, rb, avg, std, n_atoms, rc, rs, sec)
    for out in (torch.float32, torch.float64):
        em, _, _, nlist = dpb.ops.env_mat_a_cells(_t(c0), _t(t0), n_atoms, _t(avg, out),
                                                  _t(std, out), rc, rs, sec, out_dtype=out)
        got = nlist.cpu().numpy()
        ties = _compare_rows(got, n0, lambda i, js: _r2f(c0[i], c0[js]), n_atoms)
        assert ties == 0, f"{ties} rows differ by tied keys"
        tol = 1e-10 if out == torch.float64 else 1e-5 * max(1.0, float(np.abs(e0).max()))
        assert float(np.abs(em.cpu().numpy().astype(np.float64) - e0).max()) <= tol


def _batch_ext(cw, L, n):
    """Extended coordinates of one frame for the oracle: the n wrapped atoms
    first (image code 13), then every (atom, image) pair with a non-zero
    shift; returns (coords [n + 26 n, 3], packed index of every entry)."""
    codes = [c for c in range(27) if c != 13]
    sh = np.array([[c // 9 - 1, (c // 3) % 3 - 1, c % 3 - 1] for c in codes], np.float64)
    ghosts = cw[None, :, :] + sh[:, None, :] * L[None, None, :]
    ext = np.concatenate([cw, ghosts.reshape(-1, 3)])
    packed = np.concatenate([np.arange(n) * 27 + 13,
                             (np.arange(n)[None, :] * 27 + np.array(codes)[:, None]).reshape(-1)])
    return ext, packed.astype(np.int64)


def test_batched_nlist_bit_exact(dpb, checker, mods):
    """Batched env pass (k_bt_env, packed (atom, image) neighbors) on Cu and
    water frames against build_nlist_cpu -> prod_env_mat_a_cpu over the same
    periodic images (the frame's wrapped coordinates plus the 26 shifts)."""
    wl, mdl, bt = mods
    rng = np.random.default_rng(5)
    frames = [wl.cu_frame(32, rng), wl.water_frame_density(150, rng), wl.cu_frame(500, rng),
              wl.cu_frame(1100, rng), wl.water_frame_density(600, rng)]
    cfg = mdl.SeAConfig(sel=SEL3)
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=3), frames)
    ev = bt.BatchEvaluator(params, frames)
    ev.compute()
    ev.check()
    cw_all = ev.cw.cpu().numpy()
    nl_all = ev.nlist.cpu().numpy()
    em_all = ev.em.cpu().numpy().astype(np.float64)
    tied = 0
    for f, (coord, atype, box) in enumerate(frames):
        sl = ev.frame_slice(f)
        n = atype.size
        L = np.diag(np.asarray(box).reshape(3, 3)).copy()
        cw = cw_all[sl]
        ext, packed = _batch_ext(cw, L, n)
        text = np.concatenate([atype, np.tile(atype, 26)]).astype(np.int32)
        ret, il, nn, rb, _ = checker.build_nlist(ext, n, cfg.rcut, atype=text, mem_size=512)
        assert ret == 0
        e0, _, _, n0 = checker.prod_env_mat_a(ext, text, il, nn, rb, params.davg, params.dstd,
                                              n, cfg.rcut, cfg.rcut_smth, cfg.sec)
        want = np.where(n0 >= 0, packed[np.maximum(n0, 0)], -1)
        got = nl_all[sl]
        pos = {int(p): k for k, p in enumerate(packed)}

        def r2_of(i, js, ext=ext, pos=pos):
            return _r2f(ext[i], ext[[pos[int(j)] for j in js]])

        tied += _compare_rows(got.astype(np.int64), want, r2_of, n)
        # env rows slot by slot, the oracle's slots put in the batched order
        # (they differ only where two neighbors tie exactly)
        e_orig = e0.reshape(n, cfg.nnei, 4)
        e0 = e_orig.copy()
        mine = em_all[sl].reshape(n, cfg.nnei, 4).copy()
        for i, k in zip(*np.nonzero(got != want)):
            src = np.nonzero(want[i] == got[i, k])[0]
            if src.size:
                e0[i, k] = e_orig[i, int(src[0])]
            else:  # a tie at the truncation edge: only the radial column is comparable
                mine[i, k, 1:] = e0[i, k, 1:]
        scale = max(1.0, float(np.abs(e0).max()))
        err = float(np.abs(mine - e0).max())
        assert err <= 1e-5 * scale, f"frame {f}: env rows {err:.2e}"
        if atype[0] == 2 and n >= 256:  # Cu: the 60 Cu slots overflow
            assert np.mean(nn > SEL3[2]) > 0.1, f"frame {f} does not overflow sel"
    # exact float r^2 ties order by index, and the two index spaces (ghost
    # index, atom * 27 + image) differ; such rows are reported, and rare
    print(f"rows ordered differently between exactly tied keys: {tied}")
    assert tied <= 5, f"{tied} rows differ by tied keys"


# --------------------------------------------- batched frames: E / F / V ---
@pytest.mark.parametrize("fused", [True, False])
def test_batched_frames_vs_fp64_oracle(dpb, checker, mods, fused):
    """Water and Cu frames of the batched path (one persistent launch, or one
    launch per stage) against the FP64 oracle of the same compressed model
    (and the plain model)."""
    from oracle import model_ref

    wl, mdl, bt = mods
    rng = np.random.default_rng(8)
    frames = [wl.water_frame_density(420, rng), wl.cu_frame(500, rng),
              wl.water_frame_density(90, rng), wl.cu_frame(64, rng)]
    cfg = mdl.SeAConfig(sel=SEL3)
    params = mdl.prepare_frames(mdl.init_params(cfg, seed=3), frames)
    ev = bt.BatchEvaluator(params, frames, fused=fused)
    E, F, V = ev.compute()
    ev.check()
    for f, (coord, atype, box) in enumerate(frames):
        n = atype.size
        for mode, etol, ftol in (("compressed", 1e-6, 1e-5), ("plain", 1e-5, 1e-4)):
            e0, f0, v0 = model_ref.evaluate(checker, params, coord, atype, box, mode=mode)
            e_err = abs(E[f] - e0) / n
            f_rmse = float(np.sqrt(np.mean((F[ev.frame_slice(f)] - f0) ** 2)))
            v_err = float(np.abs(V[f] - v0).max())
            print(f"frame {f} ({n} atoms) vs FP64 {mode}: |dE|/N {e_err:.2e} eV/atom, "
                  f"force RMSE {f_rmse:.2e} eV/A, |dV| {v_err:.2e}")
            assert e_err <= etol, (f, mode)
            assert f_rmse <= ftol, (f, mode)
            assert v_err <= 10 * ftol * max(1.0, float(np.abs(v0).max())), (f, mode)


# ------------------------------------------ 12,288-atom water frame -------
@pytest.fixture(scope="module")
def water12288(dpb, mods):
    wl, mdl, _ = mods
    coord, atype, box = wl.water_frame(16, seed=100)
    params = mdl.init_params(mdl.SeAConfig(), seed=1)
    mdl.prepare(params, coord, atype, box)
    return coord, atype, box, params


@pytest.mark.parametrize("degree", [5, 3])
def test_water12288_compressed_vs_fp64_oracle(checker, mods, water12288, degree):
    """The benchmark frame: the mixed-precision compressed path (the
    reference's quintic table, or its cubic re-interpolation) against the FP64
    oracle of the same compressed model, every atom."""
    from oracle import model_ref

    mdl = mods[1]
    coord, atype, box, params = water12288
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed", table_degree=degree)
    E, F, V = ev.compute(coord)
    ev.check()
    e0, f0, v0 = model_ref.evaluate(checker, params, coord, atype, box, mode="compressed",
                                    chunk=2048)
    n = atype.size
    e_err = abs(E - e0) / n
    f_rmse = float(np.sqrt(np.mean((F - f0) ** 2)))
    v_err = float(np.abs(V - v0).max())
    print(f"12,288 atoms, compressed FP32 (table degree {degree}) vs FP64 oracle: "
          f"|dE|/N {e_err:.2e} eV/atom, "
          f"force RMSE {f_rmse:.2e} eV/A, max |dF| {np.abs(F - f0).max():.2e}, |dV| {v_err:.2e}")
    assert e_err <= 1e-6
    assert f_rmse <= 1e-5
    assert v_err <= 1e-5 * max(1.0, float(np.abs(v0).max()))


def test_water12288_plain_fp64_vs_fp64_oracle(checker, mods, water12288):
    """The FP64 plain GPU path (the denominator of the speed-up) against the
    FP64 plain oracle on the benchmark frame."""
    from oracle import model_ref

    mdl = mods[1]
    coord, atype, box, params = water12288
    ev = mdl.SeAEvaluator(params, atype, box, mode="plain")
    E, F, V = ev.compute(coord)
    ev.check()
    e0, f0, v0 = model_ref.evaluate(checker, params, coord, atype, box, mode="plain",
                                    chunk=1024)
    assert abs(E - e0) <= 1e-10 * abs(e0)
    np.testing.assert_allclose(F, f0, atol=1e-10, rtol=0)
    np.testing.assert_allclose(V, v0, atol=1e-8 * max(1.0, float(np.abs(v0).max())), rtol=0)
