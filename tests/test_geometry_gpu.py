"""The one-launch geometry pass (dpb_geometry_cells_f64) against the separate
kernels it replaces and against the oracle.

normalize_coord + copy_coord must agree bit for bit with the oracle's
restatement of coord.cc / neighbor_list.cc (extended coordinates, types,
mapping, nall); the cell grid must equal the separate grid build's (header,
cell starts, cell of every atom; atoms inside a cell as a set, since their
order there is not defined). Cases cover cells of <= 32, 33..256 and > 256
atoms (the three ranking paths of the ghost copy), triclinic boxes, coordinates
outside the box, and a ghost capacity smaller than nall. Given a buffer of
dpb_cell_grid_bytes_packed bytes the fused pass also writes the atoms' cell-
ordered records (position, type, index), which the cell-list env kernels
read instead of gathering: the records must equal the extended arrays, and
the env kernels' outputs must not depend on them (bit for bit).
"""

import ctypes
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HDR_BYTES = 256  # grid header, rounded up to 256 bytes in the grid buffer


def _run(dpb, coord, atype, box, rcut, mem_nall, fused, packed=False):
    cap, dev = dpb._capi, torch.device("cuda:0")
    lib = cap.lib()
    nloc = atype.size
    boxc = np.ascontiguousarray(box, np.float64).reshape(9)
    gb = int(lib.dpb_cell_grid_bytes_packed(mem_nall) if packed else lib.dpb_cell_grid_bytes(mem_nall))
    sb = int(lib.dpb_geometry_scratch_bytes(nloc, ctypes.c_float(rcut), boxc.ctypes.data))
    c = torch.tensor(coord, dtype=torch.float64, device=dev).reshape(-1, 3).contiguous()
    c0 = c.clone()
    t = torch.tensor(atype, dtype=torch.int32, device=dev)
    cext = torch.full((mem_nall, 3), np.nan, dtype=torch.float64, device=dev)
    text = torch.full((mem_nall,), -7, dtype=torch.int32, device=dev)
    mapping = torch.full((mem_nall,), -7, dtype=torch.int32, device=dev)
    nall = torch.zeros(1, dtype=torch.int32, device=dev)
    grid = torch.full((gb,), 0xAB, dtype=torch.uint8, device=dev)
    scratch = torch.full((sb,), 0xCD, dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    old = lib.dpb_tune_get(b"geometry_fused")
    cap.call("dpb_tune_set", b"geometry_fused", 1 if fused else 0)
    try:
        s = torch.cuda.current_stream().cuda_stream
        cap.call("dpb_geometry_cells_f64", cap.ptr(cext), cap.ptr(text), cap.ptr(mapping),
                 cap.ptr(nall), cap.ptr(grid), gb, cap.ptr(scratch), sb, cap.ptr(c),
                 cap.ptr(t), nloc, mem_nall, ctypes.c_float(rcut), boxc.ctypes.data,
                 cap.ptr(status), s)
        cap.call("dpb_status_check", cap.ptr(status), s)
    finally:
        cap.call("dpb_tune_set", b"geometry_fused", old)
    assert torch.equal(c, c0), "the input coordinates must not change"
    n_all = int(nall.item())
    return dict(nall=n_all, cext=cext.cpu().numpy(), text=text.cpu().numpy(),
                mapping=mapping.cpu().numpy(), grid=_grid(grid.cpu().numpy(), mem_nall,
                                                          min(n_all, mem_nall)),
                dev=dict(grid=grid, cext=cext, text=text))


def _grid(buf, mem_nall, n):
    hdr = buf[:128]
    kmin = hdr[0:24].view(np.uint64)
    kmax = hdr[24:48].view(np.uint64)
    origin = hdr[48:72].view(np.float64)
    inv_cs = hdr[72:96].view(np.float64)
    ints = hdr[96:116].view(np.int32)
    dims, ncells, natoms = ints[:3].copy(), int(ints[3]), int(ints[4])
    packed = int(hdr[116:120].view(np.int32)[0])
    max_cells = max(mem_nall, 64)
    body = buf[HDR_BYTES:].view(np.int32)
    cell_start = body[:ncells + 1].copy()
    off = (max_cells + 1) + max_cells
    cell_of = body[off:off + n].copy()
    cell_atoms = body[off + mem_nall:off + mem_nall + n].copy()
    # cell-ordered records after the grid, at grid_bytes rounded up to 256
    ints_total = (max_cells + 1) + max_cells + 3 * mem_nall + 1 + 64
    off_rec = (128 + 256 + 4 * ints_total + 255) // 256 * 256
    rec = None
    if packed == 1:
        rec = buf[off_rec:off_rec + 32 * n].view(np.float64).reshape(-1, 4).copy()
    return dict(kmin=kmin.copy(), kmax=kmax.copy(), origin=origin.copy(),
                inv_cs=inv_cs.copy(), dims=dims, ncells=ncells, natoms=natoms,
                cell_start=cell_start, cell_of=cell_of, cell_atoms=cell_atoms,
                packed=packed, rec=rec)


def _same(a, b):
    assert a["nall"] == b["nall"]
    n = min(a["nall"], a["cext"].shape[0])
    assert np.array_equal(a["cext"][:n].view(np.uint64), b["cext"][:n].view(np.uint64))
    assert np.array_equal(a["text"][:n], b["text"][:n])
    assert np.array_equal(a["mapping"][:n], b["mapping"][:n])
    ga, gb = a["grid"], b["grid"]
    for k in ("kmin", "kmax", "dims", "origin", "inv_cs", "cell_start", "cell_of"):
        assert np.array_equal(ga[k], gb[k]), k
    assert ga["ncells"] == gb["ncells"] and ga["natoms"] == gb["natoms"]
    cs = ga["cell_start"]
    assert cs[-1] == ga["natoms"]
    for c in range(ga["ncells"]):
        sa = np.sort(ga["cell_atoms"][cs[c]:cs[c + 1]])
        sb = np.sort(gb["cell_atoms"][cs[c]:cs[c + 1]])
        assert np.array_equal(sa, sb), c
        assert np.all(ga["cell_of"][sa] == c)


def _against_oracle(port, got, coord, atype, box, rcut, mem_nall):
    cn = port.normalize_coord(np.asarray(coord, np.float64).reshape(-1, 3).copy(), box)
    c_ref, t_ref, m_ref = port.copy_coord(cn, atype, rcut, box)
    n = c_ref.shape[0]
    assert got["nall"] == n
    k = min(n, mem_nall)
    assert np.array_equal(got["cext"][:k].view(np.uint64),
                          np.ascontiguousarray(c_ref.reshape(-1, 3)[:k]).view(np.uint64))
    assert np.array_equal(got["text"][:k], t_ref[:k])
    assert np.array_equal(got["mapping"][:k], m_ref[:k])


def _water(dpb, n_side, seed=0):
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    return wl.water_frame(n_side, seed)


CASES = {
    # name: (frame builder, rcut)
    "water_192": (lambda d: _water(d, 4), 6.0),
    "water_1536": (lambda d: _water(d, 8, 1), 6.0),
    "dense_one_cell": (lambda d: _water(d, 4, 2), 9.0),     # nc = 1: 192 atoms per cell
    "dense_large_cell": (lambda d: _water(d, 5, 3), 10.0),  # nc = 1: 375 atoms per cell
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_equals_separate_and_oracle(dpb, port, name):
    build, rcut = CASES[name]
    coord, atype, box = build(dpb)
    mem = int(atype.size * 30) + 64
    a = _run(dpb, coord, atype, box, rcut, mem, fused=True)
    b = _run(dpb, coord, atype, box, rcut, mem, fused=False)
    _same(a, b)
    _against_oracle(port, a, coord, atype, box, rcut, mem)


def test_triclinic_and_outside_box(dpb, port):
    rng = np.random.default_rng(5)
    coord, atype, box = _water(dpb, 6, 4)
    box = np.array([[18.6, 0.0, 0.0], [3.1, 18.2, 0.0], [-2.4, 1.7, 17.9]]).reshape(9)
    coord = coord + rng.uniform(-25.0, 25.0, size=coord.shape)  # far outside the box
    mem = int(atype.size * 30) + 64
    a = _run(dpb, coord, atype, box, 6.0, mem, fused=True)
    b = _run(dpb, coord, atype, box, 6.0, mem, fused=False)
    _same(a, b)
    _against_oracle(port, a, coord, atype, box, 6.0, mem)


def test_ghost_capacity_smaller_than_nall(dpb):
    coord, atype, box = _water(dpb, 6, 6)
    full = _run(dpb, coord, atype, box, 6.0, atype.size * 30, fused=False)
    mem = atype.size + (full["nall"] - atype.size) // 2
    a = _run(dpb, coord, atype, box, 6.0, mem, fused=True)
    b = _run(dpb, coord, atype, box, 6.0, mem, fused=False)
    assert a["nall"] == full["nall"] > mem
    _same(a, b)
    assert np.array_equal(a["cext"][:mem], full["cext"][:mem])


def test_water_12288(dpb):
    """The 12,288-atom water frame of the single-frame benchmark."""
    coord, atype, box = _water(dpb, 16)
    mem = int(atype.size * 3)
    a = _run(dpb, coord, atype, box, 6.0, mem, fused=True)
    b = _run(dpb, coord, atype, box, 6.0, mem, fused=False)
    _same(a, b)


def _check_records(r):
    g = r["grid"]
    assert g["packed"] == 1
    n = g["natoms"]
    rec = g["rec"][:n]
    j = g["cell_atoms"][:n]
    assert np.array_equal(rec[:, :3].view(np.uint64), r["cext"][j].view(np.uint64))
    w = rec[:, 3].copy().view(np.int64)
    assert np.array_equal((w & 0xFFFFFFFF).astype(np.int64), j.astype(np.int64))
    assert np.array_equal((w >> 32).astype(np.int64), r["text"][j].astype(np.int64))


@pytest.mark.parametrize("name", ["water_192", "water_1536", "dense_one_cell"])
def test_packed_records(dpb, name):
    """The fused pass with a packed-size buffer writes one record per atom in
    cell order and flags the header; without the room, or from the separate
    kernels, the flag stays 0 and the rest of the grid is unchanged."""
    build, rcut = CASES[name]
    coord, atype, box = build(dpb)
    mem = int(atype.size * 30) + 64
    a = _run(dpb, coord, atype, box, rcut, mem, fused=True, packed=True)
    _check_records(a)
    b = _run(dpb, coord, atype, box, rcut, mem, fused=True)
    c = _run(dpb, coord, atype, box, rcut, mem, fused=False, packed=True)
    assert b["grid"]["packed"] == 0 and c["grid"]["packed"] == 0
    _same(a, b)
    _same(a, c)


def _env(dpb, r, nloc, mem_nall, rcut, sel, kind):
    cap, dev = dpb._capi, torch.device("cuda:0")
    ft = torch.float64 if kind == "f64" else torch.float32
    nnei = int(sum(sel))
    sec = np.concatenate([[0], np.cumsum(sel)]).astype(np.int32)
    ntypes = len(sel)
    g = torch.Generator().manual_seed(5)
    avg = (0.1 * torch.randn(ntypes, nnei * 4, generator=g, dtype=torch.float64)).to(dev, ft)
    std = (1.0 + 0.2 * torch.rand(ntypes, nnei * 4, generator=g, dtype=torch.float64)).to(dev, ft)
    em = torch.zeros(nloc, nnei * 4, dtype=ft, device=dev)
    ed = torch.zeros(nloc, nnei * 12, dtype=ft, device=dev)
    rij = torch.zeros(nloc, nnei * 3, dtype=ft, device=dev)
    nl = torch.zeros(nloc, nnei, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    d = r["dev"]
    s = torch.cuda.current_stream().cuda_stream
    fn = "dpb_env_mat_a_cells_f64" if kind == "f64" else "dpb_env_mat_a_cells_mixed"
    cap.call(fn, cap.ptr(em), cap.ptr(ed), cap.ptr(rij), cap.ptr(nl), cap.ptr(d["cext"]),
             cap.ptr(d["text"]), cap.ptr(d["grid"]), cap.ptr(avg), cap.ptr(std), nloc, mem_nall,
             ctypes.c_float(rcut), ctypes.c_float(0.5), sec.ctypes.data, sec.size,
             cap.ptr(status), s)
    cap.call("dpb_status_check", cap.ptr(status), s)
    return [t.cpu().numpy() for t in (em, ed, rij, nl)]


@pytest.mark.parametrize("kind", ["f64", "mixed"])
def test_env_packed_equals_gathered(dpb, kind):
    """The cell-list env kernel walking the packed records gives the same
    neighbor list, env matrix, derivative and rij as walking the atom indices
    (12,288-atom water and a dense one-cell frame with a small sel)."""
    for build, rcut, sel in ((lambda d: _water(d, 16), 6.0, [46, 92]),
                             (lambda d: _water(d, 4, 2), 9.0, [20, 40])):
        coord, atype, box = build(dpb)
        mem = int(atype.size * 30) + 64 if atype.size < 1000 else int(atype.size * 3)
        a = _run(dpb, coord, atype, box, rcut, mem, fused=True, packed=True)
        b = _run(dpb, coord, atype, box, rcut, mem, fused=True)
        assert a["grid"]["packed"] == 1 and b["grid"]["packed"] == 0
        oa = _env(dpb, a, atype.size, mem, rcut, sel, kind)
        ob = _env(dpb, b, atype.size, mem, rcut, sel, kind)
        for x, y in zip(oa, ob):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
        assert (oa[3] >= 0).any()
