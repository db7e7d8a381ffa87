"""Reading the reference's serialized se_e2_a model (checkpoint.py) on CPU.

The layout is pinned by tests/golden/state_dict_golden.npz: the names,
shapes and checksums of every state-dict entry of the reference's own
compressed model (made by tests/golden/make_state_dict_golden.py with the
reference's enable_compression on the seeded weights). The writer must
produce those names and shapes with the same values (the tables to the
precision in which this package's builder reproduces the reference
compressor), and the reader must recover the model from them."""

import importlib
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                    "state_dict_golden.npz")


@pytest.fixture(scope="module")
def layout():
    with np.load(GOLD) as z:
        g = {k: z[k] for k in z.files}
    shapes, o = {}, 0
    for k, n in zip(g["keys"], g["ndim"]):
        shapes[str(k)] = tuple(int(x) for x in g["dims"][o:o + n])
        o += n
    sums = {str(k): (float(s), float(a)) for k, s, a in zip(g["keys"], g["sums"], g["abssums"])}
    return g, shapes, sums


@pytest.fixture(scope="module")
def model(dpb, layout):
    from oracle import model_ref, oracle, table_ref

    g = layout[0]
    mdl = importlib.import_module("deepmd_kit_lr_pt_b200.model")
    wl = importlib.import_module("deepmd_kit_lr_pt_b200.workload")
    cfg = mdl.SeAConfig()
    p = mdl.init_params(cfg, seed=1)
    coord, atype, box = wl.water_frame(4, seed=0)
    p.davg, p.dstd, mind = model_ref.env_stats(oracle.port(), cfg, coord, atype, box)
    assert abs(mind - float(g["min_nbor_dist"])) < 1e-12
    p.tables = table_ref.build_tables(p.emb, p.davg, p.dstd, cfg.sel, mind, cfg.rcut_smth,
                                      cfg.rcut)
    return p


def test_writer_matches_reference_layout(dpb, layout, model):
    ck = importlib.import_module("deepmd_kit_lr_pt_b200.checkpoint")
    _, shapes, sums = layout
    sd = ck.params_to_state_dict(model)
    for k, v in sd.items():
        assert k in shapes, f"{k} is not a reference state-dict entry"
        assert tuple(v.shape) == shapes[k], (k, tuple(v.shape), shapes[k])
        s, a = float(v.sum()), float(v.abs().sum())
        tol = 1e-6 if "compress_data" in k else 1e-9
        assert abs(s - sums[k][0]) <= tol * max(1.0, sums[k][1]), (k, s, sums[k][0])
        assert abs(a - sums[k][1]) <= tol * max(1.0, sums[k][1]), (k, a, sums[k][1])
    # everything the reader needs is in the reference's layout
    needed = [k for k in shapes if ".networks." in k or "compress_" in k or
              k.endswith(("sea.mean", "sea.stddev", "out_bias"))]
    assert sorted(needed) == sorted(sd), sorted(set(needed) ^ set(sd))


def test_reader_round_trip_and_prefixes(dpb, layout, model):
    ck = importlib.import_module("deepmd_kit_lr_pt_b200.checkpoint")
    g = layout[0]
    sd = ck.params_to_state_dict(model)
    # a training checkpoint: the wrapper prefix and the "_networks" copies
    wrapped = {"model": {"model.Default." + k.replace(".networks.", "._networks."): v
                         for k, v in sd.items()}}
    for src in (sd, wrapped):
        p = ck.load(src, sel=tuple(int(x) for x in g["sel"]), rcut=float(g["rcut"]))
        assert p.cfg.sel == model.cfg.sel and p.cfg.neuron == model.cfg.neuron
        assert p.cfg.axis_neuron == model.cfg.axis_neuron and p.cfg.fitting == model.cfg.fitting
        np.testing.assert_array_equal(p.davg, model.davg)
        np.testing.assert_array_equal(p.dstd, model.dstd)
        for (a, b), (c, d) in zip([x for net in p.emb for x in net],
                                  [x for net in model.emb for x in net]):
            np.testing.assert_array_equal(a, c)
            np.testing.assert_array_equal(b, d)
        for f0, f1 in zip(p.fit, model.fit):
            for (W, b, d), (W1, b1, d1) in zip(f0["layers"], f1["layers"]):
                np.testing.assert_array_equal(W, W1)
                np.testing.assert_array_equal(b, b1)
                assert (d is None) == (d1 is None)
                if d is not None:
                    np.testing.assert_array_equal(d, d1)
            np.testing.assert_array_equal(f0["out"][0], np.asarray(f1["out"][0]).reshape(-1, 1))
        assert len(p.tables) == 2
        for (t0, i0), (t1, i1) in zip(p.tables, model.tables):
            np.testing.assert_array_equal(t0, t1)
            np.testing.assert_array_equal(i0, i1)


def test_reader_from_checkpoint_file(dpb, layout, model, tmp_path):
    """A training checkpoint file as the reference writes it (the wrapper's
    state dict under "model", optimizer state and training info beside it)
    read back by path, with the default weights-only unpickling."""
    import torch

    ck = importlib.import_module("deepmd_kit_lr_pt_b200.checkpoint")
    g = layout[0]
    sd = ck.params_to_state_dict(model)
    wrapped = {"model.Default." + k.replace(".networks.", "._networks."): v
               for k, v in sd.items()}
    wrapped["_extra_state"] = {"model_params": {"type_map": ["O", "H"]},
                               "train_infos": {"lr": 1e-3, "step": 10}}
    path = str(tmp_path / "model.ckpt.pt")
    torch.save({"model": wrapped, "optimizer": {"state": {}, "param_groups": [{"lr": 1e-3}]}},
               path)
    p = ck.load(path, sel=tuple(int(x) for x in g["sel"]), rcut=float(g["rcut"]))
    np.testing.assert_array_equal(p.davg, model.davg)
    for (t0, i0), (t1, i1) in zip(p.tables, model.tables):
        np.testing.assert_array_equal(t0, t1)
        np.testing.assert_array_equal(i0, i1)
    for (a, b), (c, d) in zip([x for net in p.emb for x in net],
                              [x for net in model.emb for x in net]):
        np.testing.assert_array_equal(a, c)
        np.testing.assert_array_equal(b, d)


def _scripted_model(sd, sel, rcut):
    """A TorchScript module with the reference model's state-dict layout and
    its get_sel / get_rcut (the two facts the reader takes from a frozen or
    compressed model file besides the state dict)."""
    from typing import List

    import torch

    class Node(torch.nn.Module):
        pass

    class Frozen(torch.nn.Module):
        def __init__(self):
            super().__init__()
            for k, v in sd.items():
                parts = k.split(".")
                m = self
                for part in parts[:-1]:
                    if part not in m._modules:
                        m.add_module(part, Node())
                    m = m._modules[part]
                m.register_buffer(parts[-1], v)
            self.sel = [int(x) for x in sel]
            self.rcut = float(rcut)

        @torch.jit.export
        def get_sel(self) -> List[int]:
            return self.sel

        @torch.jit.export
        def get_rcut(self) -> float:
            return self.rcut

        def forward(self, x: torch.Tensor) -> torch.Tensor:
            return x

    return torch.jit.script(Frozen())


def test_reader_from_torchscript_file(dpb, layout, model, tmp_path):
    """A frozen / compressed TorchScript file: sel and rcut come from the
    model's own get_sel / get_rcut, the entries (tables included) from its
    state dict."""
    import torch

    ck = importlib.import_module("deepmd_kit_lr_pt_b200.checkpoint")
    g = layout[0]
    sd = ck.params_to_state_dict(model)
    path = str(tmp_path / "frozen_compressed.pth")
    torch.jit.save(_scripted_model(sd, g["sel"], g["rcut"]), path)
    p = ck.load(path)
    assert p.cfg.sel == tuple(int(x) for x in g["sel"]) and p.cfg.rcut == float(g["rcut"])
    np.testing.assert_array_equal(p.dstd, model.dstd)
    assert len(p.tables) == len(model.tables)
    for (t0, i0), (t1, i1) in zip(p.tables, model.tables):
        np.testing.assert_array_equal(t0, t1)
        np.testing.assert_array_equal(i0, i1)
    for f0, f1 in zip(p.fit, model.fit):
        for (W, b, _), (W1, b1, _) in zip(f0["layers"], f1["layers"]):
            np.testing.assert_array_equal(W, W1)
            np.testing.assert_array_equal(b, b1)


class _Opaque:
    """An object only a full unpickler can rebuild."""


def test_reader_refuses_pickled_objects_unless_trusted(dpb, model, tmp_path):
    """A file that needs arbitrary unpickling is refused by default."""
    import pickle

    import torch

    ck = importlib.import_module("deepmd_kit_lr_pt_b200.checkpoint")
    sd = ck.params_to_state_dict(model)
    path = str(tmp_path / "odd.pt")
    torch.save({"model": sd, "extra": _Opaque()}, path)
    with pytest.raises(pickle.UnpicklingError):
        ck.load(path, sel=model.cfg.sel, rcut=model.cfg.rcut)
    p = ck.load(path, sel=model.cfg.sel, rcut=model.cfg.rcut, trusted=True)
    np.testing.assert_array_equal(p.dstd, model.dstd)


def test_reader_rejects_wrong_sel(dpb, model):
    ck = importlib.import_module("deepmd_kit_lr_pt_b200.checkpoint")
    sd = ck.params_to_state_dict(model)
    with pytest.raises(ValueError):
        ck.params_from_state_dict(sd, sel=(46, 90))
    with pytest.raises(ValueError):
        ck.params_from_state_dict({"x": 1}, sel=(46, 92))


def test_trainable_names_are_the_reference_parameters(dpb, layout, model):
    """Every trainable tensor of the training step (train.param_specs, the
    flat layout's order) is a reference state-dict entry of the same shape,
    and together they are all of the reference's network weights, so trained
    weights go back into the reference's checkpoint by name."""
    tr = importlib.import_module("deepmd_kit_lr_pt_b200.train")
    _, shapes, _ = layout
    specs = tr.param_specs(model)
    names = [n for n, _ in specs]
    assert len(names) == len(set(names))
    for n, a in specs:
        assert n in shapes, n
        assert tuple(a.shape) == shapes[n], (n, a.shape, shapes[n])
    nets = {k for k in shapes if ".networks." in k}
    assert set(names) == nets, sorted(nets ^ set(names))
