#!/usr/bin/env python
"""se_e2_a energy/force/virial throughput on B200: microseconds per step per atom.

Workload: 12,288-atom water (4096 H2O in a 49.67 A box, 16^3 molecules on a
3.104 A grid with +-0.3 A jitter and random rigid rotations), seeded synthetic
data; model rcut 6.0 / rcut_smth 0.5, sel [46, 92], embedding [25, 50, 100],
axis 16, fitting [240, 240, 240], seeded random weights, statistics from the
frame, the FP64 quintic table (stride 0.01 / 0.1, 5x extrapolation).

One step = one full evaluation from coordinates: wrap, ghost copy, cell grid,
neighbor search + format + env matrix, compressed embedding + descriptor,
fitting net forward and backward, descriptor backward, force and virial.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:      the compressed FP32 path (FP64 coordinate differences and sums),
           replayed as a CUDA graph; device time per step with the L2 flushed
           between steps; e2e through SeAEvaluator.run_pinned() (pinned host
           buffers; H2D coordinates, the step and D2H energy/force/virial in
           one graph) in the timed region, compute() beside it. The FP64 plain path, per-stage times and errors are
           reported beside it.
reference: the reference's own CPU implementation (deepmd:: *_cpu functions
           compiled from the reference sources, FP64, OpenMP where the
           reference has it, the fitting net in FP64 torch on all host cores)
           on the same frame, every atom a center in every step; this arm
           does not load the project's GPU library.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "us/step/atom, se_e2_a water: mixed-precision vs FP64 plain on same B200"
UNIT = "us/step/atom"
N_SIDE = 16          # 16^3 molecules = 12,288 atoms
PARAM_SEED = 1
CPU_STEPS = 20      # steps of the CPU baseline leg (whole frame each)
L2_FLUSH_BYTES = 256 << 20


def _load():
    import importlib

    import __graft_entry__

    __graft_entry__.load_package()
    return (importlib.import_module("deepmd_kit_lr_pt_b200.model"),
            importlib.import_module("deepmd_kit_lr_pt_b200.workload"),
            importlib.import_module("deepmd_kit_lr_pt_b200.table"))


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- CPU reference --
def _workload_module():
    """The seeded input generator (numpy only) loaded on its own, without the
    package: the reference arm must not load this project's GPU library."""
    import importlib.util

    name = "dpb_workload_standalone"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "deepmd-kit-lr-pt_b200", "workload.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class CpuReference:
    """The reference CPU path (oracle/_ref: deepmd:: *_cpu compiled from the
    reference sources; the restatement where that library is absent), FP64:
    normalize_coord_cpu, copy_coord_cpu, build_nlist_cpu, prod_env_mat_a_cpu,
    tabulate_fusion_se_a_cpu per neighbor type, the descriptor and fitting
    net in FP64 torch on the host cores with autograd for dE/dD,
    tabulate_fusion_se_a_grad_cpu, prod_force_a_cpu and prod_virial_a_cpu."""

    def __init__(self, params, coord, atype, box):
        import torch

        from oracle import oracle

        self.lib = oracle.ref()
        self.kind = "reference"
        if self.lib is None:
            self.lib, self.kind = oracle.port(), "port"
        self.p, self.coord, self.atype, self.box = params, coord, atype, box
        self.threads = os.cpu_count() or 1
        torch.set_num_threads(self.threads)
        self.fit = []
        for f in params.fit:
            self.fit.append(([(torch.tensor(W), torch.tensor(b),
                               None if d is None else torch.tensor(d)) for W, b, d in f["layers"]],
                             (torch.tensor(f["out"][0]), torch.tensor(f["out"][1]))))

    def step(self):
        """One FP64 energy/force/virial evaluation of the whole frame (every
        atom a center); returns (wall seconds, energy)."""
        import torch

        p, lib, cfg = self.p, self.lib, self.p.cfg
        M = cfg.neuron[-1]
        t0 = time.perf_counter()
        cn = lib.normalize_coord(self.coord.reshape(-1), self.box).reshape(-1, 3)
        c, t, mapping = lib.copy_coord(cn, self.atype, cfg.rcut, self.box)
        nall = c.shape[0]
        S = self.atype.size
        ret, il, nn, rb, _ = lib.build_nlist(c, S, cfg.rcut, atype=t, mem_size=512)
        em, emd, rij, nlist = lib.prod_env_mat_a(c, t, il, nn, rb, p.davg, p.dstd, S,
                                                 cfg.rcut, cfg.rcut_smth, cfg.sec)
        nnei = cfg.nnei
        emv = em.reshape(S, nnei, 4)
        xyz = np.zeros((S, 4, M))
        blocks = []
        for ty in range(cfg.ntypes):
            a, b = int(cfg.sec[ty]), int(cfg.sec[ty + 1])
            e = np.ascontiguousarray(emv[:, a:b, :])
            ex = np.ascontiguousarray(e[:, :, 0])
            table, info = p.tables[ty]
            xyz += lib.tabulate(table, info, ex, e, M)
            blocks.append((a, b, e, ex, table, info))
        xt = torch.from_numpy(xyz / nnei).requires_grad_(True)
        D = (xt.transpose(1, 2) @ xt[:, :, :cfg.axis_neuron]).reshape(S, -1)
        E = torch.zeros((), dtype=torch.float64)
        for ty in range(cfg.ntypes):
            idx = torch.from_numpy(np.nonzero(self.atype == ty)[0])
            if idx.numel() == 0:
                continue
            layers, (Wo, bo) = self.fit[ty]
            h = D[idx]
            for W, b, d in layers:
                y = torch.tanh(torch.addmm(b, h, W))
                h = h + d * y if d is not None else y
            E = E + torch.addmm(bo, h, Wo).sum() + float(p.bias_atom_e[ty]) * idx.numel()
        (dxyz,) = torch.autograd.grad(E, xt)
        dy = np.ascontiguousarray(dxyz.numpy() / nnei)
        nd = np.zeros((S, nnei, 4))
        for a, b, e, ex, table, info in blocks:
            dx, de = lib.tabulate_grad(table, info, ex, e, dy, M)
            nd[:, a:b, :] = de
            nd[:, a:b, 0] += dx
        nd = nd.reshape(S, nnei * 4)
        fext = lib.prod_force_a(nd, emd, nlist, S, nall)[0]
        force = np.zeros((S, 3))
        np.add.at(force, mapping, fext)
        virial, _ = lib.prod_virial_a(nd, emd, rij, nlist, S, nall)
        del force, virial
        return time.perf_counter() - t0, float(E.detach())


# ------------------------------------------------------------ ranks (N > 1) --
# Frames are independent: each rank evaluates its own frame (seeded by its
# rank, same size), no data-path collective; the only cross-rank operations
# are the barriers around the timed region and the max of the step times.
def frame_seed(rank: int) -> int:
    """Seed of the water frame evaluated by `rank`."""
    return 100 + rank


def max_over_ranks(v: float, world: int, device) -> float:
    """The largest of every rank's `v` (all ranks call it in the same order)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_us_per_atom(ms_step: float, nloc: int, world: int) -> float:
    """Whole-job throughput: world frames of nloc atoms per step of ms_step."""
    return ms_step * 1e3 / (nloc * world)


def _setup_frame(mdl, wl, tab, rank: int, device):
    cfg = mdl.SeAConfig()
    coord, atype, box = wl.water_frame(N_SIDE, seed=frame_seed(rank))
    params = mdl.init_params(cfg, seed=PARAM_SEED)
    mdl.prepare(params, coord, atype, box, device=device)
    return cfg, params, coord, atype, box


# ------------------------------------------------- repeated evaluation (c4) --
def run_repeated(args) -> None:
    """A large frame evaluated many times with small moves, an rcut + skin
    list rebuilt every --rebuild-every steps, FP64 plain-path checks every
    --check-every steps. One GPU; prints its own JSON line."""
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    mdl, wl, tab = _load()
    rep = importlib.import_module("deepmd_kit_lr_pt_b200.repeated")
    coord, atype, box = wl.water_frame(args.n_side, seed=100)
    if args.model == "c2":
        # the compressed 3-species model of the batched workload (O, H, Cu;
        # statistics and tables from every 16th of its 512 frames); its Cu
        # net is not reached on water
        cfg = mdl.SeAConfig(sel=(46, 92, 60))
        params = mdl.init_params(cfg, seed=PARAM_SEED)
        mdl.prepare_frames(params, wl.batched_frames(512, seed=0)[::16], device=device)
    else:
        cfg = mdl.SeAConfig()
        params = mdl.init_params(cfg, seed=PARAM_SEED)
        mdl.prepare(params, coord, atype, box, device=device)
    nloc = atype.size
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed", device=device, skin=args.skin)
    tuned = None
    if not args.no_tune:
        # launch shapes timed on this frame's own step (the skin list built
        # from the starting coordinates); the loop below recaptures with them
        ev.coord.copy_(torch.as_tensor(np.asarray(coord, np.float64).reshape(-1, 3)))
        ev.rebuild()
        tuned = ev.tune()
    plain = mdl.SeAEvaluator(params, atype, box, mode="plain", device=device)
    clocks = ClockSampler(0)
    clocks.start()
    out = rep.repeated_evaluation(ev, coord, steps=args.steps, rebuild_every=args.rebuild_every,
                                  sigma=args.sigma, seed=7, check=plain.compute,
                                  check_every=args.check_every)
    clk = clocks.stop()
    us = out["wall_s"] * 1e6 / (args.steps * nloc)
    line = {"metric": "us/step/atom, se_e2_a water repeated evaluation, skin list "
                      "(compressed, mixed precision)",
            "value": us, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": 0,
            "ms_per_step": out["wall_s"] * 1e3 / args.steps, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"water {nloc} atoms ({nloc // 3} H2O, {box[0]:.2f} A box), "
                                   f"coordinates + N(0, {args.sigma}^2) A per step, list "
                                   f"rcut + {args.skin} A rebuilt every "
                                   f"{args.rebuild_every} steps",
                       "nloc": nloc, "sel": list(cfg.sel), "embedding": list(cfg.neuron),
                       "fitting": list(cfg.fitting),
                       "model": "3-species O/H/Cu model of the batched workload" if
                       args.model == "c2" else "2-species water model, statistics from the frame"},
            "rebuilds": out["rebuilds"],
            "autotune": None if tuned is None else
            {"knobs": tuned["knobs"], "tuned_ms": tuned["ms"],
             "default_shapes_ms": tuned["baseline_ms"]},
            "step_device_ms": {"mean": out["step_device_ms_mean"],
                               "max": out["step_device_ms_max"]},
            "clocks": clk,
            "checks_vs_fp64_plain": out["checks"]}
    print(json.dumps(line), flush=True)


# --------------------------------------------------- batched frames (c2) --
def run_batched(args) -> None:
    """Uneven frames (log-uniform 24..3000 atoms, half water at 1.0 g/cm^3, half
    FCC Cu with vacancies; 3-species model) in one graph per step over all
    frames; FP64 plain-path checks on a few frames. One GPU."""
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    mdl, wl, tab = _load()
    bt = importlib.import_module("deepmd_kit_lr_pt_b200.batch")
    frames = wl.batched_frames(args.frames, seed=0)
    cfg = mdl.SeAConfig(sel=(46, 92, 60))
    params = mdl.init_params(cfg, seed=PARAM_SEED)
    # statistics from a subset of the frames (every 16th)
    mdl.prepare_frames(params, frames[::16], device=device)
    ev = bt.BatchEvaluator(params, frames, device=device)
    ev.compute()
    ev.check()
    # tile shapes (atoms per CTA of the env / force and descriptor kernels,
    # fitting GEMM N tile) timed on this workload; leaves the step captured
    tuned = ev.tune(reps=5, use_cache=False) if not args.no_tune else None
    if tuned is None:
        ev.capture()
    N = ev.N
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    clocks = ClockSampler(0)
    clocks.start()
    t_end, nw = time.time() + 0.6, 0
    while nw < args.warmup or time.time() < t_end:
        ev.replay()
        nw += 1
        if nw % 16 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ev.replay()
        b.record()
        ts.append((a, b))
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = float(np.mean([a.elapsed_time(b) for a, b in ts]))
    ev.check()
    E, F, V = ev.compute()
    checks = []
    half = len(frames) // 2 - (len(frames) // 2) % 2
    for f in sorted({0, min(1, len(frames) - 1), half, min(half + 1, len(frames) - 1)}):
        coord, atype, box = frames[f]
        plain = mdl.SeAEvaluator(params, atype, box, mode="plain", device=device)
        e0, f0, v0 = plain.compute(coord)
        n = atype.size
        checks.append({"frame": f, "atoms": int(n), "species": "water" if f % 2 == 0 else "Cu",
                       "energy_err_ev_per_atom": abs(E[f] - e0) / n,
                       "force_rmse_ev_per_a": float(np.sqrt(np.mean(
                           (F[ev.frame_slice(f)] - f0) ** 2))),
                       "virial_max_abs_err": float(np.abs(V[f] - v0).max())})
        del plain
    # the same step as ONE persistent cooperative launch (dpb_bt_step_launch),
    # timed the same way, with its pass times
    one = None
    if not args.no_one_launch:
        del ev
        torch.cuda.synchronize()
        ev1 = bt.BatchEvaluator(params, frames, device=device, fused=True)
        E1, F1, V1 = ev1.compute()
        ev1.check()
        ev1.capture()
        for _ in range(max(3, args.warmup)):
            ev1.replay()
        ts1 = []
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            ev1.replay()
            b.record()
            ts1.append((a, b))
        torch.cuda.synchronize()
        ms1 = float(np.mean([a.elapsed_time(b) for a, b in ts1]))
        ev1.check()
        one = {"ms_per_step": ms1, "us_per_step_atom": ms1 * 1e3 / N, "launches_per_step": 1,
               "pass_us": ev1.pass_times_us(),
               "max_abs_diff_vs_staged": {"energy": float(np.abs(E1 - E).max()),
                                          "force": float(np.abs(F1 - F).max()),
                                          "virial": float(np.abs(V1 - V).max())}}
        del ev1
    line = {"metric": "us/step/atom, se_e2_a batched uneven frames (compressed, mixed "
                      "precision)",
            "value": ms * 1e3 / N, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(frames)} frames, {N} atoms (log-uniform 24..3000 "
                                   "atoms per frame; even frames water at 1.0 g/cm^3, odd "
                                   "frames FCC Cu a=3.615 A with vacancies)",
                       "sel": list(cfg.sel), "embedding": list(cfg.neuron),
                       "fitting": list(cfg.fitting), "graph": "one CUDA graph per step",
                       "l2": "256 MiB buffer written between timed steps"},
            "clocks": clk, "checks_vs_fp64_plain": checks, "one_launch": one,
            "autotune": None if tuned is None else {
                "knobs": tuned["knobs"], "tuned_ms": tuned["ms"],
                "default_shapes_ms": tuned["baseline_ms"], "trials": len(tuned["history"])}}
    print(json.dumps(line), flush=True)


def run_train(args) -> None:
    """Training step of the uncompressed model: 16 frames of 192-atom water,
    FP32, EnergyStdLoss (prefactors e 0.02, f 1000, v 0.02) with its gradient
    through the force (hand-written double backward) and an Adam update, one
    CUDA graph per step. The FP64 step and the oracle's FP64 torch-autograd
    step on the host cores are reported beside it. One GPU."""
    import torch

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    mdl, wl, tab = _load()
    tr = importlib.import_module("deepmd_kit_lr_pt_b200.train")
    cfg = mdl.SeAConfig()
    frames = [wl.water_frame(4, seed=100 + s) for s in range(args.frames)]
    params = mdl.init_params(cfg, seed=PARAM_SEED)
    params.davg, params.dstd, _ = mdl.env_stats_frames(params, frames[:1], device)
    prefs = (0.02, 1000.0, 0.02)
    lr = 1e-5

    def make(dtype):
        loss = tr.EnergyStdLoss(starter_learning_rate=lr, start_pref_e=prefs[0],
                                limit_pref_e=prefs[0], start_pref_f=prefs[1],
                                limit_pref_f=prefs[1], start_pref_v=prefs[2],
                                limit_pref_v=prefs[2])
        return tr.SeATrainer(params, frames, dtype=dtype, device=device, loss=loss)

    t32 = make(torch.float32)
    E, F, V = t32.compute()
    rng = np.random.default_rng(3)
    labels = (E + rng.normal(0, 1.0, E.shape), 0.5 * F, V + rng.normal(0, 1.0, V.shape))
    t32.set_labels(*labels)
    t64 = make(torch.float64)
    t64.set_labels(*labels)
    N = t32.ft.N
    # gradient accuracy of the FP32 step against the FP64 one (same weights)
    g = {}
    for name, t in (("f32", t32), ("f64", t64)):
        with torch.no_grad():
            E_, F_, V_ = t._forward()
            Eh, Fh, Vh = t.labels
            t._pref.copy_(torch.tensor(t.loss.prefactors(lr), dtype=torch.float64))
            _, gE, gF, gV = tr.loss_grads(E_, F_, V_, Eh, Fh, Vh, t._natoms_inv, t._pref)
            g[name] = t._backward(gE, gF, gV).double().clone()
    grad_rel = float(torch.linalg.norm(g["f32"] - g["f64"]) / torch.linalg.norm(g["f64"]))
    # launches of the product's kernels in one step (C-ABI calls; the batched
    # env call launches two kernels)
    calls = {"n": 0, "names": []}
    orig = tr.call

    def counting(name, *a):
        # the batched env call, the train bwd and rev calls launch two kernels
        two = ("dpb_batch_env_mat_a", "dpb_se_a_train_bwd", "dpb_se_a_train_rev")
        calls["n"] += 2 if name.startswith(two) else 1
        calls["names"].append(name)
        return orig(name, *a)

    tr.call = counting
    torch.cuda.nvtx.range_push("train_step")  # one eager step, for ncu --nvtx-include
    with torch.no_grad():
        t32._set_step_scalars(lr, 0.9, 0.999)
        t32._step_body(0.9, 0.999, 1e-8)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    tr.call = orig
    torch.cuda.synchronize()
    # stage times (eager, events on the launching stream)
    st = {"forward": [], "backward": [], "step": []}
    for _ in range(3 + args.warmup):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        with torch.no_grad():
            a.record()
            E_, F_, V_ = t32._forward()
            Eh, Fh, Vh = t32.labels
            _, gE, gF, gV = tr.loss_grads(E_, F_, V_, Eh, Fh, Vh, t32._natoms_inv, t32._pref)
            b.record()
            t32._backward(gE, gF, gV)
            c.record()
        st["forward"].append((a, b))
        st["backward"].append((b, c))
    torch.cuda.synchronize()
    stages = {k: float(np.median([x.elapsed_time(y) for x, y in v[args.warmup:]]))
              for k, v in st.items() if v}

    def timed(trainer, k, flush):
        trainer.capture()
        for _ in range(args.warmup):
            trainer.train_step(lr)
        torch.cuda.synchronize()
        ts = []
        for _ in range(k):
            flush.zero_()
            trainer._set_step_scalars(lr, 0.9, 0.999)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            trainer.graph.replay()
            b.record()
            ts.append((a, b))
        torch.cuda.synchronize()
        trainer.check()
        return float(np.mean([a.elapsed_time(b) for a, b in ts]))

    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    tuned = None
    if not args.no_tune:
        t32._set_step_scalars(lr, 0.9, 0.999)
        tuned = t32.tune(reps=5, use_cache=False)
    clocks = ClockSampler(0)
    clocks.start()
    ms = timed(t32, args.steps, flush)
    clk = clocks.stop()
    ms64 = timed(t64, max(3, args.steps // 4), flush)
    # end to end: host coordinates and labels in, loss out, every step
    pin = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64)).pin_memory()  # noqa: E731
    h_coord = pin(np.concatenate([c for c, _, _ in frames]).reshape(-1, 3))
    h_lab = [pin(x) for x in labels]
    h_loss = torch.empty(1, dtype=torch.float64).pin_memory()
    ts = []
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        t32._set_step_scalars(lr, 0.9, 0.999)  # 48 bytes: lr, bias corrections, prefactors
        t32.coord.copy_(h_coord, non_blocking=True)
        for dst, src in zip(t32.labels, h_lab):
            dst.copy_(src.view(dst.shape), non_blocking=True)
        t32.graph.replay()
        h_loss.copy_(t32._loss.double(), non_blocking=True)
        b.record()
        ts.append((a, b))
    torch.cuda.synchronize()
    e2e_ms = float(np.mean([a.elapsed_time(b) for a, b in ts]))
    h2d = h_coord.numel() * 8 + sum(x.numel() * 8 for x in h_lab) + 48
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import model_ref, oracle

        lib = oracle.ref() or oracle.port()
        torch.set_num_threads(os.cpu_count() or 1)
        sample = frames[:2]
        lab_s = (labels[0][:2], labels[1][:2 * frames[0][1].size], labels[2][:2])
        model_ref.train_loss_grads(lib, params, sample, lab_s, prefs)  # warm-up
        t0 = time.perf_counter()
        reps = 0
        while reps < 3 or time.perf_counter() - t0 < 10.0:
            model_ref.train_loss_grads(lib, params, sample, lab_s, prefs)
            reps += 1
        el = (time.perf_counter() - t0) / reps
        na = sum(a.size for _, a, _ in sample)
        cpu = {"value": el * 1e6 / na, "unit": UNIT, "cores": torch.get_num_threads(),
               "kind": "port",
               "sample": f"loss + gradient of 2 frames ({na} atoms) per step, FP64 torch autograd "
                         f"through the force on the host cores, geometry from "
                         f"{'the compiled reference library' if oracle.ref() else 'the restatement'}"
                         f", {reps} repetitions"}
    line = {"metric": "us/step/atom, se_e2_a training step (energy + force + virial loss, "
                      "double backward, Adam)",
            "value": ms * 1e3 / N, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(frames)} frames x 192 atoms water ({N} atoms), "
                                   "uncompressed se_e2_a [25, 50, 100] / fitting [240, 240, 240]"
                                   ", EnergyStdLoss prefactors (0.02, 1000, 0.02), Adam",
                       "graph": "one CUDA graph per step (forward, loss gradient, backward, "
                                "Adam)",
                       "l2": "256 MiB buffer written between timed steps"},
            "e2e": {"value": e2e_ms * 1e3 / N, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 8},
            "gpu_launches": calls["n"],
            "fp64_step": {"value": ms64 * 1e3 / N, "ms_per_step": ms64,
                          "speedup_of_f32": ms64 / ms},
            "grad_rel_err_f32_vs_f64": grad_rel,
            "stages_ms": stages, "clocks": clk, "cpu_baseline": cpu,
            "autotune": None if tuned is None else {
                "knobs": tuned["knobs"], "tuned_ms": tuned["ms"],
                "default_shapes_ms": tuned["baseline_ms"], "trials": len(tuned["history"])}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- arms -------
def run_reference(args, rank: int, world: int) -> None:
    """The reference's own CPU implementation of the path on this host's
    cores, on the same 12,288-atom frame and model: every atom a center in
    every step. Nothing of this project's GPU library is loaded: the inputs
    come from the numpy generator, the statistics from the reference library
    and the tables from the oracle's restatement of the reference compressor
    (pinned to the compressor's own output by the tests)."""
    if rank != 0:
        return
    wl = _workload_module()
    cfg = wl.SeAConfig()
    coord, atype, box = wl.water_frame(N_SIDE, seed=frame_seed(0))
    params = wl.init_params(cfg, seed=PARAM_SEED)
    from oracle import model_ref, oracle, table_ref

    lib = oracle.ref() or oracle.port()
    params.davg, params.dstd, mind = model_ref.env_stats(lib, cfg, coord, atype, box)
    params.tables = table_ref.build_tables(params.emb, params.davg, params.dstd, cfg.sel, mind,
                                           cfg.rcut_smth, cfg.rcut)
    ref = CpuReference(params, coord, atype, box)
    for _ in range(args.warmup):
        ref.step()
    ts = [ref.step()[0] for _ in range(args.steps)]
    ms = float(np.mean(ts)) * 1e3
    us = ms * 1e3 / atype.size
    line = {
        "impl": "reference", "metric": METRIC, "value": us, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"water {atype.size} atoms ({atype.size // 3} H2O, "
                               f"{box[0]:.2f} A box), se_e2_a compressed E/F/V, reference CPU path",
                   "nloc": int(atype.size), "sel": list(cfg.sel)},
        "cpu_baseline": {"value": us, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
                         "sample": f"the whole frame ({atype.size} centers) every step, "
                                   f"{args.steps} steps after {args.warmup} warm-up; deepmd:: "
                                   "CPU library compiled from the reference sources + FP64 "
                                   "torch fitting"},
        "e2e": {"value": us, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    import torch.distributed as dist

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    mdl, wl, tab = _load()
    cfg, params, coord, atype, box = _setup_frame(mdl, wl, tab, rank, device)
    nloc = atype.size
    ev = mdl.SeAEvaluator(params, atype, box, mode="compressed", device=device)
    ev.compute(coord)
    nall = ev.check()
    ev.capture()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed_steps(evl, k):
        ts = []
        for _ in range(k):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            evl.replay()
            b.record()
            ts.append((a, b))
        torch.cuda.synchronize()
        return [x.elapsed_time(y) for x, y in ts]


    # ---- device-resident timed region (CUDA graph replay, L2 flushed between).
    # The clock sampler (200 ms period) runs from the warm-up through the e2e
    # region; the warm-up lasts at least 0.6 s so the samples see the GPU
    # under this load.
    clocks = ClockSampler(local_rank)
    clocks.start()
    t_end, nw = time.time() + 0.6, 0
    while nw < args.warmup or time.time() < t_end:
        ev.replay()
        nw += 1
        if nw % 64 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.nvtx.range_push("dpb_graph_steps")
    ms = timed_steps(ev, args.steps)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier()
    ms_step = max_over_ranks(float(np.sum(ms)) / args.steps, world, device)
    value = whole_job_us_per_atom(ms_step, nloc, world)

    # ---- end to end through the public calls: pinned host in, pinned host out.
    # run_pinned(): the host-to-device copy of the coordinates, the step and
    # the device-to-host copy of energy / forces / virial as one graph;
    # compute(host_c): the same through separate copies (reported beside it)
    host_c = torch.tensor(coord, dtype=torch.float64).pin_memory()
    host_out = torch.empty(1 + 3 * nloc + 9, dtype=torch.float64).pin_memory()
    io_c, _ = ev.io_buffers()
    io_c.copy_(host_c)
    for _ in range(args.warmup):
        ev.compute(host_c, out=host_out)
        ev.run_pinned()
    barrier()
    e2e, e2e_compute = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_step = float(ev.run_pinned()[0][0])
        e2e.append(time.perf_counter() - t0)
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev.compute(host_c, out=host_out)
        e2e_compute.append(time.perf_counter() - t0)
    # the same step (up to the order of the FP32 atomic energy partials)
    assert abs(e_step - float(host_out[0])) <= 1e-8 * nloc, "run_pinned and compute disagree"
    e2e_ms = max_over_ranks(float(np.mean(e2e)) * 1e3, world, device)
    e2e_compute_ms = max_over_ranks(float(np.mean(e2e_compute)) * 1e3, world, device)
    clk = clocks.stop()
    ev.check()

    # ---- per-stage device times (eager step, same inputs) for the roofline
    stages = {}
    for _ in range(max(3, min(args.steps, 10))):
        flush.zero_()
        torch.cuda.nvtx.range_push("dpb_eager_step")
        ev.step(timers=stages)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    stage_ms = {k: float(np.mean([a.elapsed_time(b) for a, b in v[1:]])) for k, v in stages.items()}

    # kernel launches per step (CUPTI, one eager step)
    launches_per_step = None
    try:
        from torch.profiler import ProfilerActivity, profile

        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            ev.step()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events() if e.device_type.name == "CUDA"]
        launches_per_step = sum(1 for n in names if "dpb" in n)
    except Exception:  # profiler unavailable: count stays unknown
        launches_per_step = None

    # ---- FP64 plain path on the same frame, and the accuracy of both
    plain_line, acc = None, None
    if not args.no_plain:
        plain = mdl.SeAEvaluator(params, atype, box, mode="plain", device=device)
        Ep, Fp, Vp = plain.compute(coord)
        plain.check()
        plain.capture()
        for _ in range(2):
            plain.replay()
        kp = max(3, min(args.steps, 10))
        ms_plain = max_over_ranks(float(np.mean(timed_steps(plain, kp))), world, device)
        pst = {}
        for _ in range(3):
            plain.step(timers=pst)
        torch.cuda.synchronize()
        plain_stages = {k: float(np.mean([a.elapsed_time(b) for a, b in v[1:]]))
                        for k, v in pst.items()}
        Ec, Fc, Vc = ev.compute(coord)
        acc = {"vs": "FP64 plain GPU path (matches the reference PyTorch model to 1e-10 in tests)",
               "energy_err_ev_per_atom": abs(Ec - Ep) / nloc,
               "force_rmse_ev_per_a": float(np.sqrt(np.mean((Fc - Fp) ** 2))),
               "force_max_abs_err": float(np.abs(Fc - Fp).max()),
               "virial_max_abs_err": float(np.abs(Vc - Vp).max()),
               "energy": Ep, "force_rms": float(np.sqrt(np.mean(Fp ** 2)))}
        plain_line = {"ms_per_step": ms_plain, "value": ms_plain * 1e3 / nloc, "unit": UNIT,
                      "speedup_of_compressed": ms_plain / ms_step, "stages_ms": plain_stages,
                      "kernels": "hand-written FP64: geometry, env mat, embedding + descriptor "
                                 "(forward, backward), fitting GEMMs and layers, force/virial"}
        del plain

    # ---- roofline of the dominant kernel stage
    per_atom_bytes = {  # algorithmic HBM bytes per atom (FP32, nnei=138, M=100)
        "env_mat": 138 * 4 * 4 + 138 * 4,                     # em + nlist written
        "descriptor_fwd": 138 * 4 * 4 + 4 * 100 * 4 + 1600 * 4,  # em in; xyz, D out
        "descriptor_bwd": 1600 * 4 + 4 * 100 * 4 + 2 * 138 * 4 * 4,  # dD, xyz, em in; nd out
        "force_virial": 138 * 4 * 4 + 138 * 4 + 3 * 8,        # nd, nlist in; force out
    }
    ours = {k: v for k, v in stage_ms.items() if k in per_atom_bytes}
    dom = max(ours, key=ours.get)
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        with open(pk_path) as f:
            peaks = json.load(f)
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = per_atom_bytes[dom] * nloc / (ours[dom] * 1e-3) / 1e9
    # DRAM bytes per launch of the stage's kernel from the committed ncu capture
    # of this workload (profiles/ncu_dram_water12288.json)
    # (matched on the name before its template arguments, which follow the
    # tile shape the autotuner picked)
    kernel_of = {"env_mat": "dpb::k_env", "descriptor_fwd": "dpb::k_desc_fwd",
                 "descriptor_bwd": "dpb::k_desc_bwd", "force_virial": "dpb::k_force_virial_rc"}
    traffic = None
    dram_path = os.path.join(ROOT, "profiles", "ncu_dram_water12288.json")
    if nloc == 12288 and os.path.exists(dram_path):
        with open(dram_path) as f:
            kernels = json.load(f)["kernels"]
        kd = next((v for k, v in kernels.items() if k.split("<")[0] == kernel_of[dom]), None)
        if kd:
            traffic = kd["dram_read_bytes"] + kd["dram_write_bytes"]
    roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": traffic,
                "traffic_source": "profiles/ncu_dram_water12288.json" if traffic else None,
                "algorithmic_bytes_per_launch": per_atom_bytes[dom] * nloc,
                "algorithmic_bytes_per_atom": per_atom_bytes[dom],
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    # The descriptor kernels are bound by L1/TEX serving the gathers of table
    # rows (ncu: L1/TEX 76-85% busy, DRAM 6-7%), not by HBM: a second roof for
    # the dominant descriptor stage counts the algorithmic gather bytes (one
    # (degree + 1) x M FP32 coefficient row per evaluated slot: the real
    # neighbors plus one folded padding slot per type section) against the
    # nominal L1 data rate (128 B/clk/SM at the sampled SM clock).
    if dom.startswith("descriptor"):
        nl = ev.nlist.view(nloc, cfg.nnei).cpu().numpy()
        sec = cfg.sec
        slots = 0
        for t in range(cfg.ntypes):
            real = (nl[:, sec[t]:sec[t + 1]] >= 0).sum(1)
            slots += int(real.sum() + (real < (sec[t + 1] - sec[t])).sum())
        ncoef = ev.ptab.degree + 1
        gather = slots * ncoef * cfg.neuron[-1] * 4
        sm_mhz = None
        try:
            sm_mhz = float(subprocess.run(
                ["nvidia-smi", "--id=0", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits"],
                capture_output=True, text=True, timeout=10).stdout.strip().splitlines()[0])
        except (OSError, ValueError, IndexError, subprocess.TimeoutExpired):
            pass
        l1_peak = 128 * 148 * (sm_mhz or 1965.0) * 1e6 / 1e12
        roofline["l1_gather"] = {
            "bytes_per_launch": gather, "slots_evaluated": slots, "coefficients_per_channel": ncoef,
            "achieved_tbs": gather / (ours[dom] * 1e-3) / 1e12, "nominal_l1_tbs": l1_peak,
            "frac": gather / (ours[dom] * 1e-3) / 1e12 / l1_peak,
            "note": "table-row gathers through L1/TEX (ncu: L1 data-pipe wavefronts 73% of "
                    "peak and issue 62% in k_desc_bwd, L1/TEX 85% busy in k_desc_fwd, DRAM "
                    "6-7%); the HBM fraction above is low by construction"}
    # every stage against its own roof: HBM bytes for the memory stages, the
    # tensor pipe for the fitting GEMMs (split TF32: three or four TF32
    # products per FP32 multiply-add, the fit_terms knob; TF32 dense peak
    # taken as half the measured BF16 GEMM rate)
    fit = cfg.fitting
    din = cfg.neuron[-1] * cfg.axis_neuron
    mac_fit = 2 * (din * fit[0] + sum(fit[k] * fit[k + 1] for k in range(len(fit) - 1)))
    tf32_peak = float(peaks.get("bf16_tflops", 1590.0)) / 2
    stage_roofs = {}
    for k, v in stage_ms.items():
        if k in per_atom_bytes:
            gbs = per_atom_bytes[k] * nloc / (v * 1e-3) / 1e9
            stage_roofs[k] = {"bound": "hbm", "achieved_gbs": gbs, "frac": gbs / hbm_peak}
        elif k == "fitting":
            capi = importlib.import_module("deepmd_kit_lr_pt_b200._capi")
            terms = int(capi.lib().dpb_tune_get(b"fit_terms"))
            tf = terms * 2 * mac_fit * nloc / (v * 1e-3) / 1e12
            stage_roofs[k] = {"bound": "tensor", "achieved_tflops_tf32": tf, "tf32_terms": terms,
                              "peak_tflops_tf32": tf32_peak, "frac": tf / tf32_peak}

    # ---- CPU baseline: the reference CPU path on a bounded sample (rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = CpuReference(params, coord, atype, box)
        ref.step()
        ts = [ref.step()[0] for _ in range(CPU_STEPS)]
        us_cpu = float(np.mean(ts)) * 1e6 / nloc
        cpu = {"value": us_cpu, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
               "sample": f"the whole frame ({nloc} centers) every step, {CPU_STEPS} steps after "
                         "1 warm-up; FP64"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"water {nloc} atoms per GPU ({nloc // 3} H2O, "
                                   f"{box[0]:.2f} A box), se_e2_a compressed E/F/V",
                       "nloc": nloc, "nall": nall, "sel": list(cfg.sel),
                       "embedding": list(cfg.neuron), "fitting": list(cfg.fitting),
                       "precision": "FP32 table/contraction/fitting, FP64 coordinate "
                                    "differences and energy/force/virial sums",
                       "l2": "256 MiB buffer written between timed steps",
                       "graph": "one CUDA graph per step"},
            "e2e": {"value": whole_job_us_per_atom(e2e_ms, nloc, world), "unit": UNIT,
                    "h2d_bytes_per_step": nloc * 3 * 8,
                    "d2h_bytes_per_step": (1 + 3 * nloc + 9) * 8,
                    "call": "SeAEvaluator.run_pinned() (copies and step in one graph)",
                    "compute_call_value": whole_job_us_per_atom(e2e_compute_ms, nloc, world)},
            "gpu_launches": None if launches_per_step is None else launches_per_step * args.steps,
            "clocks": clk,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "plain_fp64": plain_line,
            "stages_ms": stage_ms,
            "stage_rooflines": stage_roofs,
            "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    del ev


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the tile-shape autotuner (batched and train workloads)")
    ap.add_argument("--no-one-launch", action="store_true",
                    help="batched workload: skip the one-launch form of the step")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the FP64 plain path (smaller device footprint for profiling)")
    ap.add_argument("--workload", choices=["step", "repeated", "batched", "train"],
                    default="step",
                    help="repeated: many evaluations of one large frame with a skin list; "
                         "batched: many uneven water / Cu frames per step; train: training "
                         "step with the force/virial loss on 16 water frames")
    ap.add_argument("--frames", type=int, default=None,
                    help="frame count (batched: 512, train: 16)")
    ap.add_argument("--n-side", type=int, default=48,
                    help="repeated workload: oxygen grid per box side (48: 331,776 atoms)")
    ap.add_argument("--model", choices=["water", "c2"], default="water",
                    help="repeated workload: the 2-species water model or the 3-species "
                         "model of the batched workload")
    ap.add_argument("--skin", type=float, default=2.0)
    ap.add_argument("--rebuild-every", type=int, default=10)
    ap.add_argument("--sigma", type=float, default=0.002)
    ap.add_argument("--check-every", type=int, default=100)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "repeated":
        if rank == 0:
            run_repeated(args)
        return
    if args.frames is None:
        args.frames = 16 if args.workload == "train" else 512
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "train":
        if rank == 0:
            run_train(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
