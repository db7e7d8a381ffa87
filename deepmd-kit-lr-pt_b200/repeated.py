"""Repeated evaluation of one large frame, the way an MD engine drives the
path: coordinates move a little every step, the ghosts and an rcut + skin
neighbor list are remade every ``rebuild_every`` steps, and every step in
between reuses them (ghosts moved with their owners, the list re-formatted
against rcut). Periodic checks compare energy, force and virial with an
independent evaluator (normally the FP64 plain path with fresh lists).
"""

from __future__ import annotations

import time

import numpy as np
import torch


def repeated_evaluation(ev, coord0: np.ndarray, steps: int, rebuild_every: int = 10,
                        sigma: float = 0.002, seed: int = 0, check=None,
                        check_every: int = 100) -> dict:
    """Runs ``steps`` evaluations of ``ev`` (an SeAEvaluator made with
    ``skin > 0``) from ``coord0``, adding N(0, sigma^2) Angstrom to every
    coordinate before each step (step 0 included).

    ``check(coord) -> (E, F [nloc, 3], V [9])`` is called on the host copy of
    the coordinates every ``check_every`` steps (step 0 included) and its
    result compared with ``ev``'s. Returns timings (wall time of the loop
    including rebuilds and the coordinate updates, without the checks; device
    time of the replayed steps) and the error series."""
    dev = ev.dev
    nloc = ev.nloc
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    coord = torch.tensor(np.asarray(coord0, np.float64).reshape(-1, 3), device=dev)
    ev.coord.copy_(coord)
    ev.rebuild()
    ev.capture()
    torch.cuda.synchronize()
    step_events = []
    checks = []
    n_rebuild = 0
    t_check = 0.0
    t0 = time.perf_counter()
    for k in range(steps):
        coord.add_(torch.randn(coord.shape, generator=gen, device=dev, dtype=torch.float64),
                   alpha=sigma)
        ev.coord.copy_(coord)
        if k > 0 and k % rebuild_every == 0:
            ev.rebuild()
            n_rebuild += 1
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ev.replay()
        b.record()
        step_events.append((a, b))
        if check is not None and check_every > 0 and k % check_every == 0:
            torch.cuda.synchronize()
            tc = time.perf_counter()
            c_host = coord.cpu().numpy()
            e = float(ev.energy.item())
            f = ev.force.cpu().numpy()
            v = ev.virial.cpu().numpy()
            e0, f0, v0 = check(c_host)
            checks.append({"step": k,
                           "energy_err_ev_per_atom": abs(e - e0) / nloc,
                           "force_rmse_ev_per_a": float(np.sqrt(np.mean((f - f0) ** 2))),
                           "force_max_abs_err": float(np.abs(f - f0).max()),
                           "virial_max_abs_err": float(np.abs(v - v0).max())})
            torch.cuda.synchronize()
            t_check += time.perf_counter() - tc
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0 - t_check
    ev.check()
    dev_ms = [x.elapsed_time(y) for x, y in step_events]
    return {"steps": steps, "rebuilds": n_rebuild, "wall_s": wall,
            "step_device_ms_mean": float(np.mean(dev_ms)),
            "step_device_ms_max": float(np.max(dev_ms)),
            "checks": checks}
