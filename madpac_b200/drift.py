"""Total-energy drift of a long NVE run, FP64 against the FP32-pair/FP64-accumulate form.

    python -m madpac_b200.drift [--steps 10000] [--skin 0.3] [--fcc-cells 64]

Runs the 1,048,576-molecule FCC box (rho 0.75, T 0.9, rc 3.0, dt 0.002, truncated-shifted LJ) for
`steps` Leapfrog steps in each precision from the same start and prints one JSON object: per form
the total energy per molecule (Upot + kinetic, from the per-step records of mdgpu_run) at the start,
every 1000 steps and at the end, its drift and linear slope, and the force error of the mixed form
against FP64 on the mixed run's final configuration.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import mdgpu as M
from . import workloads as W


def run(nsteps: int, skin: float, fcc_cells: int = 64, device: int = 0) -> dict:
    s = W.config_c2() if fcc_cells == 64 else W.lj_fcc_box(fcc_cells, 0.75, 0.9, 2, 3.0,
                                                          [W.Component(1.0, 1.0, 1.0, True)])
    res = {"n_molecules": int(s.n), "steps": nsteps, "dt": float(s.dt), "verlet_skin": skin}
    ends = {}
    for name, prec in (("fp64", M.FP64), ("mixed", M.MIXED)):
        lc = M.LinkedCells.from_system(s, prec, device)
        lc.update()
        u0, _, _ = lc.traversePairs()
        lc.setSkin(skin)
        k0 = 0.5 * float(np.sum(s.mass()[s.cid] * np.sum(lc.getParticles()["v"] ** 2, axis=1)))
        t0 = time.perf_counter()
        rec = lc.run(nsteps, s.dt)
        wall = time.perf_counter() - t0
        e = (rec[:, 0] + 0.5 * rec[:, 2]) / s.n
        e0 = (u0 + k0) / s.n
        res[name] = {"E0_per_molecule": e0, "E_end_per_molecule": float(e[-1]),
                     "drift_per_molecule": float(e[-1] - e0), "rel_drift": float((e[-1] - e0) / abs(e0)),
                     "max_abs_dev_per_molecule": float(np.max(np.abs(e - e0))),
                     "slope_per_molecule_per_1000_steps": float(np.polyfit(np.arange(nsteps), e, 1)[0] * 1000),
                     "T_end": float(rec[-1, 2] / (3 * s.n)), "wall_s": wall, "list_builds": lc.skinBuilds(),
                     "E_every_1000": [float(x) for x in e[999::1000]]}
        ends[name] = lc.getParticles()["r"]
        lc.close()
    a = M.LinkedCells.from_system(s, M.MIXED, device)
    b = M.LinkedCells.from_system(s, M.FP64, device)
    for x in (a, b):
        x.setState(r=ends["mixed"])
        x.update()
    ua, wa, _ = a.traversePairs()
    ub, wb, _ = b.traversePairs()
    fa, fb = a.getParticles()["F"], b.getParticles()["F"]
    rms = np.sqrt(np.mean(np.sum(fb * fb, axis=1)))
    err = np.linalg.norm(fa - fb, axis=1)
    res["mixed_force_error_at_end"] = {"rms": float(np.sqrt(np.mean(err ** 2)) / rms), "max": float(err.max() / rms),
                                       "upot_rel": abs(ua - ub) / abs(ub), "virial_rel": abs(wa - wb) / abs(wb)}
    a.close()
    b.close()
    return res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--skin", type=float, default=0.3)
    ap.add_argument("--fcc-cells", type=int, default=64)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(run(a.steps, a.skin, a.fcc_cells, a.device)))


if __name__ == "__main__":
    main()
