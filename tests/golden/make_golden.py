"""Generate the golden fixtures in this folder by running the reference MarDyn itself.

The reference sources are compiled unmodified into oracle/_ref/ref_driver (see oracle/Makefile,
target `ref`), which runs Simulation::prepare_start + simulateStep on a seeded .cfg/.inp pair and
dumps every molecule's r, v, F and LinkedCells cell index. The systems are the seeded synthetic
ones of madpac_b200.workloads. Run from the repository root:

    make -C oracle ref REF=<the reference mardyn/ directory> && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from madpac_b200 import workloads as W  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def systems():
    """name -> (system, nsteps, dump steps)"""
    out = {}
    s = W.lj_fcc_box(6, 0.8, 1.0, 11, 2.5, [W.Component(1.0, 1.0, 1.0, False)], name="fcc864_unshifted")
    out[s.name] = (s, 20, (0, 1, 20))
    s = W.lj_fcc_box(8, 0.8, 1.0, 12, 2.5, W.two_species(), [0.5, 0.5], np.array([[0.95, 1.05]]),
                     name="two_species_2048")
    out[s.name] = (s, 10, (0, 10))
    s = W.lj_fcc_box(5, 0.7, 1.0, 13, 2.5, [W.Component(1.0, 1.0, 1.0, True)], nve=False, name="thermostat_500")
    s.temperature = 1.3
    out[s.name] = (s, 10, (0, 10))
    s = W.config_c3(seed=14, n_total=8000)
    s.name = "slab_8000"
    out[s.name] = (s, 5, (0, 5))
    # molecules 2e-3 from the lower faces (and so close to the upper ones through the lattice
    # period) move across the periodic boundaries within a few steps
    s = W.lj_fcc_box(6, 0.8, 1.2, 15, 2.5, [W.Component(1.0, 1.0, 1.0, True)], name="wrap_864")
    a = s.length[0] / 6
    s.r = np.mod(s.r - (a / 4.0 - 2e-3), s.length[None, :])
    s.v *= 3.0
    out[s.name] = (s, 10, (0, 1, 5, 10))
    return out


def main():
    if not os.path.exists(O.REF_DRIVER):
        raise SystemExit("build the reference harness first: make -C oracle ref REF=<the reference mardyn/ directory>")
    meta = {}
    for name, (s, nsteps, dumps) in systems().items():
        ref = O.run_reference(s, nsteps, dumps)
        arrays = {}
        arrays["length"] = s.length
        arrays["eps"], arrays["sigma"], arrays["mass"] = s.eps(), s.sigma(), s.mass()
        arrays["do_shift"] = s.do_shift()
        arrays["mix"] = s.mix
        arrays["in_id"], arrays["in_cid"], arrays["in_r"], arrays["in_v"] = s.ids, s.cid, s.r, s.v
        sc = ref["scalars"]
        arrays["upot"] = np.array([x["upot"] for x in sc])
        arrays["virial"] = np.array([x["virial"] for x in sc])
        arrays["summv2"] = np.array([x["summv2"] for x in sc])
        for k, d in ref["dumps"].items():
            for f in ("id", "r", "v", "F", "cell"):
                arrays[f"s{k}_{f}"] = d[f]
        np.savez_compressed(os.path.join(OUT, f"ref_{name}.npz"), **arrays)
        meta[name] = dict(n=s.n, nsteps=nsteps, dumps=list(dumps), cutoff=s.cutoff, lj_cutoff=s.lj_cutoff,
                          dt=s.dt, nve=s.nve, temperature=s.temperature)
        print(name, s.n, "molecules,", nsteps, "steps")
    with open(os.path.join(OUT, "ref_systems.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
