"""Generate the checkpoint fixtures in this folder with the reference MarDyn itself.

oracle/_ref/ref_driver (the reference sources compiled unmodified, see oracle/Makefile, target
`ref`) runs a few steps of a seeded system and then writes the reference's own checkpoint
(Domain::writeCheckpoint) together with the exact FP64 state of that step. Kept here: the
checkpoint text (ck_<name>.txt) and the state and system parameters (ck_<name>.npz), from which
tests/test_phase_space.py checks the device-path writer and reader. Run from the repository root:

    make -C oracle ref REF=<the reference mardyn/ directory> && python tests/golden/make_checkpoint_golden.py
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from madpac_b200 import workloads as W  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
NSTEPS = 3


def systems():
    return [
        W.lj_fcc_box(5, 0.8, 1.0, 21, 2.5, [W.Component(1.0, 1.0, 1.0, True)], name="fcc500_shifted"),
        W.lj_fcc_box(5, 0.75, 1.2, 22, 2.5, W.two_species(), [0.5, 0.5], np.array([[0.95, 1.05]]),
                     name="two_species_500"),
    ]


def main():
    if not os.path.exists(O.REF_DRIVER):
        raise SystemExit("build the reference harness first: make -C oracle ref REF=<the reference mardyn/ directory>")
    for s in systems():
        tmp = tempfile.mkdtemp(prefix="mdck_")
        W.write_inp(s, os.path.join(tmp, "sys.inp"))
        W.write_cfg(s, os.path.join(tmp, "sys.cfg"), "sys.inp")
        subprocess.run([O.REF_DRIVER, "--checkpoint", "sys.cfg", str(NSTEPS), "ck.txt", "."], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        shutil.copy(os.path.join(tmp, "ck.txt"), os.path.join(OUT, f"ck_{s.name}.txt"))
        d = O.read_ref_dump(os.path.join(tmp, f"step{NSTEPS:06d}.bin"))
        np.savez_compressed(os.path.join(OUT, f"ck_{s.name}.npz"), id=d["id"], cid=d["cid"], r=d["r"], v=d["v"],
                            length=s.length, eps=s.eps(), sigma=s.sigma(), mass=s.mass(), do_shift=s.do_shift(),
                            mix=s.mix, cutoff=s.cutoff, lj_cutoff=s.lj_cutoff, temperature=s.temperature,
                            current_time=NSTEPS * s.dt)
        shutil.rmtree(tmp)
        print("wrote", f"ck_{s.name}.txt", f"ck_{s.name}.npz")


if __name__ == "__main__":
    main()
