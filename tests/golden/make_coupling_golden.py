"""Generate the coupling-boundary fixtures in this folder with the reference MarDyn itself.

oracle/_ref/ref_driver (the reference sources compiled unmodified, see oracle/Makefile, target
`ref`, which includes the reference's coupling/boundary classes) reads a seeded FCC box in which
some molecules have been moved just outside the box faces, edges and corners (as the drift of a
step leaves them), bins the container and runs the reference's ReflectingBoundary::applyBoundary,
then the pair forces and ForceBoundary::applyBoundary (`--boundary` mode). Kept here per case
(coupling_<name>.npz): the input, the state after the reflection (r, v), the forces before and
after ForceBoundary, and samples of ForceBoundary::calcFm. tests/test_coupling.py (oracle) and
tests/test_gpu_coupling.py (device) check against them. Run from the repository root:

    make -C oracle ref REF=<the reference mardyn/ directory> && python tests/golden/make_coupling_golden.py
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


def displaced(seed, dim):
    """An 864-molecule FCC box (rho 0.8, T 1.0, rc 2.5) and new positions for 40 of its molecules,
    0.01-0.3 sigma outside the box in one, two or three dimensions (lower and upper faces)."""
    s = W.lj_fcc_box(6, 0.8, 1.0, seed, 2.5, [W.Component(1.0, 1.0, 1.0, True)], name=f"coupling_d{dim}")
    rng = np.random.default_rng(seed)
    L = s.length
    r = s.r.copy()
    picked = rng.choice(s.n, size=40, replace=False)
    for k, i in enumerate(picked):
        dims = rng.choice(3, size=1 + (k % 3), replace=False)
        for d in dims:
            out = rng.uniform(0.01, 0.3)
            r[i, d] = -out if rng.random() < 0.5 else L[d] + out
    return s, picked, r


def cases():
    # (system, dim, streamOutDir, streamOut)
    return [(displaced(31, 3), 3, 0, 1), (displaced(32, 2), 2, 1, 1)]


def main():
    if not os.path.exists(O.REF_DRIVER):
        raise SystemExit("build the reference harness first: make -C oracle ref REF=<the reference mardyn/ directory>")
    for (s, picked, r_moved), dim, sod, so in cases():
        tmp = tempfile.mkdtemp(prefix="mdcpl_")
        W.write_inp(s, os.path.join(tmp, "sys.inp"))
        W.write_cfg(s, os.path.join(tmp, "sys.cfg"), "sys.inp")
        with open(os.path.join(tmp, "moves.txt"), "w") as f:
            for i in picked:
                x, y, z = (float(c) for c in r_moved[i])
                f.write(f"{int(s.ids[i])} {x!r} {y!r} {z!r}\n")
        subprocess.run([O.REF_DRIVER, "--boundary", "sys.cfg", str(dim), str(sod), str(so), ".", "moves.txt"], cwd=tmp,
                       check=True, stdout=subprocess.DEVNULL)
        d1, d2, d3 = (O.read_ref_dump(os.path.join(tmp, f"step{k:06d}.bin")) for k in (1, 2, 3))
        fm = np.loadtxt(os.path.join(tmp, "calcfm.txt"))
        np.savez_compressed(os.path.join(OUT, f"{s.name}.npz"), in_id=s.ids, in_r=r_moved, in_v=s.v, length=s.length,
                            cutoff=s.cutoff, dim=dim, stream_out_dir=sod, stream_out=so,
                            refl_id=d1["id"], refl_r=d1["r"], refl_v=d1["v"],
                            f_id=d2["id"], f_before=d2["F"], f_after=d3["F"], calcfm=fm)
        shutil.rmtree(tmp)
        print("wrote", f"{s.name}.npz", "molecules", len(d1["id"]), "after the reflection")


if __name__ == "__main__":
    main()
