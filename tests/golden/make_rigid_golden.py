"""Generate the rigid multi-centre fixtures in this folder with the reference MarDyn itself.

oracle/_ref/ref_driver (the reference sources compiled unmodified, see oracle/Makefile, target
`ref`) runs 10 steps of three seeded systems of rigid LJ molecules and dumps, after prepare_start
and after step 10, every molecule's r, v, F and its orientation q, angular momentum D and torque M,
with the potential energy, virial, sum m v^2 and sum I w^2 of every step. Kept here as
rigid_<name>.npz (the start state is stored too, so the fixtures do not depend on the generator):

* rigid_2clj_256:  two-centre LJ (elongation 0.5, truncated-shifted), rho 0.3, T 2.0, rc 3.0;
* rigid_mix_256:   that molecule and a linear three-centre molecule with a different middle centre,
                   50/50, xi 0.9, eta 1.05, rho 0.15, T 2.0, rc 3.0;
* rigid_bent_256:  a bent three-centre molecule with three non-zero moments, plain LJ, rho 0.25,
                   T 1.5, rc 2.5;
* rigid_charged_256: the two-centre molecule with point charges +-0.5 at z = +-0.35 (massless),
                   rho 0.3, T 2.0, rc 3.0;
* rigid_charged_mix_256: three components (the charged molecule with +-0.8, the plain two-centre
                   molecule and the bent molecule), 40/30/30, rho 0.2, T 1.5, rc 3.0;
* rigid_dipolar_256: the two-centre molecule with a point dipole 1.2 along its axis, rho 0.3,
                   T 2.0, rc 3.0 (epsilon_RF 1e10);
* rigid_polar_mix_256: quadrupolar (Q 1.0), dipolar (0.9) and charged (+-0.6) two-centre molecules,
                   40/30/30, rho 0.25, T 1.8, rc 3.0, reaction field epsilon_RF 5 (every point-polarity
                   block of PotForce and MyRF);
* rigid_far_field.json: Domain::initFarFieldCorr's UpotCorr and VirialCorr (the LJ tails of
                   unshifted centre pairs at and off the centre of mass, the reaction field's self
                   term of charged and dipolar molecules) of two systems;
* rigid_2clj_4000_energy: the per-step Upot, virial, sum m v^2 and sum I w^2 of 1000 steps
                   (dt 0.001) of workloads.config_2clj(n_cells=10, temperature=1.5), 4,000
                   molecules, with a checksum of the generated start (the energy drift of the
                   reference's quaternion Leapfrog, which the device path must follow).

Run from the repository root:

    make -C oracle ref REF=<the reference mardyn/ directory> && python tests/golden/make_rigid_golden.py
"""
import os
import shutil
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from madpac_b200 import workloads as W  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
NSTEPS = 10


def systems():
    return [
        W.rigid_fcc_box(4, 0.3, 2.0, 11, 3.0, [W.two_centre()], name="rigid_2clj_256"),
        W.rigid_fcc_box(4, 0.15, 2.0, 12, 3.0, [W.two_centre(), W.three_centre_linear()], [0.5, 0.5],
                        np.array([[0.9, 1.05]]), name="rigid_mix_256"),
        W.rigid_fcc_box(4, 0.25, 1.5, 13, 2.5, [W.bent_three_centre()], name="rigid_bent_256"),
        W.rigid_fcc_box(4, 0.3, 2.0, 14, 3.0, [W.charged_two_centre()], name="rigid_charged_256"),
        W.rigid_fcc_box(4, 0.2, 1.5, 15, 3.0, [W.charged_two_centre(0.8), W.two_centre(), W.bent_three_centre()],
                        [0.4, 0.3, 0.3], np.array([[0.9, 1.05], [1.0, 1.0], [0.95, 0.98]]),
                        name="rigid_charged_mix_256"),
        W.rigid_fcc_box(4, 0.3, 2.0, 16, 3.0, [W.dipolar_two_centre(1.2)], name="rigid_dipolar_256"),
        polar_mix(),
    ]


def polar_mix():
    s = W.rigid_fcc_box(4, 0.25, 1.8, 17, 3.0, [W.quadrupolar_two_centre(1.0), W.dipolar_two_centre(0.9),
                                               W.charged_two_centre(0.6)], [0.4, 0.3, 0.3],
                        np.array([[0.95, 1.0], [1.0, 1.02], [0.98, 1.0]]), name="rigid_polar_mix_256")
    s.epsilon_rf = 5.0
    return s


def main():
    if not os.path.exists(O.REF_DRIVER):
        raise SystemExit("build the reference harness first: make -C oracle ref REF=<the reference mardyn/ directory>")
    for s in systems():
        out = O.run_reference(s, NSTEPS, (0, NSTEPS))
        d0, d1 = out["dumps"][0], out["dumps"][NSTEPS]
        sc = out["scalars"]
        np.savez_compressed(
            os.path.join(OUT, f"{s.name}.npz"),
            length=s.length, cutoff=s.cutoff, lj_cutoff=s.lj_cutoff, dt=s.dt, mix=s.mix, epsilon_rf=s.epsilon_rf,
            ids=s.ids, cid=s.cid, r=s.r, v=s.v, q=s.q, D=s.D,
            F0=d0["F"], M0=d0["M"],
            r1=d1["r"], v1=d1["v"], q1=d1["q"], D1=d1["D"], F1=d1["F"], M1=d1["M"],
            upot=np.array([x["upot"] for x in sc]), virial=np.array([x["virial"] for x in sc]),
            summv2=np.array([x["summv2"] for x in sc]), sum_iw2=np.array([x["sum_iw2"] for x in sc]))
        print("wrote", f"{s.name}.npz")
    import json
    import subprocess
    import tempfile

    ff = {}
    for s in far_field_systems():
        tmp = tempfile.mkdtemp(prefix="mdff_")
        W.write_inp(s, os.path.join(tmp, "sys.inp"))
        W.write_cfg(s, os.path.join(tmp, "sys.cfg"), "sys.inp")
        r = subprocess.run([O.REF_DRIVER, "--farfield", "sys.cfg"], cwd=tmp, check=True, capture_output=True, text=True)
        ff[s.name] = json.loads(r.stdout.strip().splitlines()[-1])
        shutil.rmtree(tmp)
    with open(os.path.join(OUT, "rigid_far_field.json"), "w") as f:
        json.dump(ff, f, indent=1)
    print("wrote rigid_far_field.json")
    s = energy_system()
    out = O.run_reference(s, 1000)
    sc = out["scalars"]
    np.savez_compressed(os.path.join(OUT, "rigid_2clj_4000_energy.npz"), checksum=start_checksum(s),
                        upot=np.array([x["upot"] for x in sc]), virial=np.array([x["virial"] for x in sc]),
                        summv2=np.array([x["summv2"] for x in sc]), sum_iw2=np.array([x["sum_iw2"] for x in sc]))
    print("wrote rigid_2clj_4000_energy.npz")


def far_field_systems():
    """Unshifted and shifted centres, charges and dipoles, off-centre sites (TICS and TISS terms)."""
    a = W.rigid_fcc_box(4, 0.25, 1.8, 18, 3.0, [W.quadrupolar_two_centre(1.0), W.dipolar_two_centre(0.9),
                                               W.charged_two_centre(0.6), W.bent_three_centre()],
                        [0.25] * 4, np.ones((6, 2)) * np.array([0.97, 1.01]), name="ff_polar_mix")
    a.epsilon_rf = 5.0
    for comp in a.components[:2]:
        for t in comp.sites:
            t.do_shift = False
    b = W.rigid_fcc_box(4, 0.3, 2.0, 19, 3.5, [W.three_centre_linear(), W.rigid_component(
        [W.Site(0.0, 0.0, 0.0, 1.0, 1.0, 1.0, False)], charges=[W.Charge(0.0, 0.0, 0.3, 0.0, 0.4),
                                                             W.Charge(0.0, 0.0, -0.3, 0.0, -0.4)])],
                        [0.5, 0.5], np.array([[0.9, 1.1]]), name="ff_centre_site")
    for t in b.components[0].sites:
        t.do_shift = False
    b.lj_cutoff = 3.0
    return [a, b]


def energy_system():
    s = W.config_2clj(n_cells=10, temperature=1.5)
    s.dt = 0.001
    return s


def start_checksum(s):
    return np.array([s.r.sum(), s.v.sum(), s.q.sum(), s.D.sum(), float(s.n)])


if __name__ == "__main__":
    main()
