"""The rigid multi-centre oracle (oracle/rigid.py) against the reference's own numbers.

Fixtures (tests/golden/make_rigid_golden.py): the reference MarDyn run for 10 steps on five systems
of rigid molecules (two-centre LJ; a two-component mix with a three-centre molecule whose centres
differ; a bent molecule with three non-zero moments; a two-centre molecule with point charges; a
three-component mix with charged and uncharged molecules; a dipolar two-centre fluid; a mix of
quadrupolar, dipolar and charged molecules with a reaction field). The oracle restates PotForce's
LJ centre loop and its point-polarity blocks (charge, dipole, quadrupole pairs, direct torques,
MyRF), calcFM's torques and the quaternion Leapfrog, and must reproduce the forces, torques,
potential energy and virial of the start and the state after 10 steps to rounding.
"""
import os
import sys

import numpy as np
import pytest

from madpac_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import rigid as R  # noqa: E402

COMPONENTS = {
    "rigid_2clj_256": lambda: [W.two_centre()],
    "rigid_mix_256": lambda: [W.two_centre(), W.three_centre_linear()],
    "rigid_bent_256": lambda: [W.bent_three_centre()],
    "rigid_charged_256": lambda: [W.charged_two_centre()],
    "rigid_charged_mix_256": lambda: [W.charged_two_centre(0.8), W.two_centre(), W.bent_three_centre()],
    "rigid_dipolar_256": lambda: [W.dipolar_two_centre(1.2)],
    "rigid_polar_mix_256": lambda: [W.quadrupolar_two_centre(1.0), W.dipolar_two_centre(0.9), W.charged_two_centre(0.6)],
}
NAMES = sorted(COMPONENTS)


def golden_system(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    s = W.System(length=d["length"], components=COMPONENTS[name](), mix=d["mix"], ids=d["ids"], cid=d["cid"],
                 r=d["r"], v=d["v"], cutoff=float(d["cutoff"]), lj_cutoff=float(d["lj_cutoff"]), dt=float(d["dt"]),
                 q=d["q"], D=d["D"], name=name, epsilon_rf=float(d["epsilon_rf"]))
    return s, d


def energy_fixture():
    """The 4,000-molecule two-centre start of tests/golden/make_rigid_golden.py (regenerated from its
    seed, checked against the stored checksum) and the reference's 1000-step scalars."""
    d = np.load(os.path.join(GOLDEN, "rigid_2clj_4000_energy.npz"))
    s = W.config_2clj(n_cells=10, temperature=1.5)
    s.dt = 0.001
    got = np.array([s.r.sum(), s.v.sum(), s.q.sum(), s.D.sum(), float(s.n)])
    np.testing.assert_allclose(got, d["checksum"], rtol=1e-13, atol=1e-9)
    return s, d


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", NAMES)
def test_rigid_oracle_matches_reference(name):
    s, d = golden_system(name)
    out = R.run(s, 10, (0, 10))
    a, b = out["dumps"][0], out["dumps"][10]
    assert rel(a["F"], d["F0"]) < 1e-12 and rel(a["M"], d["M0"]) < 1e-12
    for key, ref in (("r", "r1"), ("q", "q1")):
        np.testing.assert_allclose(b[key], d[ref], rtol=0, atol=1e-12)
    for key, ref in (("v", "v1"), ("D", "D1"), ("F", "F1"), ("M", "M1")):
        assert rel(b[key], d[ref]) < 1e-12, key
    up = np.array([x["upot"] for x in out["scalars"]])
    vi = np.array([x["virial"] for x in out["scalars"]])
    np.testing.assert_allclose(up, d["upot"], rtol=1e-12)
    np.testing.assert_allclose(vi, d["virial"], rtol=1e-12)
    mv2 = np.array([x["summv2"] for x in out["scalars"][1:]])
    iw2 = np.array([x["sum_iw2"] for x in out["scalars"][1:]])
    np.testing.assert_allclose(mv2, d["summv2"][1:], rtol=1e-12)
    np.testing.assert_allclose(iw2, d["sum_iw2"][1:], rtol=1e-12)


def test_quaternion_rotations_are_inverse():
    rng = np.random.default_rng(1)
    q = rng.standard_normal((100, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    d = rng.standard_normal((100, 3))
    np.testing.assert_allclose(R.rotate(q, R.rotate_inv(q, d)), d, atol=1e-14)
    np.testing.assert_allclose(W.rotate_inv(q, d), R.rotate_inv(q, d), atol=0)


def test_rigid_phase_space_round_trip(tmp_path):
    s = W.rigid_fcc_box(3, 0.2, 1.0, 5, 2.5, [W.two_centre(), W.bent_three_centre(), W.dipolar_two_centre(),
                                              W.quadrupolar_two_centre(), W.charged_two_centre()],
                        [0.2] * 5, np.ones((10, 2)))
    s.epsilon_rf = 7.5
    path = str(tmp_path / "rigid.inp")
    W.write_inp(s, path)
    t = W.read_inp(path)
    assert [c.is_rigid for c in t.components] == [True] * 5 and t.epsilon_rf == 7.5
    for a, b in zip(s.components, t.components):
        np.testing.assert_array_equal(a.moments(), b.moments())
        assert a.mass == b.mass and len(a.lj_centres()) == len(b.lj_centres())
        assert a.point_charges() == b.point_charges() and a.point_dipoles() == b.point_dipoles()
        assert a.point_quadrupoles() == b.point_quadrupoles()
    for key in ("r", "v", "q", "D"):
        np.testing.assert_array_equal(getattr(t, key), getattr(s, key))
    # the rotational temperature of the start: sum I w^2 = rotDOF * T
    m = R.Model(s)
    w = R.rotate(s.q, s.D) * m.invI[s.cid]
    rot_dof = int(np.sum(m.I[s.cid] > 0))
    assert abs(float(np.sum(m.I[s.cid] * w * w)) - rot_dof * 1.0) < 1e-9


def test_energy_fixture_start_is_reproducible():
    s, d = energy_fixture()
    assert s.n == 4000 and d["upot"].shape == (1001,)


@pytest.mark.parametrize("name", ["rigid_charged_mix_256", "rigid_polar_mix_256"])
def test_both_sided_evaluation_equals_the_reference_order(name):
    """The device path evaluates every pair from both sides, each molecule taking PotForce's blocks
    with itself as mi (charge-dipole on one side, dipole-charge on the other, and so on) and keeping
    its own share; that gives the reference's forces, torques, Upot and virial."""
    s, d = golden_system(name)
    m = R.Model(s)
    one = R.forces(m, s.r, s.cid.astype(np.int64), s.q)
    two = R.forces(m, s.r, s.cid.astype(np.int64), s.q, both_sided=True)
    assert rel(two["F"], one["F"]) < 1e-12 and rel(two["M"], one["M"]) < 1e-12
    assert abs(two["upot"] - one["upot"]) <= 1e-12 * abs(one["upot"])
    assert abs(two["virial"] - one["virial"]) <= 1e-12 * abs(one["virial"])
    assert two["npairs"] == one["npairs"]
    assert rel(one["F"], d["F0"]) < 1e-12


def test_domain_temperature_and_betas_with_rotation():
    """Domain::calculateGlobalValues with rotational degrees of freedom (Domain.cpp:223-262):
    T = (sum m v^2 + sum I w^2) / (3N + rotDOF); beta_trans = (3N Ti / sum m v^2)^0.4,
    beta_rot = (rotDOF Ti / sum I w^2)^0.4 when thermostatted, 1 under NVE."""
    from madpac_b200 import mdgpu as M

    d = M.Domain(1.5, nve=False)
    d.n, d.rot_dof, d.summv2, d.sum_iw2 = 1000, 2000, 4200.0, 3100.0
    d.calculateGlobalValues()
    assert d.temperature == (4200.0 + 3100.0) / 5000.0
    assert d.beta_trans == (3000 * 1.5 / 4200.0) ** 0.4 and d.beta_rot == (2000 * 1.5 / 3100.0) ** 0.4
    nve = M.Domain(1.5, nve=True)
    nve.n, nve.rot_dof, nve.summv2, nve.sum_iw2 = 1000, 2000, 4200.0, 3100.0
    nve.calculateGlobalValues()
    assert nve.beta_trans == 1.0 and nve.beta_rot == 1.0
    # no rotational degrees of freedom: the single-centre formula
    single = M.Domain(1.0, nve=False)
    single.n, single.summv2 = 100, 310.0
    single.calculateGlobalValues()
    assert single.temperature == 310.0 / 300.0 and single.beta_rot == 1.0


def test_far_field_correction_matches_reference():
    """mdgpu_rigid_far_field_correction (host arithmetic of libmdgpu.so) gives the reference's
    Domain::initFarFieldCorr terms: the LJ tails of unshifted centre pairs at and off the centre of
    mass (TICC, TICS, TISS) and the reaction field's self term of charged and dipolar molecules."""
    import json

    from madpac_b200 import mdgpu as M

    sys.path.insert(0, GOLDEN)
    from make_rigid_golden import far_field_systems

    want = json.load(open(os.path.join(GOLDEN, "rigid_far_field.json")))
    for s in far_field_systems():
        u, w = M.rigid_far_field_correction(s)
        assert abs(u - want[s.name]["upot_corr"]) <= 1e-12 * abs(want[s.name]["upot_corr"]), s.name
        assert abs(w - want[s.name]["virial_corr"]) <= 1e-12 * abs(want[s.name]["virial_corr"]), s.name
    # two sites whose distances from the centre of mass add up to the cutoff: refused
    s = far_field_systems()[1]
    s.lj_cutoff = 1.0
    with pytest.raises(M.MdgpuError):
        M.rigid_far_field_correction(s)


def test_far_field_correction_reports_why_it_refuses():
    """The far-field entry point names the reason of each refusal: a too small LJ cutoff, a
    negative molecule count, a negative LJ cutoff."""
    import copy

    from madpac_b200 import mdgpu as M

    sys.path.insert(0, GOLDEN)
    from make_rigid_golden import far_field_systems

    s = far_field_systems()[1]
    s.lj_cutoff = 1.0
    with pytest.raises(M.MdgpuError) as e:
        M.rigid_far_field_correction(s)
    assert e.value.code == 1 and "cutoff too small" in str(e.value)
    s = copy.deepcopy(far_field_systems()[1])
    s.lj_cutoff = -1.0
    with pytest.raises(M.MdgpuError) as e:
        M.rigid_far_field_correction(s)
    assert e.value.code == 1 and "lj_cutoff" in str(e.value)
