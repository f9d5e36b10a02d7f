"""Rigid multi-centre LJ molecules on the device (mdgpu_rigid_*), against the reference and the oracle.

* The reference's own numbers (tests/golden/rigid_*.npz, made by the compiled reference): forces,
  torques, Upot and virial of the start, and the state after 10 NVE steps (r, v, q, D, F, M, and the
  per-step Upot, virial, sum m v^2, sum I w^2) for a two-centre fluid, a two-component mix with a
  three-centre molecule whose centres differ, a bent molecule with three non-zero moments, a
  two-centre molecule with point charges, a three-component mix with charged and uncharged
  molecules, a dipolar fluid, and a mix of quadrupolar, dipolar and charged molecules with a
  reaction field. FP64 agrees to rounding (1e-12 at the start, 1e-10 after 10 steps).
* Charged molecules, and a mix with dipoles, quadrupoles and a reaction field, on a larger box:
  FP64 against the oracle (1e-12), the mixed form within 1e-5.
* The oracle (oracle/rigid.py) on a larger box (more cells, the same code path at other sizes).
* Single-centre components through the rigid path give the single-centre container's forces.
* The step-by-step sequence equals mdgpu_rigid_run bit for bit; the mixed form stays within 1e-5 of
  FP64 forces and torques; over 1000 steps of a 4,000-molecule two-centre fluid the total energy
  (translational + rotational + potential) follows the reference's run step by step.
* Errors: traversal before update, two molecules at the same place, bad centre tables.
"""
import os
import sys

import numpy as np
import pytest

from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, HERE)

import rigid as R  # noqa: E402
from test_rigid_oracle import NAMES, golden_system  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def start(system, precision=M.FP64):
    lc = M.RigidLinkedCells.from_system(system, precision)
    lc.update()
    u, w, p = lc.traversePairs()
    return lc, u, w, p


@pytest.mark.parametrize("name", NAMES)
def test_rigid_start_matches_reference(name):
    s, d = golden_system(name)
    lc, u, w, p = start(s)
    st = lc.getParticles()
    np.testing.assert_array_equal(st["id"], s.ids)
    assert rel(st["F"], d["F0"]) < 1e-12
    assert rel(st["M"], d["M0"]) < 1e-12
    assert abs(u - d["upot"][0]) <= 1e-12 * abs(d["upot"][0])
    assert abs(w - d["virial"][0]) <= 1e-12 * abs(d["virial"][0])
    f = R.forces(R.Model(s), s.r, s.cid.astype(np.int64), s.q)
    assert p == f["npairs"]
    lc.close()


@pytest.mark.parametrize("name", NAMES)
def test_rigid_run_matches_reference(name):
    s, d = golden_system(name)
    lc, *_ = start(s)
    rec = lc.run(10, s.dt)
    st = lc.getParticles()
    np.testing.assert_allclose(st["r"], d["r1"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(st["q"], d["q1"], rtol=0, atol=1e-11)
    for key in ("v", "D", "F", "M"):
        assert rel(st[key], d[key + "1"]) < 1e-10, key
    np.testing.assert_allclose(rec[:, 0], d["upot"][1:], rtol=1e-10)
    np.testing.assert_allclose(rec[:, 1], d["virial"][1:], rtol=1e-10)
    np.testing.assert_allclose(rec[:, 2], d["summv2"][1:], rtol=1e-10)
    np.testing.assert_allclose(rec[:, 3], d["sum_iw2"][1:], rtol=1e-10)
    lc.close()


def test_rigid_larger_box_matches_oracle():
    s = W.rigid_fcc_box(8, 0.2, 1.5, 21, 2.5, [W.bent_three_centre(), W.two_centre(0.6, 0.9, 1.1, 1.2, True)],
                        [0.5, 0.5], np.array([[0.95, 1.02]]))
    lc, u, w, p = start(s)
    f = R.forces(R.Model(s), s.r, s.cid.astype(np.int64), s.q)
    st = lc.getParticles()
    assert rel(st["F"], f["F"]) < 1e-12 and rel(st["M"], f["M"]) < 1e-12
    assert abs(u - f["upot"]) <= 1e-12 * abs(f["upot"]) and abs(w - f["virial"]) <= 1e-12 * abs(f["virial"])
    assert p == f["npairs"]
    lc.close()


def test_single_centre_components_match_single_centre_container():
    s = W.lj_fcc_box(6, 0.8, 1.0, 31, 2.5, W.two_species(), [0.5, 0.5], np.array([[0.95, 1.05]]))
    lc, u, w, p = start(s)
    ref = M.LinkedCells.from_system(s, M.FP64)
    ref.update()
    u0, w0, p0 = ref.traversePairs()
    F0 = ref.getParticles()["F"]
    st = lc.getParticles()
    assert rel(st["F"], F0) < 1e-12
    np.testing.assert_array_equal(st["M"], 0.0)
    assert abs(u - u0) <= 1e-12 * abs(u0) and abs(w - w0) <= 1e-12 * abs(w0) and p == p0
    lc.close()
    ref.close()


def test_rigid_stepwise_equals_run():
    s, _ = golden_system("rigid_mix_256")
    a, *_ = start(s)
    b, *_ = start(s)
    rec = a.run(5, s.dt)
    for k in range(5):
        b.eventNewTimestep(s.dt)
        b.update()
        u, w, p = b.traversePairs()
        mv2, iw2 = b.eventForcesCalculated(s.dt)
        assert (u, w, mv2, iw2, p) == tuple(rec[k])
    sa, sb = a.getParticles(), b.getParticles()
    for key in ("r", "v", "q", "D", "F", "M"):
        np.testing.assert_array_equal(sa[key], sb[key])
    a.close()
    b.close()


def test_rigid_mixed_accuracy():
    s = W.config_2clj(n_cells=10)
    a, ua, wa, _ = start(s, M.FP64)
    b, ub, wb, _ = start(s, M.MIXED)
    fa, fb = a.getParticles(), b.getParticles()
    for key in ("F", "M"):
        rms = np.sqrt(np.mean(np.sum(fa[key] ** 2, axis=1)))
        err = np.sqrt(np.mean(np.sum((fb[key] - fa[key]) ** 2, axis=1))) / rms
        assert err <= 1e-5, (key, err)
    assert abs(ub - ua) <= 1e-5 * abs(ua) and abs(wb - wa) <= 1e-5 * abs(wa)
    a.close()
    b.close()


@pytest.mark.parametrize("polar", [False, True])
def test_rigid_charged_mixed_accuracy(polar):
    if polar:
        comps = [W.charged_two_centre(0.7), W.dipolar_two_centre(1.0), W.quadrupolar_two_centre(0.8),
                 W.bent_three_centre()]
        s = W.rigid_fcc_box(8, 0.25, 1.5, 42, 3.0, comps, [0.25] * 4, np.ones((6, 2)))
        s.epsilon_rf = 3.0
    else:
        s = W.rigid_fcc_box(8, 0.25, 1.5, 41, 3.0, [W.charged_two_centre(0.7), W.bent_three_centre()], [0.6, 0.4],
                            np.array([[0.95, 1.0]]))
    a, ua, wa, _ = start(s, M.FP64)
    b, ub, wb, _ = start(s, M.MIXED)
    f = R.forces(R.Model(s), s.r, s.cid.astype(np.int64), s.q)
    fa, fb = a.getParticles(), b.getParticles()
    assert rel(fa["F"], f["F"]) < 1e-12 and rel(fa["M"], f["M"]) < 1e-12
    assert abs(ua - f["upot"]) <= 1e-12 * abs(f["upot"]) and abs(wa - f["virial"]) <= 1e-12 * abs(f["virial"])
    for key in ("F", "M"):
        rms = np.sqrt(np.mean(np.sum(fa[key] ** 2, axis=1)))
        err = np.sqrt(np.mean(np.sum((fb[key] - fa[key]) ** 2, axis=1))) / rms
        assert err <= 1e-5, (key, err)
    assert abs(ub - ua) <= 1e-5 * abs(ua) and abs(wb - wa) <= 1e-5 * abs(wa)
    a.close()
    b.close()


def test_rigid_energy_follows_reference():
    """1000 NVE steps of a 4,000-molecule two-centre fluid: the total energy (translational +
    rotational kinetic + potential) of every step agrees with the reference's run of the same start,
    so its drift (about 7e-3 per molecule here: truncated-shifted forces and the quaternion
    Leapfrog) is the reference's own."""
    from test_rigid_oracle import energy_fixture

    s, d = energy_fixture()
    lc, u0, w0, _ = start(s)
    assert abs(u0 - d["upot"][0]) <= 1e-12 * abs(d["upot"][0])
    rec = lc.run(1000, s.dt)
    E = rec[:, 0] + 0.5 * (rec[:, 2] + rec[:, 3])
    Er = d["upot"][1:] + 0.5 * (d["summv2"][1:] + d["sum_iw2"][1:])
    assert np.all(np.isfinite(E))
    assert np.max(np.abs(E - Er)) / s.n < 1e-9, np.max(np.abs(E - Er)) / s.n
    np.testing.assert_allclose(rec[:, 1], d["virial"][1:], rtol=1e-6)
    lc.close()


def test_rigid_errors():
    s, _ = golden_system("rigid_2clj_256")
    lc = M.RigidLinkedCells.from_system(s)
    with pytest.raises(M.MdgpuError) as ei:
        lc.traversePairs()
    assert ei.value.code == 3
    r = s.r.copy()
    r[1] = r[0]
    lc.addParticles(s.ids, s.cid, r, s.v, s.q, s.D)
    lc.update()
    with pytest.raises(M.MdgpuError) as ei:
        lc.traversePairs()
    assert ei.value.code == 7
    lc.close()
    many = W.rigid_component([W.Site(0.1 * k, 0.0, 0.0, 0.1, 1.0, 1.0) for k in range(7)])
    with pytest.raises(M.MdgpuError) as ei:
        M.RigidLinkedCells(s.length, 3.0, [many])
    assert ei.value.code == 1
