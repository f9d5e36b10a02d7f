"""The molecule-side operations of MaDPaC's coupled step, restated in oracle/coupling.py, against
the compiled reference's own classes (tests/golden/coupling_*.npz, made by
tests/golden/make_coupling_golden.py with oracle/_ref/ref_driver --boundary):

* ReflectingBoundary::applyBoundary on boxes with molecules just outside faces, edges and corners:
  positions and velocities bit-exact, in three and in two dimensions, molecules beyond the
  stream-out face left where they are;
* ForceBoundary::calcFm bit-exact on 401 distances;
* ForceBoundary::applyBoundary leaves every force as it was in the reference (its region lists are
  filled in copies), recorded here so that the device's boundary force is understood as what the
  code computes per molecule, not what the reference applies.
CPU only."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN), "..", "oracle"))
import coupling as C  # noqa: E402

CASES = ["coupling_d3", "coupling_d2"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.mark.parametrize("name", CASES)
def test_reflection_matches_the_reference_bitwise(name):
    d = load(name)
    o = np.argsort(d["in_id"])
    r, v, nout = C.reflect(d["in_r"][o], d["in_v"][o], d["length"], int(d["dim"]), int(d["stream_out_dir"]),
                           False, bool(d["stream_out"]))
    np.testing.assert_array_equal(d["refl_id"], d["in_id"][o])
    np.testing.assert_array_equal(r, d["refl_r"])
    np.testing.assert_array_equal(v, d["refl_v"])
    # the molecules beyond the stream-out face stay outside (deleted later by deleteOuterParticles)
    L = d["length"]
    beyond = r[:, int(d["stream_out_dir"])] > L[int(d["stream_out_dir"])]
    assert nout == int(np.sum(beyond)) > 0


def test_wall_force_fit_matches_the_reference_bitwise():
    fm = load("coupling_d3")["calcfm"]
    for r, f in fm:
        assert C.calc_fm(r) == f
    # continuous at the ends of its pieces to the fit's accuracy, zero beyond 2.95
    assert C.calc_fm(2.95) == 0.0 and C.calc_fm(3.5) == 0.0


@pytest.mark.parametrize("name", CASES)
def test_reference_force_boundary_applies_no_force(name):
    d = load(name)
    np.testing.assert_array_equal(d["f_after"], d["f_before"])
    # while the force the code computes for its boundary molecules is not zero
    F = C.force_boundary(d["refl_r"], d["f_before"], d["length"], int(d["dim"]), 2.5, int(d["stream_out_dir"]), 1.0)
    assert np.max(np.abs(F - d["f_before"])) > 1.0


def test_cellwise_thermostat_restatement_hits_the_cell_temperatures():
    """After an adjusting call with gamma 1, every coupling cell's peculiar kinetic energy is
    1.5 T per molecule sample of the interval (the reference's target)."""
    rng = np.random.default_rng(3)
    n = 4000
    L = 12.0
    r = rng.uniform(0, L, size=(n, 3))
    v = rng.normal(0, 1.3, size=(n, 3)) + np.array([0.4, 0.0, 0.0])
    mass = np.ones(n)
    th = C.CellWiseThermostat([0, 0, 0], [L, L, L], 3.0, [4, 4, 4], 3, 0.9, 1.0, 2, [1, 0, 0])
    v1 = th.apply(r, v, mass, 1)
    assert np.array_equal(v1, v)          # iteration 1: velocities only sampled
    v2 = th.apply(r, v1, mass, 2)         # iteration 2: adjusted
    idx = np.array([th.index(p) for p in r])
    for k in range(64):
        m = idx == k
        vc = np.array([v[m, 0].mean(), 0.0, 0.0])   # the mean of both (equal) samples
        e = 0.5 * np.sum((v2[m] - vc) ** 2)
        target = 1.5 * (2 * m.sum()) / 2 * 0.9
        assert abs(e - target) <= 1e-9 * target
