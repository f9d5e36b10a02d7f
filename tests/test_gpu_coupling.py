"""The device's molecule-side coupling operations (madpac_b200/csrc/coupling.cu through the C ABI)
against the reference's own classes and the oracle:

* mdgpu_reflect_boundary against ReflectingBoundary::applyBoundary run by the compiled reference
  (tests/golden/coupling_*.npz): positions and velocities bit-exact, the streamed-out count equal;
* mdgpu_force_boundary against oracle/coupling.force_boundary (ForceBoundary's per-molecule force,
  its calcFm pinned bit-exact by the fixtures) on the device's own forces: bit-exact;
* the cell-wise thermostat against oracle/coupling.CellWiseThermostat over two intervals with the
  velocities changed between calls, in three and in two dimensions, directed and not: velocities
  within 1e-11 relative (the device sums in 64-bit fixed point, the oracle in doubles).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

import coupling as C

pytestmark = pytest.mark.gpu

CASES = ["coupling_d3", "coupling_d2"]
LJ = [W.Component(1.0, 1.0, 1.0, True)]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def wrapped(r, L):
    """Positions as the container reads them back: one periodic image into [0, L)."""
    return np.where(r < 0.0, r + L, np.where(r >= L, r - L, r))


def container(d, r, v, precision=M.FP64):
    lc = M.LinkedCells(d["length"], float(d["cutoff"]), LJ, precision=precision)
    lc.addParticles(d["in_id"], np.zeros(len(r), dtype=np.int32), r, v)
    return lc


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: a[o] for k, a in st.items()}


@pytest.mark.parametrize("name", CASES)
def test_reflection_matches_the_reference_bitwise(name):
    d = load(name)
    lc = container(d, d["in_r"], d["in_v"])
    nout = lc.reflectBoundary(int(d["dim"]), int(d["stream_out_dir"]), False, bool(d["stream_out"]))
    st = by_id(lc.getParticles())
    lc.close()
    np.testing.assert_array_equal(st["id"], d["refl_id"])
    np.testing.assert_array_equal(st["v"], d["refl_v"])
    np.testing.assert_array_equal(st["r"], wrapped(d["refl_r"], d["length"]))
    sod = int(d["stream_out_dir"])
    assert nout == int(np.sum(d["refl_r"][:, sod] > d["length"][sod])) > 0


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("damping", [1.0, 0.35])
def test_boundary_force_matches_the_oracle_bitwise(name, damping):
    d = load(name)
    lc = container(d, d["refl_r"], d["refl_v"])
    lc.update()
    lc.traversePairs()
    before = by_id(lc.getParticles())
    lc.forceBoundary(int(d["dim"]), 2.5, int(d["stream_out_dir"]), damping)
    after = by_id(lc.getParticles())
    lc.close()
    want = C.force_boundary(before["r"], before["F"], d["length"], int(d["dim"]), 2.5, int(d["stream_out_dir"]),
                            damping)
    np.testing.assert_array_equal(after["F"], want)
    assert np.max(np.abs(after["F"] - before["F"])) > 1.0
    # dimensions past dim keep their forces
    if int(d["dim"]) == 2:
        np.testing.assert_array_equal(after["F"][:, 2], before["F"][:, 2])


def test_coupling_operations_refuse_the_skin_mode_and_bad_arguments():
    d = load("coupling_d3")
    lc = container(d, d["refl_r"], d["refl_v"])
    with pytest.raises(M.MdgpuError):
        lc.reflectBoundary(4, 0)
    with pytest.raises(M.MdgpuError):
        lc.forceBoundary(3, -1.0, 0)
    with pytest.raises(M.MdgpuError):
        M.CellWiseThermostat(lc, [0, 0, 0], [5, 5, 5], 0.0, [2, 2, 2], 3, 1.0, 1.0, 2)
    with pytest.raises(M.MdgpuError):
        M.CellWiseThermostat(lc, [0, 0, 0], [5, 5, 1], 2.5, [2, 2, 2], 2, 1.0, 1.0, 2)
    lc.setSkin(0.3)
    with pytest.raises(M.MdgpuError):
        lc.reflectBoundary(3, 0)
    lc.close()


@pytest.mark.parametrize("dim,directed,gamma", [(3, (1, 0, 0), 1.0), (3, (0, 0, 0), 0.6), (2, (1, 1, 0), 0.8)])
def test_thermostat_matches_the_oracle(dim, directed, gamma):
    s = W.lj_fcc_box(8, 0.8, 1.4, 77 + dim, 2.5, LJ, name="thermostat")
    L = s.length
    rng = np.random.default_rng(5 + dim)
    v = s.v + np.array([0.5, -0.2, 0.1])
    lower, cell = np.array([0.7, 0.4, 0.9]), 2.1
    size = [int((L[k] - 1.0 - lower[k]) // cell) for k in range(3)]
    if dim == 2:
        size[2] = 1
    upper = lower + cell * np.array(size)
    interval = 3
    lc = M.LinkedCells.from_system(s)
    lc.setState(v=v)
    th = M.CellWiseThermostat(lc, lower, upper, cell, size, dim, 0.9, gamma, interval, directed)
    ref = C.CellWiseThermostat(lower, upper, cell, size, dim, 0.9, gamma, interval, directed)
    mass = np.ones(s.n)
    vr = v.copy()
    inside = np.array([ref.index(p) for p in s.r]) >= 0
    assert 0 < inside.sum() < s.n
    for it in range(1, 2 * interval + 1):
        th.applyThermostat(it)
        vr = ref.apply(s.r, vr, mass, it)
        got = lc.getParticles()["v"]
        scale = np.max(np.abs(vr))
        assert np.max(np.abs(got - vr)) <= 1e-11 * scale, it
        if it % interval == 0:
            assert not np.allclose(vr[inside], v[inside])
            np.testing.assert_array_equal(got[~inside], v[~inside])
        # new velocities between calls (the dynamics' part), the same on both sides
        kick = rng.normal(0.0, 0.05, size=v.shape)
        vr = vr + kick
        v = vr.copy()
        lc.setState(v=vr)
    th.close()
    lc.close()


def test_thermostat_reports_a_sum_out_of_range():
    """A cell whose velocity sum reaches the fixed-point range (2^23) fails the call instead of
    rescaling with a wrapped sum; the container stays usable."""
    s = W.lj_fcc_box(4, 0.8, 1.0, 9, 2.5, LJ, name="thermostat_range")
    lc = M.LinkedCells.from_system(s)
    v = s.v.copy()
    v[:, 0] = 1.0e6
    lc.setState(v=v)
    L = s.length
    th = M.CellWiseThermostat(lc, [0, 0, 0], L, L[0], [1, 1, 1], 3, 1.0, 1.0, 1, (1, 0, 0))
    with pytest.raises(M.MdgpuError, match="fixed-point"):
        th.applyThermostat(1)
    lc.setState(v=s.v)
    lc.update()
    lc.traversePairs()
    th.close()
    lc.close()
