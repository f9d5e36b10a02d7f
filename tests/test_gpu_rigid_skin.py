"""The Verlet-skin mode of the rigid path (mdgpu_rigid_set_skin): lists of molecule pairs within
rc + skin on cells of edge >= rc + skin, rebuilt when a molecule has moved more than skin/2, every
list entry tested with the reference's exact double cutoff.

Every pair within rc is evaluated as in the per-step sequence, in another order, so a skin run
follows the per-step run (mdgpu_rigid_run without the skin, itself pinned to the reference by
tests/test_gpu_rigid.py) to rounding: FP64 step records within 1e-10 and the same pair counts over
60 steps of a hot two-centre fluid with several rebuilds; the same with point charges, and with
dipoles, quadrupoles and a reaction field; lists that overflow fall back to the cell scan with the
same results; the mixed form within its 1e-5.
"""
import numpy as np
import pytest

from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu

SKIN = 0.3


def started(system, precision=M.FP64, skin=0.0, cap=0):
    lc = M.RigidLinkedCells.from_system(system, precision)
    lc.update()
    lc.traversePairs()
    if skin > 0.0:
        lc.setSkin(skin, cap)
    return lc


def compare(system, steps, precision=M.FP64, cap=0, tol=1e-10):
    a = started(system, precision)
    b = started(system, precision, SKIN, cap)
    ra = a.run(steps, system.dt)
    rb = b.run(steps, system.dt)
    builds = b.skinBuilds()
    sa, sb = a.getParticles(), b.getParticles()
    a.close()
    b.close()
    n = system.n
    for j in range(4):   # Upot, virial, sum m v^2, sum I w^2
        scale = np.maximum(np.abs(ra[:, j]), float(n))
        err = float(np.max(np.abs(rb[:, j] - ra[:, j]) / scale))
        assert err <= tol, (j, err)
    if precision == M.FP64:
        np.testing.assert_array_equal(rb[:, 4], ra[:, 4])
    else:
        assert np.max(np.abs(rb[:, 4] - ra[:, 4])) <= 2
    # positions come back wrapped into the box, in the caller's order
    L = np.asarray(system.length)
    assert np.all(sb["r"] >= 0.0) and np.all(sb["r"] < L)
    d = sb["r"] - sa["r"]
    d -= L * np.round(d / L)
    assert np.max(np.abs(d)) <= (1e-8 if precision == M.FP64 else 1e-4)
    # orientations, angular momenta and torques back in the caller's order (the skin mode keeps
    # them in the sorted order during the run)
    qtol = 1e-8 if precision == M.FP64 else 1e-4
    assert np.max(np.abs(sb["q"] - sa["q"])) <= qtol
    for key in ("D", "M", "v"):
        scale = max(float(np.max(np.abs(sa[key]))), 1.0)
        assert np.max(np.abs(sb[key] - sa[key])) <= (1e-7 if precision == M.FP64 else 1e-3) * scale, key
    return builds


def test_rigid_skin_two_centre_fluid_follows_the_per_step_run():
    s = W.config_2clj(n_cells=10)
    builds = compare(s, 60)
    assert builds >= 3   # the first build and rebuilds along the run


@pytest.mark.parametrize("polar", [False, True])
def test_rigid_skin_with_point_polarities(polar):
    if polar:
        comps = [W.charged_two_centre(0.7), W.dipolar_two_centre(1.0), W.quadrupolar_two_centre(0.8),
                 W.bent_three_centre()]
        s = W.rigid_fcc_box(8, 0.25, 1.5, 42, 3.0, comps, [0.25] * 4, np.ones((6, 2)))
        s.epsilon_rf = 3.0
    else:
        s = W.rigid_fcc_box(8, 0.25, 1.5, 41, 3.0, [W.charged_two_centre(0.7), W.bent_three_centre()], [0.6, 0.4],
                            np.array([[0.95, 1.0]]))
    assert compare(s, 30) >= 1


def test_rigid_skin_overflowing_lists_scan_the_cells():
    s = W.config_2clj(n_cells=8)
    assert compare(s, 40, cap=4) >= 2


def test_rigid_skin_mixed_form():
    s = W.config_2clj(n_cells=10)
    compare(s, 40, M.MIXED, tol=1e-5)


def test_rigid_skin_state_and_errors():
    s = W.config_2clj(n_cells=8)
    lc = started(s, M.FP64, SKIN)
    lc.run(10, s.dt)
    with pytest.raises(M.MdgpuError):
        lc.traversePairs()   # the cells are the skin grid's: update first
    lc.update()
    u, w, p = lc.traversePairs()
    ref = started(s)
    ref.run(10, s.dt)
    ref.update()
    u0, w0, p0 = ref.traversePairs()
    assert p == p0 and abs(u - u0) <= 1e-10 * abs(u0)
    with pytest.raises(M.MdgpuError):
        lc.setSkin(-0.1)
    with pytest.raises(M.MdgpuError):
        lc.setSkin(0.6 * s.cutoff)
    lc.setSkin(0.0)   # back to the per-step sequence
    lc.run(2, s.dt)
    lc.close()
    ref.close()
