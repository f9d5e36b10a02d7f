"""Pruned lists of the Verlet-skin mode (mdgpu_set_list_prune).

The steps evaluate inner lists, the entries of each build list within rc + prune at the last prune,
re-pruned after every build and when the summed largest per-step drifts reach prune/2. A pair left
out is beyond rc until the next prune, so the evaluated pairs are exactly those of the per-step
traversal: identical pair counts every step, FP64 step records within 1e-10 (relative) and final
forces within 1e-10 of a fresh traversal, over runs long enough for several prunes between builds.
Covered: one and two species, mdgpu_run and mdgpu_step (the drift of the pre-kick kernel), a hot
box that prunes every few steps with a thin inner skin, a slab with sparse bricks over split runs,
the mixed form against FP64, a displaced state, and the argument checks.
"""
import numpy as np
import pytest

from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu

DT = 0.002


def box(n_cells=10, rho=0.75, T=0.9, rc=3.0, seed=7, two=False):
    if two:
        return W.lj_fcc_box(n_cells, 0.8, 1.0, seed, 2.5, W.two_species(), [0.5, 0.5], np.ones((1, 2)))
    return W.lj_fcc_box(n_cells, rho, T, seed, rc, [W.Component(1.0, 1.0, 1.0, True)])


def rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def run(system, precision, skin, prune, runs, use_step=False):
    lc = M.LinkedCells.from_system(system, precision)
    lc.update()
    lc.traversePairs()
    if skin:
        lc.setSkin(skin)
        lc.setListPrune(prune)
    out = []
    for k in runs:
        if use_step:
            out.append(np.stack([lc.step(DT) for _ in range(k)]))
        else:
            out.append(lc.run(k, DT))
    st = lc.getParticles()
    counts = (lc.skinBuilds(), lc.listPrunes()) if skin else (0, 0)
    lc.close()
    return np.concatenate(out), st, counts


def forces_at(system, r, precision=M.FP64):
    lc = M.LinkedCells.from_system(system, precision)
    lc.setState(r=r)
    lc.update()
    lc.traversePairs()
    F = lc.getParticles()["F"]
    lc.close()
    return F


def check_exact(system, r0, s0, r1, s1):
    assert np.all(rel(r1[:, :3], r0[:, :3]) <= 1e-10), np.max(rel(r1[:, :3], r0[:, :3]))
    np.testing.assert_array_equal(r1[:, 3], r0[:, 3])
    np.testing.assert_array_equal(s1["id"], s0["id"])
    np.testing.assert_allclose(s1["r"], s0["r"], rtol=0, atol=1e-10)
    F = forces_at(system, s1["r"])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    assert np.max(np.linalg.norm(s1["F"] - F, axis=1)) / rms <= 1e-10


@pytest.mark.parametrize("two", [False, True])
def test_prune_fp64_follows_exact_traversal(two):
    system = box(two=two)
    runs = [80]
    r0, s0, _ = run(system, M.FP64, 0.0, 0.0, runs)
    r1, s1, (builds, prunes) = run(system, M.FP64, 0.3, 0.1, runs)
    assert 1 <= builds < 80
    assert prunes > builds   # drift prunes between the builds
    check_exact(system, r0, s0, r1, s1)


def test_prune_step_path_and_hot_box():
    """mdgpu_step (drift in the pre-kick kernel) on a box at T = 4, pruned with a thin inner skin."""
    system = box(n_cells=8, T=4.0, seed=11)
    runs = [30]
    r0, s0, _ = run(system, M.FP64, 0.0, 0.0, runs, use_step=True)
    r1, s1, (builds, prunes) = run(system, M.FP64, 0.4, 0.05, runs, use_step=True)
    assert prunes >= 8, (builds, prunes)
    check_exact(system, r0, s0, r1, s1)
    # the same steps through mdgpu_run in two pieces
    r2, s2, (b2, p2) = run(system, M.FP64, 0.4, 0.05, [13, 17])
    assert p2 >= 8
    check_exact(system, r0, s0, r2, s2)


def test_prune_slab_split_runs_and_mixed():
    system = W.config_c3(seed=5, n_total=30000)
    runs = [25, 25]
    r0, s0, _ = run(system, M.FP64, 0.0, 0.0, runs)
    r1, s1, (builds, prunes) = run(system, M.FP64, 0.3, 0.1, runs)
    assert builds >= 2 and prunes > builds
    check_exact(system, r0, s0, r1, s1)
    # the mixed form, pruned and not, on the same steps
    r2, s2, _ = run(system, M.MIXED, 0.3, 0.1, runs)
    r3, s3, _ = run(system, M.MIXED, 0.3, 0.0, runs)
    F = s1["F"]
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    for s in (s2, s3):
        err = np.sqrt(np.mean(np.sum((s["F"] - F) ** 2, axis=1))) / rms
        assert err <= 1e-5, err
    np.testing.assert_array_equal(r2[:, 3], r3[:, 3])
    assert np.all(rel(r2[:, :2], r1[:, :2]) <= 1e-5)


def test_prune_is_deterministic():
    system = box(n_cells=8)
    a = run(system, M.MIXED, 0.3, 0.1, [40])
    b = run(system, M.MIXED, 0.3, 0.1, [40])
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1]["F"], b[1]["F"])
    assert a[2] == b[2]


def test_prune_after_displacement_and_off_above_skin():
    system = box(n_cells=8)
    lc = M.LinkedCells.from_system(system, M.FP64)
    lc.update()
    lc.traversePairs()
    lc.setSkin(0.3)
    lc.setListPrune(0.1)
    lc.run(5, DT)
    b0, p0 = lc.skinBuilds(), lc.listPrunes()
    assert p0 >= 1
    st = lc.getParticles()
    lc.setState(r=st["r"] + np.array([0.2, -0.1, 0.05]))
    lc.run(1, DT)
    assert lc.skinBuilds() == b0 + 1 and lc.listPrunes() == p0 + 1
    got = lc.getParticles()
    F = forces_at(system, got["r"])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    assert np.max(np.linalg.norm(got["F"] - F, axis=1)) / rms <= 1e-10
    # an inner skin at or above the skin leaves the lists unpruned
    lc.setListPrune(0.3)
    p1 = lc.listPrunes()
    lc.run(5, DT)
    assert lc.listPrunes() == p1
    with pytest.raises(M.MdgpuError):
        lc.setListPrune(-0.1)
    with pytest.raises(M.MdgpuError):
        lc.setListPrune(3.5)
    lc.close()
