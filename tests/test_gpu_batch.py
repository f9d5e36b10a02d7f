"""Batched ensemble (mdgpu_batch_*): many independent boxes advanced by one persistent kernel per
step from a captured CUDA graph.

* Against single-box contexts running the same steps: with the same tile shape (list depth 64) the
  per-brick arithmetic and the (cell, id) order are the same, so positions, velocities and forces are
  bit-identical; per-box Upot, virial and sum m v^2 agree to 1e-12 (the box sums run in another
  order); pair counts are exact. With a Verlet skin the two build their lists at different steps
  (same pairs within rc, different entries near rc + skin), so the comparison is to rounding level.
* Against the oracle (the reference's algorithm on the CPU): FP64 step records within 1e-9 along a
  short trajectory and forces within 1e-8, as for the single-box trajectory parity.
* Every tile shape gives the same trajectory (FP64, 1e-12); the autotuner leaves the state as it
  found it; a grid-barrier wait that runs out returns MDGPU_ERR_TIMEOUT and the batch recovers.
"""
import numpy as np
import pytest

import oracle as O
from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu

DT = 0.002


def ensemble(seed=11, sizes=(256, 700, 1500, 333, 2048, 4000), shifted=True):
    rng = np.random.default_rng(seed)
    out = []
    for k, n in enumerate(sizes):
        rho = float(rng.uniform(0.6, 0.9))
        T = float(rng.uniform(0.7, 1.5))
        ncell = int(np.ceil((n / 4.0) ** (1.0 / 3.0)))
        out.append(W.lj_fcc_box(ncell, rho, T, int(rng.integers(1 << 31)), 2.5,
                                [W.Component(1.0, 1.0, 1.0, shifted)], n_atoms=n, name=f"box{k}"))
    return out


def two_species_ensemble(seed=12, sizes=(500, 1200, 2600)):
    rng = np.random.default_rng(seed)
    out = []
    for k, n in enumerate(sizes):
        ncell = int(np.ceil((n / 4.0) ** (1.0 / 3.0)))
        out.append(W.lj_fcc_box(ncell, float(rng.uniform(0.6, 0.85)), 1.0, int(rng.integers(1 << 31)), 2.5,
                                W.two_species(), [0.5, 0.5], np.ones((1, 2)), n_atoms=n, name=f"ab{k}"))
    return out


def unordered_pairs(r, length, rc):
    from scipy.spatial import cKDTree

    tree = cKDTree(np.mod(r, length), boxsize=length)
    return (tree.count_neighbors(tree, rc) - len(r)) / 2.0


def rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def single_box_run(system, precision, nsteps, skin=0.0):
    lc = M.LinkedCells.from_system(system, precision)
    lc.update()
    u, w, p = lc.traversePairs()
    lc.setSkin(skin)
    recs = lc.run(nsteps, DT)
    st = lc.getParticles()
    lc.close()
    return np.array([u, w, p]), recs, st


@pytest.mark.parametrize("skin", [0.0, 0.3])
@pytest.mark.parametrize("precision", [M.FP64, M.MIXED])
@pytest.mark.parametrize("make", [ensemble, two_species_ensemble])
def test_batch_matches_single_box_bitwise(precision, make, skin):
    systems = make()
    nsteps = 12 if skin == 0.0 else 40
    b = M.Batch.from_systems(systems, precision)
    b.setTiles(64, 2, 1)
    b.setSkin(skin)
    prep = b.prepare()
    recs = b.run(nsteps, DT)
    st = b.getParticles()
    if skin > 0.0:
        assert len(systems) <= b.skinBuilds() < len(systems) * (nsteps + 1)
    for k, s in enumerate(systems):
        p0, r1, s1 = single_box_run(s, precision, nsteps, skin)
        bk = b.box(st, k)
        np.testing.assert_array_equal(bk["id"], s1["id"])
        fp64 = precision == M.FP64
        assert np.all(rel(prep[k, :2], p0[:2]) <= (1e-12 if skin == 0.0 or fp64 else 1e-6))
        assert prep[k, 3] == p0[2]
        if skin == 0.0:
            np.testing.assert_array_equal(bk["r"], s1["r"])
            np.testing.assert_array_equal(bk["v"], s1["v"])
            np.testing.assert_array_equal(bk["F"], s1["F"])
            for step in range(nsteps):
                assert np.all(rel(recs[step, k, :3], r1[step, :3]) <= 1e-12), (k, step, recs[step, k], r1[step])
                assert recs[step, k, 3] == r1[step, 3]
            continue
        # Verlet skin: the batch builds its lists in prepare(), a single-box context at the first
        # step of run(); the lists hold the same pairs within rc but differ near rc + skin, which
        # moves entries between the partial accumulators (rounding-level differences only)
        np.testing.assert_allclose(bk["r"], s1["r"], rtol=0, atol=1e-12 if fp64 else 1e-7)
        np.testing.assert_allclose(bk["v"], s1["v"], rtol=0, atol=1e-12 if fp64 else 1e-6)
        frms = np.sqrt(np.mean(np.sum(s1["F"] ** 2, axis=1)))
        assert np.max(np.abs(bk["F"] - s1["F"])) / frms <= (1e-12 if fp64 else 1e-5)
        for step in range(nsteps):
            assert np.all(rel(recs[step, k, :3], r1[step, :3]) <= (1e-12 if fp64 else 1e-6)), (k, step)
            assert abs(recs[step, k, 3] - r1[step, 3]) <= (0 if fp64 else 2)
    b.close()


@pytest.mark.parametrize("skin", [0.0, 0.3])
def test_batch_fp64_matches_oracle(skin):
    systems = ensemble(seed=21, sizes=(256, 900, 1700))
    nsteps = 8
    b = M.Batch.from_systems(systems, M.FP64)
    b.setSkin(skin)
    prep = b.prepare()
    recs = b.run(nsteps, DT)
    st = b.getParticles()
    for k, s in enumerate(systems):
        ref = O.run_oracle(s, nsteps, dump_steps=(nsteps,))
        sc = ref["scalars"]
        assert rel(prep[k, 0], sc[0]["upot_exact"]) <= 1e-12
        assert rel(prep[k, 1], sc[0]["virial_exact"]) <= 1e-12
        # the oracle counts processPair calls (halo pairs too); ours are unordered pairs within rc
        assert prep[k, 3] == unordered_pairs(s.r, s.length, s.cutoff)
        for step in range(1, nsteps + 1):
            assert rel(recs[step - 1, k, 0], sc[step]["upot"]) <= 1e-9
            assert rel(recs[step - 1, k, 1], sc[step]["virial"]) <= 1e-9
            assert rel(recs[step - 1, k, 2], sc[step]["summv2"]) <= 1e-9
        d = ref["dumps"][nsteps]
        bk = b.box(st, k)
        o = np.argsort(bk["id"])
        np.testing.assert_array_equal(bk["id"][o], d["id"])
        np.testing.assert_allclose(bk["r"][o], d["r"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(bk["v"][o], d["v"], rtol=0, atol=1e-8)
        rms = max(np.sqrt(np.mean(np.sum(d["F"] ** 2, axis=1))), 1.0)
        assert np.max(np.linalg.norm(bk["F"][o] - d["F"], axis=1)) / rms <= 1e-8
    b.close()


def test_batch_mixed_force_error():
    systems = ensemble(seed=31, sizes=(512, 2000, 5000))
    b64 = M.Batch.from_systems(systems, M.FP64)
    b64.prepare()
    b64.run(50, DT, record=False)
    st = b64.getParticles()
    bm = M.Batch([s.length for s in systems], [s.n for s in systems], 2.5, systems[0].components,
                 precision=M.MIXED)
    bm.setParticles(st["id"], st["cid"], st["r"], st["v"])
    pm = bm.prepare()
    # FP64 forces on the same (thermalised) configuration
    b64.setParticles(st["id"], st["cid"], st["r"], st["v"])
    p64 = b64.prepare()
    F64, Fm = b64.getParticles()["F"], bm.getParticles()["F"]
    rms = np.sqrt(np.mean(np.sum(F64 ** 2, axis=1)))
    err = np.sqrt(np.mean(np.sum((Fm - F64) ** 2, axis=1))) / rms
    assert err <= 1e-5, err
    assert np.all(rel(pm[:, 0], p64[:, 0]) <= 1e-5)
    np.testing.assert_array_equal(pm[:, 3], p64[:, 3])


def test_batch_tile_shapes_agree():
    systems = ensemble(seed=41, sizes=(300, 1100, 2500, 700))
    base = None
    for cap, ctas, dyn in M.Batch.TILE_CANDIDATES:
        b = M.Batch.from_systems(systems, M.FP64)
        b.setTiles(cap, ctas, dyn)
        b.prepare()
        recs = b.run(6, DT)
        st = b.getParticles()
        b.close()
        if base is None:
            base = (recs, st)
            continue
        np.testing.assert_allclose(recs, base[0], rtol=1e-12, atol=0)
        np.testing.assert_allclose(st["r"], base[1]["r"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(st["F"], base[1]["F"], rtol=1e-9, atol=1e-9)


def test_batch_autotune_restores_state():
    systems = ensemble(seed=51, sizes=(400, 1600, 3000))
    b = M.Batch.from_systems(systems, M.MIXED)
    b.prepare()
    before = b.getParticles()
    best, ms = b.autotune(DT, trial_steps=3)
    after = b.getParticles()
    for key in ("id", "r", "v", "F"):
        np.testing.assert_array_equal(after[key], before[key])
    assert best in M.Batch.TILE_CANDIDATES and b.tiles() == best
    assert all(t > 0 for t in ms.values())
    # the tuned batch follows the same trajectory as an untuned one with the chosen tiles
    recs = b.run(5, DT)
    c = M.Batch.from_systems(systems, M.MIXED)
    c.setTiles(*best)
    c.prepare()
    np.testing.assert_array_equal(c.run(5, DT), recs)
    b.close()
    c.close()


def test_batch_autotune_skin_mode_times_one_list_depth():
    systems = ensemble(seed=53, sizes=(400, 1600, 3000))
    b = M.Batch.from_systems(systems, M.MIXED)
    b.setSkin(0.3)
    b.prepare()
    depth = b.tiles()[0]
    before = b.getParticles()
    best, ms = b.autotune(DT, trial_steps=3)
    after = b.getParticles()
    for key in ("id", "r", "v", "F"):
        np.testing.assert_array_equal(after[key], before[key])
    assert best[0] == depth and b.tiles() == best
    for (cap, _, _), t in ms.items():
        assert (t > 0) if cap == depth else (t == -1)
    b.close()


def test_batch_barrier_timeout_reports_and_recovers():
    systems = ensemble(seed=61, sizes=(256, 3000, 6000))
    b = M.Batch.from_systems(systems, M.FP64)
    b.prepare()
    b.setBarrierTimeout(0)
    with pytest.raises(M.MdgpuError) as ei:
        b.run(3, DT)
    assert ei.value.code == 9
    # prepare is required again; with the default limit the batch runs as a fresh one does
    b.setBarrierTimeout(2_000_000_000)
    with pytest.raises(M.MdgpuError):
        b.run(1, DT)
    b.setParticles(np.concatenate([s.ids for s in systems]), np.concatenate([s.cid for s in systems]),
                   np.concatenate([s.r for s in systems]), np.concatenate([s.v for s in systems]))
    b.prepare()
    recs = b.run(4, DT)
    c = M.Batch.from_systems(systems, M.FP64)
    c.prepare()
    np.testing.assert_array_equal(c.run(4, DT), recs)
    b.close()
    c.close()


def test_batch_rejects_bad_arguments():
    s = ensemble(sizes=(256,))[0]
    with pytest.raises(M.MdgpuError) as ei:
        M.Batch([[4.0, 4.0, 4.0]], [10], 2.5, s.components)
    assert ei.value.code == 5   # fewer than 2 cells per dimension
    with pytest.raises(M.MdgpuError) as ei:
        M.Batch([[60.0, 60.0, 60.0]], [70000], 2.5, s.components)
    assert ei.value.code == 10
    b = M.Batch([s.length], [s.n], 2.5, s.components)
    with pytest.raises(M.MdgpuError) as ei:
        b.run(1, DT)
    assert ei.value.code == 3
    with pytest.raises(M.MdgpuError):
        b.setTiles(48, 2, 0)
    b.close()
