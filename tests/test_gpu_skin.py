"""Verlet-skin mode of mdgpu_step / mdgpu_run (mdgpu_set_skin).

Every pair within the cutoff is still evaluated with the exact test, so a skin run follows the
per-step traversal's trajectory up to summation order: FP64 step records within 1e-10 (relative)
and identical pair counts over a short trajectory, forces at the final positions within 1e-10 of a
fresh traversal; the mixed form stays within 1e-5 of FP64 forces. Lists are reused (fewer builds
than steps) and rebuilt when molecules move more than skin/2 (a displaced state forces a build).
The same holds where the bricks are evaluated in other ways: a liquid slab with a vapour (sparse
bricks one warp each, the dense ones from a queue, over two runs so that the second knows what
the first build found) and a jittered lattice whose cells hold 27 to 64 molecules (bricks of more
than 256, whose last molecules are spread over the warps, several lanes each).
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


def run(system, precision, skin, nsteps, warm=None):
    lc = M.LinkedCells.from_system(system, precision)
    lc.update()
    lc.traversePairs()
    if skin:
        lc.setSkin(skin)
    recs = lc.run(nsteps, DT)
    st = lc.getParticles()
    builds = lc.skinBuilds()
    lc.close()
    return recs, st, builds


def forces_at(system, r, precision=M.FP64):
    lc = M.LinkedCells.from_system(system, precision)
    lc.setState(r=r)
    lc.update()
    u, w, p = lc.traversePairs()
    F = lc.getParticles()["F"]
    lc.close()
    return F, u, w, p


@pytest.mark.parametrize("two", [False, True])
def test_skin_fp64_follows_exact_traversal(two):
    system = box(two=two)
    n = 60
    r0, s0, _ = run(system, M.FP64, 0.0, n)
    r1, s1, builds = run(system, M.FP64, 0.3, n)
    assert 1 <= builds < n
    assert np.all(rel(r1[:, :3], r0[:, :3]) <= 1e-10), np.max(rel(r1[:, :3], r0[:, :3]))
    np.testing.assert_array_equal(r1[:, 3], r0[:, 3])
    np.testing.assert_array_equal(s1["id"], s0["id"])
    np.testing.assert_allclose(s1["r"], s0["r"], rtol=0, atol=1e-10)
    assert np.all((s1["r"] >= 0) & (s1["r"] < system.length))
    F, u, w, p = forces_at(system, s1["r"])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    assert np.max(np.linalg.norm(s1["F"] - F, axis=1)) / rms <= 1e-10


def jittered_lattice(n_side=24, rho=0.3, jitter=0.3, seed=9, rc=4.5):
    """A simple-cubic lattice at density rho with each site moved by up to +-jitter: the skin grid's
    cells (edge rc + 0.3) hold 3 or 4 lattice planes per dimension, 27 to 64 molecules."""
    rng = np.random.default_rng(seed)
    a = rho ** (-1.0 / 3.0)
    g = np.arange(n_side) * a
    r = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + a / 4.0
    r += rng.uniform(-jitter, jitter, r.shape)
    length = np.full(3, n_side * a)
    n = r.shape[0]
    v = rng.normal(0.0, 1.0, (n, 3))
    v -= v.mean(axis=0)
    return W.System(length=length, components=[W.Component(1.0, 1.0, 1.0, True)], mix=np.zeros((0, 2)),
                    ids=np.arange(1, n + 1, dtype=np.uint64), cid=np.zeros(n, dtype=np.int32),
                    r=np.mod(r, length), v=v, temperature=1.0, cutoff=rc, lj_cutoff=rc, name="jittered")


def run_split(system, precision, skin, runs):
    """The steps as several mdgpu_run calls (the records concatenated)."""
    lc = M.LinkedCells.from_system(system, precision)
    lc.update()
    lc.traversePairs()
    if skin:
        lc.setSkin(skin)
    recs = np.concatenate([lc.run(k, DT) for k in runs])
    st = lc.getParticles()
    builds = lc.skinBuilds()
    lc.close()
    return recs, st, builds


@pytest.mark.parametrize("kind", ["slab", "jittered"])
def test_skin_fp64_other_brick_shapes(kind):
    if kind == "slab":
        system = W.config_c3(seed=5, n_total=30000)
    else:
        system = jittered_lattice()
    runs = [12, 12]
    r0, s0, _ = run_split(system, M.FP64, 0.0, runs)
    r1, s1, builds = run_split(system, M.FP64, 0.3, runs)
    assert builds >= 2   # one forced build per run at least
    assert np.all(rel(r1[:, :3], r0[:, :3]) <= 1e-10), np.max(rel(r1[:, :3], r0[:, :3]))
    np.testing.assert_array_equal(r1[:, 3], r0[:, 3])
    np.testing.assert_allclose(s1["r"], s0["r"], rtol=0, atol=1e-10)
    F, u, w, p = forces_at(system, s1["r"])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    assert np.max(np.linalg.norm(s1["F"] - F, axis=1)) / rms <= 1e-10
    # the mixed form on the same steps
    r2, s2, _ = run_split(system, M.MIXED, 0.3, runs)
    err = np.sqrt(np.mean(np.sum((s2["F"] - s1["F"]) ** 2, axis=1))) / rms
    assert err <= 1e-5, err
    assert np.all(rel(r2[:, :2], r1[:, :2]) <= 1e-5)


def test_skin_mixed_accuracy():
    system = box()
    r1, s1, builds = run(system, M.MIXED, 0.3, 80)
    assert builds >= 1
    F, u, w, p = forces_at(system, s1["r"])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    err = np.sqrt(np.mean(np.sum((s1["F"] - F) ** 2, axis=1))) / rms
    assert err <= 1e-5, err


def test_skin_rebuilds_after_displacement():
    system = box(n_cells=8)
    lc = M.LinkedCells.from_system(system, M.FP64)
    lc.update()
    lc.traversePairs()
    lc.setSkin(0.3)
    lc.run(5, DT)
    b0 = lc.skinBuilds()
    st = lc.getParticles()
    # shift every molecule by 0.2 (more than skin/2): the next step must build again
    r = st["r"] + np.array([0.2, -0.1, 0.05])
    lc.setState(r=r)
    lc.run(1, DT)
    assert lc.skinBuilds() == b0 + 1
    got = lc.getParticles()
    F, *_ = forces_at(system, got["r"])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    assert np.max(np.linalg.norm(got["F"] - F, axis=1)) / rms <= 1e-10
    # a drop-in traversal needs an update after skin steps
    with pytest.raises(M.MdgpuError) as ei:
        lc.traversePairs()
    assert ei.value.code == 3
    lc.update()
    lc.traversePairs()
    lc.close()


def test_skin_rejects_bad_values():
    system = box(n_cells=6)
    lc = M.LinkedCells.from_system(system, M.FP64)
    with pytest.raises(M.MdgpuError):
        lc.setSkin(-0.1)
    with pytest.raises(M.MdgpuError):
        lc.setSkin(3.5)
    lc.close()
