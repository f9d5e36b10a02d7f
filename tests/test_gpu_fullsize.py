"""Parity at the stated sizes of the large workloads, against the oracle (the reference's algorithm,
bit-exact with the compiled reference on the golden fixtures):

* 1,048,576 molecules, rho 0.75, T 0.9, rc 3.0, truncated-shifted LJ (the bench's headline box):
  FP64 through the reference's step sequence (update + traversePairs every step) and through the
  Verlet-skin sequence (lists within rc + 0.3, rebuilt on the device), at step 0 and along 10 steps;
  the mixed form on the same steps and on a thermalised state of the same box.
* 4,194,304 molecules, the two-species slab (liquid rho 0.70 in the middle third, vapour 0.02,
  Lz = 3 Lx): step 0 in FP64 and mixed, and the first skin step (its vapour bricks take the
  one-warp list kernel, the liquid ones the queued dense kernel).
* 512 independent boxes of 256 to 8,192 molecules: every box at step 0 and after 5 steps, FP64 and
  mixed, with and without the skin, all boxes advanced by the persistent batched kernel; the
  oracle's boxes run on all host cores.

Tolerances are those of the small-box parity tests: FP64 forces max_i |dF_i| / max(rms F, 1) <= 1e-12
at step 0 and Upot, virial within 1e-12 of the exactly summed pair terms; step records within 1e-9
and forces within 1e-8 along a trajectory (summation order differs and molecular dynamics amplifies
last bits); the mixed form's forces within 1e-5 rms of the reference's and its records within 1e-6
(the 512 lattice-start boxes: 1e-5 of each sum's conditioning scale, the sum of its terms' magnitudes).
"""
import numpy as np
import pytest

import oracle as O
from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.fullsize]

DT = 0.002
SKIN = 0.3


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(np.asarray(b)), 1e-300)


def force_err_max(F, Fref):
    rms = max(np.sqrt(np.mean(np.sum(Fref * Fref, axis=1))), 1.0)
    return float(np.max(np.linalg.norm(F - Fref, axis=1)) / rms)


def force_err_rms(F, Fref):
    rms = np.sqrt(np.mean(np.sum(Fref * Fref, axis=1)))
    return float(np.sqrt(np.mean(np.sum((F - Fref) ** 2, axis=1))) / rms)


def by_id(st):
    o = np.argsort(st["id"], kind="stable")
    return {k: a[o] for k, a in st.items()}


def unordered_pairs(r, length, rc):
    from scipy.spatial import cKDTree

    tree = cKDTree(np.mod(r, length), boxsize=length)
    return (tree.count_neighbors(tree, rc) - len(r)) / 2.0


def pair_term_scales(r, length, rc):
    """The conditioning scales of Upot and the virial of a single-species LJ box (eps = sigma = 1):
    the sums over pairs within rc of the magnitudes of their terms, 4 (s^12 + s^6 + |shift|) and
    24 (2 s^12 + s^6). A summed error of the rounded pair terms is a fraction of these, whatever
    cancels in the sums themselves."""
    from scipy.spatial import cKDTree

    x = np.mod(r, length)
    tree = cKDTree(x, boxsize=length)
    ij = tree.query_pairs(rc, output_type="ndarray")
    d = x[ij[:, 0]] - x[ij[:, 1]]
    d -= length * np.round(d / length)
    s6 = 1.0 / np.sum(d * d, axis=1) ** 3
    shift = abs(4.0 * (rc ** -12 - rc ** -6))
    return float(np.sum(4.0 * (s6 * s6 + s6) + shift)), float(np.sum(24.0 * (2.0 * s6 * s6 + s6)))


def with_positions(system, r, v=None):
    """The same system (ids in the same order) at other positions and velocities."""
    import copy

    s = copy.copy(system)
    s.r = np.ascontiguousarray(r)
    if v is not None:
        s.v = np.ascontiguousarray(v)
    return s


# ---- 1,048,576 molecules ------------------------------------------------------------------------

C2_STEPS = 10


@pytest.fixture(scope="module")
def c2():
    """The C2 box and the oracle's step 0 and 10 steps."""
    system = W.config_c2()
    ref = O.run_oracle(system, C2_STEPS, dump_steps=(0, C2_STEPS))
    return system, ref


def _check_records(recs, sc, tol, what):
    for k in range(1, len(sc)):
        for j, key in enumerate(("upot", "virial", "summv2")):
            e = float(rel(recs[k - 1][j], sc[k][key]))
            assert e <= tol, (what, k, key, e)


def test_c2_fp64_reference_sequence_against_oracle(c2):
    system, ref = c2
    sim = M.Simulation(system, M.FP64)
    sim.prepare_start()
    st = sim.state()
    d0, sc = ref["dumps"][0], ref["scalars"]
    np.testing.assert_array_equal(st["id"], d0["id"])
    np.testing.assert_array_equal(st["cell"], d0["cell"])
    assert force_err_max(st["F"], d0["F"]) <= 1e-12
    assert rel(sim.scalars()["upot"], sc[0]["upot_exact"]) <= 1e-12
    assert rel(sim.scalars()["virial"], sc[0]["virial_exact"]) <= 1e-12
    assert sim.npairs == unordered_pairs(system.r, system.length, system.cutoff)
    recs = []
    for _ in range(C2_STEPS):
        sim.simulateStep()
        s = sim.scalars()
        recs.append((s["upot"], s["virial"], s["summv2"]))
    _check_records(recs, sc, 1e-9, "reference sequence")
    st, d = sim.state(), ref["dumps"][C2_STEPS]
    np.testing.assert_allclose(st["r"], d["r"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(st["v"], d["v"], rtol=0, atol=1e-8)
    assert force_err_max(st["F"], d["F"]) <= 1e-8
    np.testing.assert_array_equal(st["cell"], d["cell"])
    sim.container.close()


@pytest.mark.parametrize("precision", [M.FP64, M.MIXED])
def test_c2_skin_sequence_against_oracle(c2, precision):
    system, ref = c2
    lc = M.LinkedCells.from_system(system, precision)
    lc.update()
    u, w, p = lc.traversePairs()
    sc = ref["scalars"]
    tol0 = 1e-12 if precision == M.FP64 else 1e-6
    assert rel(u, sc[0]["upot_exact"]) <= tol0 and rel(w, sc[0]["virial_exact"]) <= tol0
    lc.setSkin(SKIN)
    recs = lc.run(C2_STEPS, DT)
    assert lc.skinBuilds() >= 1
    _check_records(recs, sc, 1e-9 if precision == M.FP64 else 1e-6, "skin sequence")
    st, d = by_id(lc.getParticles()), ref["dumps"][C2_STEPS]
    np.testing.assert_array_equal(st["id"], d["id"])
    if precision == M.FP64:
        np.testing.assert_allclose(st["r"], d["r"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(st["v"], d["v"], rtol=0, atol=1e-8)
        assert force_err_max(st["F"], d["F"]) <= 1e-8
    else:
        assert force_err_rms(st["F"], d["F"]) <= 1e-5
    # the pair count of the last step is the exact number of unordered pairs within rc
    assert recs[-1, 3] == unordered_pairs(st["r"], system.length, system.cutoff)
    lc.close()


def test_c2_mixed_against_oracle_on_a_thermalised_state(c2):
    system, _ = c2
    lc = M.LinkedCells.from_system(system, M.FP64)
    lc.update()
    lc.traversePairs()
    lc.setSkin(SKIN)
    lc.run(300, DT, record=False)
    st = lc.getParticles()   # in the caller's (the system's) order
    lc.close()
    np.testing.assert_array_equal(st["id"], system.ids)
    liquid = with_positions(system, st["r"])
    o = O.Oracle(liquid)
    o.init()
    o.prepare_start()
    d, so = o.state(), o.scalars()
    for precision, tol in ((M.FP64, 1e-12), (M.MIXED, 1e-5)):
        m = M.LinkedCells.from_system(liquid, precision)
        m.update()
        u, w, _ = m.traversePairs()
        F = by_id(m.getParticles())["F"]
        m.close()
        if precision == M.FP64:
            assert force_err_max(F, d["F"]) <= tol
        else:
            assert force_err_rms(F, d["F"]) <= tol
        assert rel(u, so["upot_exact"]) <= (1e-12 if precision == M.FP64 else 1e-6)
        assert rel(w, so["virial_exact"]) <= (1e-12 if precision == M.FP64 else 1e-6)


# ---- 4,194,304 molecules: the two-species slab -------------------------------------------------

def test_c3_slab_step0_and_first_skin_step_against_oracle():
    system = W.config_c3()
    ref = O.run_oracle(system, 1, dump_steps=(0, 1))
    d0, d1, sc = ref["dumps"][0], ref["dumps"][1], ref["scalars"]
    for precision in (M.FP64, M.MIXED):
        lc = M.LinkedCells.from_system(system, precision)
        lc.update()
        u, w, p = lc.traversePairs()
        st = by_id(lc.getParticles())
        np.testing.assert_array_equal(st["id"], d0["id"])
        if precision == M.FP64:
            assert force_err_max(st["F"], d0["F"]) <= 1e-12
            assert rel(u, sc[0]["upot_exact"]) <= 1e-12 and rel(w, sc[0]["virial_exact"]) <= 1e-12
            assert p == unordered_pairs(system.r, system.length, system.cutoff)
        else:
            assert force_err_rms(st["F"], d0["F"]) <= 1e-5
            assert rel(u, sc[0]["upot_exact"]) <= 1e-6 and rel(w, sc[0]["virial_exact"]) <= 1e-6
        lc.setSkin(SKIN)
        rec = lc.run(1, DT)[0]
        st = by_id(lc.getParticles())
        lc.close()
        tol = 1e-9 if precision == M.FP64 else 1e-6
        for j, key in enumerate(("upot", "virial", "summv2")):
            assert rel(rec[j], sc[1][key]) <= tol, (precision, key)
        if precision == M.FP64:
            np.testing.assert_allclose(st["r"], d1["r"], rtol=0, atol=1e-9)
            assert force_err_max(st["F"], d1["F"]) <= 1e-8
        else:
            assert force_err_rms(st["F"], d1["F"]) <= 1e-5


# ---- 512 boxes ----------------------------------------------------------------------------------

C4_STEPS = 5


@pytest.fixture(scope="module")
def c4():
    systems = W.config_c4()
    refs = O.run_oracle_many(systems, C4_STEPS, dump_steps=(C4_STEPS,))
    return systems, refs


@pytest.mark.parametrize("precision,skin", [(M.FP64, 0.0), (M.FP64, SKIN), (M.MIXED, SKIN)])
def test_c4_all_512_boxes_against_oracle(c4, precision, skin):
    systems, refs = c4
    assert len(systems) == 512
    b = M.Batch.from_systems(systems, precision)
    b.setSkin(skin)
    prep = b.prepare()
    recs = b.run(C4_STEPS, DT)
    st = b.getParticles()
    b.close()
    fp64 = precision == M.FP64
    for k, (s, ref) in enumerate(zip(systems, refs)):
        sc = ref["scalars"]
        if fp64:
            assert rel(prep[k, 0], sc[0]["upot_exact"]) <= 1e-12, k
            assert rel(prep[k, 1], sc[0]["virial_exact"]) <= 1e-12, k
        else:
            # The mixed form's Upot and virial are held to the 1e-5 of its stated accuracy, taken of
            # each sum's conditioning scale (the sum of its pair terms' magnitudes). On these lattice
            # starts every pair of a neighbour shell carries the same FP32 rounding, so the errors
            # add coherently (box 13: 0.059 in a virial of 38,649, 1.5e-6 of it, 3.8e-7 of its
            # scale of 153,395), and a lattice sum can be a small difference of large shell sums
            # (box 7: a virial of 1,826 with a scale of 195,665).
            su, sw = pair_term_scales(s.r, s.length, s.cutoff)
            assert abs(prep[k, 0] - sc[0]["upot_exact"]) <= 1e-5 * su, k
            assert abs(prep[k, 1] - sc[0]["virial_exact"]) <= 1e-5 * sw, k
        for step in range(1, C4_STEPS + 1):
            for j, key in enumerate(("upot", "virial", "summv2")):
                got, want = recs[step - 1, k, j], sc[step][key]
                if fp64:
                    e = float(rel(got, want))
                    assert e <= 1e-9, (k, step, key, e)
                else:
                    e = abs(got - want) / (abs(want) if j == 2 else (su, sw)[j])
                    assert e <= 1e-5, (k, step, key, e)
        d = ref["dumps"][C4_STEPS]
        bk = by_id(b.box(st, k))
        np.testing.assert_array_equal(bk["id"], d["id"])
        if fp64:
            np.testing.assert_allclose(bk["r"], d["r"], rtol=0, atol=1e-9)
            np.testing.assert_allclose(bk["v"], d["v"], rtol=0, atol=1e-8)
            assert force_err_max(bk["F"], d["F"]) <= 1e-8, k
        else:
            assert force_err_rms(bk["F"], d["F"]) <= 1e-5, k
