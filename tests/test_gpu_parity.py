"""GPU parity through the C ABI against the reference (golden fixtures made by the compiled
reference) and the oracle. Tolerances:
  * cell assignment and periodic wrap: bit-exact;
  * MDGPU_FP64 forces: max_i |F_i - F_i^ref| / max(rms(F^ref), 1) <= 1e-12 at step 0 (the floor of
    1 epsilon/sigma keeps the perfect-lattice starts, whose net forces are rounding noise, well
    posed); Upot and virial within 1e-12 (relative) of the same pair terms summed exactly (the
    oracle's compensated sums: the reference's own sequential sum carries ~1e-12 of rounding on a
    lattice), and within 1e-9 of the reference along a trajectory (the GPU sums the same pair terms
    in another order, and molecular dynamics amplifies the last-bit differences);
  * MDGPU_MIXED forces on a thermalised configuration: rms_i |F_i - F_i^ref| / rms(F^ref) <= 1e-5.
"""
import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN_NAMES, system_from_golden
from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu


def force_err_max(F, Fref):
    rms = max(np.sqrt(np.mean(np.sum(Fref * Fref, axis=1))), 1.0)
    return float(np.max(np.linalg.norm(F - Fref, axis=1)) / rms)


def force_err_rms(F, Fref):
    rms = np.sqrt(np.mean(np.sum(Fref * Fref, axis=1)))
    return float(np.sqrt(np.mean(np.sum((F - Fref) ** 2, axis=1))) / rms)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_step0_fp64_matches_reference(name):
    system, g, meta = system_from_golden(name)
    sim = M.Simulation(system, M.FP64)
    sim.prepare_start()
    st = sim.state()
    np.testing.assert_array_equal(st["id"], g["s0_id"])
    np.testing.assert_array_equal(st["cell"], g["s0_cell"])
    np.testing.assert_array_equal(st["r"], g["s0_r"])
    assert force_err_max(st["F"], g["s0_F"]) <= 1e-12
    sc = sim.scalars()
    o = O.Oracle(system)
    o.init()
    o.prepare_start()
    so = o.scalars()
    assert so["upot"] == g["upot"][0] and so["virial"] == g["virial"][0]
    assert rel(sc["upot"], so["upot_exact"]) <= 1e-12
    assert rel(sc["virial"], so["virial_exact"]) <= 1e-12
    assert rel(sc["upot"], g["upot"][0]) <= 1e-10


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_trajectory_fp64_matches_reference(name):
    system, g, meta = system_from_golden(name)
    sim = M.Simulation(system, M.FP64)
    sim.prepare_start()
    for k in range(1, meta["nsteps"] + 1):
        sim.simulateStep()
        sc = sim.scalars()
        assert rel(sc["upot"], g["upot"][k]) <= 1e-9, (k, sc["upot"], g["upot"][k])
        assert rel(sc["virial"], g["virial"][k]) <= 1e-9
        if k in meta["dumps"]:
            st = sim.state()
            np.testing.assert_array_equal(st["id"], g[f"s{k}_id"])
            np.testing.assert_allclose(st["r"], g[f"s{k}_r"], rtol=0, atol=1e-9)
            np.testing.assert_allclose(st["v"], g[f"s{k}_v"], rtol=0, atol=1e-8)
            assert force_err_max(st["F"], g[f"s{k}_F"]) <= 1e-8
            # the cells of the GPU's own positions are those the reference formula gives
            np.testing.assert_array_equal(st["cell"], g[f"s{k}_cell"])
        # sum m v^2 after any thermostat scaling, as the reference harness records it
        st = sim.container.getParticles()
        mv2 = float(np.sum(system.mass()[st["cid"]] * np.sum(st["v"] ** 2, axis=1)))
        assert rel(mv2, g["summv2"][k]) <= 1e-9


def test_cell_assignment_bitexact_edge_positions():
    system = W.lj_fcc_box(5, 0.8, 1.0, 21, 2.5)
    lc = M.LinkedCells.from_system(system)
    o = O.Oracle(system, add_particles=False)
    L = system.length[0]
    geo = lc.geometry()
    cl = geo["cell_length"][0]
    rng = np.random.default_rng(5)
    n = system.n
    r = rng.uniform(0, L, size=(n, 3))
    # positions on cell faces, at the box faces and just outside them (they wrap)
    edges = np.concatenate([np.arange(geo["box_cells"][0] + 1) * cl, [0.0, np.nextafter(L, 0), L,
                            -1e-9, -0.3 * cl, L + 0.3 * cl, L + 1e-12,
                            np.nextafter(cl, 0), np.nextafter(cl, 2 * L)]])
    k = min(len(edges), n)
    for d in range(3):
        r[:k, d] = rng.permutation(edges)[:k]
    lc.setState(r=r)
    lc.update()
    got = lc.getParticles()
    cells = lc.getCellIndexOfMolecule()
    wrapped = r.copy()
    for d in range(3):
        lo = r[:, d] < 0
        hi = r[:, d] >= L
        wrapped[lo, d] = r[lo, d] + L
        wrapped[hi, d] = r[hi, d] - L
    np.testing.assert_array_equal(got["r"], wrapped)
    expect = np.array([o.cell_index(x) for x in wrapped])
    np.testing.assert_array_equal(cells, expect)


def _lattice12():
    z, y, x = np.meshgrid(np.arange(1, 13), np.arange(1, 13), np.arange(1, 13), indexing="ij")
    r = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float64)
    n = r.shape[0]
    return W.System(length=np.array([12.5, 12.5, 12.5]), components=[W.Component(1.0, 1.0, 1.0, False)],
                    mix=np.zeros((0, 2)), ids=np.arange(1, n + 1, dtype=np.uint64), cid=np.zeros(n, np.int32),
                    r=r, v=np.zeros((n, 3)), temperature=0.7, cutoff=1.8, lj_cutoff=1.8)


@pytest.mark.parametrize("precision", [M.FP64, M.MIXED])
def test_pair_count_known_answer_lattice(precision):
    # mardyn/tests/RDFTest.cpp:139-178: 4752 + 8712 + 432 + 5324 pairs within rc = 1.8
    lc = M.LinkedCells.from_system(_lattice12(), precision)
    lc.update()
    u, w, npairs = lc.traversePairs()
    assert npairs == 4752 + 8712 + 432 + 5324
    o = O.Oracle(_lattice12())
    o.init()
    o.prepare_start()
    assert rel(u, o.scalars()["upot"]) <= (1e-12 if precision == M.FP64 else 1e-6)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_mixed_precision_force_error(name):
    # the last dumped step of each fixture: molecules have left their lattice sites
    system, g, meta = system_from_golden(name)
    k = max(meta["dumps"])
    o = np.argsort(system.ids)
    lc = M.LinkedCells.from_system(system, M.MIXED)
    r = np.empty_like(system.r)
    r[o] = g[f"s{k}_r"]
    lc.setState(r=r)
    lc.update()
    u, w, _ = lc.traversePairs()
    st = lc.getParticles()
    F = st["F"][np.argsort(st["id"])]
    assert force_err_rms(F, g[f"s{k}_F"]) <= 1e-5
    assert rel(u, g["upot"][k]) <= 1e-5
    assert rel(w, g["virial"][k]) <= 1e-5


def test_fp64_is_deterministic():
    system = W.config_c5()
    outs = []
    for _ in range(2):
        lc = M.LinkedCells.from_system(system)
        lc.update()
        lc.traversePairs()
        rec = lc.run(5, system.dt)
        outs.append((rec, lc.getParticles()))
        lc.close()
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    for f in ("r", "v", "F"):
        np.testing.assert_array_equal(outs[0][1][f], outs[1][1][f])


def test_run_matches_stepwise_api():
    system = W.lj_fcc_box(6, 0.75, 0.9, 31, 3.0, [W.Component(1.0, 1.0, 1.0, True)])
    a = M.LinkedCells.from_system(system)
    a.update()
    a.traversePairs()
    rec = a.run(6, system.dt)
    b = M.Simulation(system)
    b.prepare_start()
    for k in range(6):
        b.simulateStep()
        sc = b.scalars()
        assert rec[k, 0] == sc["upot"] and rec[k, 1] == sc["virial"] and rec[k, 2] == sc["summv2"]
    np.testing.assert_array_equal(a.getParticles()["r"], b.container.getParticles()["r"])


def test_c1_100_steps_against_oracle():
    """32,000 molecules, rho 0.8, T 1, rc 2.5, 100 NVE steps: GPU FP64 against the oracle."""
    system = W.config_c1()
    o = O.Oracle(system)
    o.init()
    o.prepare_start()
    sim = M.Simulation(system, M.FP64)
    sim.prepare_start()
    assert rel(sim.scalars()["upot"], o.scalars()["upot_exact"]) <= 1e-12
    assert rel(sim.scalars()["virial"], o.scalars()["virial_exact"]) <= 1e-12
    for k in range(100):
        o.step()
        sim.simulateStep()
        so, sg = o.scalars(), sim.scalars()
        assert rel(sg["upot"], so["upot"]) <= 1e-9, k
        assert rel(sg["virial"], so["virial"]) <= 1e-9, k
        assert rel(sg["summv2"], so["summv2"]) <= 1e-9, k
    a, b = sim.state(), o.state()
    np.testing.assert_allclose(a["r"], b["r"], rtol=0, atol=1e-8)
    assert force_err_max(a["F"], b["F"]) <= 1e-7


# ---- error paths: the reference's exit() codes become status codes ------------------------------

def test_box_too_small_is_rejected():
    with pytest.raises(M.MdgpuError) as e:
        M.LinkedCells([4.0, 10.0, 10.0], 2.5, [W.Component()])
    assert e.value.code == 5


def test_traverse_before_update_is_rejected():
    lc = M.LinkedCells.from_system(W.lj_fcc_box(4, 0.8, 1.0, 1, 2.5))
    with pytest.raises(M.MdgpuError) as e:
        lc.traversePairs()
    assert e.value.code == 3


def test_molecule_beyond_halo_is_reported():
    s = W.lj_fcc_box(4, 0.8, 1.0, 1, 2.5)
    lc = M.LinkedCells.from_system(s)
    r = s.r.copy()
    r[7, 0] = s.length[0] + 5.0 * 2.5
    lc.setState(r=r)
    with pytest.raises(M.MdgpuError) as e:
        lc.update()
    assert e.value.code == 6


def test_wrap_onto_upper_face_is_reported():
    # r = -5e-324 wraps to r + L == L: the reference's image lands on the upper face and
    # deleteOuterParticles drops it (the molecule is lost); here the update reports it instead.
    s = W.lj_fcc_box(4, 0.8, 1.0, 1, 2.5)
    lc = M.LinkedCells.from_system(s)
    r = s.r.copy()
    r[2, 1] = np.nextafter(0.0, -1.0)
    lc.setState(r=r)
    with pytest.raises(M.MdgpuError) as e:
        lc.update()
    assert e.value.code == 6


def test_identical_positions_are_reported():
    s = W.lj_fcc_box(4, 0.8, 1.0, 1, 2.5)
    s.r[3] = s.r[4]
    lc = M.LinkedCells.from_system(s)
    lc.update()
    with pytest.raises(M.MdgpuError) as e:
        lc.traversePairs()
    assert e.value.code == 7
