"""The oracle itself: pinned bit-for-bit to the compiled reference (golden fixtures) and to the
known answers of the reference's own unit tests (mardyn/tests/RDFTest.cpp,
mardyn/molecules/tests/MoleculeTest.cpp). CPU only."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_NAMES, system_from_golden
import oracle as O
from madpac_b200 import workloads as W


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_oracle_matches_reference_bitwise(name):
    system, g, meta = system_from_golden(name)
    o = O.Oracle(system)
    o.init()
    o.prepare_start()
    scal = [o.scalars()]
    states = {0: o.state()}
    for k in range(1, meta["nsteps"] + 1):
        o.step()
        scal.append(o.scalars())
        if k in meta["dumps"]:
            states[k] = o.state()
    np.testing.assert_array_equal(np.array([s["upot"] for s in scal]), g["upot"])
    np.testing.assert_array_equal(np.array([s["virial"] for s in scal]), g["virial"])
    np.testing.assert_array_equal(np.array([s["summv2_end"] for s in scal]), g["summv2"])
    for k in meta["dumps"]:
        st = states[k]
        np.testing.assert_array_equal(st["id"], g[f"s{k}_id"])
        for f in ("r", "v", "F", "cell"):
            np.testing.assert_array_equal(st[f], g[f"s{k}_{f}"], err_msg=f"{name} step {k} {f}")


def lattice(nx, ny, nz, length):
    """Unit-spaced lattice at integer coordinates 1..n (x fastest), zero velocities, like the
    1clj-regular-*.inp inputs of the reference's RDF test."""
    z, y, x = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    r = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float64)
    n = r.shape[0]
    return W.System(length=np.array(length, dtype=np.float64), components=[W.Component(1.0, 1.0, 1.0, False)],
                    mix=np.zeros((0, 2)), ids=np.arange(1, n + 1, dtype=np.uint64), cid=np.zeros(n, np.int32),
                    r=r, v=np.zeros((n, 3)), temperature=0.7, cutoff=1.8, lj_cutoff=1.8)


# Expected bin counts: mardyn/tests/RDFTest.cpp:70-110 (2x2x3) and :139-178 (12x12x12).
RDF_12 = {55: 4752, 78: 8712, 83: 432, 96: 5324}
RDF_2x2x3_NOHALO = {55: 20, 78: 22, 96: 8}
RDF_2x2x3_HALO = {55: 20, 78: 22, 83: 4, 96: 8}


def _expect(counts):
    e = np.zeros(100, dtype=np.uint64)
    for k, v in counts.items():
        e[k] = v
    return e


def test_rdf_known_answer_12x12x12():
    s = lattice(12, 12, 12, [12.5, 12.5, 12.5])
    o = O.Oracle(s)
    o.rdf_enable(0.018, 100)
    # ParticleContainerFactory: update + deleteOuterParticles; then balanceAndExchange and the
    # traversal (RDFTest.cpp:125-132)
    o.update()
    o.delete_outer()
    o.exchange()
    o.traverse()
    np.testing.assert_array_equal(o.rdf_counts(), _expect(RDF_12))


def test_rdf_known_answer_2x2x3_with_and_without_halo():
    s = lattice(2, 2, 3, [3.0, 3.0, 3.5])
    o = O.Oracle(s)
    o.update()
    o.delete_outer()
    o.rdf_enable(0.018, 100)
    o.update()
    o.traverse()
    np.testing.assert_array_equal(o.rdf_counts(), _expect(RDF_2x2x3_NOHALO))
    o.rdf_enable(0.018, 100)
    o.exchange()
    o.traverse()
    np.testing.assert_array_equal(o.rdf_counts(), _expect(RDF_2x2x3_HALO))


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_cross_boundary_pair_counted_once(axis):
    # A pair across a periodic face is processed from both sides through halo images; the
    # z-then-y-then-x order of Molecule::isLessThan (Molecule.cpp:439-461; MoleculeTest.cpp:21-55)
    # makes exactly one of the two a MOLECULE_MOLECULE pair.
    s = lattice(1, 1, 2, [8.0, 8.0, 8.0])
    r = np.array([[4.0, 4.0, 4.0], [4.0, 4.0, 4.0]])
    r[0, axis], r[1, axis] = 0.4, 7.7
    s.r = r
    o = O.Oracle(s)
    o.update()
    o.delete_outer()
    o.rdf_enable(0.018, 100)
    o.exchange()
    o.traverse()
    c = o.rdf_counts()
    assert int(c.sum()) == 1 and int(c[int(np.floor(0.7 / 0.018))]) == 1
    o.delete_outer()
    st = o.state()
    # both originals received equal and opposite forces
    np.testing.assert_allclose(st["F"][0], -st["F"][1], rtol=1e-12, atol=1e-9)
    assert abs(st["F"][0, axis]) > 0


def test_geometry_and_params():
    s = W.lj_fcc_box(4, 0.8, 1.0, 1, 2.5, W.two_species(), [0.5, 0.5], np.array([[0.9, 1.1]]))
    o = O.Oracle(s)
    g = o.geometry()
    L = s.length[0]
    nc = int(np.floor(L / 2.5))
    assert list(g["box_cells"]) == [nc] * 3
    assert g["cell_length"][0] == L / nc
    assert g["halo_min"][0] == 0.0 - 1 * (L / nc)
    e24, s2, sh = o.params(0, 1)
    assert e24 == 24.0 * 0.9 * np.sqrt(1.0 * 0.8)
    sig = 1.1 * 0.5 * (1.0 + 0.9)
    assert s2 == sig * sig
    # same-species entries use the component's own shift flag
    assert o.params(0, 0)[2] != 0.0


def test_golden_metadata_consistent():
    meta = json.load(open(os.path.join(GOLDEN, "ref_systems.json")))
    assert set(meta) == set(GOLDEN_NAMES)


def test_image_on_the_halo_face_is_dropped_without_changing_the_forces():
    """Box 285 of the 512-box ensemble (1,117 molecules, L = 11.30, 4 cells per dimension) has FCC
    sites exactly on a cell face; exchangeMolecules then places an image within an ulp of the halo
    box's upper face, whose cell index runs past the reference's cell array (the compiled reference
    crashes there). The oracle leaves that image out; it has no partner within the cutoff, so the
    forces, Upot and virial equal a direct minimum-image sum over all pairs."""
    s = W.config_c4()[285]
    o = O.Oracle(s)
    o.init()
    o.prepare_start()
    st, sc = o.state(), o.scalars()
    L, rc2 = s.length, s.cutoff ** 2
    r = s.r[np.argsort(s.ids)]
    n = len(r)
    eps24, sig2, shift6 = o.params(0, 0)
    F = np.zeros((n, 3))
    U6 = W6 = 0.0
    for i in range(n):
        d = r[i] - r[i + 1:]
        d -= L * np.round(d / L)
        dd = np.sum(d * d, axis=1)
        m = dd < rc2
        inv = 1.0 / dd[m]
        s6 = (sig2 * inv) ** 3
        fac = eps24 * (s6 * s6 + (s6 * s6 - s6)) * inv
        f = fac[:, None] * d[m]
        F[i] += f.sum(axis=0)
        F[i + 1:][m] -= f
        U6 += np.sum(eps24 * (s6 * s6 - s6) + shift6)
        W6 += np.sum(fac * dd[m])
    rms = np.sqrt(np.mean(np.sum(F * F, axis=1)))
    assert np.max(np.linalg.norm(st["F"] - F, axis=1)) / rms <= 1e-12
    assert abs(sc["upot_exact"] - U6 / 6.0) <= 1e-12 * abs(U6 / 6.0)
    assert abs(sc["virial_exact"] - W6) <= 1e-12 * abs(W6)
