"""Old-style phase-space files on the device path (mdgpu_write_checkpoint, mdgpu_read_phase_space).

Golden fixtures (tests/golden/make_checkpoint_golden.py): the reference MarDyn's own checkpoint
(Domain::writeCheckpoint after 3 steps) and the exact FP64 state of that step.

* CPU: the fixtures agree with each other under the reference's formatting rules (molecule lines
  at 6 significant digits, the header's fixed tokens and 9-digit values), so the rules the writer
  follows are pinned by the reference's output.
* GPU: the context loaded with the reference's state writes the reference's checkpoint, byte for
  byte in the header and line for line in the molecules (the reference writes them in its
  container's order, the context in the caller's, so they are compared sorted by id); reading the
  reference's file gives exactly its numbers; a 17-digit checkpoint reads back bit-identical; a
  file of another box or component table is refused.
"""
import os

import numpy as np
import pytest

from madpac_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
NAMES = ["fcc500_shifted", "two_species_500"]


def golden(name):
    text = open(os.path.join(GOLDEN, f"ck_{name}.txt")).read()
    d = np.load(os.path.join(GOLDEN, f"ck_{name}.npz"))
    head, _, body = text.partition(" MoleculeFormat\tICRVQD\n")
    return head + " MoleculeFormat\tICRVQD\n", body.splitlines(), d


def molecule_line(i, c, r, v, digits=6):
    g = lambda x: "%.*g" % (digits, x)  # noqa: E731
    return (f"{int(i)}\t{int(c) + 1}\t{g(r[0])} {g(r[1])} {g(r[2])}\t{g(v[0])} {g(v[1])} {g(v[2])}"
            "\t1 0 0 0\t0 0 0\t")


def components(d):
    return [W.Component(float(e), float(s), float(m), bool(sh))
            for e, s, m, sh in zip(d["eps"], d["sigma"], d["mass"], d["do_shift"])]


@pytest.mark.parametrize("name", NAMES)
def test_golden_checkpoint_formatting(name):
    head, lines, d = golden(name)
    want = sorted(molecule_line(i, c, r, v) for i, c, r, v in zip(d["id"], d["cid"], d["r"], d["v"]))
    assert sorted(lines) == want
    h = head.splitlines()
    assert h[0] == "mardyn trunk 20100321"
    assert h[1] == " currentTime\t%.6g" % float(d["current_time"])
    assert h[2] == " Length\t" + " ".join("%.9g" % x for x in d["length"])
    assert h[3] == " Temperature\t%.9g" % float(d["temperature"])
    nc = len(d["eps"])
    assert h[4] == f" NumberOfComponents\t{nc}"
    rc = float(d["lj_cutoff"])
    for k in range(nc):
        blk = h[5 + 3 * k: 8 + 3 * k]
        assert blk[0] == "1\t0\t0\t0\t0" and blk[2] == "0 0 0"
        s6 = (d["sigma"][k] / rc) ** 6
        shift6 = 24.0 * d["eps"][k] * (s6 - s6 * s6) if d["do_shift"][k] else 0.0
        assert blk[1] == "0 0 0\t%.9g\t%.9g %.9g %.9g %.9g" % (d["mass"][k], d["eps"][k], d["sigma"][k], rc, shift6)
    assert h[-2] == " NumberOfMolecules\t%d" % len(d["id"])


def _context(d, precision=None):
    from madpac_b200 import mdgpu as M

    lc = M.LinkedCells(d["length"], float(d["cutoff"]), components(d), d["mix"], float(d["lj_cutoff"]), 1.0,
                       M.FP64 if precision is None else precision)
    return lc


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_write_checkpoint_matches_reference(name, tmp_path):
    head, lines, d = golden(name)
    lc = _context(d)
    lc.addParticles(d["id"], d["cid"], d["r"], d["v"])
    path = str(tmp_path / "ck.txt")
    lc.writeCheckpoint(path, float(d["current_time"]), float(d["temperature"]))
    mine = open(path).read()
    mhead, _, mbody = mine.partition(" MoleculeFormat\tICRVQD\n")
    assert mhead + " MoleculeFormat\tICRVQD\n" == head
    assert sorted(mbody.splitlines()) == sorted(lines)
    lc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_read_reference_checkpoint(name):
    head, lines, d = golden(name)
    lc = _context(d)
    t, T = lc.readPhaseSpace(os.path.join(GOLDEN, f"ck_{name}.txt"))
    assert t == float("%.6g" % float(d["current_time"])) and T == float("%.9g" % float(d["temperature"]))
    st = lc.getParticles()
    rows = np.array([ln.split() for ln in lines])
    ids = rows[:, 0].astype(np.uint64)
    np.testing.assert_array_equal(st["id"], ids)
    np.testing.assert_array_equal(st["cid"], rows[:, 1].astype(np.int64) - 1)
    np.testing.assert_array_equal(st["r"], rows[:, 2:5].astype(np.float64))
    np.testing.assert_array_equal(st["v"], rows[:, 5:8].astype(np.float64))
    lc.close()


@pytest.mark.gpu
def test_checkpoint_round_trip_17_digits(tmp_path):
    _, _, d = golden("two_species_500")
    lc = _context(d)
    lc.addParticles(d["id"], d["cid"], d["r"], d["v"])
    lc.update()
    lc.traversePairs()
    lc.run(5, 0.002, record=False)
    before = lc.getParticles()
    path = str(tmp_path / "ck17.txt")
    lc.writeCheckpoint(path, 0.01, 1.2, digits=17)
    other = _context(d)
    other.readPhaseSpace(path)
    after = other.getParticles()
    for key in ("id", "cid", "r", "v"):
        np.testing.assert_array_equal(after[key], before[key])
    lc.close()
    other.close()


@pytest.mark.gpu
def test_read_phase_space_formats_and_mismatch(tmp_path):
    from madpac_b200 import mdgpu as M

    s = W.lj_fcc_box(4, 0.8, 1.0, 23, 2.5, [W.Component(1.0, 1.0, 1.0, True)])
    lc = M.LinkedCells.from_system(s, M.FP64)
    for fmt in ("ICRV", "ICRVQD"):
        path = str(tmp_path / f"s_{fmt}.inp")
        W.write_inp(s, path, fmt=fmt)
        t, T = lc.readPhaseSpace(path)
        st = lc.getParticles()
        np.testing.assert_array_equal(st["id"], s.ids)
        np.testing.assert_array_equal(st["r"], s.r)
        np.testing.assert_array_equal(st["v"], s.v)
        assert T == s.temperature
    other = W.lj_fcc_box(4, 0.7, 1.0, 24, 2.5, [W.Component(1.0, 1.0, 1.0, True)])
    path = str(tmp_path / "other.inp")
    W.write_inp(other, path)
    with pytest.raises(M.MdgpuError) as ei:
        lc.readPhaseSpace(path)
    assert ei.value.code == 1 and "box" in str(ei.value)
    lc.close()
