"""Seeded workloads and the old-style phase-space format (CPU)."""
import os

import numpy as np

from madpac_b200 import workloads as W


def test_fcc_box_density_temperature_momentum():
    s = W.lj_fcc_box(6, 0.8, 1.2, 3, 2.5)
    assert s.n == 864
    assert abs(s.n / np.prod(s.length) - 0.8) < 1e-12
    assert np.all(s.r >= 0) and np.all(s.r < s.length)
    mv2 = np.sum(s.v * s.v)
    assert abs(mv2 / (3 * s.n) - 1.2) < 1e-12
    assert np.abs(s.v.sum(axis=0)).max() < 1e-9


def test_configs_shapes():
    c1 = W.config_c1()
    assert c1.n == 32000 and abs(c1.length[0] - 34.199518933533936) < 1e-9
    c5 = W.config_c5()
    assert c5.n == 16384 and len(c5.components) == 2
    assert abs(np.mean(c5.cid) - 0.5) < 1e-9
    boxes = W.config_c4(n_boxes=16)
    assert all(256 <= b.n <= 8192 for b in boxes)


def test_inp_round_trip(tmp_path):
    s = W.lj_fcc_box(3, 0.8, 1.0, 5, 2.5, W.two_species(), [0.5, 0.5], np.array([[0.9, 1.1]]))
    p = os.path.join(tmp_path, "x.inp")
    W.write_inp(s, p)
    t = W.read_inp(p)
    np.testing.assert_array_equal(t.ids, s.ids)
    np.testing.assert_array_equal(t.cid, s.cid)
    np.testing.assert_array_equal(t.r, s.r)
    np.testing.assert_array_equal(t.v, s.v)
    np.testing.assert_array_equal(t.length, s.length)
    np.testing.assert_array_equal(t.mix, s.mix)
    assert [c.do_shift for c in t.components] == [True, True]
