"""Deck generator / .dat reader host logic (CPU)."""
import os

import numpy as np

from fast_b200 import decks


def test_cantilever_hex8_counts():
    d = decks.cantilever_hex8()
    assert (d.num_nodes, d.num_elems, d.num_eq()) == (525, 320, 1500)
    assert 3 * d.num_nodes == 1575
    assert len(d.face_elem) == 16


def test_hex20_box_counts():
    d = decks.box_hex20_lognormal(8, 8, 4)
    assert d.num_elems == 256
    # serendipity node count of an a x b x c box
    a, b, c = 8, 8, 4
    full = (2 * a + 1) * (2 * b + 1) * (2 * c + 1)
    face_c = a * b * (c + 1) + a * c * (b + 1) + b * c * (a + 1)
    assert d.num_nodes == full - face_c - a * b * c


def test_hex20_full_size_counts():
    d = decks.box_hex20_lognormal()
    assert (d.num_nodes, d.num_elems, d.num_eq()) == (549185, 131072, 1609920)
    E = d.E
    assert abs(np.median(E) / 1000 - 1) < 0.01
    assert abs(np.std(np.log(E)) - 0.5) < 0.01


def test_positive_jacobian_orientation():
    from oracle import fem_oracle as fo
    for d in (decks.cantilever_hex8(2, 2, 2), decks.box_hex20_lognormal(2, 2, 1)):
        K, rc = fo.elem_stiff(d.nn, d.ngp, d.coords[d.conn[0]], 1000.0, 0.3)
        assert rc == 0


def test_dat_round_trip(tmp_path):
    d = decks.box_hex20_lognormal(3, 2, 2, seed=5)
    base = str(tmp_path / "deck")
    decks.write_dat(d, base)
    r = decks.read_dat(base + ".dat")
    np.testing.assert_array_equal(r.conn, d.conn)
    np.testing.assert_array_equal(r.coords, d.coords)
    np.testing.assert_array_equal(r.E, d.E)
    np.testing.assert_array_equal(r.node_eq(), d.node_eq())
    np.testing.assert_array_equal(r.face_nodes(), d.face_nodes())
    assert r.ngp == d.ngp and r.matrix_type == "sparse"
