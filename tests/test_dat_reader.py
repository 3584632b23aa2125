"""The library's parallel .dat reader (fast_dat_*, include/fast_dat.h) on the
CPU: every hex deck of the golden set read back equal to the Python reader
and giving the reference's equation numbering and load vector; layout,
number-format and thread-count independence; the reference's record
semantics; deck errors reported with their line."""
import ctypes
import os
import re

import numpy as np
import pytest

from fast_b200 import build as fbuild
from fast_b200 import datfile, decks, gpu
from oracle import fem_oracle as fo
from tests import golden_io as gio

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEX = [n for n in gio.names() if gio.load(n)[0].kind in ("hex8", "hex20")]
BSP = [n for n in gio.names() if gio.load(n)[0].kind == "bsp"]
FIELDS = ["coords", "conn", "E", "nu", "fixed", "face_elem", "face_corners", "face_q", "face_local", "rho",
          "solver_rank"]


@pytest.fixture(scope="module", autouse=True)
def lib():
    fbuild.build()
    return datfile._lib()


def same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert (x is None) == (y is None), f
        if x is not None:
            assert np.array_equal(np.asarray(x), np.asarray(y)), f
    assert a.kind == b.kind and tuple(a.ngp) == tuple(b.ngp) and a.total_lagrangian == b.total_lagrangian
    for f in ("algorithm", "matrix_type", "tol", "maxit", "maxstep", "step_factor"):
        assert getattr(a, f) == getattr(b, f), f


def test_header_lists_every_export(lib):
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "fast_dat.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(fast_dat_[a-z_]+)\s*\(", txt)))
    assert names == sorted(datfile.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


@pytest.mark.parametrize("name", HEX)
def test_golden_decks_match_python_reader_and_reference(name, tmp_path):
    d, g = gio.load(name)
    p = decks.write_dat(d, str(tmp_path / name))
    nat = datfile.read_dat(p)
    same(nat, decks.read_dat(p))
    np.testing.assert_array_equal(nat.node_eq(), g["ref_node_eq"])
    if "ref_f" in g and not name.startswith(("nr_", "arc_", "modal_")):
        assert gio.rel(fo.face_loads(nat), g["ref_f"]) < 1e-13
    if nat.face_elem is not None:
        np.testing.assert_array_equal(datfile_face_nodes(p), nat.face_nodes())


def datfile_face_nodes(path):
    L = datfile._lib()
    h = ctypes.c_void_p()
    assert L.fast_dat_read(os.fsencode(path), 0, ctypes.byref(h)) == 0
    try:
        info = datfile.DatInfo()
        L.fast_dat_get_info(h, ctypes.byref(info))
        out = np.empty((info.num_faces, info.nodes_per_face), np.int32)
        assert L.fast_dat_get_faces(h, None, None, out.ctypes.data_as(ctypes.c_void_p), None, None) == 0
    finally:
        L.fast_dat_free(h)
    return out


def test_analysis_header_and_loads_round_trip(tmp_path):
    d = decks.cantilever_hex8(6, 3, 2)
    d.algorithm, d.tol, d.maxit, d.maxstep, d.step_factor = "newmark", 1e-9, 17, 40, 0.125
    d.time_step, d.newmark, d.print_step = 2.5e-3, (0.6, 0.3025), 1
    d.arc_load_coeff, d.target_iter = 1.0, 4
    d.rho = np.full(d.num_elems, 7.85e-9)
    rng = np.random.default_rng(3)
    d.nodal_f = np.zeros((d.num_nodes, 3))
    d.nodal_f[rng.choice(d.num_nodes, 5, replace=False)] = rng.standard_normal((5, 3))
    d.solver_rank = rng.permutation(d.num_nodes) + 1
    p = decks.write_dat(d, str(tmp_path / "hdr"))
    nat = datfile.read_dat(p)
    assert nat.algorithm == "newmark" and nat.tol == 1e-9 and nat.maxit == 17 and nat.maxstep == 40
    assert nat.step_factor == 0.125 and nat.time_step == 2.5e-3 and nat.newmark == (0.6, 0.3025)
    assert nat.arc_load_coeff == 1.0 and nat.target_iter == 4
    np.testing.assert_array_equal(nat.rho, d.rho)
    np.testing.assert_array_equal(nat.nodal_f, d.nodal_f)
    np.testing.assert_array_equal(nat.solver_rank, d.solver_rank)
    np.testing.assert_array_equal(nat.node_eq(), d.node_eq())


def _reflow(text, mode):
    """The same deck with another token layout (labels kept on their own line)."""
    out = []
    for line in text.split("\n"):
        if line.startswith("%") or "'" in line:
            out.append(line)
            continue
        toks = line.split()
        if mode == "one_per_line":
            out.extend(toks)
        elif mode == "tabs_crlf":
            out.append("\t ".join(toks) + "\r")
        elif mode == "signs":
            out.append(" ".join(("+" + t if re.fullmatch(r"\d[\d.eE+-]*", t) else t) for t in toks))
    if mode == "joined":
        return re.sub(r"(?<=[0-9])\n(?=[0-9-])", "  ", text)
    return "\n".join(out)


@pytest.mark.parametrize("mode", ["one_per_line", "tabs_crlf", "signs", "joined"])
def test_token_layout_does_not_matter(mode, tmp_path):
    d, _ = gio.load("cfg_hex20_lognormal_4x4x2")
    p = decks.write_dat(d, str(tmp_path / "base"))
    base = datfile.read_dat(p)
    q = tmp_path / f"{mode}.dat"
    q.write_text(_reflow(open(p).read(), mode))
    same(datfile.read_dat(str(q)), base)


def test_exponent_forms_parse_to_the_same_doubles(tmp_path):
    d = decks.cantilever_hex8(3, 2, 2)
    p = decks.write_dat(d, str(tmp_path / "e"))
    text = open(p).read()
    # rewrite every coordinate as %.17E and as a plain decimal: same binary values
    lines = text.split("\n")
    i = lines.index("%NODE.COORD") + 2
    for k in range(d.num_nodes):
        lab, x, y, z = lines[i + k].split()
        lines[i + k] = f"{lab} {float(x):.17E} {float(y):.17e} {repr(float(z))}"
    q = tmp_path / "e2.dat"
    q.write_text("\n".join(lines))
    np.testing.assert_array_equal(datfile.read_dat(str(q)).coords, datfile.read_dat(p).coords)


def test_thread_count_does_not_change_the_deck(tmp_path):
    d = decks.box_hex20_lognormal(24, 24, 18)
    p = decks.write_dat(d, str(tmp_path / "box"))
    assert os.path.getsize(p) > 3 << 20  # several parallel chunks per large block
    ref = datfile.read_dat(p, threads=1)
    same(ref, decks.read_dat(p))
    for t in (2, 3, 8):
        same(datfile.read_dat(p, threads=t), ref)


def test_node_records_are_numbered_by_position(tmp_path):
    # cNode::ReadCoord: the i-th record becomes node i+1 whatever label it states
    d = decks.cantilever_hex8(3, 2, 2)
    p = decks.write_dat(d, str(tmp_path / "lab"))
    lines = open(p).read().split("\n")
    i = lines.index("%NODE.COORD") + 2
    for k in range(d.num_nodes):
        t = lines[i + k].split()
        lines[i + k] = " ".join([str(1000 + k)] + t[1:])
    q = tmp_path / "lab2.dat"
    q.write_text("\n".join(lines))
    same(datfile.read_dat(str(q)), datfile.read_dat(p))


def _edit(tmp_path, fn):
    d = decks.cantilever_hex8(3, 2, 2)
    p = decks.write_dat(d, str(tmp_path / "x"))
    q = tmp_path / "bad.dat"
    q.write_text(fn(open(p).read()))
    return str(q)


def _err(path):
    with pytest.raises(datfile.DatError) as ei:
        datfile.read_dat(path)
    return ei.value


def test_deck_errors_are_reported_with_their_line(tmp_path):
    def bad_number(t):
        lines = t.split("\n")
        i = lines.index("%NODE.COORD") + 3
        lines[i] = lines[i].replace(" ", " 1.2.3 ", 1)
        return "\n".join(lines)
    e = _err(_edit(tmp_path, bad_number))
    assert e.rc == -1 and "not a number" in str(e) and "line" in str(e)

    def bad_node(t):
        lines = t.split("\n")
        i = lines.index("%ELEMENT.BRICK8") + 2
        tok = lines[i].split()
        tok[3] = "99999"
        lines[i] = " ".join(tok)
        return "\n".join(lines)
    assert "invalid node" in str(_err(_edit(tmp_path, bad_node)))

    def twice(t):
        lines = t.split("\n")
        i = lines.index("%ELEMENT.BRICK8") + 2
        tok = lines[i + 1].split()
        tok[0] = lines[i].split()[0]
        lines[i + 1] = " ".join(tok)
        return "\n".join(lines)
    assert "exactly once" in str(_err(_edit(tmp_path, twice)))

    def short(t):
        i = t.index("%ELEMENT.BRICK8")
        j = t.index("%", i + 1)
        return t[:j - 30] + "\n" + t[j:]
    assert "expected" in str(_err(_edit(tmp_path, short)))

    def bad_section(t):
        lines = t.split("\n")
        i = lines.index("%ELEMENT.BRICK8") + 2
        tok = lines[i].split()
        tok[1] = "7"
        lines[i] = " ".join(tok)
        return "\n".join(lines)
    assert "section" in str(_err(_edit(tmp_path, bad_section)))

    assert _err(str(tmp_path / "missing.dat")).rc == -1


def test_decks_outside_the_subset_are_refused(tmp_path):
    d, _ = gio.load("iga_p2_box")
    p = decks.write_dat(d, str(tmp_path / "bsp"))
    txt = open(p).read()
    q = tmp_path / "bsp_patch_kind.dat"
    q.write_text(txt.replace("'bspsol'", "'bspsurf'"))
    assert _err(str(q)).rc == -7

    def two_types(t):
        return t.replace("%END", "%ELEMENT.BRICK20\n0\n\n%END")
    assert _err(_edit(tmp_path, two_types)).rc == -7


def test_bucket_points_into_the_deck(tmp_path):
    d = decks.cantilever_hex8(4, 2, 2)
    p = decks.write_dat(d, str(tmp_path / "b"))
    L = datfile._lib()
    L.fast_dat_bucket.argtypes = [ctypes.c_void_p, ctypes.POINTER(gpu.Bucket)]
    h = ctypes.c_void_p()
    assert L.fast_dat_read(os.fsencode(p), 2, ctypes.byref(h)) == 0
    try:
        b = gpu.Bucket()
        assert L.fast_dat_bucket(h, ctypes.byref(b)) == 0
        assert b.elem_type == 1 and tuple(b.ngp) == tuple(d.ngp) and b.num_elems == d.num_elems
        conn = np.ctypeslib.as_array(b.conn, shape=(d.num_elems, 8))
        np.testing.assert_array_equal(conn, d.conn)
        np.testing.assert_array_equal(np.ctypeslib.as_array(b.E, shape=(d.num_elems,)), d.E)
        assert not b.rho and b.formulation == 0
    finally:
        L.fast_dat_free(h)


def same_patch(P, Q):
    assert P.degree == Q.degree and tuple(P.grid) == tuple(Q.grid) and P.rational == Q.rational
    for k in range(3):
        np.testing.assert_array_equal(P.knots[k], Q.knots[k])
    np.testing.assert_array_equal(P.span, Q.span)
    np.testing.assert_array_equal(P.cps, Q.cps)
    assert (P.weights is None) == (Q.weights is None)
    if P.weights is not None:
        np.testing.assert_array_equal(P.weights, Q.weights)


@pytest.mark.parametrize("name", BSP)
def test_bspline_decks_match_python_reader_and_reference(name, tmp_path):
    """%PATCH / %CONTROL.POINT.WEIGHT / %ELEMENT.BSPLINE.SOLID(TL): the native
    reader builds the same patch, spans and control-point incidence as the
    Python reader, and the reference's equation numbering."""
    d, g = gio.load(name)
    p = decks.write_dat(d, str(tmp_path / name))
    nat = datfile.read_dat(p)
    py = decks.read_dat(p)
    same(nat, py)
    same_patch(nat.patch, py.patch)
    np.testing.assert_array_equal(nat.node_eq(), g["ref_node_eq"])
    # the bucket view carries the patch
    L = datfile._lib()
    L.fast_dat_bucket.argtypes = [ctypes.c_void_p, ctypes.POINTER(gpu.Bucket)]
    h = ctypes.c_void_p()
    assert L.fast_dat_read(os.fsencode(p), 2, ctypes.byref(h)) == 0
    try:
        b = gpu.Bucket()
        assert L.fast_dat_bucket(h, ctypes.byref(b)) == 0
        assert b.elem_type == 3 and bool(b.patch)
        assert tuple(b.patch.contents.degree) == tuple(d.patch.degree)
        span = np.ctypeslib.as_array(b.patch.contents.span, shape=(d.num_elems, 3))
        np.testing.assert_array_equal(span, d.patch.span)
    finally:
        L.fast_dat_free(h)
