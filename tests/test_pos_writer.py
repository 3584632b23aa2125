"""The library's .pos writer (fast_pos_*, include/fast_pos.h) on the CPU:
byte for byte the files the reference's `fast` binary wrote, from the
numbers of the same runs (tests/golden/pos_output.npz, made by
tests/golden/make_golden.py pos)."""
import ctypes
import os
import re

import numpy as np
import pytest

from fast_b200 import build as fbuild
from fast_b200 import datfile
from oracle import fem_oracle as fo

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
G = dict(np.load(os.path.join(ROOT, "tests", "golden", "pos_output.npz")))


@pytest.fixture(scope="module", autouse=True)
def lib():
    fbuild.build()
    return datfile._lib()


def test_header_lists_every_export(lib):
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "fast_pos.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(fast_pos_[a-z_]+)\s*\(", txt)))
    assert names == sorted(datfile.POS_EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def _text(key):
    return G[key].tobytes()


def _node_displ(prefix):
    eq = G[prefix + "_ref_node_eq"].reshape(-1, 3)
    u = G[prefix + "_ref_u"]
    out = np.zeros(eq.shape)
    m = eq > 0
    out[m] = u[eq[m] - 1]
    return out


@pytest.mark.parametrize("prefix", ["hex8", "hex20"])
@pytest.mark.parametrize("threads", [1, 3])
def test_linear_static_file_is_the_reference_file(prefix, threads, tmp_path):
    dat = tmp_path / "deck.dat"
    dat.write_bytes(_text(prefix + "_dat"))
    ref = _text(prefix + "_pos")
    header = ref.split(b"\n")[1].decode()
    en = G[prefix + "_ref_elm_nodal_stress"]
    conn = G[prefix + "_conn"]
    avg = fo.averaged_nodal_stress(len(G[prefix + "_coords"]), conn, en)
    out = tmp_path / "out.pos"
    datfile.write_pos(str(out), str(dat), [dict(factor=1.0, displ=_node_displ(prefix),
                                               gauss_stress=G[prefix + "_ref_elm_stress"], elem_nodal=en,
                                               nodal_avg=avg)],
                      precision=15, max_steps=1, print_average=True, header_line=header, threads=threads)
    assert out.read_bytes() == ref


def _parse_steps(text):
    """Every printed step of a .pos: factor, displacements [n][3], Gauss and
    element-nodal stresses."""
    lines = text.decode().split("\n")
    steps, i = [], 0
    while i < len(lines):
        t = lines[i]
        if t == "%RESULT.CASE.STEP.FACTOR":
            steps.append({"factor": float(lines[i + 1])})
        elif t in ("%RESULT.CASE.STEP.NODAL.DISPLACEMENT", "%RESULT.CASE.STEP.VELOCITY",
                   "%RESULT.CASE.STEP.ACCELERATION"):
            n = int(lines[i + 1].split()[0])
            key = {"DISPLACEMENT": "displ", "VELOCITY": "velocity", "ACCELERATION": "acceleration"}[t.split(".")[-1]]
            steps[-1][key] = np.array([[float(v) for v in lines[i + 2 + k].split()[1:4]] for k in range(n)])
        elif t == "%RESULT.CASE.STEP.NODAL.REACTIONS":
            n = int(lines[i + 1].split()[0])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            steps[-1]["reaction_nodes"] = np.array([int(r[0]) - 1 for r in rows])
            steps[-1]["reactions"] = np.array([[float(v) for v in r[1:4]] for r in rows])
        elif t in ("%RESULT.CASE.STEP.ELEMENT.GAUSS.SCALAR.DATA", "%RESULT.CASE.STEP.ELEMENT.NODAL.SCALAR.DATA"):
            ne, j, blocks = int(lines[i + 1]), i + 2, []
            gauss = "GAUSS" in t
            for _ in range(ne):
                j += 1
                npt = int(lines[j]) if gauss else None
                j += 1 if gauss else 0
                rows = []
                while lines[j].startswith(("+", "-")):
                    rows.append([float(v) for v in lines[j].split()])
                    j += 1
                assert npt is None or npt == len(rows)
                blocks.append(rows)
            steps[-1]["gauss_stress" if gauss else "elem_nodal"] = np.array(blocks)
        i += 1
    return steps


def test_three_step_newton_file_is_the_reference_file(tmp_path):
    """Per-step blocks and the step list over the reserved area; every value
    read back from the reference's own print (precision 14) and re-printed."""
    dat = tmp_path / "deck.dat"
    dat.write_bytes(_text("steps_dat"))
    ref = _text("steps_pos")
    steps = _parse_steps(ref)
    assert len(steps) == 3
    out = tmp_path / "out.pos"
    datfile.write_pos(str(out), str(dat), steps, precision=14, max_steps=3, header_line=ref.split(b"\n")[1].decode())
    assert out.read_bytes() == ref


def test_step_list_longer_than_one_line_per_step(tmp_path):
    # 12 printed steps with max_steps 10: 1.1 * 10 gives 12 reserved lines,
    # the list needs 13 and overwrites the start of the first step header,
    # as the reference's seekp does
    dat = tmp_path / "d.dat"
    dat.write_text("%HEADER\nx\n\n%END\n")
    out = tmp_path / "o.pos"
    datfile.write_pos(str(out), str(dat), [dict(factor=0.1 * k, displ=np.zeros((1, 3))) for k in range(12)],
                      precision=3, max_steps=10, header_line="h")
    txt = out.read_bytes().decode()
    head = txt.split("%RESULT.CASE\n", 1)[1]
    listing = "1   12\n" + "".join(f"{i:<2}  'step{i}'\n" for i in range(1, 13))
    reserved = "             \n" * 12
    expect = listing + (reserved + "%RESULT.CASE.STEP\n1\n")[len(listing):]
    assert head.startswith(expect)
    assert txt.endswith("\n%END\n")


def test_number_format_is_iostream_scientific_showpos(tmp_path):
    dat = tmp_path / "d.dat"
    dat.write_text("%HEADER\nt\n%END\n")
    vals = np.array([[0.0, -0.0, 1.0], [-1.5e-300, 9.999999e99, 123456.789], [5e-324, -2.5, 1e100]])
    out = tmp_path / "o.pos"
    datfile.write_pos(str(out), str(dat), [dict(factor=0.5, displ=vals)], precision=5, header_line="h")
    rows = out.read_text().split("%RESULT.CASE.STEP.NODAL.DISPLACEMENT\n")[1].split("\n")[1:4]
    for r, v in zip(rows, vals):
        toks = r.split()
        assert toks[1:4] == [("%+.5e" % x) if not (x == 0 and np.signbit(x)) else "-0.00000e+00" for x in v]
        assert toks[4:] == ["+0.00000e+00"] * 3
    assert "%RESULT.CASE.STEP.FACTOR\n5.00000e-01\n" in out.read_text()


def test_echo_without_end_keeps_the_reference_quirk(tmp_path):
    # InpCopyData reads past the final newline and copies one empty line more
    dat = tmp_path / "d.dat"
    dat.write_text("%HEADER\nline one\n%NODE\n1\n")
    out = tmp_path / "o.pos"
    datfile.write_pos(str(out), str(dat), [], header_line="h")
    assert out.read_text() == "%HEADER\nh\nline one\n%NODE\n1\n\n\n%END\n1   0\n"


def test_bad_arguments(tmp_path):
    with pytest.raises(datfile.DatError):
        datfile.write_pos(str(tmp_path / "o.pos"), str(tmp_path / "missing.dat"), [])


def _parse_modes(text):
    lines = text.decode().split("\n")
    vals, shapes, kind = [], [], None
    for i, t in enumerate(lines):
        if t in ("%RESULT.CASE.STEP.NATURAL.FREQUENCY", "%RESULT.CASE.STEP.BUCKLING.FACTOR"):
            kind = datfile.POS_VIBRATION if "NATURAL" in t else datfile.POS_BUCKLING
            vals.append(float(lines[i + 1].split()[1]))
        elif t == "%RESULT.CASE.STEP.NODAL.EIGENVECTOR":
            n = int(lines[i + 1].split()[0])
            shapes.append([[float(v) for v in lines[i + 2 + k].split()[1:4]] for k in range(n)])
    return dict(kind=kind, values=np.array(vals), shapes=np.array(shapes))


@pytest.mark.parametrize("key", ["modal", "buck"])
def test_eigen_analysis_file_is_the_reference_file(key, tmp_path):
    """Modal (modes only, the step list after %END) and linear buckling (the
    linear step, then the modes): every value read back from the
    reference's print at precision 14 and re-printed."""
    dat = tmp_path / "deck.dat"
    dat.write_bytes(_text(key + "_dat"))
    ref = _text(key + "_pos")
    steps = _parse_steps(ref)
    modes = _parse_modes(ref)
    assert len(modes["values"]) == 3
    out = tmp_path / "out.pos"
    datfile.write_pos(str(out), str(dat), steps, precision=14, max_steps=1, modes=modes,
                      header_line=ref.split(b"\n")[1].decode())
    assert out.read_bytes() == ref


def test_newmark_file_is_the_reference_file(tmp_path):
    """Three printed Newmark steps: displacements, stresses, velocities and
    accelerations (cCtrlNewmark::PrintVelAcc), re-printed from the values."""
    dat = tmp_path / "deck.dat"
    dat.write_bytes(_text("newmark_dat"))
    ref = _text("newmark_pos")
    steps = _parse_steps(ref)
    assert len(steps) == 3 and all("velocity" in st and "acceleration" in st for st in steps)
    out = tmp_path / "out.pos"
    datfile.write_pos(str(out), str(dat), steps, precision=14, max_steps=3, header_line=ref.split(b"\n")[1].decode())
    assert out.read_bytes() == ref


def test_support_reactions_file_is_the_reference_file(tmp_path):
    """%HEADER.PRINT.SUPPORT.REACTIONS: the reactions block (five digits,
    right-aligned) after the displacements, and the step list padded the way
    the stream's alignment leaves it."""
    dat = tmp_path / "deck.dat"
    dat.write_bytes(_text("reac_dat"))
    ref = _text("reac_pos")
    steps = _parse_steps(ref)
    assert "reactions" in steps[0]
    out = tmp_path / "out.pos"
    datfile.write_pos(str(out), str(dat), steps, precision=14, max_steps=1, header_line=ref.split(b"\n")[1].decode())
    assert out.read_bytes() == ref
