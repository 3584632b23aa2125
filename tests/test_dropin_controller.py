"""The drop-in, end to end: the reference's own, unmodified FAST program
(every object file of its sources, main included) linked with the device
binding fast_b200/shim/fast_shim.cpp and libfastgpu.so (`oracle/_ref/fastgpu`,
built by `make -C oracle gpu`).

* CPU: for decks that do not ask for the device matrix, the binding hands
  every call back to the reference's functions, so its .pos files are byte
  for byte those of the plain `fast` binary.
* GPU: a deck with %HEADER.ANALYSIS.MATRIX.TYPE 'gpu' runs cLinStat::Solver
  (ctrl/ctrllins.cpp:46-99) unchanged: ExtLoadVector and the printing on the
  host, CreateMatrix / StiffnessMatrix / Solve on the device; the printed
  displacements equal the reference's own solution (1e-9 relative).
"""
import os
import subprocess

import numpy as np
import pytest

from fast_b200 import decks
from tests import golden_io as gio

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
FAST = os.path.join(ROOT, "oracle", "_ref", "fast")
FASTGPU = os.path.join(ROOT, "oracle", "_ref", "fastgpu")
TOL_U = 1e-9

CASES = [("cfg_hex8_cantilever", "skyline"), ("cfg_hex20_lognormal_4x4x2", "sparse")]


def _require_binaries():
    for b in (FAST, FASTGPU):
        assert os.path.exists(b), f"{b} missing: build it with make -C oracle FAST_REF=<reference tree> ref gpu"


def _run(binary, deck, base):
    decks.write_dat(deck, base)
    r = subprocess.run([binary, base, "-silent"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (binary, r.stdout[-2000:], r.stderr[-2000:])
    with open(base + ".pos", "rb") as fh:
        return fh.read()


def _deck(name, matrix_type):
    d, g = gio.load(name)
    d.matrix_type = matrix_type
    d.tol = 1e-12
    d.maxit = 100000
    return d, g


@pytest.mark.parametrize("name,cpu_type", CASES)
def test_binding_is_transparent_for_other_matrix_types(name, cpu_type, tmp_path):
    _require_binaries()
    d, _ = _deck(name, cpu_type)
    a = _run(FAST, d, str(tmp_path / "plain"))
    b = _run(FASTGPU, d, str(tmp_path / "bound"))
    assert a == b


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,cpu_type", CASES)
def test_unmodified_linear_static_controller_on_the_device_matrix(name, cpu_type, precision, tmp_path, monkeypatch):
    _require_binaries()
    monkeypatch.setenv("FAST_GPU_PRECISION", precision)
    d, g = _deck(name, "gpu")
    _run(FASTGPU, d, str(tmp_path / "gpu"))
    u_gpu = decks.read_pos_displacements(str(tmp_path / "gpu.pos"))[-1]
    dc, _ = _deck(name, cpu_type)
    _run(FAST, dc, str(tmp_path / "cpu"))
    u_cpu = decks.read_pos_displacements(str(tmp_path / "cpu.pos"))[-1]
    # the reference's own solution (fixture) mapped to nodes
    eq = g["ref_node_eq"].reshape(-1, 3)
    u_ref = np.where(eq > 0, g["ref_u"][np.maximum(eq, 1) - 1], 0.0)
    assert gio.rel(u_gpu, u_ref) < TOL_U
    assert gio.rel(u_gpu, u_cpu) < TOL_U
