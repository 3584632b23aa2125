"""CPU-only checks of the C ABI library: it builds for sm_100a, loads, exports
every entry point include/fast_gpu.h declares, and its host-only routines
agree with the reference.  No device compute is called here."""
import ctypes
import os
import re

import numpy as np
import pytest

from fast_b200 import build as fbuild
from fast_b200 import gpu
from tests import golden_io as gio

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


@pytest.fixture(scope="module")
def lib():
    fbuild.build()
    return gpu.load_library()


def header_functions():
    txt = open(os.path.join(ROOT, "include", "fast_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fast_gpu_[a-z0-9_]+)\s*\(", txt)))


def test_header_matches_binding_list():
    assert header_functions() == sorted(gpu.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_library_is_sm100a(lib):
    # the fatbin section carries sm_100a code; cuobjdump is not used, only the build flags
    assert "arch=compute_100a,code=sm_100a" in " ".join(fbuild.ARCH)


def test_abi_version(lib):
    assert lib.fast_gpu_version() == 1


@pytest.mark.parametrize("name", [n for n in gio.names() if not n.startswith(("nr_", "iga_", "arc_", "modal_"))])
def test_face_load_vector_matches_reference(lib, name):
    d, g = gio.load(name)
    f = gpu.face_load_vector(d)
    assert gio.rel(f, g["ref_f"]) < 1e-13


def test_face_load_rejects_bad_input(lib):
    f = np.zeros(3)
    rc = lib.fast_gpu_face_load_vector(1, None, None, 3, 0, 4, None, None, None, 2, f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == -1


def test_create_without_device_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    ctx = ctypes.c_void_p()
    rc = lib.fast_gpu_create(0, ctypes.byref(ctx))
    assert rc == -3 and not ctx.value


@pytest.mark.parametrize("name", ["cfg_hex8_cantilever", "cfg_hex20_lognormal_4x4x2", "ref_beamb20", "iga_p2_box",
                                  "iga_p3_box", "iga_scordelis_deg3"])
def test_host_pattern_matches_reference_structure(lib, name):
    """Node-block pattern covers exactly the reference's stored lower triangle,
    and no two elements of one colour share a node."""
    d, g = gio.load(name)
    p = gpu.inspect_pattern(d)
    assert p["nnz_lower_eq"] == (len(g["ref_K_data"]) if "ref_K_data" in g else p["nnz_lower_eq"])
    rp, col = p["rowptr"], p["col"]
    # rows sorted, diagonal present, symmetric
    for n in range(d.num_nodes):
        r = col[rp[n]:rp[n + 1]]
        assert np.all(np.diff(r) > 0) and n in r
    pairs = set()
    for n in range(d.num_nodes):
        for m in col[rp[n]:rp[n + 1]]:
            pairs.add((n, int(m)))
    assert all((m, n) in pairs for (n, m) in pairs)
    # colouring: elements of a colour are node-disjoint
    color = p["color"]
    for c in range(p["num_colors"]):
        nodes = d.conn[color == c].ravel()
        assert len(nodes) == len(np.unique(nodes))


def test_host_pattern_full_size_colours(lib):
    from fast_b200 import decks
    d = decks.box_hex20_lognormal(16, 16, 8)
    p = gpu.inspect_pattern(d)
    assert p["num_colors"] == 8
    assert p["nnz_blocks"] == len(p["col"])
