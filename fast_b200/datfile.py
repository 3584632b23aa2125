"""FAST ``.dat`` decks (hex8 / hex20 / B-spline solids) read by the library's
parallel reader (fast_dat_*),
and ``.pos`` result files written by its parallel writer (fast_pos_*).

``read_dat(path)`` returns the same :class:`fast_b200.decks.Deck` as the
pure-Python reader, for hex8 / hex20 (small-strain or total-Lagrangian)
decks, with the reference's record semantics (the i-th %NODE.COORD record is
node i+1; sections, materials and elements by label; integration orders by
position).  Decks outside that subset raise :class:`DatError` with the
library's status (``rc == -7`` for B-spline patches, ties, mixed types).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import decks, gpu


class DatInfo(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int64), ("num_elems", ctypes.c_int64), ("num_faces", ctypes.c_int64),
                ("nodes_per_face", ctypes.c_int32), ("elem_type", ctypes.c_int32),
                ("nodes_per_elem", ctypes.c_int32), ("formulation", ctypes.c_int32),
                ("ngp", ctypes.c_int32 * 3), ("has_density", ctypes.c_int32), ("has_solver_order", ctypes.c_int32),
                ("has_nodal_forces", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("max_steps", ctypes.c_int32),
                ("target_iter", ctypes.c_int32), ("print_step", ctypes.c_int32), ("has_arc_length", ctypes.c_int32),
                ("tol", ctypes.c_double), ("step_factor", ctypes.c_double), ("arc_load_coeff", ctypes.c_double),
                ("time_step", ctypes.c_double), ("newmark", ctypes.c_double * 2),
                ("algorithm", ctypes.c_char * 32), ("matrix_type", ctypes.c_char * 32), ("title", ctypes.c_char * 128),
                ("patch_degree", ctypes.c_int32 * 3), ("patch_num_knots", ctypes.c_int32 * 3),
                ("patch_rational", ctypes.c_int32), ("has_weights", ctypes.c_int32), ("patch_num_cps", ctypes.c_int64)]


class PosOpts(ctypes.Structure):
    _fields_ = [("header_line", ctypes.c_char_p), ("precision", ctypes.c_int32), ("max_steps", ctypes.c_int32),
                ("print_average", ctypes.c_int32), ("threads", ctypes.c_int32)]


POS_EXPORTS = ["fast_pos_open", "fast_pos_step", "fast_pos_reactions", "fast_pos_velacc", "fast_pos_modes", "fast_pos_finish", "fast_pos_error",
               "fast_pos_free"]
POS_VIBRATION, POS_BUCKLING = 0, 1

EXPORTS = ["fast_dat_read", "fast_dat_error", "fast_dat_free", "fast_dat_get_info", "fast_dat_get_nodes",
           "fast_dat_get_elements", "fast_dat_get_faces", "fast_dat_get_patch", "fast_dat_bucket"]


class DatError(RuntimeError):
    def __init__(self, rc, msg):
        super().__init__(f"fast_dat_read failed ({rc}): {msg}")
        self.rc = rc


def _lib():
    L = gpu.load_library()
    if getattr(L, "_dat_bound", False):
        return L
    vp = ctypes.c_void_p
    L.fast_dat_read.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(vp)]
    L.fast_dat_error.argtypes = [vp]
    L.fast_dat_error.restype = ctypes.c_char_p
    L.fast_dat_free.argtypes = [vp]
    L.fast_dat_free.restype = None
    L.fast_dat_get_info.argtypes = [vp, ctypes.POINTER(DatInfo)]
    L.fast_dat_get_nodes.argtypes = [vp, vp, vp, vp, vp]
    L.fast_dat_get_elements.argtypes = [vp, vp, vp, vp, vp]
    L.fast_dat_get_faces.argtypes = [vp, vp, vp, vp, vp, vp]
    L.fast_dat_get_patch.argtypes = [vp, vp, vp, vp, vp]
    L.fast_pos_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(PosOpts), ctypes.POINTER(vp)]
    L.fast_pos_step.argtypes = [vp, ctypes.c_double, ctypes.c_int64, vp, ctypes.c_int64, ctypes.c_int32, vp,
                                ctypes.c_int32, vp, vp]
    L.fast_pos_velacc.argtypes = [vp, ctypes.c_int64, vp, vp]
    L.fast_pos_reactions.argtypes = [vp, ctypes.c_int64, vp, vp]
    L.fast_pos_modes.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int64, vp]
    L.fast_pos_finish.argtypes = [vp]
    L.fast_pos_error.argtypes = [vp]
    L.fast_pos_error.restype = ctypes.c_char_p
    L.fast_pos_free.argtypes = [vp]
    L.fast_pos_free.restype = None
    L._dat_bound = True
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def read_dat(path: str, threads: int = 0) -> decks.Deck:
    """Read a hex8 / hex20 FAST deck with ``threads`` host threads (0: all)."""
    L = _lib()
    h = ctypes.c_void_p()
    rc = L.fast_dat_read(os.fsencode(path), int(threads), ctypes.byref(h))
    try:
        if rc != 0:
            msg = L.fast_dat_error(h).decode(errors="replace") if h else "out of memory"
            raise DatError(rc, msg)
        I = DatInfo()
        L.fast_dat_get_info(h, ctypes.byref(I))
        n, ne, nf, nn = I.num_nodes, I.num_elems, I.num_faces, I.nodes_per_elem
        coords = np.empty((n, 3))
        fixed = np.empty((n, 3), np.uint8)
        rank = np.empty(n, np.int64)
        nodal = np.empty((n, 3))
        L.fast_dat_get_nodes(h, _ptr(coords), _ptr(fixed), _ptr(rank), _ptr(nodal))
        conn = np.empty((ne, nn), np.int32)
        E, nu, rho = np.empty(ne), np.empty(ne), np.empty(ne)
        L.fast_dat_get_elements(h, _ptr(conn), _ptr(E), _ptr(nu), _ptr(rho))
        patch = None
        if I.elem_type == 3:
            nk = list(I.patch_num_knots)
            knots = np.empty(sum(nk))
            span = np.empty((ne, 3), np.int32)
            wts = np.empty(n)
            cps = np.empty(I.patch_num_cps, np.int32)
            L.fast_dat_get_patch(h, _ptr(knots), _ptr(span), _ptr(wts), _ptr(cps))
            deg = tuple(int(v) for v in I.patch_degree)
            kv = [knots[sum(nk[:k]):sum(nk[:k + 1])].copy() for k in range(3)]
            grid = tuple(len(kv[k]) - deg[k] - 1 for k in range(3))
            patch = decks.Patch(deg, kv, span, grid, cps.astype(np.int64), wts if I.has_weights else None,
                                bool(I.patch_rational))
        fe = fc = fq = fl = None
        if nf:
            fe = np.empty(nf, np.int32)
            fc = np.empty((nf, 3), np.int32)
            fnodes = np.empty((nf, I.nodes_per_face), np.int32)
            fl = np.empty(nf, np.int32)
            fq = np.empty((nf, 3))
            L.fast_dat_get_faces(h, _ptr(fe), _ptr(fc), _ptr(fnodes), _ptr(fl), _ptr(fq))
    finally:
        if h:
            L.fast_dat_free(h)
    kind = {gpu_elem: k for k, gpu_elem in (("hex8", 1), ("hex20", 2), ("bsp", 3))}[I.elem_type]
    return decks.Deck(kind, coords, conn, E, nu, tuple(int(v) for v in I.ngp), fixed.astype(bool), fe, fc, fq, fl,
                      rho if I.has_density else None, bool(I.formulation == 1),
                      algorithm=I.algorithm.decode() or "linear", matrix_type=I.matrix_type.decode() or "skyline",
                      tol=I.tol, maxit=I.max_iter, maxstep=I.max_steps, step_factor=I.step_factor,
                      time_step=I.time_step, arc_load_coeff=I.arc_load_coeff if I.has_arc_length else None,
                      target_iter=I.target_iter if I.target_iter >= 0 else None,
                      newmark=(I.newmark[0], I.newmark[1]), print_step=I.print_step,
                      node_labels=np.arange(1, n + 1, dtype=np.int64), title=os.path.basename(path),
                      nodal_f=nodal if I.has_nodal_forces else None,
                      solver_rank=rank if I.has_solver_order else None, patch=patch)


def _arr(a, shape=None):
    if a is None:
        return None, None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a, a.ctypes.data_as(ctypes.c_void_p)


def write_pos(pos_path: str, dat_path: str, steps, precision: int = 5, max_steps: int = 1,
              print_average: bool = False, header_line: str = None, threads: int = 0, modes=None) -> None:
    """Write a FAST ``.pos`` file: the deck's echo, then one printed step per
    entry of ``steps`` (dicts with ``factor``, ``displ`` [nnode][3] and
    optionally ``gauss_stress`` [ne][points][6], ``elem_nodal`` [ne][nn][6],
    ``nodal_avg`` [nnode][6], ``reaction_nodes`` [k] with ``reactions``
    [k][3], and for Newmark ``velocity`` and ``acceleration`` [nnode][3]),
    then, when ``modes`` is given, the modes of an
    eigen analysis: a dict with ``kind`` (POS_VIBRATION / POS_BUCKLING),
    ``values`` [p] (frequencies or buckling factors) and ``shapes``
    [p][nnode][3]."""
    L = _lib()
    o = PosOpts(header_line.encode() if header_line is not None else None, int(precision), int(max_steps),
                int(bool(print_average)), int(threads))
    h = ctypes.c_void_p()
    try:
        rc = L.fast_pos_open(os.fsencode(pos_path), os.fsencode(dat_path), ctypes.byref(o), ctypes.byref(h))
        if rc != 0:
            raise DatError(rc, L.fast_pos_error(h).decode(errors="replace") if h else "out of memory")
        for st in steps:
            if st.get("reactions") is not None:
                rn = np.ascontiguousarray(st["reaction_nodes"], dtype=np.int64)
                rv, rp_ = _arr(st["reactions"])
                rc = L.fast_pos_reactions(h, len(rn), rn.ctypes.data_as(ctypes.c_void_p), rp_)
                if rc != 0:
                    raise DatError(rc, L.fast_pos_error(h).decode(errors="replace"))
            u, up = _arr(st["displ"])
            gs, gp = _arr(st.get("gauss_stress"))
            en, ep = _arr(st.get("elem_nodal"))
            av, ap = _arr(st.get("nodal_avg"))
            ne = gs.shape[0] if gs is not None else (en.shape[0] if en is not None else 0)
            rc = L.fast_pos_step(h, float(st["factor"]), u.shape[0], up, ne, gs.shape[1] if gs is not None else 0,
                                 gp, en.shape[1] if en is not None else 0, ep, ap)
            if rc != 0:
                raise DatError(rc, L.fast_pos_error(h).decode(errors="replace"))
            if st.get("velocity") is not None:
                v, vp2 = _arr(st["velocity"])
                a, ap2 = _arr(st["acceleration"])
                rc = L.fast_pos_velacc(h, v.shape[0], vp2, ap2)
                if rc != 0:
                    raise DatError(rc, L.fast_pos_error(h).decode(errors="replace"))
        if modes is not None:
            vals, vp_ = _arr(modes["values"])
            shp, sp_ = _arr(modes["shapes"])
            rc = L.fast_pos_modes(h, int(modes["kind"]), len(vals), vp_, shp.shape[1], sp_)
            if rc != 0:
                raise DatError(rc, L.fast_pos_error(h).decode(errors="replace"))
        rc = L.fast_pos_finish(h)
        if rc != 0:
            raise DatError(rc, L.fast_pos_error(h).decode(errors="replace"))
    finally:
        if h:
            L.fast_pos_free(h)
