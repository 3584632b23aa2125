"""ctypes binding of libfastgpu.so (the C ABI in include/fast_gpu.h).

:class:`GpuSystem` mirrors the part of FAST's interface the C ABI replaces:

* ``upload(deck)``           - cControl::Init's equation/profile set-up
                               (ctrl/ctrl.cpp:2004-2157) for the device matrix;
* ``assemble()``             - cControl::StiffnessMatrix (ctrl/ctrl.cpp:886-975);
* ``assemble_mass()``        - cControl::MassMatrix (ctrl/ctrl.cpp:979-1027);
* ``add/get/mult_vect``      - cSysMatrix::Add/Get/MultVect (mlib/sysmat.h:60-99);
* ``solve(f)``               - cSysMatrix::Solve -> PCGSolver (mlib/sysmat.cpp:1061-1125);
* ``ext_load(deck)``         - cControl::ExtLoadVector for face tractions.

There is no CPU fallback: if the library is missing or no CUDA device is
present, constructing a :class:`GpuSystem` raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import decks as _decks

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfastgpu.so")

FAST_GPU_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ESTATE", -5: "ENONCONV", -6: "EDETJ", -7: "ENOTSUP",
          -8: "ENOTFOUND", -9: "ETOOBIG"}
ELEM = {"hex8": 1, "hex20": 2, "bsp": 3}
ASM_K, ASM_M, ASM_G, ASM_K_TF32 = 1, 2, 3, 4
FORM_SMALL, FORM_TL = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
PRECOND_JACOBI, PRECOND_BLOCK_JACOBI = 0, 1

# Every entry point the header declares; the CPU test checks the library exports all of them.
EXPORTS = [
    "fast_gpu_create", "fast_gpu_destroy", "fast_gpu_last_error", "fast_gpu_version", "fast_gpu_set_stream",
    "fast_gpu_synchronize", "fast_gpu_upload_mesh", "fast_gpu_pattern_info", "fast_gpu_update_coords",
    "fast_gpu_update_material", "fast_gpu_zero", "fast_gpu_assemble", "fast_gpu_add", "fast_gpu_add_mat", "fast_gpu_get",
    "fast_gpu_mult_vect", "fast_gpu_solve", "fast_gpu_solve_device", "fast_gpu_face_load_vector",
    "fast_gpu_get_lower_csr", "fast_gpu_element_matrices", "fast_gpu_launch_count", "fast_gpu_kernel_timing", "fast_gpu_kernel_stats",
    "fast_gpu_inspect_pattern", "fast_gpu_pcg_solve_noalloc", "fast_gpu_set_displacement",
    "fast_gpu_set_displacement_device", "fast_gpu_internal_force", "fast_gpu_internal_force_device",
    "fast_gpu_nr_solve", "fast_gpu_ws_create", "fast_gpu_ws_destroy", "fast_gpu_ws_add_trajectory",
    "fast_gpu_ws_build_basis", "fast_gpu_ws_train", "fast_gpu_ws_predict", "fast_gpu_ws_report", "fast_gpu_autotune", "fast_gpu_set_face_loads", "fast_gpu_gauss_stress",
    "fast_gpu_face_load_device", "fast_gpu_arclength_solve", "fast_gpu_nodal_stress", "fast_gpu_modal", "fast_gpu_buckling", "fast_gpu_support_reactions",
    "fast_gpu_ws_get_basis", "fast_gpu_ws_get_samples", "fast_gpu_mlp_params", "fast_gpu_mlp_forward",
    "fast_gpu_mlp_loss_grad", "fast_gpu_mlp_gemm", "fast_gpu_ws_configure", "fast_gpu_ws_last_input",
    "fast_gpu_set_option", "fast_gpu_set_problems", "fast_gpu_solve_batch", "fast_gpu_newmark",
]
OPT_PERSISTENT_MAX_NODES, OPT_SPMV_LANES_FP32, OPT_SPMV_LANES_FP64, OPT_GRAPH_STEPS = 1, 2, 3, 4
OPT_SPMV_BULK_FP32 = 5
OPT_ELEM_SHAPE = 6
OPT_ZERO_FILL = 7
OPT_PERSISTENT_ASSEMBLY = 8
OPT_SPMV_STREAM_FP32 = 9
OPT_SPMV_COL16_FP32 = 10
OPT_FORCE_GATHER = 11


def elem_shape(bucket: int, ctas: int = 0, split: int = 0, tc_ctas: int = 0, kernel: int = 0) -> int:
    """The value of OPT_ELEM_SHAPE for one bucket (each field 0..255, 0 = default;
    kernel 1: the FP64 hex stiffness with one warp per element)."""
    for v in (ctas, split, tc_ctas):
        assert 0 <= v <= 255
    assert kernel in (0, 1)
    return (int(kernel) << 32) | (int(bucket) << 24) | (tc_ctas << 16) | (split << 8) | ctas
KERNEL_SPMV_FP64, KERNEL_SPMV_FP32, KERNEL_ASSEMBLE = 0, 1, 2
KERNEL_PREDICT_NET, KERNEL_PREDICT_GALERKIN, KERNEL_INTERNAL_FORCE, KERNEL_LINEAR_SOLVE = 3, 4, 5, 6
KERNEL_ASSEMBLE_TF32 = 7


class FastGpuError(RuntimeError):
    def __init__(self, rc, msg=""):
        super().__init__(f"{ERRORS.get(rc, rc)}: {msg}")
        self.rc = rc


class Patch(ctypes.Structure):
    _fields_ = [("degree", ctypes.c_int32 * 3), ("num_knots", ctypes.c_int32 * 3),
                ("knots", ctypes.POINTER(ctypes.c_double) * 3), ("span", ctypes.POINTER(ctypes.c_int32)),
                ("weights", ctypes.POINTER(ctypes.c_double)), ("rational", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Bucket(ctypes.Structure):
    _fields_ = [("elem_type", ctypes.c_int32), ("ngp", ctypes.c_int32 * 3), ("num_elems", ctypes.c_int64),
                ("conn", ctypes.POINTER(ctypes.c_int32)), ("E", ctypes.POINTER(ctypes.c_double)),
                ("nu", ctypes.POINTER(ctypes.c_double)), ("rho", ctypes.POINTER(ctypes.c_double)),
                ("formulation", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("patch", ctypes.POINTER(Patch))]


class Ties(ctypes.Structure):
    _fields_ = [("num_slaves", ctypes.c_int64), ("slave", ctypes.POINTER(ctypes.c_int64)),
                ("ptr", ctypes.POINTER(ctypes.c_int64)), ("master", ctypes.POINTER(ctypes.c_int64)),
                ("weight", ctypes.POINTER(ctypes.c_double))]


class Mesh(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int64), ("coords", ctypes.POINTER(ctypes.c_double)),
                ("node_eq", ctypes.POINTER(ctypes.c_int32)), ("num_eq", ctypes.c_int32),
                ("num_buckets", ctypes.c_int32), ("buckets", ctypes.POINTER(Bucket)),
                ("ties", ctypes.POINTER(Ties))]


class SolveOpts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("precond", ctypes.c_int32), ("maxit", ctypes.c_int32),
                ("warm_start", ctypes.c_int32), ("tol", ctypes.c_double), ("inner_tol", ctypes.c_double),
                ("max_outer", ctypes.c_int32), ("check_every", ctypes.c_int32)]


class SolveReport(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int32), ("iterations", ctypes.c_int32), ("outer", ctypes.c_int32),
                ("escalated", ctypes.c_int32), ("rel_residual", ctypes.c_double),
                ("true_rel_residual", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ModalOpts(ctypes.Structure):
    _fields_ = [("num_modes", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("tol", ctypes.c_double),
                ("lin", SolveOpts)]


class ModalReport(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int32), ("iterations", ctypes.c_int32), ("linear_iterations", ctypes.c_int32),
                ("subspace", ctypes.c_int32), ("max_err", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


ARC_INITIAL_NORMAL, ARC_UPDATED_NORMAL, ARC_LINEARIZED = 1, 2, 3
ARC_METHODS = {"ioal": ARC_INITIAL_NORMAL, "uoal": ARC_UPDATED_NORMAL, "clinal": ARC_LINEARIZED}


class ArcOpts(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("steps", ctypes.c_int32), ("max_iter", ctypes.c_int32),
                ("target_iter", ctypes.c_int32), ("step_factor", ctypes.c_double), ("tol", ctypes.c_double),
                ("load_coeff", ctypes.c_double), ("lin", SolveOpts)]


class ArcReport(ctypes.Structure):
    _fields_ = [("converged_steps", ctypes.c_int32), ("failed_step", ctypes.c_int32),
                ("iterations", ctypes.c_int32), ("linear_iterations", ctypes.c_int32),
                ("last_err", ctypes.c_double), ("arc_length", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NrOpts(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("step_factor", ctypes.c_double),
                ("tol", ctypes.c_double), ("predictor", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("lin", SolveOpts), ("lin_tol_rel", ctypes.c_double), ("lin_tol_min", ctypes.c_double),
                ("lin_tol_max", ctypes.c_double)]


class NrReport(ctypes.Structure):
    _fields_ = [("converged_steps", ctypes.c_int32), ("failed_step", ctypes.c_int32),
                ("iterations", ctypes.c_int32), ("linear_iterations", ctypes.c_int32),
                ("secant_starts", ctypes.c_int32), ("predictions", ctypes.c_int32),
                ("predictions_accepted", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("last_err", ctypes.c_double), ("last_rel_residual", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# int (*)(void *user, int32 step, double lambda, const double *d_u_last, const double *d_u_prev, const double *d_f,
#         double *d_u_pred)
NR_PREDICTOR = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)
PREDICT_NONE, PREDICT_SECANT, PREDICT_CALLBACK = 0, 1, 2


class NewmarkOpts(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("damping", ctypes.c_int32), ("dt", ctypes.c_double),
                ("gamma", ctypes.c_double), ("beta", ctypes.c_double), ("lin", SolveOpts), ("mass", SolveOpts),
                ("omega1", ctypes.c_double), ("omega2", ctypes.c_double), ("xi1", ctypes.c_double),
                ("xi2", ctypes.c_double)]


class NewmarkReport(ctypes.Structure):
    _fields_ = [("steps_done", ctypes.c_int32), ("failed_step", ctypes.c_int32),
                ("linear_iterations", ctypes.c_int32), ("max_step_iterations", ctypes.c_int32),
                ("mass_iterations", ctypes.c_int32), ("escalated_steps", ctypes.c_int32),
                ("umax", ctypes.c_double), ("vmax", ctypes.c_double), ("amax", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneReport(ctypes.Structure):
    _fields_ = [("lanes_fp32", ctypes.c_int32), ("lanes_fp64", ctypes.c_int32), ("ms_fp32", ctypes.c_double * 4),
                ("ms_fp64", ctypes.c_double * 4), ("persistent_max_nodes", ctypes.c_int64),
                ("us_iter_persistent", ctypes.c_double), ("us_iter_kernels", ctypes.c_double),
                ("ms_fp32_bulk", ctypes.c_double * 2), ("bulk_fp32", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("elem_buckets", ctypes.c_int32), ("elem_tc", ctypes.c_int32), ("elem_ctas", ctypes.c_int32 * 8),
                ("elem_split", ctypes.c_int32 * 8), ("elem_tc_ctas", ctypes.c_int32 * 8),
                ("elem_ms_default", ctypes.c_double * 8), ("elem_ms_tuned", ctypes.c_double * 8),
                ("elem_tc_ms_default", ctypes.c_double * 8), ("elem_tc_ms_tuned", ctypes.c_double * 8),
                ("ms_fp32_stream", ctypes.c_double * 2), ("stream_fp32", ctypes.c_int32), ("reserved2", ctypes.c_int32),
                ("us_iter_mixed", ctypes.c_double * 6), ("us_iter_mixed_col16", ctypes.c_double * 2),
                ("col16_fp32", ctypes.c_int32), ("reserved3", ctypes.c_int32), ("elem_kernel", ctypes.c_int32 * 8)]

    def as_dict(self):
        return {"lanes_fp32": self.lanes_fp32, "lanes_fp64": self.lanes_fp64,
                "ms_fp32_lanes_4_8_16_32": list(self.ms_fp32), "ms_fp64_lanes_4_8_16_32": list(self.ms_fp64),
                "ms_fp32_bulk_lanes_8_16": list(self.ms_fp32_bulk), "bulk_fp32": bool(self.bulk_fp32),
                "persistent_max_nodes": self.persistent_max_nodes, "us_iter_persistent": self.us_iter_persistent,
                "us_iter_kernels": self.us_iter_kernels,
                "elements": [{"kernel": "warp" if self.elem_kernel[b] == 1 else "cta",
                              "ctas_per_sm": self.elem_ctas[b], "split": self.elem_split[b],
                              "ms_default": self.elem_ms_default[b], "ms_tuned": self.elem_ms_tuned[b],
                              "tc_ctas_per_sm": self.elem_tc_ctas[b], "tc_ms_default": self.elem_tc_ms_default[b],
                              "tc_ms_tuned": self.elem_tc_ms_tuned[b]} for b in range(self.elem_buckets)],
                "elements_tensor_core_timed": bool(self.elem_tc),
                "ms_fp32_stream_lanes_8_16": list(self.ms_fp32_stream), "stream_fp32": bool(self.stream_fp32),
                "us_per_mixed_iteration_plain_8_16_stream_8_16_bulk_8_16": list(self.us_iter_mixed),
                "us_per_mixed_iteration_col16_8_16": list(self.us_iter_mixed_col16),
                "col16_fp32": bool(self.col16_fp32)}


class ProblemReport(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int32), ("iterations", ctypes.c_int32), ("rel_residual", ctypes.c_double)]


class WsOpts(ctypes.Structure):
    _fields_ = [("modes", ctypes.c_int32), ("history", ctypes.c_int32), ("width", ctypes.c_int32),
                ("hidden", ctypes.c_int32), ("oversample", ctypes.c_int32), ("power_iters", ctypes.c_int32),
                ("seed", ctypes.c_uint64)]


class WsStats(ctypes.Structure):
    _fields_ = [("trajectories", ctypes.c_int32), ("snapshots", ctypes.c_int32), ("samples", ctypes.c_int32),
                ("modes", ctypes.c_int32), ("input_dim", ctypes.c_int32), ("output_dim", ctypes.c_int32),
                ("epochs", ctypes.c_int32), ("reserved", ctypes.c_int32), ("params", ctypes.c_int64),
                ("captured_energy", ctypes.c_double), ("basis_ms", ctypes.c_double), ("train_ms", ctypes.c_double),
                ("first_loss", ctypes.c_float), ("last_loss", ctypes.c_float), ("launches", ctypes.c_int64),
                ("predictions", ctypes.c_int64), ("galerkin_iterations", ctypes.c_int64),
                ("predict_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lp = ctypes.POINTER(ctypes.c_int64)


def load_library(path: str = LIB_PATH):
    """Load libfastgpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FastGpuError(-4, f"{path} is missing: build it with `python -m fast_b200.build`")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.fast_gpu_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.fast_gpu_destroy.argtypes = [vp]
    L.fast_gpu_last_error.argtypes = [vp]
    L.fast_gpu_last_error.restype = ctypes.c_char_p
    L.fast_gpu_set_stream.argtypes = [vp, vp]
    L.fast_gpu_synchronize.argtypes = [vp]
    L.fast_gpu_set_option.argtypes = [vp, ctypes.c_int32, ctypes.c_int64]
    L.fast_gpu_autotune.argtypes = [vp, vp]
    L.fast_gpu_gauss_stress.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, vp, vp]
    L.fast_gpu_nodal_stress.argtypes = [vp, ctypes.c_int32, vp, vp]
    L.fast_gpu_support_reactions.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_int32, vp,
                                             ctypes.c_double, vp]
    L.fast_gpu_set_face_loads.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_int32]
    L.fast_gpu_face_load_device.argtypes = [vp, ctypes.c_double, vp]
    L.fast_gpu_set_problems.argtypes = [vp, ctypes.c_int32, _lp]
    L.fast_gpu_newmark.argtypes = [vp, _dp, ctypes.POINTER(NewmarkOpts), _dp, _dp, _dp, ctypes.c_int32, _ip, _dp,
                                   ctypes.POINTER(NewmarkReport)]
    L.fast_gpu_solve_batch.argtypes = [vp, _dp, _dp, ctypes.POINTER(SolveOpts), ctypes.POINTER(ProblemReport)]
    L.fast_gpu_upload_mesh.argtypes = [vp, ctypes.POINTER(Mesh)]
    L.fast_gpu_pattern_info.argtypes = [vp, _lp, _lp, _ip, _dp]
    L.fast_gpu_update_coords.argtypes = [vp, _dp]
    L.fast_gpu_update_material.argtypes = [vp, ctypes.c_int32, _dp, _dp]
    L.fast_gpu_zero.argtypes = [vp, ctypes.c_int32]
    L.fast_gpu_assemble.argtypes = [vp, ctypes.c_int32]
    L.fast_gpu_add.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double]
    L.fast_gpu_add_mat.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_int32]
    L.fast_gpu_get.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _dp]
    L.fast_gpu_mult_vect.argtypes = [vp, ctypes.c_int32, _dp, _dp]
    L.fast_gpu_solve.argtypes = [vp, _dp, _dp, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveReport)]
    L.fast_gpu_solve_device.argtypes = [vp, vp, vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveReport)]
    L.fast_gpu_face_load_vector.argtypes = [ctypes.c_int64, _dp, _ip, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            _ip, _dp, _ip, ctypes.c_int32, _dp]
    L.fast_gpu_get_lower_csr.argtypes = [vp, ctypes.c_int32, _lp, _lp, _ip, _dp]
    L.fast_gpu_element_matrices.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, _dp]
    L.fast_gpu_launch_count.argtypes = [vp, _lp]
    L.fast_gpu_pcg_solve_noalloc.argtypes = [ctypes.c_int32, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int32, vp,
                                             ctypes.POINTER(SolveReport)]
    L.fast_gpu_inspect_pattern.argtypes = [ctypes.POINTER(Mesh), _lp, _lp, _ip, _ip, _ip, _ip]
    L.fast_gpu_set_displacement.argtypes = [vp, _dp]
    L.fast_gpu_set_displacement_device.argtypes = [vp, vp]
    L.fast_gpu_internal_force.argtypes = [vp, _dp]
    L.fast_gpu_internal_force_device.argtypes = [vp, vp]
    L.fast_gpu_nr_solve.argtypes = [vp, _dp, ctypes.POINTER(NrOpts), NR_PREDICTOR, vp, _dp, _ip,
                                    ctypes.POINTER(NrReport)]
    L.fast_gpu_modal.argtypes = [vp, ctypes.POINTER(ModalOpts), _dp, _dp, ctypes.POINTER(ModalReport)]
    L.fast_gpu_buckling.argtypes = [vp, _dp, ctypes.POINTER(ModalOpts), _dp, _dp, _dp, ctypes.POINTER(ModalReport)]
    L.fast_gpu_arclength_solve.argtypes = [vp, _dp, ctypes.POINTER(ArcOpts), _dp, _dp, _ip,
                                           ctypes.POINTER(ArcReport)]
    _fp = ctypes.POINTER(ctypes.c_float)
    L.fast_gpu_ws_create.argtypes = [vp, ctypes.POINTER(WsOpts), ctypes.POINTER(vp)]
    L.fast_gpu_ws_destroy.argtypes = [vp]
    L.fast_gpu_ws_destroy.restype = None
    L.fast_gpu_ws_add_trajectory.argtypes = [vp, ctypes.c_int32, _dp, _dp]
    L.fast_gpu_ws_build_basis.argtypes = [vp, _dp]
    L.fast_gpu_ws_train.argtypes = [vp, ctypes.c_int32, ctypes.c_float, _fp]
    L.fast_gpu_ws_predict.argtypes = [vp, ctypes.c_int32, ctypes.c_double, vp, vp, vp, vp]
    L.fast_gpu_ws_configure.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double]
    L.fast_gpu_ws_last_input.argtypes = [vp, _fp]
    L.fast_gpu_ws_report.argtypes = [vp, ctypes.POINTER(WsStats)]
    L.fast_gpu_ws_get_basis.argtypes = [vp, _dp]
    L.fast_gpu_ws_get_samples.argtypes = [vp, _fp, _fp]
    L.fast_gpu_mlp_params.argtypes = [vp, _fp, _fp, _lp]
    L.fast_gpu_mlp_forward.argtypes = [vp, ctypes.c_int32, _fp, _fp]
    L.fast_gpu_mlp_loss_grad.argtypes = [vp, ctypes.c_int32, _fp, _fp, _fp, _fp]
    L.fast_gpu_mlp_gemm.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _fp, ctypes.c_int32, _fp,
                                    ctypes.c_int32, _fp]
    L.fast_gpu_kernel_timing.argtypes = [vp, ctypes.c_int32]
    L.fast_gpu_kernel_stats.argtypes = [vp, ctypes.c_int32, _lp, _dp, _dp]
    _lib = L
    return L


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def face_load_vector(deck: _decks.Deck) -> np.ndarray:
    """External load vector of the deck's face tractions (library host routine)."""
    L = load_library()
    neq = deck.num_eq()
    f = np.zeros(neq)
    if deck.face_elem is None or not len(deck.face_elem):
        return f
    fn = np.ascontiguousarray(deck.face_nodes(), dtype=np.int32)
    X = np.ascontiguousarray(deck.coords, dtype=np.float64)
    eq = np.ascontiguousarray(deck.node_eq(), dtype=np.int32)
    q = np.ascontiguousarray(deck.face_q, dtype=np.float64)
    loc = np.ascontiguousarray(deck.face_local, dtype=np.int32)
    rc = L.fast_gpu_face_load_vector(deck.num_nodes, _p(X), _p(eq, _ip), neq, fn.shape[0], fn.shape[1], _p(fn, _ip),
                                     _p(q), _p(loc, _ip), int(max(deck.ngp)), _p(f))
    if rc != FAST_GPU_OK:
        raise FastGpuError(rc, "face_load_vector")
    return f


def _bucket_struct(b: _decks.Deck, keep: list) -> Bucket:
    conn = np.ascontiguousarray(b.conn, dtype=np.int32)
    E = np.ascontiguousarray(b.E, dtype=np.float64)
    nu = np.ascontiguousarray(b.nu, dtype=np.float64)
    rho = None if b.rho is None else np.ascontiguousarray(b.rho, dtype=np.float64)
    keep += [conn, E, nu, rho]
    pat = ctypes.POINTER(Patch)()
    if b.kind == "bsp":
        P = b.patch
        knots = [np.ascontiguousarray(k, dtype=np.float64) for k in P.knots]
        span = np.ascontiguousarray(P.span, dtype=np.int32)
        w = None if P.weights is None else np.ascontiguousarray(P.weights, dtype=np.float64)
        ps = Patch((ctypes.c_int32 * 3)(*P.degree), (ctypes.c_int32 * 3)(*[len(k) for k in knots]),
                   (ctypes.POINTER(ctypes.c_double) * 3)(*[_p(k) for k in knots]), _p(span, _ip),
                   _p(w) if w is not None else ctypes.POINTER(ctypes.c_double)(), int(bool(P.rational)), 0)
        keep += [knots, span, w, ps]
        pat = ctypes.pointer(ps)
    return Bucket(ELEM[b.kind], (ctypes.c_int32 * 3)(*b.ngp), b.num_elems, _p(conn, _ip), _p(E), _p(nu),
                  _p(rho) if rho is not None else ctypes.POINTER(ctypes.c_double)(),
                  FORM_TL if b.total_lagrangian else FORM_SMALL, 0, pat)


def _mesh_struct(deck: _decks.Deck):
    coords = np.ascontiguousarray(deck.coords, dtype=np.float64)
    eq = np.ascontiguousarray(deck.node_eq(), dtype=np.int32)
    keep = []
    bl = deck.buckets()
    buckets = (Bucket * len(bl))(*[_bucket_struct(b, keep) for b in bl])
    tp = ctypes.POINTER(Ties)()
    if deck.ties is not None and len(deck.ties.slave):
        t = deck.ties
        arrs = [np.ascontiguousarray(a, dtype=np.int64) for a in (t.slave, t.ptr, t.master)]
        w = np.ascontiguousarray(t.weight, dtype=np.float64)
        ts = Ties(len(arrs[0]), _p(arrs[0], _lp), _p(arrs[1], _lp), _p(arrs[2], _lp), _p(w))
        keep += [arrs, w, ts]
        tp = ctypes.pointer(ts)
    m = Mesh(deck.num_nodes, _p(coords), _p(eq, _ip), int(eq.max(initial=0)), len(bl), buckets, tp)
    return m, (coords, eq, keep, buckets)


def inspect_pattern(deck: _decks.Deck) -> dict:
    """Host-only pattern and colouring of a deck (no device needed)."""
    L = load_library()
    m, keep = _mesh_struct(deck)
    nnzb, nlow, ncol = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    rc = L.fast_gpu_inspect_pattern(ctypes.byref(m), ctypes.byref(nnzb), ctypes.byref(nlow), ctypes.byref(ncol),
                                    _ip(), _ip(), _ip())
    if rc != FAST_GPU_OK:
        raise FastGpuError(rc, "inspect_pattern")
    rp = np.zeros(deck.num_nodes + 1, np.int32)
    col = np.zeros(nnzb.value, np.int32)
    color = np.zeros(deck.num_elems, np.int32)
    rc = L.fast_gpu_inspect_pattern(ctypes.byref(m), ctypes.byref(nnzb), ctypes.byref(nlow), ctypes.byref(ncol),
                                    _p(rp, _ip), _p(col, _ip), _p(color, _ip))
    if rc != FAST_GPU_OK:
        raise FastGpuError(rc, "inspect_pattern")
    return {"nnz_blocks": nnzb.value, "nnz_lower_eq": nlow.value, "num_colors": ncol.value, "rowptr": rp,
            "col": col, "color": color}


class GpuSystem:
    """One device context holding one mesh, its matrices and solver state."""

    def __init__(self, device: int = 0):
        self.L = load_library()
        self.ctx = ctypes.c_void_p()
        rc = self.L.fast_gpu_create(device, ctypes.byref(self.ctx))
        if rc != FAST_GPU_OK:
            raise FastGpuError(rc, "fast_gpu_create (is a CUDA device present?)")
        self.neq = 0
        self._keep = []

    # -- plumbing
    def _ck(self, rc, what=""):
        if rc != FAST_GPU_OK:
            msg = self.L.fast_gpu_last_error(self.ctx).decode(errors="replace")
            raise FastGpuError(rc, f"{what}: {msg}")

    def close(self):
        if self.ctx:
            self.L.fast_gpu_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def newmark(self, q, steps, dt, gamma=0.5, beta=0.25, precision=PREC_FP64, precond=PRECOND_JACOBI, tol=1e-10,
                warm=True, mass_tol=1e-12, probes=None, check_every=0, rayleigh=None):
        """Linear Newmark (cCtrlNewmark::Solver) under the step load q, with
        Rayleigh damping when rayleigh = (omega1, omega2, xi1, xi2).
        Returns (u, v, a) at the last step, u at the probe equations per step
        ([steps][len(probes)], or None) and the report."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        lin = SolveOpts(precision, precond, 0, int(bool(warm)), float(tol), 0.0, 0, int(check_every))
        mass = SolveOpts(PREC_FP64, PRECOND_JACOBI, 0, 0, float(mass_tol), 0.0, 0, 0)
        ray = tuple(float(v) for v in rayleigh) if rayleigh is not None else (0.0, 1.0, 0.0, 0.0)
        o = NewmarkOpts(int(steps), int(rayleigh is not None), float(dt), float(gamma), float(beta), lin, mass, *ray)
        u, v, a = np.zeros(self.neq), np.zeros(self.neq), np.zeros(self.neq)
        pr = np.ascontiguousarray(probes if probes is not None else [], dtype=np.int32)
        hist = np.zeros((steps, len(pr))) if len(pr) else None
        rep = NewmarkReport()
        self._ck(self.L.fast_gpu_newmark(self.ctx, _p(q), ctypes.byref(o), _p(u), _p(v), _p(a), len(pr),
                                         _p(pr, _ip) if len(pr) else _ip(), _p(hist) if hist is not None else _dp(),
                                         ctypes.byref(rep)), "newmark")
        return (u, v, a), hist, rep.as_dict()

    def set_problems(self, node_offsets):
        """Mark the uploaded mesh as independent problems over node ranges."""
        off = np.ascontiguousarray(node_offsets, dtype=np.int64)
        self._ck(self.L.fast_gpu_set_problems(self.ctx, len(off) - 1, _p(off, _lp)), "set_problems")
        self.nprob = len(off) - 1

    def solve_batch(self, f, tol=1e-8, precond=PRECOND_JACOBI, maxit=0, u0=None, raise_on_nonconv=True):
        """Solve every problem to its own stopping test in one launch;
        returns u and per-problem (converged, iterations, rel_residual) arrays."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        u = np.zeros(self.neq) if u0 is None else np.array(u0, dtype=np.float64)
        o = SolveOpts(PREC_FP64, precond, int(maxit), int(u0 is not None), float(tol), 0.0, 0, 0)
        reps = (ProblemReport * self.nprob)()
        rc = self.L.fast_gpu_solve_batch(self.ctx, _p(f), _p(u), ctypes.byref(o), reps)
        if rc != FAST_GPU_OK and (raise_on_nonconv or rc != -5):
            self._ck(rc, "solve_batch")
        conv = np.array([r.converged for r in reps], bool)
        its = np.array([r.iterations for r in reps], np.int32)
        res = np.array([r.rel_residual for r in reps])
        return u, conv, its, res

    def set_face_loads(self, deck: _decks.Deck = None):
        """Store the deck's face tractions on the device (fast_gpu_set_face_loads)."""
        deck = self.deck if deck is None else deck
        if deck.face_elem is None or not len(deck.face_elem):
            self._ck(self.L.fast_gpu_set_face_loads(self.ctx, 0, 4, None, None, None, 2), "set_face_loads")
            return
        fn = np.ascontiguousarray(deck.face_nodes(), dtype=np.int32)
        q = np.ascontiguousarray(deck.face_q, dtype=np.float64)
        loc = np.ascontiguousarray(deck.face_local, dtype=np.int32)
        self._ck(self.L.fast_gpu_set_face_loads(self.ctx, fn.shape[0], fn.shape[1], fn.ctypes.data, q.ctypes.data,
                                                loc.ctypes.data, int(max(deck.ngp))), "set_face_loads")

    def face_load_device(self, d_f_ptr: int, scale: float = 1.0):
        """scale * f into the device vector at d_f_ptr (num_eq doubles)."""
        self._ck(self.L.fast_gpu_face_load_device(self.ctx, float(scale), ctypes.c_void_p(d_f_ptr)),
                 "face_load_device")

    def gauss_stress(self, first=0, count=None, bucket=0):
        """Gauss-point (strain, stress) [count][points][6] at the current
        displacements (fast_gpu_gauss_stress)."""
        b = self.deck.buckets()[bucket]
        count = b.num_elems - first if count is None else count
        ng = int(np.prod(b.ngp))
        st = np.zeros((count, ng, 6))
        ss = np.zeros((count, ng, 6))
        self._ck(self.L.fast_gpu_gauss_stress(self.ctx, bucket, int(first), int(count), st.ctypes.data,
                                              ss.ctypes.data), "gauss_stress")
        return st, ss

    def support_reactions(self, load_factor=1.0, supported=None):
        """Support reactions [nnode][3] at the current displacements under the
        deck's face and nodal loads scaled by load_factor (fast_gpu_support_reactions)."""
        d = self.deck
        R = np.zeros((d.num_nodes, 3))
        sup = None if supported is None else np.ascontiguousarray(supported, dtype=np.uint8)
        nf = 0 if d.face_elem is None else len(d.face_elem)
        fn = q = loc = None
        if nf:
            fn = np.ascontiguousarray(d.face_nodes(), dtype=np.int32)
            q = np.ascontiguousarray(d.face_q, dtype=np.float64)
            loc = np.ascontiguousarray(d.face_local, dtype=np.int32)
        nod = None if d.nodal_f is None else np.ascontiguousarray(d.nodal_f, dtype=np.float64)
        ptr = lambda a: None if a is None else a.ctypes.data
        self._ck(self.L.fast_gpu_support_reactions(self.ctx, ptr(sup), nf, fn.shape[1] if nf else 4, ptr(fn), ptr(q),
                                                   ptr(loc), int(d.ngp[0]), ptr(nod), float(load_factor),
                                                   R.ctypes.data), "support_reactions")
        return R

    def nodal_stress(self, bucket=0):
        """(element-nodal [ne][nn][6], averaged nodal [nnode][6]) stresses at the
        current displacements (fast_gpu_nodal_stress)."""
        b = self.deck.buckets()[bucket]
        en = np.zeros((b.num_elems, b.nn, 6))
        avg = np.zeros((self.deck.num_nodes, 6))
        self._ck(self.L.fast_gpu_nodal_stress(self.ctx, bucket, en.ctypes.data, avg.ctypes.data), "nodal_stress")
        return en, avg

    def autotune(self) -> dict:
        """Measure the element kernels' launch shapes (bucket by bucket), the
        SpMV lanes-per-row choices and the PCG iteration path on this
        (assembled) system and keep the fastest (fast_gpu_autotune); K is
        re-assembled with the chosen shapes."""
        r = TuneReport()
        self._ck(self.L.fast_gpu_autotune(self.ctx, ctypes.byref(r)), "autotune")
        return r.as_dict()

    def set_option(self, option: int, value: int):
        self._ck(self.L.fast_gpu_set_option(self.ctx, int(option), int(value)), "set_option")

    def mlp_gemm(self, A, B, ta=False, tb=False):
        """The tensor-core GEMM alone: C = opA(A) opB(B)^T with opA = A^T when ta
        (A given as [K][M]) and opB = B^T when tb (B given as [K][N])."""
        A = np.ascontiguousarray(A, dtype=np.float32)
        B = np.ascontiguousarray(B, dtype=np.float32)
        M = A.shape[1] if ta else A.shape[0]
        K = A.shape[0] if ta else A.shape[1]
        N = B.shape[1] if tb else B.shape[0]
        assert (B.shape[0] if tb else B.shape[1]) == K
        C = np.zeros((M, N), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self._ck(self.L.fast_gpu_mlp_gemm(self.ctx, M, N, K, _p(A, fp), int(ta), _p(B, fp), int(tb), _p(C, fp)),
                 "mlp_gemm")
        return C

    def set_stream(self, stream_ptr: Optional[int]):
        self._ck(self.L.fast_gpu_set_stream(self.ctx, ctypes.c_void_p(stream_ptr or 0)), "set_stream")

    def synchronize(self):
        self._ck(self.L.fast_gpu_synchronize(self.ctx), "synchronize")

    # -- mesh
    def upload(self, deck: _decks.Deck):
        self.deck = deck
        m, keep = _mesh_struct(deck)
        self.neq = int(m.num_eq)
        self.nbuckets = int(m.num_buckets)
        self._ck(self.L.fast_gpu_upload_mesh(self.ctx, ctypes.byref(m)), "upload_mesh")
        self.node_eq = keep[1]
        return self

    def pattern_info(self):
        a, b, c, d = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_double()
        self._ck(self.L.fast_gpu_pattern_info(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                              ctypes.byref(d)))
        return {"nnz_blocks": a.value, "nnz_lower_eq": b.value, "num_colors": c.value, "pattern_seconds": d.value}

    def update_coords(self, coords):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        self._ck(self.L.fast_gpu_update_coords(self.ctx, _p(coords)), "update_coords")

    def update_material(self, E=None, nu=None, bucket=0):
        Ep = _p(np.ascontiguousarray(E, dtype=np.float64)) if E is not None else _dp()
        nup = _p(np.ascontiguousarray(nu, dtype=np.float64)) if nu is not None else _dp()
        self._ck(self.L.fast_gpu_update_material(self.ctx, bucket, Ep, nup), "update_material")

    # -- displacement state and internal force
    def set_displacement(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self._ck(self.L.fast_gpu_set_displacement(self.ctx, _p(u)), "set_displacement")

    def internal_force(self):
        g = np.zeros(self.neq)
        self._ck(self.L.fast_gpu_internal_force(self.ctx, _p(g)), "internal_force")
        return g

    # -- load-control Newton-Raphson (cCtrlNR::Solver)
    def nr_solve(self, q, steps, step_factor, tol=1e-8, max_iter=30, predictor=PREDICT_NONE, callback=None,
                 precision=PREC_FP64, precond=PRECOND_JACOBI, lin_tol=1e-12, lin_tol_rel=0.0, lin_tol_min=1e-12,
                 lin_tol_max=1e-2, keep_history=True, raise_on_fail=True, learned=None, lin_check_every=0):
        """Load-control Newton-Raphson.  ``learned``: a trained
        :class:`LearnedPredictor` used as the caller predictor (implies
        ``predictor=PREDICT_CALLBACK``).  ``lin_check_every``: PCG iterations
        per chunk of the inner solves (0: the library's default)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        lin = SolveOpts(precision, precond, 0, 0, float(lin_tol), 0.0, 0, int(lin_check_every))
        o = NrOpts(int(steps), int(max_iter), float(step_factor), float(tol), int(predictor), 0, lin,
                   float(lin_tol_rel), float(lin_tol_min), float(lin_tol_max))
        hist = np.zeros((steps, self.neq)) if keep_history else None
        iters = np.zeros(steps, np.int32)
        rep = NrReport()
        user = None
        if learned is not None:
            o.predictor = PREDICT_CALLBACK
            callback = NR_PREDICTOR(("fast_gpu_ws_predict", self.L))
            user = learned.handle
        cb = callback if callback is not None else NR_PREDICTOR()
        rc = self.L.fast_gpu_nr_solve(self.ctx, _p(q), ctypes.byref(o), cb, user,
                                      _p(hist) if hist is not None else _dp(), _p(iters, _ip), ctypes.byref(rep))
        if rc != FAST_GPU_OK and raise_on_fail:
            self._ck(rc, "nr_solve")
        return hist, iters, rep.as_dict()

    # -- modal analysis (cCtrlModal::Solver, subspace iteration)
    def modal(self, num_modes=5, tol=1e-6, max_iter=200, lin_tol=1e-12, precision=PREC_FP64, precond=PRECOND_JACOBI,
              raise_on_fail=True):
        """(eigenvalues [num_modes], M-normalised modes [num_modes][neq], report)."""
        lin = SolveOpts(precision, precond, 0, 0, float(lin_tol), 0.0, 0, 0)
        o = ModalOpts(int(num_modes), int(max_iter), float(tol), lin)
        lam = np.zeros(num_modes)
        modes = np.zeros((num_modes, self.neq))
        rep = ModalReport()
        rc = self.L.fast_gpu_modal(self.ctx, ctypes.byref(o), _p(lam), _p(modes), ctypes.byref(rep))
        if rc != FAST_GPU_OK and raise_on_fail:
            self._ck(rc, "modal")
        return lam, modes, rep.as_dict()

    def buckling(self, f, num_modes=5, tol=1e-6, max_iter=200, lin_tol=1e-12, precision=PREC_FP64,
                 precond=PRECOND_JACOBI, raise_on_fail=True):
        """Linear buckling under the reference load f: (factors [num_modes],
        modes [num_modes][neq], linear solution u [neq], report)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        lin = SolveOpts(precision, precond, 0, 0, float(lin_tol), 0.0, 0, 0)
        o = ModalOpts(int(num_modes), int(max_iter), float(tol), lin)
        lam = np.zeros(num_modes)
        modes = np.zeros((num_modes, self.neq))
        u = np.zeros(self.neq)
        rep = ModalReport()
        rc = self.L.fast_gpu_buckling(self.ctx, _p(f), ctypes.byref(o), _p(lam), _p(modes), _p(u), ctypes.byref(rep))
        if rc != FAST_GPU_OK and raise_on_fail:
            self._ck(rc, "buckling")
        return lam, modes, u, rep.as_dict()

    # -- path following (cCtrlPath::Solver with the arc-length rules)
    def arclength_solve(self, q, method, steps, step_factor, tol=1e-8, max_iter=30, load_coeff=0.0, target_iter=1,
                        precision=PREC_FP64, precond=PRECOND_JACOBI, lin_tol=1e-12, raise_on_fail=True):
        """Arc-length path following.  ``method``: "ioal", "uoal" or "clinal"
        (the reference's cIniOrtArcLength, cUpOrtArcLength, cConLinArcLength).
        Returns (displacements [steps][neq], load factors [steps], iterations
        per step, report)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        lin = SolveOpts(precision, precond, 0, 0, float(lin_tol), 0.0, 0, 0)
        o = ArcOpts(ARC_METHODS.get(method, method), int(steps), int(max_iter), int(target_iter), float(step_factor),
                    float(tol), float(load_coeff), lin)
        hist = np.zeros((steps, self.neq))
        lams = np.zeros(steps)
        iters = np.zeros(steps, np.int32)
        rep = ArcReport()
        rc = self.L.fast_gpu_arclength_solve(self.ctx, _p(q), ctypes.byref(o), _p(hist), _p(lams), _p(iters, _ip),
                                             ctypes.byref(rep))
        if rc != FAST_GPU_OK and raise_on_fail:
            self._ck(rc, "arclength_solve")
        n = rep.converged_steps
        return hist[:n], lams[:n], iters[:n], rep.as_dict()

    # -- cSysMatrix
    def zero(self, what=ASM_K):
        self._ck(self.L.fast_gpu_zero(self.ctx, what), "zero")

    def assemble(self, what=ASM_K):
        self._ck(self.L.fast_gpu_assemble(self.ctx, what), "assemble")

    def assemble_mass(self):
        self.assemble(ASM_M)

    def add(self, i, j, v, what=ASM_K):
        self._ck(self.L.fast_gpu_add(self.ctx, what, int(i), int(j), float(v)), "add")

    def add_mat(self, a, dst=ASM_K, src=ASM_M):
        """cSysMatrix::AddMat(a, M): K += a M on the device."""
        self._ck(self.L.fast_gpu_add_mat(self.ctx, dst, float(a), src), "add_mat")

    def get(self, i, j, what=ASM_K):
        v = ctypes.c_double()
        self._ck(self.L.fast_gpu_get(self.ctx, what, int(i), int(j), ctypes.byref(v)), "get")
        return v.value

    def mult_vect(self, x, what=ASM_K):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.neq)
        self._ck(self.L.fast_gpu_mult_vect(self.ctx, what, _p(x), _p(y)), "mult_vect")
        return y

    def solve(self, f, tol=1e-8, precision=PREC_FP64, precond=PRECOND_JACOBI, maxit=0, u0=None,
              inner_tol=0.0, max_outer=0, check_every=0, raise_on_nonconv=True):
        f = np.ascontiguousarray(f, dtype=np.float64)
        u = np.zeros(self.neq) if u0 is None else np.array(u0, dtype=np.float64)
        o = SolveOpts(precision, precond, int(maxit), int(u0 is not None), float(tol), float(inner_tol),
                      int(max_outer), int(check_every))
        rep = SolveReport()
        rc = self.L.fast_gpu_solve(self.ctx, _p(f), _p(u), ctypes.byref(o), ctypes.byref(rep))
        if rc != FAST_GPU_OK and (raise_on_nonconv or rc != -5):
            self._ck(rc, "solve")
        return u, rep.as_dict()

    def solve_device(self, d_f_ptr: int, d_u_ptr: int, tol=1e-8, precision=PREC_FP64, precond=PRECOND_JACOBI,
                     maxit=0, warm=False, inner_tol=0.0, max_outer=0, check_every=0):
        o = SolveOpts(precision, precond, int(maxit), int(warm), float(tol), float(inner_tol), int(max_outer),
                      int(check_every))
        rep = SolveReport()
        self._ck(self.L.fast_gpu_solve_device(self.ctx, ctypes.c_void_p(d_f_ptr), ctypes.c_void_p(d_u_ptr),
                                              ctypes.byref(o), ctypes.byref(rep)), "solve_device")
        return rep.as_dict()

    # -- measurement
    def launch_count(self) -> int:
        n = ctypes.c_int64()
        self._ck(self.L.fast_gpu_launch_count(self.ctx, ctypes.byref(n)), "launch_count")
        return n.value

    def kernel_timing(self, enable: bool = True):
        self._ck(self.L.fast_gpu_kernel_timing(self.ctx, int(enable)), "kernel_timing")

    def kernel_stats(self, which: int):
        """(timed launches, summed device ms, algorithmic bytes per launch) since timing was enabled.

        Launches issued after convergence return at once and are counted here;
        divide the summed time by the number of real launches for a mean."""
        n, ms, b = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        self._ck(self.L.fast_gpu_kernel_stats(self.ctx, which, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b)),
                 "kernel_stats")
        return n.value, ms.value, b.value

    # -- parity
    def lower_csr(self, what=ASM_K):
        import scipy.sparse as sp
        nnz = ctypes.c_int64()
        self._ck(self.L.fast_gpu_get_lower_csr(self.ctx, what, ctypes.byref(nnz), _lp(), _ip(), _dp()), "lower_csr")
        rp = np.zeros(self.neq + 1, np.int64)
        ci = np.zeros(nnz.value, np.int32)
        v = np.zeros(nnz.value)
        self._ck(self.L.fast_gpu_get_lower_csr(self.ctx, what, ctypes.byref(nnz), _p(rp, _lp), _p(ci, _ip), _p(v)),
                 "lower_csr")
        return sp.csr_matrix((v, ci, rp), shape=(self.neq, self.neq))

    def element_matrices(self, first=0, count=None, what=ASM_K, bucket=0):
        b = self.deck.buckets()[bucket]
        nn = b.nn
        if count is None:
            count = b.num_elems - first
        out = np.zeros((count, 3 * nn) if what == ASM_G else (count, 3 * nn, 3 * nn))
        self._ck(self.L.fast_gpu_element_matrices(self.ctx, what, bucket, int(first), int(count), _p(out)),
                 "element_matrices")
        return out


_fp = ctypes.POINTER(ctypes.c_float)


class LearnedPredictor:
    """The learned load-step predictor (fast_gpu_ws_*): POD basis of converged
    displacements plus a tanh MLP trained on the device with BF16 tensor-core
    GEMMs.  Pass it as ``GpuSystem.nr_solve(..., learned=p)``."""

    def __init__(self, system: "GpuSystem", modes=32, history=4, width=256, hidden=2, oversample=16,
                 power_iters=2, seed=0):
        self.sys = system
        self.L = system.L
        o = WsOpts(int(modes), int(history), int(width), int(hidden), int(oversample), int(power_iters), int(seed))
        h = ctypes.c_void_p()
        system._ck(self.L.fast_gpu_ws_create(system.ctx, ctypes.byref(o), ctypes.byref(h)), "ws_create")
        self.handle = h
        self.modes, self.history, self.width, self.hidden = modes, history, width, hidden

    def close(self):
        if self.handle:
            self.L.fast_gpu_ws_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, use_network=True, galerkin_iters=0, galerkin_tol=1e-3):
        """Start from the network's prediction (or the secant start) and refine
        it with `galerkin_iters` reduced Newton corrections in the basis."""
        self.sys._ck(self.L.fast_gpu_ws_configure(self.handle, int(bool(use_network)), int(galerkin_iters),
                                                  float(galerkin_tol)), "ws_configure")

    def last_input(self):
        """Network input of the last prediction (scaled features)."""
        x = np.zeros(self.dims()[0], np.float32)
        self.sys._ck(self.L.fast_gpu_ws_last_input(self.handle, _p(x, _fp)), "ws_last_input")
        return x

    def add_trajectory(self, lambdas, u_steps):
        lam = np.ascontiguousarray(lambdas, dtype=np.float64)
        u = np.ascontiguousarray(u_steps, dtype=np.float64)
        assert u.shape == (len(lam), self.sys.neq)
        self.sys._ck(self.L.fast_gpu_ws_add_trajectory(self.handle, len(lam), _p(lam), _p(u)), "ws_add_trajectory")

    def build_basis(self):
        e = ctypes.c_double()
        self.sys._ck(self.L.fast_gpu_ws_build_basis(self.handle, ctypes.byref(e)), "ws_build_basis")
        return e.value

    def train(self, epochs=2000, lr=2e-3):
        h = np.zeros(max(1, epochs), np.float32)
        self.sys._ck(self.L.fast_gpu_ws_train(self.handle, int(epochs), float(lr), _p(h, _fp)), "ws_train")
        return h[:epochs]

    def report(self):
        r = WsStats()
        self.sys._ck(self.L.fast_gpu_ws_report(self.handle, ctypes.byref(r)), "ws_report")
        return r.as_dict()

    def basis(self):
        k = self.report()["modes"]
        phi = np.zeros((self.sys.neq, k))
        self.sys._ck(self.L.fast_gpu_ws_get_basis(self.handle, _p(phi)), "ws_get_basis")
        return phi

    def samples(self):
        r = self.report()
        x = np.zeros((r["samples"], r["input_dim"]), np.float32)
        t = np.zeros((r["samples"], r["output_dim"]), np.float32)
        self.sys._ck(self.L.fast_gpu_ws_get_samples(self.handle, _p(x, _fp), _p(t, _fp)), "ws_get_samples")
        return x, t

    # -- the network alone
    def params(self, set_to=None):
        n = ctypes.c_int64()
        self.sys._ck(self.L.fast_gpu_mlp_params(self.handle, None, None, ctypes.byref(n)), "mlp_params")
        if set_to is not None:
            p = np.ascontiguousarray(set_to, dtype=np.float32)
            assert p.size == n.value
            self.sys._ck(self.L.fast_gpu_mlp_params(self.handle, None, _p(p, _fp), None), "mlp_params")
        out = np.zeros(n.value, np.float32)
        self.sys._ck(self.L.fast_gpu_mlp_params(self.handle, _p(out, _fp), None, None), "mlp_params")
        return out

    def dims(self):
        return [1 + self.history * self.modes] + [self.width] * self.hidden + [self.modes]

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.modes), np.float32)
        self.sys._ck(self.L.fast_gpu_mlp_forward(self.handle, x.shape[0], _p(x, _fp), _p(y, _fp)), "mlp_forward")
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.params().size, np.float32)
        self.sys._ck(self.L.fast_gpu_mlp_loss_grad(self.handle, x.shape[0], _p(x, _fp), _p(t, _fp), _p(loss, _fp),
                                                   _p(g, _fp)), "mlp_loss_grad")
        return float(loss[0]), g
