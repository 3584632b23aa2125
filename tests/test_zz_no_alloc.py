"""The allocation-free solve entry point (fast_gpu_pcg_solve_noalloc).

It exists for callers that cannot let a library allocate device memory (a
memory pool of their own owns the device, or the implicit device
synchronisation of cudaMalloc/cudaFree would stall their other streams).  It
is checked here against the regular entry point, fast_gpu_solve with FP64
Jacobi PCG, through the C ABI, on two calls in a row (the second call reuses
the shared static scratch the first one left behind).  This file is collected
last on purpose.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from fast_b200 import gpu
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

TOL_U = 1e-9          # displacement bound used by the device parity tests
MAX_EQ = 500000       # the entry point's static-scratch limit


def _full_csr(lower):
    """Equation-space full symmetric CSR from the lower triangle."""
    K = (lower + lower.T - sp.diags(lower.diagonal())).tocsr()
    K.sort_indices()
    return K


def test_noalloc_solve_matches_regular_solve_twice():
    import torch
    d, g = gio.load("cfg_hex20_lognormal_8x8x4")
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    f = g["ref_f"]
    tol = 1e-12
    u_ref, rep_ref = s.solve(f, tol=tol, precision=gpu.PREC_FP64, precond=gpu.PRECOND_JACOBI)
    K = _full_csr(s.lower_csr())
    dev = torch.device("cuda", 0)
    rowptr = torch.from_numpy(K.indptr.astype(np.int64)).to(dev)
    col = torch.from_numpy(K.indices.astype(np.int32)).to(dev)
    val = torch.from_numpy(K.data.astype(np.float64)).to(dev)
    d_f = torch.from_numpy(np.ascontiguousarray(f)).to(dev)
    L = gpu.load_library()
    for call in range(2):
        d_u = torch.full((K.shape[0],), float("nan"), dtype=torch.float64, device=dev)
        rep = gpu.SolveReport()
        torch.cuda.synchronize()
        rc = L.fast_gpu_pcg_solve_noalloc(K.shape[0], rowptr.data_ptr(), col.data_ptr(), val.data_ptr(),
                                          d_f.data_ptr(), d_u.data_ptr(), tol, 0, None, ctypes.byref(rep))
        assert rc == 0, gpu.ERRORS.get(rc, rc)
        u = d_u.cpu().numpy()
        assert rep.converged
        assert abs(rep.iterations - rep_ref["iterations"]) <= 2, (call, rep.iterations, rep_ref)
        assert gio.rel(u, u_ref) < TOL_U, call
        assert gio.rel(u, g["ref_u"]) < TOL_U, call
    s.close()


def test_noalloc_rejects_systems_above_its_limit():
    L = gpu.load_library()
    dummy = ctypes.c_void_p(1)
    rc = L.fast_gpu_pcg_solve_noalloc(MAX_EQ + 1, dummy, dummy, dummy, dummy, dummy, 1e-8, 10, None, None)
    assert rc == -9  # FAST_GPU_ETOOBIG, returned before any device work
