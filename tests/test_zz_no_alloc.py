"""The allocation-free solve entry point (fast_gpu_pcg_solve_noalloc).

It exists for callers that cannot let a library allocate device memory (a
memory pool of their own owns the device, or the implicit device
synchronisation of cudaMalloc/cudaFree would stall their other streams).  It
is checked here against the regular entry point, fast_gpu_solve with FP64
Jacobi PCG, through the C ABI, on two calls in a row (the second call reuses
the shared static scratch the first one left behind), and the second call is
checked to leave the device's free memory unchanged.  This file is collected
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
EINVAL, ENONCONV, ETOOBIG = -1, -5, -9


def _full_csr(lower):
    """Equation-space full symmetric CSR from the lower triangle."""
    K = (lower + lower.T - sp.diags(lower.diagonal())).tocsr()
    K.sort_indices()
    return K


def _device_csr(K, dev):
    import torch
    return (torch.from_numpy(K.indptr.astype(np.int64)).to(dev),
            torch.from_numpy(K.indices.astype(np.int32)).to(dev),
            torch.from_numpy(K.data.astype(np.float64)).to(dev))


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
    n = K.shape[0]
    dev = torch.device("cuda", 0)
    rowptr, col, val = _device_csr(K, dev)
    d_f = torch.from_numpy(np.ascontiguousarray(f)).to(dev)
    L = gpu.load_library()
    free_change = []
    for call in range(2):
        d_u = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        rep = gpu.SolveReport()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        rc = L.fast_gpu_pcg_solve_noalloc(n, rowptr.data_ptr(), col.data_ptr(), val.data_ptr(),
                                          d_f.data_ptr(), d_u.data_ptr(), tol, 20 * n, None, ctypes.byref(rep))
        torch.cuda.synchronize()
        free_change.append(free_before - torch.cuda.mem_get_info(0)[0])
        assert rc == 0, gpu.ERRORS.get(rc, rc)
        u = d_u.cpu().numpy()
        assert rep.converged
        assert abs(rep.iterations - rep_ref["iterations"]) <= 2, (call, rep.iterations, rep_ref)
        assert gio.rel(u, u_ref) < TOL_U, call
        assert gio.rel(u, g["ref_u"]) < TOL_U, call
    # the first call on this device may have loaded the scratch array (lazy
    # module loading); the second allocates nothing
    print("device memory taken by the first call: %d B, by the second: %d B" % tuple(free_change))
    assert free_change[1] == 0, free_change
    s.close()


def test_noalloc_setup_call_and_diagonal_check():
    import torch
    L = gpu.load_library()
    # num_eq = 0: set-up only (loads the scratch array onto this device)
    assert L.fast_gpu_pcg_solve_noalloc(0, None, None, None, None, None, 1e-8, 0, None, None) == 0
    # a 3x3 system whose middle row stores no diagonal: Jacobi is undefined
    K = sp.csr_matrix(np.array([[4.0, 1.0, 0.0], [1.0, 0.0, 1.0], [0.0, 1.0, 4.0]]))
    K.eliminate_zeros()
    K.sort_indices()
    assert K[1, 1] == 0 and 1 not in K.indices[K.indptr[1]:K.indptr[2]]
    dev = torch.device("cuda", 0)
    rowptr, col, val = _device_csr(K, dev)
    d_f = torch.ones(3, dtype=torch.float64, device=dev)
    d_u = torch.zeros(3, dtype=torch.float64, device=dev)
    rep = gpu.SolveReport()
    rc = L.fast_gpu_pcg_solve_noalloc(3, rowptr.data_ptr(), col.data_ptr(), val.data_ptr(), d_f.data_ptr(),
                                      d_u.data_ptr(), 1e-10, 0, None, ctypes.byref(rep))
    assert rc == EINVAL and not rep.converged
    # and a well-posed 3x3 system right after it converges with the default maxit (n)
    K2 = sp.csr_matrix(np.array([[4.0, 1.0, 0.0], [1.0, 3.0, 1.0], [0.0, 1.0, 4.0]]))
    rowptr, col, val = _device_csr(K2, dev)
    rc = L.fast_gpu_pcg_solve_noalloc(3, rowptr.data_ptr(), col.data_ptr(), val.data_ptr(), d_f.data_ptr(),
                                      d_u.data_ptr(), 1e-12, 0, None, ctypes.byref(rep))
    assert rc == 0 and rep.converged and rep.iterations <= 3
    assert np.abs(d_u.cpu().numpy() - np.linalg.solve(K2.toarray(), np.ones(3))).max() < 1e-12


def test_noalloc_rejects_systems_above_its_limit():
    L = gpu.load_library()
    dummy = ctypes.c_void_p(1)
    rc = L.fast_gpu_pcg_solve_noalloc(MAX_EQ + 1, dummy, dummy, dummy, dummy, dummy, 1e-8, 10, None, None)
    assert rc == ETOOBIG  # returned before any device work
