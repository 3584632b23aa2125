"""Python side of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/libfem_oracle.so`` (the C restatement in
``fem_oracle.c``) and offers whole-deck helpers built from it: element
matrices, the assembled equation-space matrix, the external load vector and
FAST's Jacobi PCG.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as a checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfem_oracle.so")

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.fo_elem_stiff.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_double, ctypes.c_double, _dp]
        L.fo_elems_stiff.argtypes = [ctypes.c_int, _ip, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32), _dp, _dp, _dp, _dp]
        L.fo_elem_intforce.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.fo_elem_stress.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
        L.fo_elem_mass.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_double, _dp]
        L.fo_extrap_matrix.argtypes = [ctypes.c_int, _ip, _dp]
        L.fo_elem_geom.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.fo_elem_tl.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
        L.fo_face_load.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp]
        L.fo_pcg.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32), _dp,
                             _dp, _dp, ctypes.c_int, ctypes.c_double, _ip, _dp]
        L.fo_pcg_threaded.argtypes = L.fo_pcg.argtypes
        L.fo_spmv.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32), _dp, _dp, _dp]
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _ngp(ngp):
    return (ctypes.c_int * 3)(*[int(v) for v in ngp])


def elem_stiff(nn, ngp, X, E, nu):
    K = np.zeros((3 * nn, 3 * nn))
    X = np.ascontiguousarray(X, dtype=np.float64)
    rc = lib().fo_elem_stiff(nn, _ngp(ngp), _p(X), float(E), float(nu), _p(K))
    return K, rc


def elems_stiff(deck, elems=None):
    nn = deck.nn
    conn = deck.conn if elems is None else deck.conn[elems]
    E = deck.E if elems is None else deck.E[elems]
    nu = deck.nu if elems is None else deck.nu[elems]
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    X = np.ascontiguousarray(deck.coords, dtype=np.float64)
    E = np.ascontiguousarray(E, dtype=np.float64)
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    Ke = np.zeros((conn.shape[0], 3 * nn, 3 * nn))
    rc = lib().fo_elems_stiff(nn, _ngp(deck.ngp), conn.shape[0], _p(conn, ctypes.POINTER(ctypes.c_int32)),
                              _p(X), _p(E), _p(nu), _p(Ke))
    return Ke, rc


def elem_intforce(nn, ngp, X, E, nu, ue):
    g = np.zeros(3 * nn)
    X = np.ascontiguousarray(X, dtype=np.float64)
    ue = np.ascontiguousarray(ue, dtype=np.float64)
    rc = lib().fo_elem_intforce(nn, _ngp(ngp), _p(X), float(E), float(nu), _p(ue), _p(g))
    return g, rc


def elem_stress(nn, ngp, X, E, nu, ue):
    """Gauss-point strains and stresses [ngp][6] (Voigt xx yy zz xy xz yz)."""
    n = int(np.prod(ngp))
    e = np.zeros((n, 6))
    s = np.zeros((n, 6))
    X = np.ascontiguousarray(X, dtype=np.float64)
    ue = np.ascontiguousarray(ue, dtype=np.float64)
    rc = lib().fo_elem_stress(nn, _ngp(ngp), _p(X), float(E), float(nu), _p(ue), _p(e), _p(s))
    return e, s, rc


def elem_geom(nn, ngp, X, E, nu, ue):
    """Element geometric stiffness [3nn][3nn] at displacements ue (cElmParam::GeomStiff)."""
    G = np.zeros((3 * nn, 3 * nn))
    X = np.ascontiguousarray(X, dtype=np.float64)
    ue = np.ascontiguousarray(ue, dtype=np.float64)
    rc = lib().fo_elem_geom(nn, _ngp(ngp), _p(X), float(E), float(nu), _p(ue), _p(G))
    return G, rc


def geom_matrix(d, u):
    """Assembled geometric stiffness (equation space, scipy CSR) of a deck at
    the equation vector u (cControl::GeomStiffMatrix, ctrl/ctrl.cpp:1031-1063)."""
    import scipy.sparse as sp
    eq = d.node_eq()
    neq = d.num_eq()
    dofs = eq[d.conn].reshape(d.num_elems, -1)
    unode = np.zeros((d.num_nodes, 3))
    m = eq > 0
    unode[m] = u[eq[m] - 1]
    I, J, V = [], [], []
    for e in range(d.num_elems):
        Ge, rc = elem_geom(d.nn, d.ngp, d.coords[d.conn[e]], d.E[e], d.nu[e], unode[d.conn[e]].ravel())
        dd = dofs[e]
        mm = dd > 0
        ii = np.repeat(dd, len(dd)) - 1
        jj = np.tile(dd, len(dd)) - 1
        keep = np.repeat(mm, len(dd)) & np.tile(mm, len(dd))
        I.append(ii[keep]); J.append(jj[keep]); V.append(Ge.ravel()[keep])
    return sp.csr_matrix((np.concatenate(V), (np.concatenate(I), np.concatenate(J))), shape=(neq, neq))


def extrap_matrix(nn, ngp):
    """TR [nn][ngp] of cElmParam::CompTRMatrix: element-nodal = TR @ Gauss-point values."""
    TR = np.zeros((nn, int(np.prod(ngp))))
    rc = lib().fo_extrap_matrix(nn, _ngp(ngp), _p(TR))
    return TR, rc


def averaged_nodal_stress(num_nodes, conn, elem_nodal):
    """cControl::PrintAvrNodalStress (ctrl/ctrl.cpp:2397-2440): every node's
    element-nodal values summed over its elements in element order, divided
    by their count; 0 at nodes of no element.  elem_nodal [ne][nn][6]."""
    s = np.zeros((num_nodes, elem_nodal.shape[2]))
    c = np.zeros(num_nodes)
    for e in range(conn.shape[0]):
        for a, n in enumerate(conn[e]):
            s[n] += elem_nodal[e, a]
            c[n] += 1
    m = c > 0
    s[m] /= c[m][:, None]
    return s


def elem_mass(nn, ngp, X, rho):
    M = np.zeros((3 * nn, 3 * nn))
    X = np.ascontiguousarray(X, dtype=np.float64)
    rc = lib().fo_elem_mass(nn, _ngp(ngp), _p(X), float(rho), _p(M))
    return M, rc


def elem_tl(nn, ngp, X, E, nu, ue):
    K = np.zeros((3 * nn, 3 * nn))
    g = np.zeros(3 * nn)
    X = np.ascontiguousarray(X, dtype=np.float64)
    ue = np.ascontiguousarray(ue, dtype=np.float64)
    rc = lib().fo_elem_tl(nn, _ngp(ngp), _p(X), float(E), float(nu), _p(ue), _p(K), _p(g))
    return K, g, rc


def elem_dofs(deck):
    """[ne][3nn] 1-based equations (cElement::GetElmDofs order: node-major, x y z)."""
    eq = deck.node_eq()
    return eq[deck.conn].reshape(deck.num_elems, -1)


def assemble(deck, Ke=None):
    """Equation-space K (scipy CSR, full symmetric) from element matrices."""
    import scipy.sparse as sp
    if Ke is None:
        Ke, _ = elems_stiff(deck)
    dofs = elem_dofs(deck)
    neq = deck.num_eq()
    nd = dofs.shape[1]
    I = np.repeat(dofs, nd, axis=1).ravel()
    J = np.tile(dofs, (1, nd)).ravel()
    V = Ke.reshape(len(dofs), -1).ravel()
    m = (I > 0) & (J > 0)
    K = sp.csr_matrix((V[m], (I[m] - 1, J[m] - 1)), shape=(neq, neq))
    K.sum_duplicates()
    K.sort_indices()
    return K


def face_loads(deck):
    """External load vector (cControl::ExtLoadVector, ctrl/ctrl.cpp:668-715)."""
    neq = deck.num_eq()
    f = np.zeros(neq)
    if deck.face_elem is None or not len(deck.face_elem):
        return f
    eq = deck.node_eq()
    fn = deck.face_nodes()
    nf = fn.shape[1]
    ngp1d = max(deck.ngp)
    for k in range(len(fn)):
        Xf = np.ascontiguousarray(deck.coords[fn[k]])
        fe = np.zeros(3 * nf)
        q = np.ascontiguousarray(deck.face_q[k], dtype=np.float64)
        lib().fo_face_load(nf, ngp1d, _p(Xf), _p(q), int(deck.face_local[k]), _p(fe))
        dofs = eq[fn[k]].ravel()
        for i in range(3 * nf):
            if dofs[i]:
                f[dofs[i] - 1] += fe[i]
    return f


def support_reactions(deck, u, load_factor=1.0):
    """cControl::SuppReactions (ctrl/ctrl.cpp:844-882) at the equation vector
    u: internal forces of the elements with a supported node added to all
    their nodes, minus the face and nodal loads with a supported node.
    [nnode][3]; supported = a node with a DOF without an equation."""
    eq = deck.node_eq()
    sup = (eq == 0).any(axis=1)
    unode = np.zeros((deck.num_nodes, 3))
    m = eq > 0
    unode[m] = u[eq[m] - 1]
    R = np.zeros((deck.num_nodes, 3))
    for e in range(deck.num_elems):
        en = deck.conn[e]
        if not sup[en].any():
            continue
        ge, rc = elem_intforce(deck.nn, deck.ngp, deck.coords[en], deck.E[e], deck.nu[e], unode[en].ravel())
        R[en] += ge.reshape(-1, 3)
    if deck.face_elem is not None and len(deck.face_elem):
        fn = deck.face_nodes()
        nf = fn.shape[1]
        for k in range(len(fn)):
            if not sup[fn[k]].any():
                continue
            fe = np.zeros(3 * nf)
            q = np.ascontiguousarray(deck.face_q[k], dtype=np.float64)
            lib().fo_face_load(nf, max(deck.ngp), _p(np.ascontiguousarray(deck.coords[fn[k]])), _p(q),
                               int(deck.face_local[k]), _p(fe))
            R[fn[k]] -= load_factor * fe.reshape(-1, 3)
    if deck.nodal_f is not None:
        R[sup] -= load_factor * deck.nodal_f[sup]
    return R


def pcg(K, f, tol, maxit):
    """FAST's Jacobi PCG on a scipy CSR matrix; returns (u, converged, iters, err)."""
    n = K.shape[0]
    rp = np.ascontiguousarray(K.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(K.indices, dtype=np.int32)
    v = np.ascontiguousarray(K.data, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    u = np.zeros(n)
    it = ctypes.c_int(0)
    err = ctypes.c_double(0)
    ok = lib().fo_pcg(n, _p(rp, ctypes.POINTER(ctypes.c_int64)), _p(ci, ctypes.POINTER(ctypes.c_int32)), _p(v),
                      _p(f), _p(u), int(maxit), float(tol), ctypes.byref(it), ctypes.byref(err))
    return u, bool(ok), it.value, err.value


def pcg_threaded(K, f, tol, maxit):
    """pcg() with the SpMV and vector operations on all host threads;
    returns (u, iterations, recurrence error)."""
    n = K.shape[0]
    rp = np.ascontiguousarray(K.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(K.indices, dtype=np.int32)
    v = np.ascontiguousarray(K.data, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    u = np.zeros(n)
    it = ctypes.c_int(0)
    err = ctypes.c_double(0)
    ok = lib().fo_pcg_threaded(n, _p(rp, ctypes.POINTER(ctypes.c_int64)), _p(ci, ctypes.POINTER(ctypes.c_int32)),
                               _p(v), _p(f), _p(u), int(maxit), float(tol), ctypes.byref(it), ctypes.byref(err))
    if not ok:
        raise RuntimeError("pcg_threaded: no convergence in %d iterations (err %.3e)" % (it.value, err.value))
    return u, it.value, err.value


def assemble_chunked(deck, chunk=16384, threads=None):
    """assemble() for large meshes: element matrices computed in chunks on
    all host threads (the C restatement releases the GIL), each chunk summed
    into the equation-space CSR matrix as it is produced."""
    import scipy.sparse as sp
    from concurrent.futures import ThreadPoolExecutor
    neq = deck.num_eq()
    dofs_all = elem_dofs(deck)
    nd = dofs_all.shape[1]
    ne = deck.num_elems
    starts = list(range(0, ne, chunk))

    def work(a):
        b = min(ne, a + chunk)
        Ke, rc = elems_stiff(deck, np.arange(a, b))
        if rc != 0:
            raise RuntimeError("element stiffness failed in elements %d..%d" % (a, b))
        dofs = dofs_all[a:b]
        I = np.repeat(dofs, nd, axis=1).ravel()
        J = np.tile(dofs, (1, nd)).ravel()
        m = (I > 0) & (J > 0)
        C = sp.csr_matrix((Ke.reshape(b - a, -1).ravel()[m], (I[m] - 1, J[m] - 1)), shape=(neq, neq))
        C.sum_duplicates()
        return C

    K = None
    with ThreadPoolExecutor(max_workers=threads or os.cpu_count()) as ex:
        for C in ex.map(work, starts):
            K = C if K is None else K + C
    K.sum_duplicates()
    K.sort_indices()
    return K


def mass_matrix(deck):
    """Equation-space consistent mass matrix (scipy CSR) from elem_mass."""
    Me = np.array([elem_mass(deck.nn, deck.ngp, deck.coords[deck.conn[e]], deck.rho[e])[0]
                   for e in range(deck.num_elems)])
    return assemble(deck, Me)


def newmark(K, M, f, dt, steps, gamma=0.5, beta=0.25):
    """Linear Newmark of cCtrlNewmark::Solver (ctrl/ctrlnewmark.cpp:79-254),
    without damping, under the constant (step) load f from t = 0, with direct
    solves: a(0) from M a = f, K_eff = K + a0 M, then per step
    f_eff = f + M (a0 u + a2 v + a3 a), u = K_eff^-1 f_eff,
    a <- -a3 a + a0 du - a2 v, v <- v + a6 a_old + a7 a.
    Returns u, v, a per step: three [steps][neq] arrays."""
    import scipy.sparse.linalg as sla
    a0 = 1.0 / (beta * dt * dt)
    a2 = 1.0 / (beta * dt)
    a3 = 0.5 / beta - 1.0
    a6 = (1.0 - gamma) * dt
    a7 = gamma * dt
    n = K.shape[0]
    u = np.zeros(n)
    v = np.zeros(n)
    a = sla.spsolve(M.tocsc(), f)
    lu = sla.splu((K + a0 * M).tocsc())
    U, V, A = [], [], []
    for _ in range(steps):
        fe = f + M @ (a0 * u + a2 * v + a3 * a)
        un = lu.solve(fe)
        du = un - u
        a_old = a
        a = -a3 * a + a0 * du - a2 * v
        v = v + a6 * a_old + a7 * a
        u = un
        U.append(u.copy())
        V.append(v.copy())
        A.append(a.copy())
    return np.array(U), np.array(V), np.array(A)
