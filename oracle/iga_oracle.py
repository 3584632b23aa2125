"""B-spline / NURBS solid element stiffness on the CPU (TEST INFRASTRUCTURE ONLY).

A numpy restatement of what FAST computes for %ELEMENT.BSPLINE.SOLID:
cElmParam::StiffMat (elc/elmparam.cpp:539-597) on the shape functions of
cShapeBspSolid::DrvShpRST (shp/shpbsp.cpp:985-1067), with B and C as
cSolid::BMatrix / QMatrix (elc/anmodel.cpp:1418-1447, 1286-1298):

    K_e = sum_g w_g detJ_g B_g^T C B_g .

The univariate B-splines are evaluated directly from the knot vector by the
Cox-de Boor recurrence (no Bezier extraction), so this checker shares no code
path with the library, which contracts extraction operators with Bernstein
polynomials.  The parameter of the knot span is mapped from the Gauss
coordinate t in [-1, 1] as u = U_k + (t+1)/2 (U_{k+1} - U_k), and the natural
derivative is dN/dt = (U_{k+1} - U_k)/2 dN/du, which is what the reference's
extraction form (Bernstein derivative halved, shp/shpbsp.cpp:277-300) equals.
Rational patches use the quotient N_a = B_a w_a / W; non-rational patches the
plain tensor product (the reference's non-rational derivative branch,
shp/shpbsp.cpp:1015-1030, does not advance its node index, so the reference
itself is only usable as an oracle through its rational branch).

Only ``tests/`` and the golden-fixture script import this module.
"""
from __future__ import annotations

import numpy as np

# FAST's 15-digit Gauss tables (elc/intpoint.cpp:742-800) as numbers
_GR = {2: [-0.577350269189626, 0.577350269189626],
       3: [-0.774596669241483, 0.0, 0.774596669241483],
       4: [-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053],
       5: [-0.906179845938664, -0.538469310105683, 0.0, 0.538469310105683, 0.906179845938664],
       6: [-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197, 0.661209386466264,
           0.932469514203152]}
_GW = {2: [1.0, 1.0],
       3: [0.555555555555556, 0.888888888888889, 0.555555555555556],
       4: [0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454],
       5: [0.236926885056189, 0.478628670499367, 0.568888888888889, 0.478628670499367, 0.236926885056189],
       6: [0.171324492379170, 0.360761573048139, 0.467913934572691, 0.467913934572691, 0.360761573048139,
           0.171324492379170]}


def spans(U):
    """Left knot index of every non-zero span (gap above 1e-5, as the reference)."""
    return [i - 1 for i in range(1, len(U)) if U[i] - U[i - 1] > 1e-5]


def basis(U, p, k, u):
    """Values and u-derivatives of the p+1 B-splines non-zero on span k at u."""
    def N(i, q, x):
        if q == 0:
            return 1.0 if i == k else 0.0
        a = 0.0
        if U[i + q] - U[i] > 0:
            a += (x - U[i]) / (U[i + q] - U[i]) * N(i, q - 1, x)
        if U[i + q + 1] - U[i + 1] > 0:
            a += (U[i + q + 1] - x) / (U[i + q + 1] - U[i + 1]) * N(i + 1, q - 1, x)
        return a

    def dN(i, q, x):
        # dN_{i,q}/du = q/(U_{i+q}-U_i) N_{i,q-1} - q/(U_{i+q+1}-U_{i+1}) N_{i+1,q-1}
        d = 0.0
        if U[i + q] - U[i] > 0:
            d += q / (U[i + q] - U[i]) * N(i, q - 1, x)
        if U[i + q + 1] - U[i + 1] > 0:
            d -= q / (U[i + q + 1] - U[i + 1]) * N(i + 1, q - 1, x)
        return d

    idx = range(k - p, k + 1)
    return np.array([N(i, p, u) for i in idx]), np.array([dN(i, p, u) for i in idx])


def _points(deck, e):
    """(c_g = w_g detJ_g, dN/dx [3][nn]) at every Gauss point of element e of
    a "bsp" deck, points in the rule's order (r fastest)."""
    P = deck.patch
    deg = P.degree
    ng = deck.ngp
    X = deck.coords[deck.conn[e]]
    w = np.ones(len(X)) if (P.weights is None or not P.rational) else P.weights[deck.conn[e]]
    tabs = []
    for d in range(3):
        U = np.asarray(P.knots[d], dtype=np.float64)
        k = spans(U)[int(P.span[e, d])]
        h = U[k + 1] - U[k]
        vals = []
        for t in _GR[ng[d]]:
            n, dn = basis(U, deg[d], k, U[k] + 0.5 * (t + 1.0) * h)
            vals.append((n, 0.5 * h * dn))
        tabs.append(vals)
    for gt in range(ng[2]):
        for gs in range(ng[1]):
            for gr in range(ng[0]):
                wg = _GW[ng[0]][gr] * _GW[ng[1]][gs] * _GW[ng[2]][gt]
                nr, dr = tabs[0][gr]
                ns, ds = tabs[1][gs]
                nt, dt = tabs[2][gt]
                # a = i + Qr j + Qr Qs k (r fastest)
                B = np.einsum("k,j,i->kji", nt, ns, nr).ravel()
                dB = np.stack([np.einsum("k,j,i->kji", nt, ns, dr).ravel(),
                               np.einsum("k,j,i->kji", nt, ds, nr).ravel(),
                               np.einsum("k,j,i->kji", dt, ns, nr).ravel()])
                if P.rational:
                    Bw, dBw = B * w, dB * w
                    W, dW = Bw.sum(), dBw.sum(axis=1)
                    N = Bw / W
                    dN = (dBw - np.outer(dW, N)) / W
                else:
                    dN = dB
                J = dN @ X
                yield wg * np.linalg.det(J), np.linalg.solve(J, dN)


def _cmatrix(E, nu):
    dd = (1 + nu) * (1 - 2 * nu)
    C = np.zeros((6, 6))
    C[:3, :3] = E * nu / dd
    np.fill_diagonal(C[:3, :3], E * (1 - nu) / dd)
    C[3, 3] = C[4, 4] = C[5, 5] = E / (2 * (1 + nu))
    return C


def elem_stiff(deck, e):
    """Stiffness matrix of element e of a "bsp" deck (local DOFs node-major, x y z)."""
    C = _cmatrix(float(deck.E[e]), float(deck.nu[e]))
    nn = deck.conn.shape[1]
    K = np.zeros((3 * nn, 3 * nn))
    for c, dx in _points(deck, e):
        Bm = np.zeros((6, 3 * nn))
        Bm[0, 0::3] = dx[0]
        Bm[1, 1::3] = dx[1]
        Bm[2, 2::3] = dx[2]
        Bm[3, 0::3] = dx[1]
        Bm[3, 1::3] = dx[0]
        Bm[4, 0::3] = dx[2]
        Bm[4, 2::3] = dx[0]
        Bm[5, 1::3] = dx[2]
        Bm[5, 2::3] = dx[1]
        K += c * Bm.T @ C @ Bm
    return K


def elem_stress(deck, e, ue):
    """Gauss-point strains and stresses [ngp][6] (Voigt xx yy zz xy xz yz,
    engineering shears) of element e of a "bsp" deck at element displacements
    ue (cElmParam::IntPntStress, elc/elmparam.cpp:859-935)."""
    C = _cmatrix(float(deck.E[e]), float(deck.nu[e]))
    nn = deck.conn.shape[1]
    U = np.asarray(ue, dtype=np.float64).reshape(nn, 3)
    st, ss = [], []
    for c, dx in _points(deck, e):
        H = U.T @ dx.T
        ev = np.array([H[0, 0], H[1, 1], H[2, 2], H[0, 1] + H[1, 0], H[0, 2] + H[2, 0], H[1, 2] + H[2, 1]])
        st.append(ev)
        ss.append(C @ ev)
    return np.array(st), np.array(ss)


def elem_tl(deck, e, ue):
    """Total-Lagrangian tangent and internal force of element e of a "bsp"
    deck at element displacements ue (cElmParamTL::StiffMat / IntForce,
    elc/elmparam.cpp:1615-1807, with cSolid::BlMatrix / BnlMatrix / SMatrix,
    elc/anmodel.cpp:1451-1568): F = I + grad u, Green strain E = (F^T F - I)/2,
    S = C E, B_L the strain variation (rows xx yy zz xy xz yz, engineering
    shears), K = sum c (B_L^T C B_L + grad N^T S grad N (x) I), g = sum c B_L^T S."""
    C = _cmatrix(float(deck.E[e]), float(deck.nu[e]))
    nn = deck.conn.shape[1]
    U = np.asarray(ue, dtype=np.float64).reshape(nn, 3)
    K = np.zeros((3 * nn, 3 * nn))
    g = np.zeros(3 * nn)
    voigt = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    for c, dx in _points(deck, e):
        F = np.eye(3) + U.T @ dx.T
        Eg = 0.5 * (F.T @ F - np.eye(3))
        ev = np.array([Eg[0, 0], Eg[1, 1], Eg[2, 2], 2 * Eg[0, 1], 2 * Eg[0, 2], 2 * Eg[1, 2]])
        sv = C @ ev
        S = np.array([[sv[0], sv[3], sv[4]], [sv[3], sv[1], sv[5]], [sv[4], sv[5], sv[2]]])
        BL = np.zeros((6, 3 * nn))
        for r, (j, k) in enumerate(voigt):
            for i in range(3):
                if j == k:
                    BL[r, i::3] = F[i, j] * dx[j]
                else:
                    BL[r, i::3] = F[i, j] * dx[k] + F[i, k] * dx[j]
        Gn = dx.T @ S @ dx
        K += c * (BL.T @ C @ BL + np.kron(Gn, np.eye(3)))
        g += c * BL.T @ sv
    return K, g


def elems_stiff(deck, elems=None):
    elems = range(deck.num_elems) if elems is None else elems
    return np.array([elem_stiff(deck, int(e)) for e in elems])


def extrapolation_matrix(degree, ngp):
    """TR [nn][ng] of cElmParam::CompTRMatrix (elc/elmparam.cpp:1444-1535)
    for a B-spline solid element: the least-squares linear field in (r, s, t)
    through the Gauss points (rule order, r fastest) evaluated at the control
    points' natural coordinates, the uniform grid of p+1 points per
    direction over [-1, 1] (cShapeBspSolid::NodeNatCoord,
    shp/shpbsp.cpp:906-923, r fastest); the point average for a one-point
    rule."""
    nb = [int(p) + 1 for p in degree]
    gp = [(r, s, t) for t in _GR.get(ngp[2], [0.0]) for s in _GR.get(ngp[1], [0.0]) for r in _GR.get(ngp[0], [0.0])]
    ng = len(gp)
    nn = nb[0] * nb[1] * nb[2]
    if ngp[0] == 1:
        return np.full((nn, ng), 1.0 / ng)
    U = np.array([[1.0, r, s, t] for r, s, t in gp])
    A = U.T @ U
    Q = np.linalg.solve(A, U.T)                     # [4][ng]: A^-1 u_g for every point
    CN = np.array([[1.0, -1.0 + 2.0 * k / degree[0], -1.0 + 2.0 * j / degree[1], -1.0 + 2.0 * i / degree[2]]
                   for i in range(nb[2]) for j in range(nb[1]) for k in range(nb[0])])
    return CN @ Q
