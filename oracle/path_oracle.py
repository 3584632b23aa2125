"""Path following (arc-length) on the CPU (TEST INFRASTRUCTURE ONLY).

A restatement of cCtrlPath::Solver (ctrl/ctrlpath.cpp:63-265) with the load
increment rules of cIniOrtArcLength, cUpOrtArcLength and cConLinArcLength
(ctrl/ctrlarclen.cpp:95-250), for total-Lagrangian hex8 meshes, with the C
oracle's TL element and a direct solve:

  per iteration:  K du1 = q,  K du2 = r,  dlf = IncLoadFac(du1, du2, Du),
                  du = dlf du1 - du2,  u += du,  lambda += dlf,
                  r = g(u) - lambda q,  converged when |r| / max(1, |q|) < tol
  first iteration of a step: the arc length (step 1: StepFactor (|du1| +
  LoadCoeff), later steps scaled by sqrt(TargetIter / PrevIter)) fixes dlf,
  signed by du1 . Du of the previous step;
  later iterations:  ioal  dlf = (Du0 . du2) / (Du0 . du1 + c Dlf)
                     uoal  dlf = (Du . du2) / (Du . du1 + c Dlf)
                     clinal dlf = (Du . du2 - r0/2) / (Du . du1 + c Dlf),
                            r0 = Du . Du + c Dlf^2 - ArcLen^2
  (c = LoadCoeff, Dlf the load increment of the step so far).

Only ``tests/`` imports this module.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from . import fem_oracle as fo


def tl_state(d, u):
    """(tangent K, internal force g) of a TL hex8 deck at equation vector u."""
    eq = d.node_eq()
    neq = d.num_eq()
    dofs = eq[d.conn].reshape(d.num_elems, -1)
    unode = np.zeros((d.num_nodes, 3))
    m = eq > 0
    unode[m] = u[eq[m] - 1]
    I, J, V, g = [], [], [], np.zeros(neq)
    for e in range(d.num_elems):
        Kt, ge, rc = fo.elem_tl(8, d.ngp, d.coords[d.conn[e]], d.E[e], d.nu[e], unode[d.conn[e]].ravel())
        dd = dofs[e]
        mm = dd > 0
        ii = np.repeat(dd, len(dd)) - 1
        jj = np.tile(dd, len(dd)) - 1
        keep = np.repeat(mm, len(dd)) & np.tile(mm, len(dd))
        I.append(ii[keep]); J.append(jj[keep]); V.append(Kt.ravel()[keep])
        np.add.at(g, dd[mm] - 1, ge[mm])
    K = sp.csr_matrix((np.concatenate(V), (np.concatenate(I), np.concatenate(J))), shape=(neq, neq))
    return K, g


def arclength(d, q, method, steps, step_factor, max_iter, tol, load_coeff=0.0, target_iter=1):
    """Displacements [steps][neq], load factors [steps] and iterations per step."""
    neq = len(q)
    lenq = np.linalg.norm(q)
    u = np.zeros(neq)
    r = np.zeros(neq)
    Du = np.zeros(neq)
    Du0 = np.zeros(neq)
    lam = 0.0
    c = float(load_coeff)
    arclen = 0.0
    prev_iter = 0
    sp0, csp1 = 1.0, 1.0
    us, lams, its = [], [], []
    for step in range(1, steps + 1):
        conv = False
        Dlf = 0.0
        for it in range(1, max_iter + 1):
            K, _ = tl_state(d, u)
            lu = sla.splu(K.tocsc())
            du1 = lu.solve(q)
            du2 = lu.solve(r) if np.any(r) else np.zeros(neq)
            # IncLoadFac
            if step == 1 and it == 1:
                arclen = step_factor * (np.linalg.norm(du1) + c)
                dlf = step_factor
                if method == "ioal":
                    Du0 = dlf * du1
            elif it == 1:
                if target_iter:
                    arclen *= np.sqrt(float(target_iter) / float(prev_iter))
                if c == 1.0 and (abs(csp1) < 0.3 or np.linalg.norm(Du) > tol):
                    arclen = np.linalg.norm(Du)
                    c = 0.0
                dlf = arclen / (np.linalg.norm(du1) + c)
                if du1 @ Du < 0.0:
                    dlf = -dlf
                if method == "ioal":
                    Du0 = dlf * du1
            else:
                if method == "ioal":
                    dlf = (Du0 @ du2) / (Du0 @ du1 + c * Dlf)
                elif method == "uoal":
                    dlf = (Du @ du2) / (Du @ du1 + c * Dlf)
                else:
                    r0 = Du @ Du + c * Dlf * Dlf - arclen * arclen
                    dlf = (Du @ du2 - 0.5 * r0) / (Du @ du1 + c * Dlf)
            if it == 1:
                Dlf = 0.0
                Du = np.zeros(neq)
            Dlf += dlf
            du = dlf * du1 - du2
            lam += dlf
            u = u + du
            Du = Du + du
            _, g = tl_state(d, u)
            r = g - lam * q
            if np.linalg.norm(r) / max(1.0, lenq) < tol:
                conv = True
                break
        if not conv:
            break
        d2 = du1 @ du1
        spv = (q @ du1) / d2 if np.sqrt(d2) > 1e-12 else 1.0
        if step == 1:
            sp0 = spv
        else:
            csp1 = spv / sp0
        prev_iter = it
        us.append(u.copy())
        lams.append(lam)
        its.append(it)
    return np.array(us), np.array(lams), np.array(its)
