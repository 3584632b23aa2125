"""Pin the CPU oracle (oracle/fem_oracle.c) against golden vectors dumped
from the reference FAST program.  CPU only."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fem_oracle as fo
from tests import golden_io as gio

CASES = [n for n in gio.names() if not n.startswith(("nr_", "nm_", "iga_", "arc_", "modal_"))]


@pytest.mark.parametrize("name", CASES)
def test_equation_numbering(name):
    d, g = gio.load(name)
    assert d.num_eq() == int(g["ref_neq"][0])
    np.testing.assert_array_equal(d.node_eq(), g["ref_node_eq"])
    np.testing.assert_array_equal(fo.elem_dofs(d), g["ref_elm_dofs"])


@pytest.mark.parametrize("name", [c for c in CASES if not c.endswith("tl_state")])
def test_element_stiffness(name):
    d, g = gio.load(name)
    el = g["ref_elems"]
    Ke, rc = fo.elems_stiff(d, el)
    assert rc == 0
    for k in range(len(el)):
        assert gio.rel(Ke[k], g["ref_elm_K"][k]) < 1e-13, (name, k)


@pytest.mark.parametrize("name", CASES)
def test_load_vector(name):
    d, g = gio.load(name)
    f = fo.face_loads(d)
    assert gio.rel(f, g["ref_f"]) < 1e-13


@pytest.mark.parametrize("name", [c for c in CASES if "ref_K_data" in gio.load(c)[1]])
def test_assembled_matrix(name):
    d, g = gio.load(name)
    K = fo.assemble(d)
    Kl = sp.tril(K).tocsr()
    R = gio.lower_K(g)
    diff = (Kl - R)
    assert abs(diff).max() / abs(R).max() < 1e-13
    assert Kl.nnz == R.nnz


# Displacement tolerance per deck.  ref_testb8 is singular (the rotation about
# x is not restrained; only its x-displacements are the published answer) and
# is checked by test_known_answer_testb8.  ref_beamb20 is a slender 2x2x50
# cantilever whose reference (skyline Crout) solution itself has a relative
# residual of 4e-8, so agreement is bounded by conditioning, not arithmetic.
U_TOL = {"ref_beamb20": 1e-6}
R_TOL = {"ref_beamb20": 1e-6}


@pytest.mark.parametrize("name", [c for c in CASES if "ref_u" in gio.load(c)[1] and c != "ref_testb8"])
def test_displacements(name):
    d, g = gio.load(name)
    K = fo.assemble(d)
    f = fo.face_loads(d)
    u, ok, it, err = fo.pcg(K, f, 1e-14, 20 * K.shape[0])
    assert ok, (it, err)
    assert np.linalg.norm(K @ u - f) / np.linalg.norm(f) < R_TOL.get(name, 1e-9)
    assert gio.rel(u, g["ref_u"]) < U_TOL.get(name, 1e-9)


def test_known_answer_testb8():
    # Bar sigma=100 MPa, L=5, E=200e9: u = sigma L / E = 2.5e-3 at x=5 (dat/continuum/TestB8.dat:2)
    d, g = gio.load("ref_testb8")
    eq = g["ref_node_eq"]
    u = g["ref_u"]
    for node in (1, 2, 5, 6):  # labels 2, 3, 6, 7
        assert abs(u[eq[node, 0] - 1] - 2.5e-3) < 1e-12


def test_known_answer_beamb20():
    # FEM tip displacements at node 1643 (dat/continuum/BeamB20.dat:5-8)
    d, g = gio.load("ref_beamb20")
    lab = list(g["node_labels"])
    i = lab.index(1643)
    eq = g["ref_node_eq"][i]
    u = g["ref_u"]
    assert abs(u[eq[0] - 1] - 5.001008e-02) < 5e-9
    assert abs(u[eq[1] - 1] - 5.001205e-02) < 5e-9


def test_mass_matrix():
    d, g = gio.load("cfg_hex8_mass")
    for k in g["ref_elems"]:
        X = d.coords[d.conn[k]]
        M, rc = fo.elem_mass(8, d.ngp, X, d.rho[k])
        assert gio.rel(M, g["ref_elm_M"][k]) < 1e-13


def test_total_lagrangian_state():
    d, g = gio.load("cfg_hex8_tl_state")
    eq = d.node_eq()
    u = g["u_state"]
    unode = np.zeros((d.num_nodes, 3))
    m = eq > 0
    unode[m] = u[eq[m] - 1]
    for k in g["ref_elems"]:
        X = d.coords[d.conn[k]]
        ue = unode[d.conn[k]].ravel()
        Kt, ge, rc = fo.elem_tl(8, d.ngp, X, d.E[k], d.nu[k], ue)
        assert gio.rel(Kt, g["ref_elm_K"][k]) < 1e-12
        assert gio.rel(ge, g["ref_elm_g"][k]) < 1e-12


def test_internal_force_linear():
    d, g = gio.load("cfg_hex20_lognormal_4x4x2")
    eq = d.node_eq()
    u = g["ref_u"]
    unode = np.zeros((d.num_nodes, 3))
    m = eq > 0
    unode[m] = u[eq[m] - 1]
    gg = np.zeros(d.num_eq())
    for k in range(d.num_elems):
        ge, rc = fo.elem_intforce(20, d.ngp, d.coords[d.conn[k]], d.E[k], d.nu[k], unode[d.conn[k]].ravel())
        dofs = eq[d.conn[k]].ravel()
        for i, q in enumerate(dofs):
            if q:
                gg[q - 1] += ge[i]
    assert gio.rel(gg, g["ref_g_of_u"]) < 1e-10


def _oracle_tl_newton(d, q, steps, step_factor, tol, maxit):
    """Load-control Newton (cCtrlNR::Solver, ctrl/ctrlnr.cpp:47-270) with the
    oracle's TL element and a direct solve."""
    import scipy.sparse.linalg as sla
    eq = d.node_eq()
    neq = d.num_eq()
    dofs = eq[d.conn].reshape(d.num_elems, -1)
    u = np.zeros(neq)
    out = []

    def state(u):
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

    lam = 0.0
    K, g = state(u)
    for step in range(steps):
        lam += step_factor
        f = lam * q
        r = f - g
        for it in range(maxit):
            K, _ = state(u)
            u = u + sla.spsolve(K.tocsc(), r)
            _, g = state(u)
            r = f - g
            if np.linalg.norm(r) / max(1.0, np.linalg.norm(f)) < tol:
                break
        out.append(u.copy())
    return np.array(out)


def test_oracle_newton_matches_reference_nr():
    """The oracle's TL element inside FAST's Newton loop reproduces the
    displacements the reference's own cCtrlNR printed for every step."""
    d, g = gio.load("nr_plate_tl")
    us = _oracle_tl_newton(d, g["ref_f"], int(g["steps"]), float(g["step_factor"]), float(g["tol"]), int(g["maxit"]))
    eq = d.node_eq()
    m = eq > 0
    for k in range(len(us)):
        unode = np.zeros((d.num_nodes, 3))
        unode[m] = us[k][eq[m] - 1]
        assert gio.rel(unode, g["ref_u_steps"][k]) < 1e-8, k


def test_oracle_newmark_matches_reference():
    """The oracle's restatement of cCtrlNewmark::Solver (with the oracle's K
    and consistent M) reproduces the displacements, velocities and
    accelerations the reference's own `fast` binary printed for every step."""
    d, g = gio.load("nm_hex20_box")
    K = fo.assemble(d)
    M = fo.mass_matrix(d)
    U, V, A = fo.newmark(K, M, g["ref_f"], float(g["time_step"]), int(g["steps"]), float(g["gamma"]),
                         float(g["beta"]))
    eq = g["ref_node_eq"].reshape(-1, 3)
    m = eq > 0
    for name, X, R in (("u", U, g["ref_u_steps"]), ("v", V, g["ref_v_steps"]), ("a", A, g["ref_a_steps"])):
        for s in range(X.shape[0]):
            node = np.zeros(eq.shape)
            node[m] = X[s][eq[m] - 1]
            assert gio.rel(node, R[s]) < 1e-9, (name, s, gio.rel(node, R[s]))


@pytest.mark.parametrize("name", [c for c in CASES if "ref_elm_stress" in gio.load(c)[1]])
def test_gauss_point_stresses(name):
    """Strains and stresses at the Gauss points of the reference's solution
    (cElement::IntPntStress) from the C restatement."""
    d, g = gio.load(name)
    eq = d.node_eq()
    u = g["ref_u"]
    for k, e in enumerate(g["ref_elems"]):
        dofs = eq[d.conn[e]].ravel()
        ue = np.where(dofs > 0, u[np.maximum(dofs - 1, 0)], 0.0)
        st, ss, rc = fo.elem_stress(d.nn, d.ngp, d.coords[d.conn[e]], d.E[e], d.nu[e], ue)
        assert rc == 0
        assert np.abs(st - g["ref_elm_strain"][k]).max() <= 1e-12 * np.abs(g["ref_elm_strain"]).max()
        assert np.abs(ss - g["ref_elm_stress"][k]).max() <= 1e-12 * np.abs(g["ref_elm_stress"]).max()


@pytest.mark.parametrize("name", [c for c in CASES if "ref_elm_nodal_stress" in gio.load(c)[1]])
def test_extrapolated_and_averaged_nodal_stresses(name):
    """cElmParam::NodalStress (TR x Gauss-point stresses, CompTRMatrix) and
    cControl::PrintAvrNodalStress from the oracle at the reference's
    solution, against the harness dump and the `fast` binary's .pos print."""
    d, g = gio.load(name)
    assert list(g["ref_pos_stress_labels"]) == ["STRESS_XX", "STRESS_YY", "STRESS_ZZ", "STRESS_XY", "STRESS_XZ",
                                                "STRESS_YZ"]
    TR, rc = fo.extrap_matrix(d.nn, d.ngp)
    assert rc == 0
    np.testing.assert_allclose(TR.sum(axis=1), 1.0, rtol=0, atol=1e-14)  # constants extrapolate exactly
    eq = d.node_eq()
    u = g["ref_u"]
    en = np.zeros((d.num_elems, d.nn, 6))
    for e in range(d.num_elems):
        dofs = eq[d.conn[e]].ravel()
        ue = np.where(dofs > 0, u[np.maximum(dofs - 1, 0)], 0.0)
        _, ss, rc = fo.elem_stress(d.nn, d.ngp, d.coords[d.conn[e]], d.E[e], d.nu[e], ue)
        en[e] = TR @ ss
    scale = np.abs(g["ref_elm_nodal_stress"]).max()
    assert np.abs(en[g["ref_elems"]] - g["ref_elm_nodal_stress"]).max() <= 1e-12 * scale
    assert np.abs(en - g["ref_pos_elm_nodal_stress"]).max() <= 1e-12 * scale
    avg = fo.averaged_nodal_stress(d.num_nodes, d.conn, en)
    assert np.abs(avg - g["ref_pos_nodal_stress_avg"]).max() <= 1e-12 * scale


@pytest.mark.parametrize("method", ["ioal", "uoal", "clinal"])
def test_oracle_arclength_matches_reference(method):
    """The oracle's restatement of cCtrlPath with the arc-length rules
    reproduces the displacements and load factors that the reference's own
    `fast` binary printed for every step."""
    from oracle import path_oracle as po
    d, g = gio.load("arc_plate_tl")
    us, lams, its = po.arclength(d, g["ref_f"], method, int(g["steps"]), float(g["step_factor"]), int(g["maxit"]),
                                 float(g["tol"]), float(g["load_coeff"]), int(g["target_iter"]))
    assert len(lams) == len(g["ref_lam_" + method])
    assert np.abs(lams - g["ref_lam_" + method]).max() < 1e-10
    eq = d.node_eq()
    m = eq > 0
    for k in range(len(us)):
        unode = np.zeros((d.num_nodes, 3))
        unode[m] = us[k][eq[m] - 1]
        assert gio.rel(unode, g["ref_u_steps_" + method][k]) < 1e-9, k


@pytest.mark.parametrize("name", ["modal_hex8_cantilever", "modal_hex20_block"])
def test_oracle_modal_matches_reference(name):
    """The oracle's subspace iteration (cGenEigSubSpaces) on the oracle's K
    and M reproduces the natural frequencies and mode shapes the reference's
    `fast` binary printed (ModalAnalysis, SubspaceIteration)."""
    from oracle import eig_oracle as eo
    d, g = gio.load(name)
    K = fo.assemble(d)
    M = fo.mass_matrix(d)
    lam, X, it, ok = eo.subspace(K, M, int(g["num_modes"]), float(g["tol"]), int(g["maxit"]))
    assert ok
    assert np.abs(np.sqrt(lam) / g["ref_freq"] - 1.0).max() < 1e-11
    eq = d.node_eq()
    m = eq > 0
    for k in range(len(lam)):
        node = np.zeros((d.num_nodes, 3))
        node[m] = X[k][eq[m] - 1]
        R = g["ref_modes"][k]
        sgn = np.sign(np.sum(node * R))
        assert np.abs(sgn * node - R).max() <= 1e-5 * np.abs(R).max(), k


@pytest.mark.parametrize("name", ["buck_hex8_column", "buck_hex20_column"])
def test_element_geometric_stiffness(name):
    """cElmParam::GeomStiff at the reference's linear solution."""
    d, g = gio.load(name)
    eq = d.node_eq()
    unode = np.zeros((d.num_nodes, 3))
    m = eq > 0
    unode[m] = g["ref_u"][eq[m] - 1]
    for k, e in enumerate(g["ref_elems"]):
        Ge, rc = fo.elem_geom(d.nn, d.ngp, d.coords[d.conn[e]], d.E[e], d.nu[e], unode[d.conn[e]].ravel())
        assert rc == 0
        assert gio.rel(Ge, g["ref_elm_G"][k]) < 1e-13, e


@pytest.mark.parametrize("name", ["buck_hex8_column", "buck_hex20_column"])
def test_oracle_buckling_matches_reference(name):
    """Linear buckling (cCtrlLinStab): the oracle's subspace iteration on K and
    minus the geometric stiffness at the linear solution reproduces the
    buckling factors and modes the reference's `fast` binary printed."""
    import scipy.sparse.linalg as sla
    from oracle import eig_oracle as eo
    d, g = gio.load(name)
    K = fo.assemble(d)
    u = sla.spsolve(K.tocsc(), fo.face_loads(d))
    G = fo.geom_matrix(d, u)
    lam, X, it, ok = eo.subspace(K, -G, int(g["num_modes"]), float(g["tol"]), int(g["maxit"]), swapped=True)
    assert ok
    assert np.abs(lam / g["ref_lambda"] - 1.0).max() < 1e-9
    eq = d.node_eq()
    m = eq > 0
    for k in range(len(lam)):
        node = np.zeros((d.num_nodes, 3))
        node[m] = X[k][eq[m] - 1]
        R = g["ref_modes"][k]
        sgn = np.sign(np.sum(node * R))
        assert np.abs(sgn * node - R).max() <= 1e-5 * np.abs(R).max(), k


@pytest.mark.parametrize("name", [c for c in CASES if "ref_reactions" in gio.load(c)[1]])
def test_support_reactions(name):
    """cControl::SuppReactions at the reference's solution from the oracle's
    element forces and face loads, against the reference's own."""
    d, g = gio.load(name)
    R = fo.support_reactions(d, g["ref_u"])
    ref = g["ref_reactions"][:, :3]
    assert np.abs(R - ref).max() <= 1e-13 * np.abs(ref).max()
