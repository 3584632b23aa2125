"""Regenerate the golden fixtures in this directory from the reference FAST
program itself.

Run where the reference tree is present, with FAST_REF set to it:

    FAST_REF=<reference tree> python tests/golden/make_golden.py          (all fixtures)
    python tests/golden/make_golden.py iga      (B-spline solid fixtures only)
    python tests/golden/make_golden.py stress   (the two fixtures with Gauss-point stresses)
    python tests/golden/make_golden.py arc      (the path-following fixture)
    python tests/golden/make_golden.py pos      (.pos files next to the numbers they print)
    python tests/golden/make_golden.py modal    (natural frequencies and mode shapes)
    python tests/golden/make_golden.py buckling (buckling factors, modes, geometric stiffness)
    python tests/golden/make_golden.py damped   (Newmark with Rayleigh damping)
    python tests/golden/make_golden.py bspmass  (consistent mass of B-spline solids)
    python tests/golden/make_golden.py variants (cCtrlNR on the learned predictor's training variants)

It builds ``oracle/_ref/fastref`` (the reference's own sources compiled by
``oracle/Makefile``, plus a dump harness), writes each deck with
``fast_b200.decks.write_dat`` (or copies a deck shipped with the reference),
runs the harness on it and stores the reference's element matrices, recorded
global-matrix Add calls, load vector and displacements as ``.npz``.  Nothing
here is hand-written data: every number comes out of the reference run.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from fast_b200 import decks  # noqa: E402
from oracle import refdump  # noqa: E402

FAST_REF = os.environ.get("FAST_REF", "")
if __name__ == "__main__" and not os.path.isdir(FAST_REF):
    sys.exit("set FAST_REF to the reference FAST source tree")


def deck_arrays(d: decks.Deck) -> dict:
    out = dict(kind=np.array(d.kind), coords=d.coords, conn=d.conn, E=d.E, nu=d.nu,
               ngp=np.array(d.ngp, np.int32), fixed=d.fixed, tl=np.array(int(d.total_lagrangian)))
    if d.face_elem is not None:
        out.update(face_elem=d.face_elem, face_corners=d.face_corners, face_q=d.face_q,
                   face_local=d.face_local)
    if d.rho is not None:
        out["rho"] = d.rho
    if d.node_labels is not None:
        out["node_labels"] = d.node_labels
    if d.nodal_f is not None:
        out["nodal_f"] = d.nodal_f
    if d.solver_rank is not None:
        out["solver_rank"] = d.solver_rank
    if d.patch is not None:
        P = d.patch
        out.update(patch_degree=np.array(P.degree, np.int32), patch_span=P.span, patch_grid=np.array(P.grid),
                   patch_cps=P.cps, patch_rational=np.array(int(bool(P.rational))),
                   **{f"patch_knots{k}": np.asarray(P.knots[k]) for k in range(3)})
        if P.weights is not None:
            out["patch_weights"] = P.weights
    return out


def lower_csr(ref: dict):
    n = int(ref["neq"][0])
    K = refdump.lower_csr_from_triplets(n, ref["K_i"], ref["K_j"], ref["K_v"])
    return dict(K_indptr=K.indptr.astype(np.int64), K_indices=K.indices.astype(np.int32), K_data=K.data)


def run_case(name, deck, tmp, keep_elems=None, triplets=True, extra=(), uvec=None, mass=False, stress=False):
    base = os.path.join(tmp, name)
    decks.write_dat(deck, base)
    opts = list(extra)
    if stress:
        opts += ["--stress", "--nodal", "--reactions"]
    if not triplets:
        opts.append("--no-triplets")
    if mass:
        opts.append("--mass")
    if uvec is not None:
        upath = base + ".u.f8"
        np.asarray(uvec, "<f8").tofile(upath)
        opts += ["--u", upath]
    ref = refdump.run_dump(base, base + ".bin", *opts)
    out = deck_arrays(deck)
    out["ref_neq"] = ref["neq"]
    out["ref_node_eq"] = ref["node_eq"]
    sel = slice(None) if keep_elems is None else np.asarray(keep_elems)
    out["ref_elems"] = np.arange(deck.num_elems)[sel]
    out["ref_elm_K"] = ref["elm_K"][sel]
    out["ref_elm_g"] = ref["elm_g"][sel]
    out["ref_elm_dofs"] = ref["elm_dofs"]
    if "elm_M" in ref:
        out["ref_elm_M"] = ref["elm_M"][sel]
    if "elm_stress" in ref:
        out["ref_elm_strain"] = ref["elm_strain"][sel]
        out["ref_elm_stress"] = ref["elm_stress"][sel]
        if "elm_nodal_stress" in ref:
            out["ref_elm_nodal_stress"] = ref["elm_nodal_stress"][sel]
    if "elm_G" in ref:
        out["ref_elm_G"] = ref["elm_G"][sel]
    if "reactions" in ref:
        out["ref_reactions"] = ref["reactions"]
    out["ref_f"] = ref["f"]
    if triplets:
        out.update({"ref_" + k: v for k, v in lower_csr(ref).items()})
    if "u" in ref:
        out["ref_u"] = ref["u"]
        out["ref_g_of_u"] = ref["g_of_u"]
    if uvec is not None:
        out["u_state"] = np.asarray(uvec)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: neq={int(ref['neq'][0])} ne={deck.num_elems} "
          f"-> {os.path.getsize(os.path.join(HERE, name + '.npz')) / 1e6:.2f} MB")


def iga_cases(tmp):
    """B-spline solids: two seeded blocks with jittered control points (rational
    flag with unit weights, the reference's usable shape branch) solved by the
    reference's sparse PCG, and the reference's own NURBS deck
    dat/iga/ScordelisLoDeg3.dat (weights, degrees 3 x 3 x 2)."""
    d = decks.bspline_box(2, (3, 2, 2), L=(3.0, 2.0, 1.0), jitter=0.05, seed=1)
    d.tol = 1e-13
    d.maxit = 100000
    run_case("iga_p2_box", d, tmp, extra=("--stress", "--nodal"))
    d = decks.bspline_box(3, (2, 2, 1), L=(2.0, 2.0, 0.5), jitter=0.05, seed=2)
    d.tol = 1e-13
    d.maxit = 100000
    run_case("iga_p3_box", d, tmp, keep_elems=np.array([0, 3]))
    src = os.path.join(FAST_REF, "dat/iga/ScordelisLoDeg3.dat")
    d = decks.read_dat(src)
    base = os.path.join(tmp, "iga_scordelis_deg3")
    shutil.copy(src, base + ".dat")
    os.chmod(base + ".dat", 0o644)
    ref = refdump.run_dump(base, base + ".bin")
    out = deck_arrays(d)
    keep = np.array([0, 9, 63])
    out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_elems=keep, ref_elm_K=ref["elm_K"][keep],
               ref_elm_dofs=ref["elm_dofs"], ref_f=ref["f"], ref_u=ref["u"])
    out.update({"ref_" + k: v for k, v in lower_csr(ref).items()})
    np.savez_compressed(os.path.join(HERE, "iga_scordelis_deg3.npz"), **out)
    print("iga_scordelis_deg3 written")
    # the reference's higher-degree NURBS cylinders: degrees (4, 2, 4) with a
    # 5-point rule and (5, 2, 5) with a 6-point rule
    for nm, deck, keep in (("iga_pincyl_deg4", "PinCylDeg4.dat", np.array([0, 31, 63])),
                           ("iga_thincyl_deg5", "ThinCylinderDeg5.dat", np.array([0, 40, 79]))):
        iga_reference_deck(tmp, nm, deck, keep)
    iga_tl_cases(tmp)


def plate_variant_cases(tmp, variants=2, steps=4):
    """The learned predictor's training data come from seeded pressure /
    stiffness variants of one plate (fast_b200.learned.trajectories): the
    reference's own cCtrlNR (unmodified `fast` binary) on the same variants,
    every printed step, to check those trajectories against."""
    base_deck = dict(nx=8, ny=8, nz=2, L=4.0, t=0.4, pressure=8.0, steps=steps, tol=1e-10, maxit=30)
    d0 = decks.plate_tl_hex8(**base_deck)
    out = deck_arrays(d0)
    base0 = os.path.join(tmp, "plate_variant_base")
    decks.write_dat(d0, base0)
    ref = refdump.run_dump(base0, base0 + ".bin", "--no-solve", "--no-triplets")
    out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_f=ref["f"])
    us = []
    for v in range(variants):
        ps, E = decks.plate_variant_params(v, d0.num_elems, float(np.median(d0.E)))
        d = decks.plate_tl_hex8(**{**base_deck, "pressure": base_deck["pressure"] * ps})
        d.E = E
        base = os.path.join(tmp, "plate_variant_%d" % v)
        decks.write_dat(d, base)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        us.append(decks.read_pos_displacements(base + ".pos"))
    out.update(ref_u_steps=np.stack(us), variants=np.array(variants), steps=np.array(steps),
               tol=np.array(base_deck["tol"]), maxit=np.array(base_deck["maxit"]))
    np.savez_compressed(os.path.join(HERE, "nr_plate_variants.npz"), **out)
    print("nr_plate_variants:", out["ref_u_steps"].shape)


def bspline_mass_cases(tmp):
    """Consistent mass of B-spline solids (cElmParam::MassMat on the
    cShapeBspSolid basis): jittered degree-2 and degree-3 blocks with density."""
    for name, p, n, L, seed in (("iga_p2_mass", 2, (3, 2, 2), (3.0, 2.0, 1.0), 4),
                                ("iga_p3_mass", 3, (2, 2, 1), (2.0, 2.0, 0.5), 5)):
        d = decks.bspline_box(p, n, L=L, jitter=0.05, seed=seed)
        d.rho = np.full(d.num_elems, 1.3e-3)   # one material: one density
        run_case(name, d, tmp, mass=True, triplets=False, keep_elems=np.arange(6 if p == 2 else 2))


def iga_tl_cases(tmp):
    """dat/iga/CurvedBeamDeg4.dat: total-Lagrangian NURBS solid (degrees
    4, 2, 2, 5-point rule) under load control.  The unmodified `fast`
    binary's displacements and load factor of every printed step (15 digits),
    and from
    the harness the element tangents and internal forces at one of those
    states, the load vector and the equation numbering."""
    src = os.path.join(FAST_REF, "dat/iga/CurvedBeamDeg4.dat")
    d = decks.read_dat(src)
    base = os.path.join(tmp, "iga_curvedbeam_tl")
    # the deck as shipped, with 15 printed digits (it asks for the default 5)
    text = open(src).read().replace("%END", "%HEADER.OUTPUT.PRECISION\n15\n\n%END")
    with open(base + ".dat", "w") as fp:
        fp.write(text)
    subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
    us = decks.read_pos_displacements(base + ".pos")
    lam = decks.read_pos_factors(base + ".pos")
    ref0 = refdump.run_dump(base, base + "0.bin", "--no-solve", "--no-triplets")
    eq = ref0["node_eq"].reshape(-1, 3)
    k = len(us) // 2
    u_state = np.zeros(int(ref0["neq"][0]))
    m = eq > 0
    u_state[eq[m] - 1] = us[k][m]
    upath = base + ".u.f8"
    u_state.astype("<f8").tofile(upath)
    ref = refdump.run_dump(base, base + ".bin", "--u", upath, "--no-triplets")
    out = deck_arrays(d)
    out.update(ref_neq=ref0["neq"], ref_node_eq=ref0["node_eq"], ref_elm_dofs=ref0["elm_dofs"], ref_f=ref0["f"],
               ref_elems=np.arange(d.num_elems), ref_elm_K0=ref0["elm_K"], u_state=u_state,
               ref_elm_K=ref["elm_K"], ref_elm_g=ref["elm_g"], ref_u_steps=us, ref_lam=lam, state_step=np.array(k),
               steps=np.array(200), step_factor=np.array(0.005), tol=np.array(1e-8), maxit=np.array(100))
    np.savez_compressed(os.path.join(HERE, "iga_curvedbeam_tl.npz"), **out)
    print("iga_curvedbeam_tl:", us.shape, lam[:3], lam[-1])


def iga_reference_deck(tmp, name, deck, keep):
    """A deck shipped with the reference under dat/iga, with the harness's
    element matrices (elements ``keep``), load and solution (the recorded K
    of these dense patches would be megabytes: the assembled K is checked
    against the oracle's assembly of element matrices pinned here)."""
    src = os.path.join(FAST_REF, "dat/iga", deck)
    d = decks.read_dat(src)
    base = os.path.join(tmp, name)
    shutil.copy(src, base + ".dat")
    os.chmod(base + ".dat", 0o644)
    ref = refdump.run_dump(base, base + ".bin")
    out = deck_arrays(d)
    out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_elems=keep, ref_elm_K=ref["elm_K"][keep],
               ref_elm_dofs=ref["elm_dofs"], ref_f=ref["f"], ref_u=ref["u"])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "written", d.patch.degree, d.ngp, d.num_elems, int(ref["neq"][0]))


def arc_cases(tmp):
    """The reference's own path-following controller (cCtrlPath with the
    'ioal', 'uoal' and 'clinal' arc-length rules, unmodified `fast` binary) on
    a small TL plate: displacements and load factors of every step."""
    out = None
    for alg in ("ioal", "uoal", "clinal"):
        d = decks.plate_tl_hex8(6, 6, 2, L=4.0, t=0.4, pressure=8.0, steps=8, tol=1e-10, maxit=30)
        d.algorithm = alg
        d.step_factor = 0.15
        d.arc_load_coeff = 0.0
        d.target_iter = 4
        base = os.path.join(tmp, "arc_" + alg)
        decks.write_dat(d, base)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        us = decks.read_pos_displacements(base + ".pos")
        lam = decks.read_pos_factors(base + ".pos")
        if out is None:
            ref = refdump.run_dump(base, base + ".bin", "--no-solve", "--no-triplets")
            out = deck_arrays(d)
            out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_f=ref["f"], steps=np.array(d.maxstep),
                       step_factor=np.array(d.step_factor), tol=np.array(d.tol), maxit=np.array(d.maxit),
                       load_coeff=np.array(d.arc_load_coeff), target_iter=np.array(d.target_iter))
        out["ref_u_steps_" + alg] = us
        out["ref_lam_" + alg] = lam
    np.savez_compressed(os.path.join(HERE, "arc_plate_tl.npz"), **out)
    print("arc_plate_tl:", out["ref_u_steps_clinal"].shape, out["ref_lam_clinal"])


def read_pos_nodal_stresses(path):
    """The last step's element-nodal stresses (%RESULT.CASE.STEP.ELEMENT.NODAL.
    SCALAR.DATA, cControl::PrintNodalStress ctrl/ctrl.cpp:2264-2320) and averaged
    nodal stresses (%RESULT.CASE.STEP.NODAL.SCALAR.DATA, PrintAvrNodalStress
    :2397-2470) of a .pos file, with their scalar labels."""
    lines = open(path).read().splitlines()
    out = {}
    for i, ln in enumerate(lines):
        t = ln.strip()
        if t in ("%RESULT.CASE.STEP.ELEMENT.NODAL.SCALAR", "%RESULT.CASE.STEP.NODAL.SCALAR"):
            out[t[18:] + ".labels"] = lines[i + 2].replace("'", " ").split()
        elif t == "%RESULT.CASE.STEP.ELEMENT.NODAL.SCALAR.DATA":
            ne = int(lines[i + 1].split()[0])
            rows, j = [], i + 2
            for _ in range(ne):
                j += 1  # element label
                blk = []
                while j < len(lines) and lines[j].strip() and not lines[j].strip().lstrip("+-").isdigit():
                    blk.append([float(v) for v in lines[j].split()])
                    j += 1
                rows.append(blk)
            out["ELEMENT.NODAL"] = np.array(rows)
        elif t == "%RESULT.CASE.STEP.NODAL.SCALAR.DATA":
            n = int(lines[i + 1].split()[0])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            lab = np.array([int(r[0]) for r in rows])
            out["NODAL"] = np.array([[float(v) for v in r[1:]] for r in rows])[np.argsort(lab)]
    return out


def stress_cases(tmp):
    """Decks whose fixtures also hold the reference's Gauss-point strains and
    stresses at its solution (cElement::IntPntStress), its extrapolated
    element-nodal stresses (cElmParam::NodalStress) and, from the unmodified
    `fast` binary's .pos with %HEADER.PRINT.AVERAGE.NODAL.STRESS, the printed
    element-nodal and averaged nodal stresses."""
    # hex8 cantilever 20x4x4 (1500 equations), skyline + Crout
    cases = [("cfg_hex8_cantilever", decks.cantilever_hex8())]
    # hex20 lognormal boxes (sparse Jacobi-PCG in the reference), small enough for full dumps
    d = decks.box_hex20_lognormal(4, 4, 2, seed=7)
    d.tol = 1e-13
    cases.append(("cfg_hex20_lognormal_4x4x2", d))
    for name, d in cases:
        run_case(name, d, tmp, stress=True)
        base = os.path.join(tmp, name + "_pos")
        path = decks.write_dat(d, base)
        text = open(path).read().replace("%END", "%HEADER.PRINT.AVERAGE.NODAL.STRESS\n1\n\n%END")
        open(path, "w").write(text)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        pos = read_pos_nodal_stresses(base + ".pos")
        f = os.path.join(HERE, name + ".npz")
        z = dict(np.load(f))
        z["ref_pos_elm_nodal_stress"] = pos["ELEMENT.NODAL"]
        z["ref_pos_nodal_stress_avg"] = pos["NODAL"]
        z["ref_pos_stress_labels"] = np.array(pos["NODAL.SCALAR.labels"])
        np.savez_compressed(f, **z)
        print(name, "pos stresses", pos["ELEMENT.NODAL"].shape, pos["NODAL"].shape, pos["NODAL.SCALAR.labels"])


def pos_cases(tmp):
    """The unmodified `fast` binary's .pos files next to the numbers they
    print: two linear static decks with every stress block (the harness's
    displacements and stresses of the same run), and a three-step Newton run
    on small-strain bricks whose numbers are read back from the file
    (precision 14, so every printed value survives the round trip)."""
    out = {}
    for name, d in (("hex8", decks.cantilever_hex8(3, 2, 2)),
                    ("hex20", decks.box_hex20_lognormal(2, 2, 1, seed=3))):
        base = os.path.join(tmp, "pos_" + name)
        path = decks.write_dat(d, base)
        text = open(path).read().replace("%END", "%HEADER.PRINT.AVERAGE.NODAL.STRESS\n1\n\n%END")
        open(path, "w").write(text)
        ref = refdump.run_dump(base, base + ".bin", "--stress", "--no-triplets")
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        for k, v in deck_arrays(d).items():
            out[f"{name}_{k}"] = v
        out[f"{name}_dat"] = np.frombuffer(open(path, "rb").read(), np.uint8)
        out[f"{name}_pos"] = np.frombuffer(open(base + ".pos", "rb").read(), np.uint8)
        out[f"{name}_ref_node_eq"] = ref["node_eq"]
        out[f"{name}_ref_u"] = ref["u"]
        out[f"{name}_ref_elm_stress"] = ref["elm_stress"]
        out[f"{name}_ref_elm_nodal_stress"] = ref["elm_nodal_stress"]
    d = decks.cantilever_hex8(3, 2, 2)
    d.algorithm, d.maxstep, d.step_factor, d.maxit, d.tol = "lcm", 3, 1.0 / 3.0, 10, 1e-10
    base = os.path.join(tmp, "pos_steps")
    path = decks.write_dat(d, base)
    text = open(path).read().replace("%HEADER.OUTPUT.PRECISION\n15", "%HEADER.OUTPUT.PRECISION\n14")
    open(path, "w").write(text)
    subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
    out["steps_dat"] = np.frombuffer(open(path, "rb").read(), np.uint8)
    out["steps_pos"] = np.frombuffer(open(base + ".pos", "rb").read(), np.uint8)
    # eigen analyses: modal (no printed step) and linear buckling (the linear
    # step, then the modes), precision 14
    dm = decks.cantilever_hex8(6, 2, 3, L=(6.0, 1.0, 1.6))
    dm.rho = np.full(dm.num_elems, 2.0)
    dm.algorithm, dm.tol, dm.maxit = "ModalAnalysis", 1e-6, 200
    db = decks.cantilever_hex8(12, 2, 3, L=(12.0, 1.0, 1.6), q=(-1.0, 0.0, 0.0))
    db.algorithm, db.tol, db.maxit = "LinearStability", 1e-6, 200
    for key, d in (("modal", dm), ("buck", db)):
        base = os.path.join(tmp, "pos_" + key)
        path = decks.write_dat(d, base)
        text = open(path).read().replace("%HEADER.OUTPUT.PRECISION\n15", "%HEADER.OUTPUT.PRECISION\n14").replace(
            "%END", "%HEADER.ANALYSIS.EIGEN.ALGORITHM\n'SubspaceIteration'\n\n"
                    "%HEADER.ANALYSIS.EIGEN.NUMBER.MODES\n3\n\n%END")
        open(path, "w").write(text)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        out[key + "_dat"] = np.frombuffer(open(path, "rb").read(), np.uint8)
        out[key + "_pos"] = np.frombuffer(open(base + ".pos", "rb").read(), np.uint8)
    # support reactions (%HEADER.PRINT.SUPPORT.REACTIONS), precision 14
    dr = decks.cantilever_hex8(3, 2, 2)
    base = os.path.join(tmp, "pos_reac")
    path = decks.write_dat(dr, base)
    text = open(path).read().replace("%HEADER.OUTPUT.PRECISION\n15", "%HEADER.OUTPUT.PRECISION\n14").replace(
        "%END", "%HEADER.PRINT.SUPPORT.REACTIONS\n1\n\n%END")
    open(path, "w").write(text)
    subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
    out["reac_dat"] = np.frombuffer(open(path, "rb").read(), np.uint8)
    out["reac_pos"] = np.frombuffer(open(base + ".pos", "rb").read(), np.uint8)
    # Newmark: three printed steps with velocities and accelerations
    dn = decks.cantilever_hex8(4, 2, 2)
    dn.rho = np.full(dn.num_elems, 1e-3)
    dn.algorithm, dn.maxstep, dn.time_step, dn.print_step, dn.matrix_type = "newmark", 3, 1e-3, 1, "skyline"
    base = os.path.join(tmp, "pos_newmark")
    path = decks.write_dat(dn, base)
    text = open(path).read().replace("%HEADER.OUTPUT.PRECISION\n15", "%HEADER.OUTPUT.PRECISION\n14")
    open(path, "w").write(text)
    subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
    out["newmark_dat"] = np.frombuffer(open(path, "rb").read(), np.uint8)
    out["newmark_pos"] = np.frombuffer(open(base + ".pos", "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "pos_output.npz"), **out)
    print("pos_output:", {k: v.shape for k, v in out.items() if k.endswith("pos")})


def read_pos_modes(path):
    """Natural frequencies and eigenvectors of a modal .pos
    (cCtrlModal::PrintMode, ctrl/ctrlmodal.cpp:128-155): [modes], [modes][nnode][3]."""
    lines = open(path).read().splitlines()
    freq, modes = [], []
    for i, ln in enumerate(lines):
        if ln.strip() == "%RESULT.CASE.STEP.NATURAL.FREQUENCY":
            freq.append(float(lines[i + 1].split()[1]))
        elif ln.strip() == "%RESULT.CASE.STEP.NODAL.EIGENVECTOR":
            n = int(lines[i + 1].split()[0])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            lab = np.array([int(r[0]) for r in rows])
            modes.append(np.array([[float(v) for v in r[1:4]] for r in rows])[np.argsort(lab)])
    return np.array(freq), np.array(modes)


def modal_cases(tmp):
    """The reference's modal analysis (cCtrlModal with cGenEigSubSpaces,
    unmodified `fast` binary): natural frequencies and mode shapes of a
    cantilever with an oblong section (distinct modes) and of a hex20 block."""
    d8 = decks.cantilever_hex8(6, 2, 3, L=(6.0, 1.0, 1.6))
    d8.rho = np.full(d8.num_elems, 2.0)
    d20 = decks.box_hex20_lognormal(3, 2, 2, L=(3.0, 2.0, 1.3), seed=5)
    d20.rho = np.full(d20.num_elems, 1.5)
    for name, d, nm in (("modal_hex8_cantilever", d8, 5), ("modal_hex20_block", d20, 6)):
        d.algorithm, d.tol, d.maxit = "ModalAnalysis", 1e-6, 200
        base = os.path.join(tmp, name)
        path = decks.write_dat(d, base)
        text = open(path).read().replace(
            "%END", f"%HEADER.ANALYSIS.EIGEN.ALGORITHM\n'SubspaceIteration'\n\n"
                    f"%HEADER.ANALYSIS.EIGEN.NUMBER.MODES\n{nm}\n\n%END")
        open(path, "w").write(text)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        freq, modes = read_pos_modes(base + ".pos")
        ref = refdump.run_dump(base, base + ".bin", "--no-solve", "--no-triplets")
        out = deck_arrays(d)
        out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_freq=freq, ref_modes=modes,
                   num_modes=np.array(nm), tol=np.array(d.tol), maxit=np.array(d.maxit))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, freq)


def buckling_cases(tmp):
    """The reference's linear buckling (cCtrlLinStab with cGenEigSubSpaces,
    unmodified `fast` binary) of two compressed columns: buckling factors and
    modes from its .pos, and from the harness the linear solution and the
    element geometric stiffness at it (cElmParam::GeomStiff)."""
    d8 = decks.cantilever_hex8(12, 2, 3, L=(12.0, 1.0, 1.6), q=(-1.0, 0.0, 0.0))
    d20 = decks.box_hex20_lognormal(2, 2, 10, L=(1.0, 1.3, 10.0), seed=9)
    d20.matrix_type = "skyline"  # the linear solve direct, as for the eigen solves
    for name, d, nm, keep in (("buck_hex8_column", d8, 3, np.array([0, 5, 40, 71])),
                              ("buck_hex20_column", d20, 3, np.array([0, 7, 39]))):
        d.algorithm, d.tol, d.maxit = "LinearStability", 1e-6, 200
        run_case(name, d, tmp, keep_elems=keep, triplets=False, extra=("--geom",))
        base = os.path.join(tmp, name + "_buck")
        path = decks.write_dat(d, base)
        text = open(path).read().replace(
            "%END", f"%HEADER.ANALYSIS.EIGEN.ALGORITHM\n'SubspaceIteration'\n\n"
                    f"%HEADER.ANALYSIS.EIGEN.NUMBER.MODES\n{nm}\n\n%END")
        open(path, "w").write(text)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        lines = open(base + ".pos").read().splitlines()
        lam = [float(lines[i + 1].split()[1]) for i, ln in enumerate(lines)
               if ln.strip() == "%RESULT.CASE.STEP.BUCKLING.FACTOR"]
        _, modes = read_pos_modes(base + ".pos")
        f = os.path.join(HERE, name + ".npz")
        z = dict(np.load(f))
        z.update(ref_lambda=np.array(lam), ref_modes=modes, num_modes=np.array(nm), tol=np.array(d.tol),
                 maxit=np.array(d.maxit))
        np.savez_compressed(f, **z)
        print(name, lam)


def newmark_case(tmp, name, rayleigh=None):
    """The reference's own linear Newmark (cCtrlNewmark, unmodified `fast`
    binary, skyline): displacements, velocities and accelerations of every
    step of a hex20 box with density under a step load, optionally with
    Rayleigh damping (omega1, omega2, xi1, xi2)."""
    d = decks.box_hex20_lognormal(4, 4, 2, seed=7)
    d.rho = np.full(d.num_elems, 1e-3)
    d.algorithm = "newmark"
    d.time_step = 2e-4
    d.maxstep = 20
    d.rayleigh = rayleigh
    base = os.path.join(tmp, name)
    decks.write_dat(d, base)
    subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
    # read the printed steps before the harness reuses the deck's output file
    blocks = {k: decks.read_pos_block(base + ".pos", k) for k in ("NODAL.DISPLACEMENT", "VELOCITY", "ACCELERATION")}
    ref = refdump.run_dump(base, base + ".bin", "--no-solve", "--no-triplets")
    out = deck_arrays(d)
    out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_f=ref["f"],
               ref_u_steps=blocks["NODAL.DISPLACEMENT"], ref_v_steps=blocks["VELOCITY"],
               ref_a_steps=blocks["ACCELERATION"],
               steps=np.array(d.maxstep), time_step=np.array(d.time_step),
               gamma=np.array(d.newmark[0]), beta=np.array(d.newmark[1]))
    if rayleigh is not None:
        out["rayleigh"] = np.array(rayleigh, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name + ":", out["ref_u_steps"].shape)


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"FAST_REF={FAST_REF}", "ref"], check=True)
    tmp = tempfile.mkdtemp(prefix="golden_")
    if len(sys.argv) > 1 and sys.argv[1] == "variants":
        try:
            plate_variant_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "bspmass":
        try:
            bspline_mass_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "damped":
        try:
            newmark_case(tmp, "nm_hex20_box_damped", rayleigh=(10.0, 200.0, 0.02, 0.05))
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "buckling":
        try:
            buckling_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "modal":
        try:
            modal_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "pos":
        try:
            pos_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "arc":
        try:
            arc_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "stress":
        try:
            stress_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "iga":
        try:
            iga_cases(tmp)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        return
    try:
        iga_cases(tmp)
        # known-answer decks shipped with the reference
        for nm, rel in [("ref_testb8", "dat/continuum/TestB8.dat"), ("ref_beamb20", "dat/continuum/BeamB20.dat")]:
            src = os.path.join(FAST_REF, rel)
            d = decks.read_dat(src)
            base = os.path.join(tmp, nm)
            shutil.copy(src, base + ".dat")
            os.chmod(base + ".dat", 0o644)
            ref = refdump.run_dump(base, base + ".bin")
            out = deck_arrays(d)
            keep = np.arange(min(4, d.num_elems))
            out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_elems=keep,
                       ref_elm_K=ref["elm_K"][keep], ref_elm_dofs=ref["elm_dofs"], ref_f=ref["f"],
                       ref_u=ref["u"], ref_g_of_u=ref["g_of_u"])
            if d.num_elems <= 8:
                out.update({"ref_" + k: v for k, v in lower_csr(ref).items()})
            np.savez_compressed(os.path.join(HERE, nm + ".npz"), **out)
            print(nm, "written")

        stress_cases(tmp)
        arc_cases(tmp)
        pos_cases(tmp)
        modal_cases(tmp)
        buckling_cases(tmp)
        d = decks.box_hex20_lognormal(8, 8, 4, seed=11)
        d.tol = 1e-12
        run_case("cfg_hex20_lognormal_8x8x4", d, tmp, keep_elems=np.arange(0, 256, 17), triplets=False)

        # hex8 with density: consistent mass matrices
        d = decks.cantilever_hex8(4, 2, 2)
        d.rho = np.full(d.num_elems, 1e-3)
        run_case("cfg_hex8_mass", d, tmp, mass=True)

        # total-Lagrangian hex8 plate evaluated at a seeded displacement state
        d = decks.cantilever_hex8(4, 4, 2, L=(4.0, 4.0, 0.4))
        d.total_lagrangian = True
        d.algorithm = "lcm"
        rng = np.random.default_rng(3)
        neq = d.num_eq()
        u = 0.05 * rng.standard_normal(neq)
        run_case("cfg_hex8_tl_state", d, tmp, uvec=u, triplets=False)

        # the reference's own load-control Newton-Raphson (cCtrlNR, unmodified
        # `fast` binary) on a small TL plate: displacements of every step
        d = decks.plate_tl_hex8(6, 6, 2, L=4.0, t=0.4, pressure=8.0, steps=4, tol=1e-10, maxit=30)
        base = os.path.join(tmp, "nr_plate_tl")
        decks.write_dat(d, base)
        subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
        us = decks.read_pos_displacements(base + ".pos")
        ref = refdump.run_dump(base, base + ".bin", "--no-solve", "--no-triplets")
        out = deck_arrays(d)
        out.update(ref_neq=ref["neq"], ref_node_eq=ref["node_eq"], ref_f=ref["f"], ref_u_steps=us,
                   steps=np.array(d.maxstep), step_factor=np.array(d.step_factor), tol=np.array(d.tol),
                   maxit=np.array(d.maxit))
        np.savez_compressed(os.path.join(HERE, "nr_plate_tl.npz"), **out)
        print("nr_plate_tl:", us.shape, "max |w|", np.abs(us[..., 2]).max())

        newmark_case(tmp, "nm_hex20_box")
        newmark_case(tmp, "nm_hex20_box_damped", rayleigh=(10.0, 200.0, 0.02, 0.05))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
