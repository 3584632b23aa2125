#!/usr/bin/env python
"""Linear-static benchmark of the element-integration -> assembly -> K.u solve
path on a hex20 box (64x64x32 elements on 4x4x2, 3x3x3 Gauss points,
lognormal Young's modulus per element, z=0 clamped, unit pressure on top:
131,072 elements, 1,609,920 equations).

One step = assemble K from the element integrals (FP64, colour-scheduled
scatter) and solve K u = f to |r|/|f| <= 1e-8.  The headline value is
equations solved per second (DOF/s = num_eq / step time).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64] [--precond jacobi|block] [--no-newton]

The line also carries "newton_plate": the geometrically nonlinear TL plate
(40x40x4 hex8, 40 load steps) solved by the device Newton driver with the
reference's start and FP64 PCG, with the secant start, and with the learned
start (POD + MLP + one POD-Galerkin correction) and mixed-precision PCG; see
newton_plate().

--impl reference runs the reference FAST program's own CPU code (built from
its sources into oracle/_ref by oracle/Makefile) on the same workload: it
assembles the full matrix once with cControl::StiffnessMatrix into its sparse
matrix, then times samples of PCGSolver iterations; its solve time is the
assembly time plus the per-iteration time times the iteration count of the
reference's PCGSolver algorithm on this workload (from the oracle's FP64
restatement).  The same line checks that model against a real converged
reference solve of a 16x16x8 box.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 64, 64, 32
TOL = 1e-8
SEED = 0
METRIC = "linear static hex20 box 64x64x32 (assemble K + solve to |r|/|f|<=1e-8): equations solved per second"
UNIT = "DOF/s"
FALLBACK_HBM_GBS = 6650.0


def workload_config(args, deck_neq=None):
    return {"workload": f"hex20 box {NX}x{NY}x{NZ} on 4x4x2, 3x3x3 Gauss, lognormal E (median 1000, sigma 0.5, "
                        f"seed {SEED}), nu 0.3, z=0 clamped, unit pressure on z=2; assemble K then solve to "
                        f"|r|/|f|<={TOL:g}",
            "elements": NX * NY * NZ, "equations": deck_neq, "precision": args.precision,
            "precond": args.precond, "l2": "inputs larger than L2 (block matrix 2.2 GB FP64)",
            "parallelism": "replicas" if args.gpus > 1 else "single"}


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fp:
            return float(json.load(fp)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


GOLDEN = os.path.join(ROOT, "tests", "golden")
CHECK_SEED, NCHECK = 12345, 4   # checksum weights of the full-size fixtures


def oracle_errors(u, z, k=None):
    """Error of a displacement vector against a full-size oracle fixture
    (tests/golden/full_*.npz, made by tests/golden/make_full_size.py): the
    largest error over the fixture's seeded sample of entries relative to the
    largest displacement, and the largest relative error of its seeded
    weighted sums over every entry (an estimate of the relative 2-norm error).
    k selects a load step of a multi-step fixture."""
    u = np.asarray(u, dtype=np.float64).ravel()
    pick = (lambda a: a[k]) if k is not None else (lambda a: a)
    W = np.random.default_rng(CHECK_SEED).uniform(-1.0, 1.0, size=(NCHECK, u.size))
    e_sample = float(np.abs(u[z["idx"]] - pick(z["u_idx"])).max() / float(pick(z["amax"])))
    e_check = float((np.abs(W @ u - pick(z["checks"])) / (np.linalg.norm(W, axis=1) * float(pick(z["norm2"])))).max())
    return {"u_rel_err_vs_oracle": e_check, "u_sample_err_vs_oracle": e_sample}


def load_fixture(name):
    p = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(p):
        return None
    z = np.load(p)
    return {k: z[k] for k in z.files}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def reference_iterations():
    """Iterations of the reference's PCGSolver algorithm (Jacobi PCG from
    u = 0, mlib/sysmat.cpp:1061-1125) to |r|/|f| < 1e-8 on the benchmark box:
    the oracle's FP64 restatement of that iteration on the restated K (pinned
    to the reference's StiffnessMatrix), recorded in the full-size fixture for
    the 64x64x32 box and computed here for other sizes."""
    z = load_fixture("full_hex20_64x64x32") if (NX, NY, NZ) == (64, 64, 32) else None
    if z is not None and "iterations_1e-8" in z:
        return int(z["iterations_1e-8"]), "oracle restatement of PCGSolver (full-size fixture)"
    from fast_b200 import decks
    from oracle import fem_oracle as fo
    d = decks.box_hex20_lognormal(NX, NY, NZ, seed=SEED)
    _, it, _ = fo.pcg_threaded(fo.assemble_chunked(d), fo.face_loads(d), TOL, 10 ** 6)
    return int(it), "oracle restatement of PCGSolver (computed)"


def pcg_split(r, warm):
    """(set-up, per-iteration) seconds of PCGSolver from a fastref bench run
    that timed calls of 1 and of r["pcg_iters2"] iterations in turn (the
    first `warm` pairs left out)."""
    t1 = statistics.mean(r["pcg_rep_s"][warm:])
    t2 = statistics.mean(r["pcg_rep2_s"][warm:])
    t_iter = (t2 - t1) / (r["pcg_iters2"] - r["pcg_iters"])
    return max(0.0, t1 - r["pcg_iters"] * t_iter), t_iter


def reference_cpu_time(pairs, warm):
    """The reference FAST program's own CPU code (oracle/_ref/fastref, one host
    thread: the reference's OpenMP build does not compile) on the full
    benchmark deck: cControl::StiffnessMatrix into its cSymSprsMatrix once,
    then `pairs` pairs of PCGSolver calls of 1 and of 3 iterations, each
    timed; their difference gives the cost of one iteration apart from the
    solver's set-up.  Solve time = assembly + set-up + the reference
    algorithm's iteration count x the iteration time."""
    from fast_b200 import decks
    from oracle import refdump
    iters, iters_src = reference_iterations()
    d = decks.box_hex20_lognormal(NX, NY, NZ, seed=SEED)
    d.tol = TOL
    t0 = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        base = os.path.join(tmp, "box")
        decks.write_dat(d, base)
        r = refdump.run_bench(base, 1, pairs, 3)
    wall = time.time() - t0
    w = min(warm, pairs - 1)
    setup, t_iter = pcg_split(r, w)
    T = r["assembly_s"] + setup + iters * t_iter
    return {"T": T, "neq": r["neq"], "iters": iters, "iters_source": iters_src, "t_iter": t_iter, "setup_s": setup,
            "samples": pairs - w, "assembly_s": r["assembly_s"], "integration_s": r["integration_s"],
            "read_s": r["read_s"], "nnz_lower": r["nnz_lower"], "wall_s": wall}


def reference_model_check(n=16):
    """The timing model above against a real converged run of the reference:
    on the n x n x n/2 box the reference solves to 1e-8 with its own sparse
    PCGSolver (fastref dump: K->Solve as cLinStat::Solver calls it), and the
    model's prediction (set-up + the oracle's iteration count x the timed
    iteration) is compared with that measured solve time."""
    from fast_b200 import decks
    from oracle import fem_oracle as fo
    from oracle import refdump
    d = decks.box_hex20_lognormal(n, n, n // 2, seed=SEED)
    d.tol = TOL
    d.maxit = 10 ** 6
    _, iters, _ = fo.pcg_threaded(fo.assemble_chunked(d), fo.face_loads(d), TOL, 10 ** 6)
    with tempfile.TemporaryDirectory() as tmp:
        base = os.path.join(tmp, "small")
        decks.write_dat(d, base)
        real = refdump.run_dump(base, base + ".bin", "--no-triplets")
        b = refdump.run_bench(base, 1, 6, 3)
    setup, t_iter = pcg_split(b, 1)
    model = setup + iters * t_iter
    solve = float(real["solve_seconds"][0])
    return {"box": f"{n}x{n}x{n // 2}", "equations": int(real["neq"][0]), "converged": bool(real["solve_ok"][0]),
            "oracle_iterations": iters, "real_solve_s": solve, "model_solve_s": model,
            "model_error": (model - solve) / solve}


def cpu_baseline(neq_full):
    """cpu_baseline of the bench line: the reference arm's method
    (reference_cpu_time) with two timed iterations, on one host thread."""
    from oracle import refdump
    if not refdump.available():
        return None
    r = reference_cpu_time(1, 0)
    return {"value": neq_full / r["T"], "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": (f"reference FAST (oracle/_ref), 1 thread, full {NX}x{NY}x{NZ} deck: StiffnessMatrix into "
                       f"cSymSprsMatrix once ({r['assembly_s']:.1f} s), PCGSolver calls of 1 and 3 iterations "
                       f"({r['t_iter']:.3f} s per iteration, {r['setup_s']:.3f} s set-up); solve time = assembly + "
                       f"set-up + {r['iters']} iterations ({r['iters_source']})"),
            "seconds_per_solve": r["T"]}


def newton_plate(local, args):
    """Geometrically nonlinear load-control Newton on the total-Lagrangian
    (St. Venant-Kirchhoff) hex8 plate 40x40x4 on 10x10x1 (E 1000, nu 0.3, sides
    pinned, pressure ramped over 40 steps to 40: centre deflection 2.1 t),
    Newton to |r|/max(1,|f|) <= 1e-8 at every step.  Times, on the device:
      plain:   the reference's iteration (start from the last converged u,
               FP64 Jacobi PCG to 1e-10 per Newton iteration);
      secant:  secant start, mixed-precision PCG, inexact Newton;
      learned: the learned start (POD + MLP trained on 64 seeded
               pressure/stiffness variants, one POD-Galerkin correction),
               mixed-precision PCG, inexact Newton;
      learned, network only: the same without the Galerkin correction;
      learned, two corrections: the same with two.
    Each solve is timed 3 times (minimum reported); training is timed once."""
    from fast_b200 import decks, gpu, learned
    d = decks.plate_tl_hex8(40, 40, 4, L=10.0, t=1.0, pressure=40.0, steps=40, tol=1e-8)
    S = gpu.GpuSystem(local)
    S.upload(d)
    q = gpu.face_load_vector(d)
    t0 = time.perf_counter()
    pred, info = learned.train_predictor(S, d, q, variants=64, seed=0, steps=40, epochs=3000, lr=2e-3)
    train_s = time.perf_counter() - t0
    pred.configure(use_network=True, galerkin_iters=1, galerkin_tol=1e-3)
    runs = {
        "plain_fp64": dict(predictor=gpu.PREDICT_NONE, precision=gpu.PREC_FP64, lin_tol=1e-10),
        "secant_mixed": dict(predictor=gpu.PREDICT_SECANT, precision=gpu.PREC_MIXED, lin_tol=1e-10,
                             lin_tol_rel=1e-3),
        "learned_mixed": dict(learned=pred, precision=gpu.PREC_MIXED, lin_tol=1e-10, lin_tol_rel=1e-3),
        "learned_mixed_network_only": dict(learned=pred, precision=gpu.PREC_MIXED, lin_tol=1e-10,
                                           lin_tol_rel=1e-3),
        "learned_mixed_two_corrections": dict(learned=pred, precision=gpu.PREC_MIXED, lin_tol=1e-10,
                                              lin_tol_rel=1e-3),
        # the same starts with FP64 inner solves (inexact Newton alike)
        "secant_fp64_inexact": dict(predictor=gpu.PREDICT_SECANT, precision=gpu.PREC_FP64, lin_tol=1e-10,
                                    lin_tol_rel=1e-3),
        "learned_fp64_inexact": dict(learned=pred, precision=gpu.PREC_FP64, lin_tol=1e-10, lin_tol_rel=1e-3),
    }
    # Galerkin corrections of the learned start per run (the network-only run has none)
    galerkin = {"learned_mixed": 1, "learned_mixed_network_only": 0, "learned_mixed_two_corrections": 2,
                "learned_fp64_inexact": 1}
    times = {k: [] for k in runs}
    out = {}
    clocks = ClockSampler(local)
    clocks.start()
    n0 = S.launch_count()
    for rep in range(3):
        for k, kw in runs.items():
            if k in galerkin:
                pred.configure(use_network=True, galerkin_iters=galerkin[k], galerkin_tol=1e-3)
            t = time.perf_counter()
            h, it, r = S.nr_solve(q, 40, 1.0 / 40, tol=1e-8, max_iter=30, **kw)
            times[k].append(time.perf_counter() - t)
            out[k] = (h[-1].copy(), r, h.copy())
    n1 = S.launch_count()
    clk = clocks.stop()
    # the same secant / mixed solve launched kernel by kernel (no graph replay)
    S.set_option(gpu.OPT_GRAPH_STEPS, 0)
    t_nog = []
    for rep in range(2):
        t = time.perf_counter()
        S.nr_solve(q, 40, 1.0 / 40, tol=1e-8, max_iter=30, **runs["secant_mixed"])
        t_nog.append(time.perf_counter() - t)
    S.set_option(gpu.OPT_GRAPH_STEPS, 1)
    # the predictor's two phases per load step (live spans, one learned run)
    pred.configure(use_network=True, galerkin_iters=1, galerkin_tol=1e-3)
    S.kernel_timing(True)
    S.nr_solve(q, 40, 1.0 / 40, tol=1e-8, max_iter=30, **runs["learned_mixed"])
    S.synchronize()
    pn_n, pn_ms, _ = S.kernel_stats(gpu.KERNEL_PREDICT_NET)
    pg_n, pg_ms, _ = S.kernel_stats(gpu.KERNEL_PREDICT_GALERKIN)
    # where the device time of that (kernel-by-kernel) learned run goes
    brk = {}
    for name, kind in (("linear_solves", gpu.KERNEL_LINEAR_SOLVE), ("internal_forces", gpu.KERNEL_INTERNAL_FORCE),
                       ("tangent_assemblies", gpu.KERNEL_ASSEMBLE)):
        kn, kms, _ = S.kernel_stats(kind)
        brk[name] = {"count": int(kn), "ms": kms}
    S.kernel_timing(False)
    pred_ms = {"network_ms_per_step": pn_ms / max(1, pn_n), "galerkin_ms_per_step": pg_ms / max(1, pg_n),
               "steps": int(pn_n), "device_time_of_a_learned_run_without_graphs": brk}
    u_ref = out["plain_fp64"][0]
    zplate = load_fixture("full_plate_tl_40x40x4")
    eqn = d.node_eq()
    mask = eqn > 0
    res = {}
    for k in runs:
        u, r, hist = out[k]
        res[k] = {"ms": min(times[k]) * 1e3, "ms_all": [round(x * 1e3, 1) for x in times[k]],
                  "newton_iterations": r["iterations"], "pcg_iterations": r["linear_iterations"],
                  "predictions": r["predictions"], "predictions_accepted": r["predictions_accepted"],
                  "final_err": r["last_err"],
                  "u_rel_diff_vs_plain": float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref))}
        if zplate is not None:
            # every load step against the reference fast binary's cCtrlNR (run to 1e-10)
            worst = {"u_rel_err_vs_oracle": 0.0, "u_sample_err_vs_oracle": 0.0}
            for step in range(hist.shape[0]):
                un = np.zeros((d.num_nodes, 3))
                un[mask] = hist[step][eqn[mask] - 1]
                e = oracle_errors(un, zplate, step)
                worst = {kk: max(worst[kk], e[kk]) for kk in worst}
            res[k]["worst_step_vs_reference_cctrlnr"] = worst
    eq = d.node_eq()
    c = int(np.argmin(np.linalg.norm(d.coords - np.array([5.0, 5.0, 1.0]), axis=1)))
    rep = pred.report()
    pred.close()
    S.close()
    return {
        "workload": "TL (St. Venant-Kirchhoff) hex8 plate 40x40x4 on 10x10x1, 2x2x2 Gauss, E 1000, nu 0.3, "
                    "sides pinned, pressure 40 in 40 load steps, Newton to |r|/max(1,|f|) <= 1e-8",
        "equations": d.num_eq(), "centre_deflection_over_t": float(-u_ref[eq[c, 2] - 1]),
        "runs": res,
        "speedup_learned_vs_plain": res["plain_fp64"]["ms"] / res["learned_mixed"]["ms"],
        "speedup_secant_vs_plain": res["plain_fp64"]["ms"] / res["secant_mixed"]["ms"],
        "speedup_learned_vs_secant": res["secant_mixed"]["ms"] / res["learned_mixed"]["ms"],
        "speedup_learned_network_only_vs_secant": res["secant_mixed"]["ms"] / res["learned_mixed_network_only"]["ms"],
        "secant_mixed_without_graphs_ms": min(t_nog) * 1e3,
        "predictor": pred_ms,
        "training": {"seconds": train_s, "variants": info["converged_variants"], "samples": rep["samples"],
                     "modes": rep["modes"], "params": rep["params"], "captured_energy": rep["captured_energy"],
                     "first_loss": rep["first_loss"], "last_loss": rep["last_loss"],
                     "trajectory_seconds": info["data_seconds"], "basis_ms": rep["basis_ms"],
                     "train_ms": rep["train_ms"]},
        "gpu_launches": int(n1 - n0), "clocks": clk,
    }


def ensemble_members(rank, world, count=1024, seed=0):
    """This rank's members (index, deck) of the cantilever ensemble: member k
    (n x n x 2n hex8 cantilever, n uniform in [6, 20], lognormal E per element,
    random tip traction, all drawn in member order from one seeded stream)
    belongs to rank k mod world.  No exchange is needed between ranks."""
    from fast_b200 import decks
    rng = np.random.default_rng(seed)
    ns = rng.integers(6, 21, size=count)
    out = []
    for k, n in enumerate(ns):
        m = decks.cantilever_hex8(2 * int(n), int(n), int(n), L=(2.0, 1.0, 1.0), q=tuple(rng.standard_normal(3)))
        m.E = 1000.0 * np.exp(0.5 * rng.standard_normal(m.num_elems))
        if k % world == rank:
            out.append((k, m))
    return out


def reduce_over_ranks(values, op, world, dev):
    """All-reduce a list of numbers over the ranks (op "max" or "sum"); the
    identity for one rank.  Every rank must call it at the same point."""
    if world == 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def ensemble_and_dynamics(local, rank, world, args, dev):
    """Ensemble and dynamics: (a) 1024 independent hex8 cantilevers n x n x 2n, n uniform
    in [6, 20], lognormal E per element, random tip traction: assembled in one
    pass and solved in one launch (one thread-block cluster per problem) to
    |r_k|/|f_k| <= 1e-8 each; with N ranks the members are split by index
    (rank k takes members k, k+N, ...), no exchange, max over ranks;
    (b) linear Newmark (beta 0.25, gamma 0.5) of the hex20 64x64x32 box with
    density 1e-3 under the step load (unit pressure), dt 1e-4, 500 steps,
    mixed-precision PCG warm-started from the last step (rank 0)."""
    import torch
    import torch.distributed as dist
    from fast_b200 import decks, gpu
    out = {}
    members = [m for _, m in ensemble_members(rank, world)]
    d, noff, _ = decks.concat_decks(members)
    f = gpu.face_load_vector(d)
    S = gpu.GpuSystem(local)
    S.upload(d)
    S.set_problems(noff)
    S.assemble()
    S.solve_batch(f, tol=1e-8)
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    ta, ts = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        S.assemble()
        S.synchronize()
        t1 = time.perf_counter()
        u, conv, its, res = S.solve_batch(f, tol=1e-8)
        t2 = time.perf_counter()
        ta.append(t1 - t0)
        ts.append(t2 - t1)
    clk = clocks.stop()
    tot = min(a + b for a, b in zip(ta, ts))
    tot = reduce_over_ranks([tot], "max", world, dev)[0]
    nconv, neq_total = (int(v) for v in reduce_over_ranks([int(conv.sum()), int(d.num_eq())], "sum", world, dev))
    out["ensemble"] = {
        "workload": "1024 hex8 cantilevers n x n x 2n on 2x1x1, n uniform in [6, 20] (seed 0), 2x2x2 Gauss, "
                    "lognormal E (median 1000, sigma 0.5) per element, random tip traction; assemble all, solve "
                    "each to |r|/|f| <= 1e-8 (one launch, one thread-block cluster per problem)",
        "members_this_rank": len(members), "elements_this_rank": int(d.num_elems), "equations_this_rank": int(d.num_eq()),
        "converged": nconv, "ms": tot * 1e3, "assemble_ms": min(ta) * 1e3, "solve_ms": min(ts) * 1e3,
        "iterations_min_mean_max": [int(its.min()), float(its.mean()), int(its.max())],
        "equations_per_s": neq_total / tot, "elements_per_s_assembly": d.num_elems / min(ta),
        "scaling": "strong (members split across ranks)", "clocks": clk}
    S.close()
    if rank == 0:
        box = decks.box_hex20_lognormal(NX, NY, NZ, seed=SEED)
        box.rho = np.full(box.num_elems, 1e-3)
        q = gpu.face_load_vector(box)
        S = gpu.GpuSystem(local)
        S.upload(box)
        eq = box.node_eq()
        c = int(np.argmin(np.linalg.norm(box.coords - np.array([2.0, 2.0, 2.0]), axis=1)))
        probe = [int(eq[c, 2]) - 1]
        clocks = ClockSampler(local)
        clocks.start()
        t0 = time.perf_counter()
        _, hist, rep = S.newmark(q, 500, 1e-4, precision=gpu.PREC_MIXED, tol=1e-8, warm=True, probes=probe,
                                 mass_tol=1e-10)
        t_mixed = time.perf_counter() - t0
        clk = clocks.stop()
        t0 = time.perf_counter()
        _, hist64, rep64 = S.newmark(q, 50, 1e-4, precision=gpu.PREC_FP64, tol=1e-8, warm=True, probes=probe,
                                     mass_tol=1e-10)
        t_fp64 = time.perf_counter() - t0
        # the first 50 mixed steps launched kernel by kernel (no graph replay)
        S.set_option(gpu.OPT_GRAPH_STEPS, 0)
        t0 = time.perf_counter()
        _, hist_ng, rep_ng = S.newmark(q, 50, 1e-4, precision=gpu.PREC_MIXED, tol=1e-8, warm=True, probes=probe,
                                       mass_tol=1e-10)
        t_nog = time.perf_counter() - t0
        S.set_option(gpu.OPT_GRAPH_STEPS, 1)
        out["newmark"] = {
            "workload": f"linear Newmark (beta 0.25, gamma 0.5) of the hex20 {NX}x{NY}x{NZ} box, density 1e-3, unit "
                        "pressure applied at t=0 (step load), dt 1e-4; each step K_eff u = f_eff by PCG to 1e-8, "
                        "warm-started from the last step",
            "equations": box.num_eq(), "steps": 500,
            "mixed": {"seconds": t_mixed, "ms_per_step": t_mixed / 500 * 1e3, **rep},
            "fp64_50_steps": {"seconds": t_fp64, "ms_per_step": t_fp64 / 50 * 1e3,
                              "pcg_iterations": rep64["linear_iterations"]},
            "mixed_50_steps_without_graphs": {"ms_per_step": t_nog / 50 * 1e3,
                                              "pcg_iterations": rep_ng["linear_iterations"]},
            "top_centre_w": {"step_100": float(hist[99, 0]), "step_500": float(hist[-1, 0]),
                             "fp64_vs_mixed_step_50": float(abs(hist64[-1, 0] - hist[49, 0]) / abs(hist64[-1, 0]))},
            "clocks": clk}
        S.close()
    return out


def tied_blocks(local, args):
    """Tied multi-block model: four blocks joined by tied interfaces (a
    B-spline p=2 patch 32x32x8 with 3^3 Gauss points, a hex8 box 40x40x20 with
    2^3, a hex20 box 24x24x12 with 3^3 and a B-spline p=3 patch 24x24x6 with
    4^3, control points jittered by uniform[-0.05h, 0.05h]); the slave DOFs
    of the non-matching interfaces are eliminated (K~ = T^T K T assembled
    directly).  Assembly of all buckets, then the mixed-precision solve (FP32
    PCG, FP64 residual replacement) to |r|/|f| <= 1e-8, its error against the
    FP64 device solve to 1e-12, and the FP64 solve to 1e-8 for comparison."""
    from fast_b200 import decks, gpu
    t0 = time.perf_counter()
    d = decks.tied_column(seed=SEED)
    f = decks.nodal_load_vector(d)
    gen_s = time.perf_counter() - t0
    S = gpu.GpuSystem(local)
    t0 = time.perf_counter()
    S.upload(d)
    setup_s = time.perf_counter() - t0
    pinfo = S.pattern_info()
    S.assemble()
    tune = S.autotune()
    S.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    S.kernel_timing(True)
    for _ in range(3):
        S.assemble()
    S.synchronize()
    a_n, a_ms, a_bytes = S.kernel_stats(gpu.KERNEL_ASSEMBLE)
    S.kernel_timing(False)
    a_ms /= max(1, a_n)
    runs = {}
    # the 84,647-node system iterates per kernel by default; the persistent
    # cooperative iteration is also measured with its node limit raised
    tuned = tune["persistent_max_nodes"]
    for name, prec, tol, persist in (("mixed", gpu.PREC_MIXED, 1e-8, tuned), ("fp64", gpu.PREC_FP64, 1e-8, tuned),
                                     ("mixed_persistent", gpu.PREC_MIXED, 1e-8, 1 << 20),
                                     ("fp64_persistent", gpu.PREC_FP64, 1e-8, 1 << 20),
                                     ("fp64_1e-12", gpu.PREC_FP64, 1e-12, tuned)):
        S.set_option(gpu.OPT_PERSISTENT_MAX_NODES, persist)
        best = None
        for _ in range(2 if name != "fp64_1e-12" else 1):
            t1 = time.perf_counter()
            u, rep = S.solve(f, tol=tol, precision=prec, maxit=400000)
            dt = time.perf_counter() - t1
            if best is None or dt < best[0]:
                best = (dt, u, rep)
        runs[name] = best
    S.set_option(gpu.OPT_PERSISTENT_MAX_NODES, tuned)
    # the mixed path on the tensor-core stiffness (B-spline and hex buckets on
    # tcgen05 (TF32 operands split in three), tied elements' FP64 matrices, FP64 residuals element
    # by element)
    tc = None
    try:
        S.assemble(gpu.ASM_K_TF32)
        S.synchronize()
        S.kernel_timing(True)
        for _ in range(3):
            S.assemble(gpu.ASM_K_TF32)
        S.synchronize()
        tn, tms, tbytes = S.kernel_stats(gpu.KERNEL_ASSEMBLE_TF32)
        S.kernel_timing(False)
        tms /= max(1, tn)
        best = None
        for _ in range(2):
            t1 = time.perf_counter()
            u, rep = S.solve(f, tol=1e-8, precision=gpu.PREC_MIXED, maxit=400000)
            dt = time.perf_counter() - t1
            if best is None or dt < best[0]:
                best = (dt, u, rep)
        runs["mixed_tf32"] = best
        tc = {"assembly_ms": tms, "assembly_GB_per_s": tbytes / (tms / 1e3) / 1e9}
        # every bucket in one persistent cooperative launch (colour phases)
        S.set_option(gpu.OPT_PERSISTENT_ASSEMBLY, 1)
        S.assemble(gpu.ASM_K_TF32)
        S.synchronize()
        n0 = S.launch_count()
        S.kernel_timing(True)
        for _ in range(3):
            S.assemble(gpu.ASM_K_TF32)
        S.synchronize()
        pn, pms, _ = S.kernel_stats(gpu.KERNEL_ASSEMBLE_TF32)
        S.kernel_timing(False)
        pl = (S.launch_count() - n0) // 3
        S.set_option(gpu.OPT_PERSISTENT_ASSEMBLY, 0)
        n0 = S.launch_count()
        S.assemble(gpu.ASM_K_TF32)
        S.synchronize()
        tc.update({"launches_per_colour": S.launch_count() - n0, "persistent_launches": pl,
                   "persistent_assembly_ms": pms / max(1, pn),
                   "persistent_speedup": tms / (pms / max(1, pn))})
    except Exception as ex:  # reported, not fatal
        tc = {"error": str(ex)[:300]}
    clk = clocks.stop()
    u_ref = runs["fp64_1e-12"][1]
    err = {k: float(np.abs(v[1] - u_ref).max() / np.abs(u_ref).max()) for k, v in runs.items() if k != "fp64_1e-12"}
    ztied = load_fixture("full_tied_column")
    oerr = {k: oracle_errors(v[1], ztied) for k, v in runs.items()} if ztied is not None else {}
    hbm, _ = measured_hbm()
    kinds = {b.kind if b.kind != "bsp" else f"bsp p={b.patch.degree[0]}": b.num_elems for b in d.buckets()}
    S.close()
    return {
        "workload": "tied column: B-spline p=2 32x32x8 (3^3 Gauss) | hex8 40x40x20 (2^3) | hex20 24x24x12 (3^3) | "
                    "B-spline p=3 24x24x6 (4^3) on a 1x1 footprint stacked in z, control points jittered by "
                    "uniform[-0.05h, 0.05h] (seed 0), E 1000, nu 0.3, p=2 patch clamped at z=0, unit total load "
                    "on the p=3 patch's top control points; non-matching interfaces tied (slave DOFs eliminated)",
        "elements": kinds, "nodes": int(d.num_nodes), "equations": int(d.num_eq()),
        "tied_slave_nodes": int(len(d.ties.slave)), "pattern": pinfo, "generate_s": gen_s, "setup_s": setup_s,
        "autotune": tune,
        "assembly": {"ms": a_ms, "launches_timed": int(a_n), "elements_per_s": sum(kinds.values()) / (a_ms / 1e3),
                     "algorithmic_bytes": a_bytes, "GB_per_s": a_bytes / (a_ms / 1e3) / 1e9,
                     "frac": a_bytes / (a_ms / 1e3) / 1e9 / hbm},
        "solve": {k: {"ms": v[0] * 1e3, "iterations": v[2]["iterations"], "outer": v[2]["outer"],
                      "escalated": v[2]["escalated"], "true_rel_residual": v[2]["true_rel_residual"],
                      "u_rel_err_vs_fp64_1e-12": err.get(k), **oerr.get(k, {})} for k, v in runs.items()},
        "oracle": ("tests/golden/full_tied_column.npz: restated element matrices, ties eliminated on the CPU, "
                   "Jacobi PCG to 1e-13") if ztied is not None else None,
        "mixed_speedup_vs_fp64": runs["fp64"][0] / runs["mixed"][0],
        "tensor_core_assembly": tc,
        "clocks": clk}


def deck_io_and_output(S, deck, u, args):
    """The host side around the hot path, on this box: the .dat deck of the
    workload read by the library's parallel reader (beside the pure-Python
    reader), and the printing step: Gauss-point and nodal stresses on the
    device, then the .pos blocks formatted on all host cores (written to
    /dev/null, so the figure is formatting, not disk)."""
    from fast_b200 import datfile, decks
    out = {"threads": os.cpu_count()}
    with tempfile.TemporaryDirectory() as td:
        path = decks.write_dat(deck, os.path.join(td, "deck"))
        out["deck_bytes"] = os.path.getsize(path)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            dn = datfile.read_dat(path)
            ts.append(time.perf_counter() - t0)
        out["native_read_s"] = min(ts)
        t0 = time.perf_counter()
        dp = decks.read_dat(path)
        out["python_read_s"] = time.perf_counter() - t0
        out["readers_agree"] = bool(np.array_equal(dn.conn, dp.conn) and np.array_equal(dn.coords, dp.coords)
                                    and np.array_equal(dn.E, dp.E))
        S.set_displacement(u)
        t0 = time.perf_counter()
        _, gs = S.gauss_stress()
        out["gauss_stress_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        en, avg = S.nodal_stress()
        out["nodal_stress_s"] = time.perf_counter() - t0
        eq = deck.node_eq()
        displ = np.zeros((deck.num_nodes, 3))
        m = eq > 0
        displ[m] = u[eq[m] - 1]
        t0 = time.perf_counter()
        datfile.write_pos(os.devnull, path, [dict(factor=1.0, displ=displ, gauss_stress=gs, elem_nodal=en,
                                                  nodal_avg=avg)], precision=15, print_average=True)
        out["pos_format_s"] = time.perf_counter() - t0
        out["pos_numbers"] = int(6 * (2 * deck.num_nodes + gs.shape[0] * gs.shape[1] + en.shape[0] * en.shape[1]))
    out["note"] = ("stress times include the device-to-host copy of the results; the reference prints the same "
                   "blocks through iostream one number at a time")
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import refdump
    if not refdump.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/fastref was not built "
                          "(the reference sources are needed to build it)"}))
        return 0
    # pairs of timed PCGSolver calls (about 10 s each on the full deck), so the
    # run ends in a few minutes whatever --steps asks for
    reps = max(2, min(args.warmup + args.steps, 6))
    warm = min(args.warmup, 1)
    r = reference_cpu_time(reps, warm)
    check = None
    try:
        check = reference_model_check()
    except Exception as ex:  # reported, not fatal
        check = {"error": str(ex)[:200]}
    T = r["T"]
    value = r["neq"] / T
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": r["samples"],
            "warmup": warm, "ms_per_step": T * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload_config(args, r["neq"]), "precision": "fp64 (reference CPU)",
                       "precond": "jacobi (PCGSolver)"}, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": (f"reference FAST (oracle/_ref), 1 thread, full {NX}x{NY}x{NZ} deck: "
                                        f"StiffnessMatrix into cSymSprsMatrix once ({r['assembly_s']:.1f} s), then "
                                        f"{r['samples']} timed pairs of PCGSolver calls of 1 and 3 iterations "
                                        f"({r['t_iter']:.3f} s per iteration, {r['setup_s']:.3f} s set-up, "
                                        f"{r['nnz_lower']} stored nonzeros); solve time = assembly + set-up + "
                                        f"{r['iters']} iterations ({r['iters_source']})")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_detail": {"assembly_s": r["assembly_s"], "integration_s": r["integration_s"],
                                 "read_s": r["read_s"], "pcg_iter_s": r["t_iter"], "pcg_setup_s": r["setup_s"],
                                 "iterations": r["iters"],
                                 "wall_s": r["wall_s"], "model_check": check}}
    print(json.dumps(line))
    return 0


def spmv_kernel_name(tune, which):
    """The SpMV form the autotuner left in place for the timed solve."""
    if which != gpu_const("KERNEL_SPMV_FP32"):
        return "spmv_f64<0, %d> (FP64 PCG K.p)" % tune["lanes_fp64"]
    if tune.get("col16_fp32"):
        return "spmv_f32_c16<%d> (FP32 PCG K.p, 16-bit column offsets)" % tune["lanes_fp32"]
    if tune.get("bulk_fp32"):
        return "spmv_f32_bulk<%d> (FP32 PCG K.p, bulk-staged)" % tune["lanes_fp32"]
    if tune.get("stream_fp32"):
        return "spmv_f32<0, %d, 1> (FP32 PCG K.p, streamed matrix loads)" % tune["lanes_fp32"]
    return "spmv_f32<0, %d> (FP32 PCG K.p)" % tune["lanes_fp32"]


def spmv_profile_file(tune, which):
    """The ncu summary under profiles/ that holds the DRAM traffic of that form."""
    if which != gpu_const("KERNEL_SPMV_FP32"):
        return "spmv_soa_fp64_hex20_64x64x32.txt"
    return "spmv_c16_fp32_hex20_64x64x32.txt" if tune.get("col16_fp32") else "spmv_soa_fp32_hex20_64x64x32.txt"


def gpu_const(name):
    from fast_b200 import gpu
    return getattr(gpu, name)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from fast_b200 import decks, gpu

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    prec = gpu.PREC_MIXED if args.precision == "mixed" else gpu.PREC_FP64
    pc = gpu.PRECOND_BLOCK_JACOBI if args.precond == "block" else gpu.PRECOND_JACOBI

    deck = decks.box_hex20_lognormal(NX, NY, NZ, seed=SEED)
    f = gpu.face_load_vector(deck)
    neq = deck.num_eq()
    S = gpu.GpuSystem(local)
    t0 = time.time()
    S.upload(deck)
    setup_s = time.time() - t0
    pinfo = S.pattern_info()
    # the library runs on an explicit (non-NULL) torch stream so that the CUDA
    # events recorded below bracket its kernels
    stream = torch.cuda.Stream(dev)
    d_f = torch.from_numpy(f).to(dev)
    d_u = torch.zeros(neq, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    S.set_stream(stream.cuda_stream)

    def step(precision=prec, precond=pc):
        S.assemble()
        return S.solve_device(d_f.data_ptr(), d_u.data_ptr(), tol=TOL, precision=precision, precond=precond)

    # launch shapes measured on this system before the warm-up (untimed)
    S.assemble()
    tune = S.autotune()
    for _ in range(args.warmup):
        rep = step()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_over_ranks([x], "max", world, dev)[0]

    # ---- timed region: device-resident inputs, no instrumentation
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    n0 = S.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    reps = []
    for _ in range(args.steps):
        reps.append(step())
    e1.record(stream)
    torch.cuda.synchronize(dev)
    n1 = S.launch_count()
    clk = clocks.stop()
    # ---- the same steps again with CUDA events around every SpMV and assembly
    # (live kernel timing replays no CUDA graphs, so it is kept out of the timed region)
    S.kernel_timing(True)
    reps_t = [step() for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    spmv_which = gpu.KERNEL_SPMV_FP32 if prec == gpu.PREC_MIXED else gpu.KERNEL_SPMV_FP64
    # mean device time per real launch: launches issued past convergence return
    # at once; their few microseconds stay in the sum (a conservative mean)
    its = sum(r["iterations"] for r in reps_t)
    outs = sum(r["outer"] for r in reps_t)
    k_span, k_tot, k_bytes = S.kernel_stats(spmv_which)
    k_n = its
    k_ms = k_tot / k_n
    r_span, r_tot, r_bytes = S.kernel_stats(gpu.KERNEL_SPMV_FP64)
    r_n = outs if spmv_which != gpu.KERNEL_SPMV_FP64 else its
    r_ms = r_tot / r_n if r_n else None
    a_n, a_tot, a_bytes = S.kernel_stats(gpu.KERNEL_ASSEMBLE)
    a_ms = a_tot / a_n
    S.kernel_timing(False)
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms)
    value = world * neq / (ms / 1e3)
    u_main = d_u.cpu().numpy().copy()
    last = reps[-1]

    # ---- plain FP64 GPU path (the reference's Jacobi PCG) for comparison, timed once
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    rep64 = step(gpu.PREC_FP64, gpu.PRECOND_JACOBI)
    eb.record(stream)
    torch.cuda.synchronize(dev)
    ms64 = ea.elapsed_time(eb)
    u64 = d_u.cpu().numpy().copy()
    rel_u = float(np.abs(u_main - u64).max() / np.abs(u64).max())

    # ---- the same step to |r|/|f| <= 1e-10 (the box configuration's Jacobi-PCG
    # tolerance; the metric's is 1e-8), mixed and plain FP64, timed once each
    tight, u_tight = {}, {}
    for name, pr in (("mixed", prec), ("fp64", gpu.PREC_FP64)):
        ta, tb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ta.record(stream)
        S.assemble()
        rr = S.solve_device(d_f.data_ptr(), d_u.data_ptr(), tol=1e-10, precision=pr, precond=pc)
        tb.record(stream)
        torch.cuda.synchronize(dev)
        tight[name] = {"ms_per_step": ta.elapsed_time(tb), "iterations": rr["iterations"],
                       "true_rel_residual": rr["true_rel_residual"]}
        u_tight[name] = d_u.cpu().numpy().copy()
    tight["speedup_mixed_vs_fp64"] = tight["fp64"]["ms_per_step"] / tight["mixed"]["ms_per_step"]

    # ---- the mixed path on the tensor-core stiffness: element products in
    # three-part TF32 products on tcgen05 (FP32 blocks), FP32 PCG, FP64 residuals element by
    # element; timed like the value path, after two untimed steps
    def step_tc():
        S.assemble(gpu.ASM_K_TF32)
        return S.solve_device(d_f.data_ptr(), d_u.data_ptr(), tol=TOL, precision=gpu.PREC_MIXED, precond=pc)

    tc = None
    try:
        for _ in range(2):
            step_tc()
        torch.cuda.synchronize(dev)
        et0, et1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        et0.record(stream)
        reps_tc = [step_tc() for _ in range(args.steps)]
        et1.record(stream)
        torch.cuda.synchronize(dev)
        ms_tc = et0.elapsed_time(et1) / args.steps
        u_tc = d_u.cpu().numpy().copy()
        S.kernel_timing(True)
        step_tc()
        torch.cuda.synchronize(dev)
        ta_n, ta_tot, ta_bytes = S.kernel_stats(gpu.KERNEL_ASSEMBLE_TF32)
        S.kernel_timing(False)
        ta_ms = ta_tot / max(1, ta_n)
        tc = {"ms_per_step": ms_tc, "equations_per_s": neq / (ms_tc / 1e3), "iterations": reps_tc[-1]["iterations"],
              "fp64_residuals": reps_tc[-1]["outer"], "true_rel_residual": reps_tc[-1]["true_rel_residual"],
              "assembly": {"ms": ta_ms, "elements_per_s": deck.num_elems / (ta_ms / 1e3),
                           "algorithmic_bytes": ta_bytes, "GB_per_s": ta_bytes / (ta_ms / 1e3) / 1e9}}
    except Exception as ex:  # reported, not fatal
        tc = {"error": str(ex)[:300]}
        u_tc = None

    # ---- every solution against the full-size oracle (C restatement of the
    # reference's K, the reference's PCG iteration to 1e-13)
    zbox = load_fixture("full_hex20_64x64x32") if (NX, NY, NZ) == (64, 64, 32) else None
    oracle = None
    if zbox is not None:
        oracle = {"oracle": "tests/golden/full_hex20_64x64x32.npz: C restatement of the reference's K, Jacobi "
                            "PCG (PCGSolver's iteration) to 1e-13, true residual %.1e" % float(zbox["true_rel_residual"]),
                  "value_path": oracle_errors(u_main, zbox), "plain_fp64": oracle_errors(u64, zbox)}
        if u_tc is not None:
            oracle["tensor_core_mixed"] = oracle_errors(u_tc, zbox)
            tc.update(oracle["tensor_core_mixed"])
        for name in u_tight:
            tight[name].update(oracle_errors(u_tight[name], zbox))
        if "rel_diff_1e-8" in zbox:
            oracle["oracle_pcg_stopped_at_1e-8"] = {"iterations": int(zbox["iterations_1e-8"]),
                                                    "u_rel_diff": float(zbox["rel_diff_1e-8"])}

    # ---- dominant kernel and assembly: CUDA events around each launch in the timed region
    hbm, hbm_kind = measured_hbm()
    # (a zero duration only happens under a profiler that replays the kernels)
    achieved = k_bytes / (k_ms / 1e3) / 1e9 if k_ms > 0 else 0.0
    a_gbs = a_bytes / (a_ms / 1e3) / 1e9 if a_ms > 0 else 0.0
    traffic = None
    tp = os.path.join(ROOT, "profiles", spmv_profile_file(tune, spmv_which))
    if os.path.exists(tp):
        for ln in open(tp):
            if ln.startswith("dram_bytes_per_launch:"):
                traffic = float(ln.split(":")[1])

    # ---- end to end through the public API with host buffers (pinned)
    e2e = None
    if not args.no_e2e:
        coords_h = torch.from_numpy(np.ascontiguousarray(deck.coords)).pin_memory().numpy()
        E_h = torch.from_numpy(np.ascontiguousarray(deck.E)).pin_memory().numpy()
        f_h = torch.from_numpy(f).pin_memory().numpy()
        S.update_coords(coords_h)
        S.update_material(E=E_h)
        S.assemble()
        S.solve(f_h, tol=TOL, precision=prec, precond=pc)
        barrier()
        torch.cuda.synchronize(dev)
        ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        ee0.record(stream)
        for _ in range(args.steps):
            S.update_coords(coords_h)
            S.update_material(E=E_h)
            S.assemble()
            u_h, _ = S.solve(f_h, tol=TOL, precision=prec, precond=pc)
        ee1.record(stream)
        torch.cuda.synchronize(dev)
        wall = (time.perf_counter() - w0) / args.steps
        e_ms = max(ee0.elapsed_time(ee1) / args.steps, wall * 1e3)
        e_ms = max_over_ranks(e_ms)
        e2e = {"value": world * neq / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(coords_h.nbytes + E_h.nbytes + f_h.nbytes),
               "d2h_bytes_per_step": int(u_h.nbytes), "ms_per_step": e_ms}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = cpu_baseline(neq)
        except Exception as ex:  # reported, not fatal
            base = {"value": None, "error": str(ex)[:200]}

    io = None
    if rank == 0 and world == 1 and not args.no_io:
        try:
            io = deck_io_and_output(S, deck, u_main, args)
        except Exception as ex:  # reported, not fatal
            io = {"error": str(ex)[:300]}
    S.close()
    cfg4 = None
    if not args.no_ensemble:
        try:
            cfg4 = ensemble_and_dynamics(local, rank, world, args, dev)
        except Exception as ex:  # reported, not fatal
            cfg4 = {"error": str(ex)[:300]}
    cfg2 = None
    if rank == 0 and world == 1 and not args.no_tied:
        try:
            cfg2 = tied_blocks(local, args)
        except Exception as ex:  # reported, not fatal
            cfg2 = {"error": str(ex)[:300]}
    plate = None
    if rank == 0 and world == 1 and not args.no_newton:
        try:
            plate = newton_plate(local, args)
        except Exception as ex:  # reported, not fatal
            plate = {"error": str(ex)[:300]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32" if prec == gpu.PREC_MIXED else "f64", "data": "synthetic",
            "config": workload_config(args, neq),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "kernel": spmv_kernel_name(tune, spmv_which),
                         "bytes_per_launch": k_bytes, "ms_per_launch": k_ms, "launches_timed": k_n,
                         "spans_timed": k_span,
                         "peak_kind": hbm_kind},
            "cpu_baseline": base,
            "e2e": e2e,
            "gpu_launches": int(n1 - n0),
            "clocks": clk,
            "spmv_fp64_in_timed_region": ({"launches": r_n, "ms_per_launch": r_ms, "spans": r_span,
                                           "GB_per_s": r_bytes / (r_ms / 1e3) / 1e9 if r_ms else None}
                                          if spmv_which != gpu.KERNEL_SPMV_FP64 else None),
            "u_rel_err_vs_oracle": oracle["value_path"]["u_rel_err_vs_oracle"] if oracle else None,
            "solve": {"iterations": last["iterations"], "outer": last["outer"], "escalated": last["escalated"],
                      "rel_residual": last["rel_residual"], "true_rel_residual": last["true_rel_residual"],
                      "u_rel_diff_vs_fp64_jacobi": rel_u},
            "oracle_errors": oracle,
            "tensor_core_path": tc,
            "solve_to_1e-10": tight,
            "plain_fp64_gpu": {"ms_per_step": ms64, "iterations": rep64["iterations"],
                               "true_rel_residual": rep64["true_rel_residual"], "speedup_of_value_path": ms64 / ms},
            "assembly": {"ms": a_ms, "launches_timed": a_n, "elements_per_s": deck.num_elems / (a_ms / 1e3),
                         "algorithmic_bytes": a_bytes, "GB_per_s": a_gbs, "frac": a_gbs / hbm},
            "pattern": {**pinfo, "setup_s": setup_s},
            "autotune": tune,
            "tied_blocks": cfg2,
            "newton_plate": plate,
            "ensemble_and_dynamics": cfg4,
            "deck_io_and_output": io,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "block"])
    ap.add_argument("--size", type=int, default=64, help="elements along x and y (z = size/2)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-newton", action="store_true", help="skip the nonlinear plate (learned start) section")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble + Newmark section")
    ap.add_argument("--no-tied", action="store_true", help="skip the tied multi-block (hex8, hex20, B-spline) section")
    ap.add_argument("--no-io", action="store_true", help="skip the deck reading / result formatting section")
    args = ap.parse_args()
    global NX, NY, NZ
    NX = NY = args.size
    NZ = args.size // 2
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
