"""Small, self-contained workloads for profiling single kernels of libfastgpu
under ncu (each one GPU, a few hundred MB at most):

    python -m fast_b200.profile_cases plate_solve   # persistent PCG on the TL plate 40x40x4 tangent
    python -m fast_b200.profile_cases mlp_grad      # tcgen05 BF16 GEMMs: MLP forward + backward,
                                                    #   batch 2496, 129 -> 256 -> 256 -> 32
    python -m fast_b200.profile_cases box N         # hex20 box N x N x N/2: assemble + mixed solve
    python -m fast_b200.profile_cases tied          # tied four-block column (B-spline p=2, hex8, hex20,
                                                    #   B-spline p=3): two assemblies
    python -m fast_b200.profile_cases ensemble N    # N hex8 cantilevers (n in [6, 20]): assemble + batch solve
    python -m fast_b200.profile_cases newmark       # hex20 box 16x16x8 with density: 20 Newmark steps (mixed)

Each prints one line of results; none measures anything itself.
"""
from __future__ import annotations

import sys

import numpy as np

from . import decks, gpu


def plate_solve():
    d = decks.plate_tl_hex8(40, 40, 4, L=10.0, t=1.0, pressure=40.0, steps=40, tol=1e-8)
    s = gpu.GpuSystem(0)
    s.upload(d)
    q = gpu.face_load_vector(d)
    s.assemble()
    u, r = s.solve(q, tol=1e-10, precision=gpu.PREC_FP64, check_every=64)
    print("plate_solve", r)


def mlp_grad():
    d = decks.plate_tl_hex8(10, 10, 2)
    s = gpu.GpuSystem(0)
    s.upload(d)
    p = gpu.LearnedPredictor(s, modes=32, history=4, width=256, hidden=2, seed=1)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2496, p.dims()[0])).astype(np.float32)
    t = rng.standard_normal((2496, 32)).astype(np.float32)
    for _ in range(3):
        loss, g = p.loss_grad(x, t)
    print("mlp_grad", loss, float(np.linalg.norm(g)))


def box(n):
    d = decks.box_hex20_lognormal(n, n, n // 2, seed=0)
    s = gpu.GpuSystem(0)
    s.upload(d)
    f = gpu.face_load_vector(d)
    s.assemble()
    u, r = s.solve(f, tol=1e-8, precision=gpu.PREC_MIXED)
    print("box", n, r)


def tied():
    d = decks.tied_column()
    s = gpu.GpuSystem(0)
    s.upload(d)
    for _ in range(2):
        s.assemble()
    s.synchronize()
    print("tied", d.num_eq())


def ensemble(count):
    d, noff, _ = decks.ensemble_cantilevers(count, 6, 20, seed=0)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.set_problems(noff)
    f = gpu.face_load_vector(d)
    s.assemble()
    u, conv, its, res = s.solve_batch(f, tol=1e-8)
    print("ensemble", count, int(conv.sum()), int(its.max()))


def newmark():
    d = decks.box_hex20_lognormal(16, 16, 8, seed=0)
    d.rho = np.full(d.num_elems, 1e-3)
    q = gpu.face_load_vector(d)
    s = gpu.GpuSystem(0)
    s.upload(d)
    _, _, rep = s.newmark(q, 20, 1e-4, precision=gpu.PREC_MIXED, tol=1e-8, warm=True, mass_tol=1e-10)
    print("newmark", rep)


if __name__ == "__main__":
    case = sys.argv[1] if len(sys.argv) > 1 else "plate_solve"
    if case == "plate_solve":
        plate_solve()
    elif case == "mlp_grad":
        mlp_grad()
    elif case == "tied":
        tied()
    elif case == "ensemble":
        ensemble(int(sys.argv[2]) if len(sys.argv) > 2 else 128)
    elif case == "newmark":
        newmark()
    elif case == "box":
        box(int(sys.argv[2]) if len(sys.argv) > 2 else 40)
    else:
        raise SystemExit(f"unknown case {case}")
