"""Training driver of the learned Newton load-step predictor.

The reference has no learned part: cCtrlNR::Solver (ctrl/ctrlnr.cpp:47-270)
starts every load step from the last converged displacements.  This module
produces training trajectories with the device Newton driver (the same
load-control iteration as cCtrlNR, run to the deck's tolerance) on seeded
pressure/stiffness variants of one mesh, and trains the device predictor
(:class:`fast_b200.gpu.LearnedPredictor`) on them.  Every numerical step runs
in libfastgpu; this file only sequences the calls.
"""
from __future__ import annotations

import time

import numpy as np

from . import decks as _decks
from . import gpu as _gpu


def trajectories(system: "_gpu.GpuSystem", deck: "_decks.Deck", q: np.ndarray, variants: int, seed: int = 0,
                 steps: int = 40, tol: float = 1e-8, max_iter: int = 30, p_range=(0.75, 1.25),
                 e_range=(0.8, 1.25), e_sigma=0.1, precision=_gpu.PREC_MIXED):
    """Converged load-step displacements of `variants` seeded variants
    (pressure scale, element moduli) of the uploaded mesh.  Yields
    (lambdas, u_steps [steps][neq], report) per variant; restores the deck's
    own moduli afterwards."""
    lam = np.arange(1, steps + 1) / steps
    try:
        for v in range(variants):
            ps, E = _decks.plate_variant_params(seed * 100003 + v, deck.num_elems, float(np.median(deck.E)),
                                                p_range, e_range, e_sigma)
            system.update_material(E=E)
            h, _, rep = system.nr_solve(ps * q, steps, 1.0 / steps, tol=tol, max_iter=max_iter,
                                        predictor=_gpu.PREDICT_SECANT, precision=precision, lin_tol=1e-10,
                                        lin_tol_rel=1e-3, raise_on_fail=False)
            if rep["converged_steps"] != steps:
                continue
            yield lam, h, rep
    finally:
        system.update_material(E=deck.E)


def train_predictor(system, deck, q, variants=64, seed=0, steps=40, tol=1e-8, modes=32, history=4, width=256,
                    hidden=2, epochs=3000, lr=2e-3, **variant_kw):
    """Generate the trajectories, build the POD basis and train the network.
    Returns (predictor, info)."""
    t0 = time.perf_counter()
    pred = _gpu.LearnedPredictor(system, modes=modes, history=history, width=width, hidden=hidden, seed=seed)
    used = 0
    newton = 0
    for lam, h, rep in trajectories(system, deck, q, variants, seed, steps, tol, **variant_kw):
        pred.add_trajectory(lam, h)
        used += 1
        newton += rep["iterations"]
    t1 = time.perf_counter()
    energy = pred.build_basis()
    losses = pred.train(epochs, lr)
    t2 = time.perf_counter()
    info = dict(variants=variants, converged_variants=used, newton_iterations=newton,
                data_seconds=t1 - t0, basis_train_seconds=t2 - t1, captured_energy=energy,
                first_loss=float(losses[0]) if len(losses) else None,
                last_loss=float(losses[-1]) if len(losses) else None)
    info.update({"report": pred.report()})
    return pred, info
