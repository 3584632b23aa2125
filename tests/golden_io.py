"""Load the golden fixtures (made by tests/golden/make_golden.py from the
reference FAST program) as a Deck plus the reference outputs."""
import os

import numpy as np

from fast_b200 import decks

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# fixtures that hold no deck (.pos files with the numbers they print)
NOT_DECKS = {"pos_output", "full_hex20_64x64x32", "full_plate_tl_40x40x4", "full_tied_column"}


def names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f[:-4] not in NOT_DECKS)


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = {k: z[k] for k in z.files}
    fq = g.get("face_q")
    d = decks.Deck(str(g["kind"]), g["coords"], g["conn"].astype(np.int32), g["E"], g["nu"],
                   tuple(int(v) for v in g["ngp"]), g["fixed"].astype(bool),
                   g.get("face_elem"), g.get("face_corners"), fq, g.get("face_local"),
                   g.get("rho"), bool(int(g["tl"])), node_labels=g.get("node_labels"), title=name,
                   nodal_f=g.get("nodal_f"), solver_rank=g.get("solver_rank"))
    if "patch_degree" in g:
        d.patch = decks.Patch(tuple(int(v) for v in g["patch_degree"]), [g[f"patch_knots{k}"] for k in range(3)],
                              g["patch_span"].astype(np.int32), tuple(int(v) for v in g["patch_grid"]),
                              g["patch_cps"], g.get("patch_weights"), bool(int(g["patch_rational"])))
    return d, g


def lower_K(g):
    import scipy.sparse as sp
    n = int(g["ref_neq"][0])
    return sp.csr_matrix((g["ref_K_data"], g["ref_K_indices"], g["ref_K_indptr"]), shape=(n, n))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
