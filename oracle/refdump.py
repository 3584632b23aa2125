"""Reader for dumps written by the reference harness ``oracle/_ref/fastref``
(TEST INFRASTRUCTURE ONLY; see ``oracle/ref_harness.cpp`` for the format).

``run_dump`` and ``run_bench`` execute the harness, which is the reference
FAST program's own code compiled from its sources by ``oracle/Makefile``.
"""
from __future__ import annotations

import json
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FASTREF = os.path.join(HERE, "_ref", "fastref")
FAST = os.path.join(HERE, "_ref", "fast")


def available() -> bool:
    return os.path.exists(FASTREF)


def read(path: str) -> dict:
    b = open(path, "rb").read()
    if b[:4] != b"FREF":
        raise ValueError(f"{path}: not a reference dump")
    o, d = 4, {}
    while o < len(b):
        nl = struct.unpack_from("<I", b, o)[0]
        o += 4
        name = b[o:o + nl].decode()
        o += nl
        dt = b[o:o + 4].rstrip(b"\0").decode()
        o += 4
        nd = struct.unpack_from("<I", b, o)[0]
        o += 4
        shape = struct.unpack_from("<%dq" % nd, b, o)
        o += 8 * nd
        cnt = int(np.prod(shape))
        a = np.frombuffer(b, dtype="<" + dt, count=cnt, offset=o).reshape(shape).copy()
        o += cnt * a.itemsize
        d[name] = a
    return d


def run_dump(deck_base: str, out_path: str, *opts: str) -> dict:
    subprocess.run([FASTREF, "dump", deck_base, out_path, *opts], check=True,
                   stdout=subprocess.DEVNULL)
    return read(out_path)


def run_bench(deck_base: str, pcg_iters: int, reps: int = 1, pcg_iters2: int = 0) -> dict:
    r = subprocess.run([FASTREF, "bench", deck_base, str(pcg_iters), str(reps), str(pcg_iters2)], check=True,
                       capture_output=True, text=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def lower_csr_from_triplets(neq: int, I, J, V):
    """Sum the recorded cSysMatrix::Add calls into a lower-triangular CSR."""
    import scipy.sparse as sp
    K = sp.csr_matrix((V, (I, J)), shape=(neq, neq))
    K.sum_duplicates()
    K.sort_indices()
    return K
