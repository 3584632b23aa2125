"""Seeded solid-mesh decks in FAST's neutral-file (.dat) format.

A :class:`Deck` holds what FAST's reader builds for the solid hot path, as
flat arrays: node coordinates, 0-based element incidence in FAST's local node
order, per-element isotropic material, Gauss order, supports and uniform face
tractions.  It can be written as a ``.dat`` deck that the reference program
reads unchanged, and read back from one.

Reference conventions restated here (FAST, paths inside its tree):

* keyword blocks ``%NODE.COORD``, ``%NODE.SUPPORT``, ``%MATERIAL.ISOTROPIC``,
  ``%SECTION.HOMOGENEOUS.ISOTROPIC.3D``, ``%INTEGRATION.ORDER``,
  ``%ELEMENT.BRICK8/BRICK20(TL)``, ``%LOAD.CASE.AREA.UNIFORM`` and
  ``%HEADER.ANALYSIS.*`` (main/input.cpp:76-330; readers node/node.cpp:78-102,
  289-320, mat/material.cpp:95-119,824-830, sec/section.cpp:96-120,794-806,
  elc/element.cpp:194-228,1985-2101, elc/elmparam.cpp:221-245,
  load/load.cpp:229-248,1440-1480);
* hex8 local order: nodes 1-4 on t=+1, 5-8 on t=-1, counter-clockwise in
  (r, s) (shp/shpsolid.cpp:173-184); hex20 order shp/shpsolid.cpp:301-325;
* equation numbers: node order, translational DOFs x, y, z, 1-based, 0 for a
  fixed or unused DOF (ctrl/ctrl.cpp:2004-2104, cControl::InitDofs/CompEqs);
* face loads name three corner nodes of the loaded face; the face is the
  first face of the element whose corner set contains all three
  (shp/shape.cpp:461-488).
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np

# Natural coordinates of the local nodes, in FAST's order.
HEX8_NAT = np.array([
    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1],
    [-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1]], dtype=np.int64)
HEX20_NAT = np.array([
    [-1, -1, 1], [0, -1, 1], [1, -1, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1], [-1, 1, 1], [-1, 0, 1],
    [-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0],
    [-1, -1, -1], [0, -1, -1], [1, -1, -1], [1, 0, -1], [1, 1, -1], [0, 1, -1], [-1, 1, -1],
    [-1, 0, -1]], dtype=np.int64)

# Faces: (corner local nodes, face-shape local nodes) (shp/shpsolid.cpp:264-276, 459-471).
HEX8_FACES = [
    ((0, 1, 2, 3), (0, 1, 2, 3)), ((3, 2, 6, 7), (3, 2, 6, 7)), ((1, 5, 6, 2), (1, 5, 6, 2)),
    ((0, 4, 5, 1), (0, 4, 5, 1)), ((0, 3, 7, 4), (0, 3, 7, 4)), ((4, 7, 6, 5), (4, 7, 6, 5))]
HEX20_FACES = [
    ((0, 2, 4, 6), (0, 1, 2, 3, 4, 5, 6, 7)),
    ((2, 0, 12, 14), (2, 1, 0, 8, 12, 13, 14, 9)),
    ((4, 2, 14, 16), (4, 3, 2, 9, 14, 15, 16, 10)),
    ((6, 4, 16, 18), (6, 5, 4, 10, 16, 17, 18, 11)),
    ((12, 18, 16, 14), (12, 19, 18, 17, 16, 15, 14, 13)),
    ((18, 6, 0, 12), (18, 11, 6, 7, 0, 8, 12, 19))]

KINDS = {"hex8": (8, HEX8_NAT, HEX8_FACES), "hex20": (20, HEX20_NAT, HEX20_FACES)}


@dataclasses.dataclass
class Patch:
    """A B-spline solid patch (cBspPat, geom/patch.cpp:1459-1484) and the knot
    spans of its elements (%ELEMENT.BSPLINE.SOLID, shp/shpbsp.cpp:57-116)."""
    degree: tuple                   # polynomial degree in r, s and t
    knots: list                     # three knot vectors, multiplicities expanded
    span: np.ndarray                # [ne, 3] 0-based non-zero span per direction
    grid: tuple                     # control points per direction (r fastest in the patch list)
    cps: np.ndarray                 # [grid product] node index of each patch control point
    weights: Optional[np.ndarray] = None  # [nnode] control-point weights, None = 1
    rational: bool = True           # the reference deck's rational flag


@dataclasses.dataclass
class Ties:
    """Slave nodes tied to master surfaces: u_s = sum_k w_k u_(m_k) in x, y
    and z (three %NODE.MULTI-POINT.CONSTRAINT equations per slave,
    node/node.cpp:459-509)."""
    slave: np.ndarray               # [ns] node index
    ptr: np.ndarray                 # [ns+1] offsets into master / weight
    master: np.ndarray              # master node indices
    weight: np.ndarray              # interpolation weights


@dataclasses.dataclass
class Deck:
    kind: str                       # "hex8" | "hex20" | "bsp" (B-spline solid)
    coords: np.ndarray              # [nnode, 3] float64
    conn: np.ndarray                # [ne, nn] int32, 0-based node index
    E: np.ndarray                   # [ne] float64
    nu: np.ndarray                  # [ne] float64
    ngp: tuple = (2, 2, 2)          # Gauss order per direction
    fixed: Optional[np.ndarray] = None   # [nnode, 3] bool, support flags
    face_elem: Optional[np.ndarray] = None   # [nf] int32 element index
    face_corners: Optional[np.ndarray] = None  # [nf, 3] int32 node index
    face_q: Optional[np.ndarray] = None      # [nf, 3] float64 traction
    face_local: Optional[np.ndarray] = None  # [nf] int32 Local flag
    rho: Optional[np.ndarray] = None         # [ne] float64 density
    total_lagrangian: bool = False
    algorithm: str = "linear"
    matrix_type: str = "skyline"
    tol: float = 1e-5
    maxit: int = 0
    maxstep: int = 1
    step_factor: float = 1.0
    time_step: float = 0.0                    # Newmark: %HEADER.ANALYSIS.TIME.STEP
    arc_load_coeff: Optional[float] = None    # arc-length: %HEADER.ANALYSIS.ARC-LENGTH (load coefficient)
    target_iter: Optional[int] = None         # %HEADER.ANALYSIS.TARGET.ITERATIONS (reference default 1)
    newmark: tuple = (0.5, 0.25)              # Newmark: (gamma, beta), cCtrlNewmark defaults
    rayleigh: Optional[tuple] = None          # Newmark: (omega1, omega2, xi1, xi2), %HEADER.ANALYSIS.RAYLEIGH.DAMPING
    print_step: int = 1                       # %HEADER.ANALYSIS.PRINT.STEPS
    node_labels: Optional[np.ndarray] = None  # [nnode] labels used in a .dat
    title: str = "deck"
    patch: Optional[Patch] = None             # kind "bsp": the element patch
    nodal_f: Optional[np.ndarray] = None      # [nnode, 3] nodal forces (%LOAD.CASE.NODAL.FORCE)
    blocks: list = dataclasses.field(default_factory=list)  # further element buckets on the same nodes
    solver_rank: Optional[np.ndarray] = None  # [nnode] %NODE.SOLVER.ORDER position of each node (1-based)
    ties: Optional["Ties"] = None             # tied interfaces (slave nodes follow master surfaces)

    @property
    def nn(self) -> int:
        if self.kind == "bsp":
            d = self.patch.degree
            return (d[0] + 1) * (d[1] + 1) * (d[2] + 1)
        return KINDS[self.kind][0]

    def buckets(self) -> list:
        """This deck's own elements followed by its extra blocks."""
        return [self] + list(self.blocks)

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def num_elems(self) -> int:
        return int(self.conn.shape[0])

    def labels(self) -> np.ndarray:
        if self.node_labels is None:
            return np.arange(1, self.num_nodes + 1, dtype=np.int64)
        return self.node_labels

    def node_eq(self) -> np.ndarray:
        """1-based equation number per (node, direction); 0 = fixed or unused.

        Follows cControl::InitDofs/CompEqs (ctrl/ctrl.cpp:2004-2104): DOFs
        are activated by the elements that use the node, supports remove
        them, and numbering runs over nodes in solver order, x, y, z.
        """
        active = np.zeros((self.num_nodes, 3), dtype=bool)
        for b in self.buckets():
            active[np.unique(b.conn.ravel())] = True
        if self.fixed is not None:
            active &= ~self.fixed
        # nodes in solver order (cNode::GetNodeInSolverOrder, node/node.cpp:543-552):
        # ascending %NODE.SOLVER.ORDER position when given, else label order
        order = np.argsort(self.labels() if self.solver_rank is None else self.solver_rank, kind="stable")
        eq = np.zeros((self.num_nodes, 3), dtype=np.int32)
        flat = active[order].ravel()
        nums = np.cumsum(flat, dtype=np.int64)
        eq_sorted = np.where(flat, nums, 0).reshape(-1, 3)
        eq[order] = eq_sorted
        return eq

    def num_eq(self) -> int:
        return int(self.node_eq().max(initial=0))

    def face_nodes(self) -> np.ndarray:
        """[nf, nface] node indices of each loaded face in face-shape order."""
        nn, _, faces = KINDS[self.kind]
        out = []
        for e, cs in zip(self.face_elem, self.face_corners):
            en = self.conn[e]
            for corner, fnodes in faces:
                cn = set(int(en[c]) for c in corner)
                if all(int(c) in cn for c in cs):
                    out.append([int(en[k]) for k in fnodes])
                    break
            else:
                raise ValueError(f"face load on element {e}: corners {cs} match no face")
        return np.asarray(out, dtype=np.int32)


# --------------------------------------------------------------------------
# structured boxes

def box_mesh(kind: str, n, L, origin=(0.0, 0.0, 0.0), fastest=None) -> tuple:
    """Structured box of hex8 or hex20 elements.

    Returns ``(coords, conn, grid)``; ``grid`` maps node index -> integer grid
    coordinate (on the doubled grid for hex20).  Nodes are numbered with the
    axis of fewest elements varying fastest (a banded numbering), elements in
    the same axis order.
    """
    nx, ny, nz = (int(v) for v in n)
    Lx, Ly, Lz = (float(v) for v in L)
    if fastest is None:
        fastest = tuple(int(a) for a in np.argsort([nx, ny, nz], kind="stable"))
    m = 1 if kind == "hex8" else 2
    G = (m * nx + 1, m * ny + 1, m * nz + 1)
    ii = np.indices(G).reshape(3, -1).T  # all grid points
    if kind == "hex20":
        keep = (ii % 2).sum(axis=1) <= 1
        ii = ii[keep]
    # sort nodes: key = slowest..fastest axis
    a0, a1, a2 = fastest
    okey = np.lexsort((ii[:, a0], ii[:, a1], ii[:, a2]))
    ii = ii[okey]
    lut = -np.ones(G, dtype=np.int64)
    lut[ii[:, 0], ii[:, 1], ii[:, 2]] = np.arange(len(ii))
    h = np.array([Lx / (m * nx), Ly / (m * ny), Lz / (m * nz)])
    coords = np.asarray(origin, dtype=np.float64)[None, :] + ii * h[None, :]

    nat = KINDS[kind][1]
    e = np.indices((nx, ny, nz)).reshape(3, -1).T
    ekey = np.lexsort((e[:, a0], e[:, a1], e[:, a2]))
    e = e[ekey]
    base = m * e  # lower corner on the (doubled) grid
    off = (nat + 1) * m // 2 if kind == "hex20" else (nat + 1) // 2
    pts = base[:, None, :] + off[None, :, :]
    conn = lut[pts[..., 0], pts[..., 1], pts[..., 2]]
    assert (conn >= 0).all()
    return coords, conn.astype(np.int32), ii


def boundary_faces(kind: str, coords, conn, axis: int, value: float, tol=1e-9):
    """(element, three corner nodes) for every element face lying on x[axis]==value."""
    nn, nat, faces = KINDS[kind]
    elems, corners = [], []
    for e in range(conn.shape[0]):
        en = conn[e]
        for corner, _ in faces:
            xs = coords[en[list(corner)], axis]
            if np.all(np.abs(xs - value) < tol):
                elems.append(e)
                corners.append([en[corner[0]], en[corner[1]], en[corner[2]]])
    return np.asarray(elems, np.int32), np.asarray(corners, np.int32)


def _boundary_faces_fast(kind, coords, conn, axis, value, tol=1e-9):
    nn, nat, faces = KINDS[kind]
    out_e, out_c = [], []
    for corner, _ in faces:
        cidx = list(corner)
        xs = coords[conn[:, cidx], axis]
        hit = np.all(np.abs(xs - value) < tol, axis=1)
        es = np.nonzero(hit)[0]
        out_e.append(es)
        out_c.append(conn[es][:, cidx[:3]])
    e = np.concatenate(out_e)
    c = np.concatenate(out_c)
    o = np.argsort(e, kind="stable")
    return e[o].astype(np.int32), c[o].astype(np.int32)


def lognormal_E(ne: int, median=1000.0, sigma=0.5, seed=0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return median * np.exp(sigma * rng.standard_normal(ne))


def cantilever_hex8(nx=20, ny=4, nz=4, L=(10.0, 1.0, 1.0), E=1000.0, nu=0.3, q=(0.0, 0.0, -1.0)) -> Deck:
    """hex8 cantilever: x=0 face clamped, uniform traction on the x=L face.

    Default sizes are the 20x4x4 box on 10x1x1 with 2x2x2 Gauss points,
    E=1000, nu=0.3 and a traction of -1 in z (1575 DOFs).
    """
    coords, conn, _ = box_mesh("hex8", (nx, ny, nz), L)
    ne = conn.shape[0]
    fixed = np.zeros((coords.shape[0], 3), bool)
    fixed[np.abs(coords[:, 0]) < 1e-12] = True
    fe, fc = _boundary_faces_fast("hex8", coords, conn, 0, L[0])
    return Deck("hex8", coords, conn, np.full(ne, E), np.full(ne, nu), (2, 2, 2), fixed,
                fe, fc, np.tile(np.asarray(q, float), (len(fe), 1)), np.zeros(len(fe), np.int32),
                title=f"hex8 cantilever {nx}x{ny}x{nz}")


def concat_decks(members) -> tuple:
    """One deck holding independent decks side by side (disjoint node and
    element ranges, same element kind and Gauss rule).  Returns (deck,
    node_offsets [m+1], element_offsets [m+1]); equation numbers of member k
    are then contiguous, in member order."""
    d0 = members[0]
    noff, eoff = [0], [0]
    for m in members:
        assert m.kind == d0.kind and tuple(m.ngp) == tuple(d0.ngp)
        noff.append(noff[-1] + m.num_nodes)
        eoff.append(eoff[-1] + m.num_elems)
    coords = np.concatenate([m.coords for m in members])
    conn = np.concatenate([m.conn + o for m, o in zip(members, noff)]).astype(np.int32)
    fixed = np.concatenate([m.fixed for m in members])
    has_face = [m.face_elem is not None for m in members]
    fe = fc = fq = fl = None
    if any(has_face):
        fe = np.concatenate([m.face_elem + o for m, o in zip(members, eoff) if m.face_elem is not None]).astype(np.int32)
        fc = np.concatenate([m.face_corners + o for m, o in zip(members, noff) if m.face_elem is not None]).astype(np.int32)
        fq = np.concatenate([m.face_q for m in members if m.face_elem is not None])
        fl = np.concatenate([m.face_local for m in members if m.face_elem is not None]).astype(np.int32)
    rho = np.concatenate([m.rho for m in members]) if all(m.rho is not None for m in members) else None
    d = Deck(d0.kind, coords, conn, np.concatenate([m.E for m in members]), np.concatenate([m.nu for m in members]),
             d0.ngp, fixed, fe, fc, fq, fl, rho=rho, title=f"{len(members)} independent decks")
    return d, np.asarray(noff, np.int64), np.asarray(eoff, np.int64)


def ensemble_cantilevers(count=1024, nmin=6, nmax=20, seed=0, median=1000.0, sigma=0.5, nu=0.3):
    """Independent hex8 cantilevers with uneven meshes: member k is n x n x 2n
    elements (n uniform in [nmin, nmax]) on a 2 x 1 x 1 bar (2n along x),
    2x2x2 Gauss points, x=0 clamped, its own lognormal Young's modulus per
    element (median, sigma) and a random uniform traction (standard normal
    components) on the x=2 face.  Returns (deck, node_offsets, sizes n)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=count)
    members = []
    for k, n in enumerate(ns):
        m = cantilever_hex8(2 * int(n), int(n), int(n), L=(2.0, 1.0, 1.0), nu=nu,
                            q=tuple(rng.standard_normal(3)))
        m.E = median * np.exp(sigma * rng.standard_normal(m.num_elems))
        members.append(m)
    d, noff, _ = concat_decks(members)
    d.title = f"{count} hex8 cantilevers n x n x 2n, n in [{nmin}, {nmax}], seed {seed}"
    return d, noff, ns


def box_hex20_lognormal(nx=64, ny=64, nz=32, L=(4.0, 4.0, 2.0), median=1000.0, sigma=0.5, seed=0,
                        nu=0.3, ngp=3, pressure=1.0) -> Deck:
    """hex20 box with a lognormal Young's modulus per element.

    z=0 face clamped, unit pressure (traction -p in z) on the top face.  The
    default 64x64x32 box on 4x4x2 with 3x3x3 Gauss points has 131,072
    elements and 1,609,920 free equations.
    """
    coords, conn, _ = box_mesh("hex20", (nx, ny, nz), L)
    ne = conn.shape[0]
    fixed = np.zeros((coords.shape[0], 3), bool)
    fixed[np.abs(coords[:, 2]) < 1e-12] = True
    fe, fc = _boundary_faces_fast("hex20", coords, conn, 2, L[2])
    E = lognormal_E(ne, median, sigma, seed)
    return Deck("hex20", coords, conn, E, np.full(ne, nu), (ngp, ngp, ngp), fixed,
                fe, fc, np.tile([0.0, 0.0, -pressure], (len(fe), 1)), np.zeros(len(fe), np.int32),
                matrix_type="sparse", tol=1e-10, maxit=100000,
                title=f"hex20 lognormal box {nx}x{ny}x{nz} seed {seed}")


def plate_tl_hex8(nx=40, ny=40, nz=4, L=10.0, t=1.0, E=1000.0, nu=0.3, pressure=1.0, steps=40,
                  tol=1e-8, maxit=30) -> Deck:
    """Total-Lagrangian (St. Venant-Kirchhoff) hex8 plate under transverse pressure.

    L x L x t plate of nx x ny x nz hex8 elements (%ELEMENT.BRICK8TL), 2x2x2
    Gauss points; every node on the four side faces pinned (u = v = w = 0);
    uniform pressure on the top face (traction -pressure in z).  Load-control
    Newton-Raphson ('lcm', proportional loading) over `steps` equal steps to
    the full pressure.
    """
    coords, conn, _ = box_mesh("hex8", (nx, ny, nz), (L, L, t))
    ne = conn.shape[0]
    fixed = np.zeros((coords.shape[0], 3), bool)
    side = ((np.abs(coords[:, 0]) < 1e-12) | (np.abs(coords[:, 0] - L) < 1e-12) |
            (np.abs(coords[:, 1]) < 1e-12) | (np.abs(coords[:, 1] - L) < 1e-12))
    fixed[side] = True
    fe, fc = _boundary_faces_fast("hex8", coords, conn, 2, t)
    return Deck("hex8", coords, conn, np.full(ne, E), np.full(ne, nu), (2, 2, 2), fixed,
                fe, fc, np.tile([0.0, 0.0, -pressure], (len(fe), 1)), np.zeros(len(fe), np.int32),
                total_lagrangian=True, algorithm="lcm", matrix_type="skyline", tol=tol, maxit=maxit,
                maxstep=steps, step_factor=1.0 / steps,
                title=f"TL hex8 plate {nx}x{ny}x{nz}, pressure {pressure}, {steps} steps")


def plate_variant_params(seed: int, num_elems: int, E: float = 1000.0, p_range=(0.75, 1.25), e_range=(0.8, 1.25),
                         e_sigma: float = 0.1):
    """One seeded pressure/stiffness variant of a plate: (pressure scale,
    Young's modulus per element).  The pressure scale is U[p_range]; the
    modulus is E times a plate-wide factor U[e_range] times an element-wise
    lognormal factor exp(e_sigma N(0, 1))."""
    rng = np.random.default_rng(seed)
    ps = float(rng.uniform(*p_range))
    es = float(rng.uniform(*e_range))
    return ps, E * es * np.exp(e_sigma * rng.standard_normal(num_elems))


def open_knots(p: int, n: int) -> np.ndarray:
    """Open uniform knot vector of degree p with n unit spans: p+1 zeros,
    1..n-1, p+1 values n (multiplicities expanded)."""
    return np.concatenate([np.zeros(p), np.arange(n + 1, dtype=np.float64), np.full(p, float(n))])


def bspline_box(p: int, n=(4, 4, 2), L=(4.0, 4.0, 2.0), origin=(0.0, 0.0, 0.0), jitter=0.05, seed=0,
                E=1000.0, nu=0.3, ngp=None, clamp_axis=0, load=(0.0, 0.0, -1.0)) -> Deck:
    """B-spline solid block of degree p with n[d] elements (knot spans) per
    direction on open uniform knot vectors.

    Control points sit on a uniform grid of (n[d] + p) points per direction
    over the box, each coordinate moved by uniform[-jitter h, jitter h]
    (h = L[d]/n[d], the element size) except along the direction in which the
    point is on a face of the box, so the faces stay plane.  The face
    x[clamp_axis] = origin is clamped and the opposite face carries nodal
    forces summing to ``load``.  Elements are numbered with the r span
    fastest; local nodes are the element's (p+1)^3 control points, r index
    fastest (cShapeBspSolid::Init, shp/shpbsp.cpp:873-902).
    """
    n = tuple(int(v) for v in n)
    nb = tuple(v + p for v in n)
    rng = np.random.default_rng(seed)
    axes = [origin[d] + L[d] * np.arange(nb[d]) / (nb[d] - 1) for d in range(3)]
    I, J, K = np.meshgrid(np.arange(nb[0]), np.arange(nb[1]), np.arange(nb[2]), indexing="ij")
    idx = np.stack([I.ravel(order="F"), J.ravel(order="F"), K.ravel(order="F")], axis=1)  # r fastest
    coords = np.stack([axes[d][idx[:, d]] for d in range(3)], axis=1)
    for d in range(3):
        h = L[d] / n[d]
        inner = (idx[:, d] > 0) & (idx[:, d] < nb[d] - 1)
        coords[inner, d] += rng.uniform(-jitter * h, jitter * h, int(inner.sum()))
    ids = np.arange(len(coords)).reshape(nb[2], nb[1], nb[0])  # [k][j][i]
    Q = p + 1
    el = []
    span = []
    for ek in range(n[2]):
        for ej in range(n[1]):
            for ei in range(n[0]):
                el.append(ids[ek:ek + Q, ej:ej + Q, ei:ei + Q].ravel())
                span.append((ei, ej, ek))
    conn = np.asarray(el, dtype=np.int32)
    ne = len(conn)
    fixed = np.zeros((len(coords), 3), bool)
    fixed[idx[:, clamp_axis] == 0] = True
    nodal = np.zeros((len(coords), 3))
    far = idx[:, clamp_axis] == nb[clamp_axis] - 1
    nodal[far] = np.asarray(load, dtype=np.float64) / int(far.sum())
    patch = Patch((p, p, p), [open_knots(p, n[d]) for d in range(3)], np.asarray(span, dtype=np.int32), nb,
                  np.arange(len(coords), dtype=np.int64))
    g = (p + 1,) * 3 if ngp is None else tuple(ngp)
    return Deck("bsp", coords, conn, np.full(ne, float(E)), np.full(ne, float(nu)), g, fixed,
                matrix_type="sparse", patch=patch, nodal_f=nodal, title=f"bspline p={p} {n}")


def hex_shape(kind: str, r: float, s: float, t: float) -> np.ndarray:
    """hex8 / hex20 shape functions at (r, s, t) in FAST's local node order
    (cShapeBrick8 / cShapeBrick20, shp/shpsolid.cpp:188-238, 329-433)."""
    nat = KINDS[kind][1]
    N = np.zeros(len(nat))
    for a, (ri, si, ti) in enumerate(nat):
        fr, fs, ft = 1 + ri * r, 1 + si * s, 1 + ti * t
        if kind == "hex8":
            N[a] = 0.125 * fr * fs * ft
        elif ri and si and ti:
            N[a] = 0.125 * fr * fs * ft * (ri * r + si * s + ti * t - 2.0)
        elif ri == 0:
            N[a] = 0.25 * (1 - r * r) * fs * ft
        elif si == 0:
            N[a] = 0.25 * fr * (1 - s * s) * ft
        else:
            N[a] = 0.25 * fr * fs * (1 - t * t)
    return N


def bspline_eval(U: np.ndarray, p: int, u: float):
    """(first basis index, values, u-derivatives) of the p+1 B-splines that are
    non-zero at u on the open knot vector U (Cox-de Boor recurrence)."""
    U = np.asarray(U, dtype=np.float64)
    nb = len(U) - p - 1
    k = int(np.searchsorted(U, u, side="right")) - 1
    k = min(max(k, p), nb - 1)

    def table(q):
        # degree-q functions N_{k-q..k}
        N = np.array([1.0])
        for d in range(1, q + 1):
            M = np.zeros(d + 1)
            for t in range(d + 1):
                i = k - d + t
                v = 0.0
                if t >= 1 and U[i + d] > U[i]:
                    v += (u - U[i]) / (U[i + d] - U[i]) * N[t - 1]
                if t <= d - 1 and U[i + d + 1] > U[i + 1]:
                    v += (U[i + d + 1] - u) / (U[i + d + 1] - U[i + 1]) * N[t]
                M[t] = v
            N = M
        return N

    N = table(p)
    Nm = table(p - 1)
    dN = np.zeros(p + 1)
    for t in range(p + 1):
        i = k - p + t
        if t >= 1 and U[i + p] > U[i]:
            dN[t] += p / (U[i + p] - U[i]) * Nm[t - 1]
        if t <= p - 1 and U[i + p + 1] > U[i + 1]:
            dN[t] -= p / (U[i + p + 1] - U[i + 1]) * Nm[t]
    return k - p, N, dN


def _hex_face_weights(kind, coords, conn, n, L, origin, pts, top):
    """(masters, weights) of each point (x, y) on the z-top / z-bottom face of a
    structured hex block made by box_mesh (its elements in (x, y, z) cells)."""
    nx, ny, nz = n
    # cell -> element: the element whose lower corner node sits at the cell corner
    X = coords[conn]                       # [ne, nn, 3]
    lo = X.min(axis=1)
    h = np.array([L[0] / nx, L[1] / ny, L[2] / nz])
    cell = np.rint((lo - np.asarray(origin)) / h).astype(np.int64)
    lut = {tuple(c): e for e, c in enumerate(cell)}
    res = []
    for x, y in pts:
        fx = (x - origin[0]) / h[0]
        fy = (y - origin[1]) / h[1]
        ix = min(max(int(np.floor(fx)), 0), nx - 1)
        iy = min(max(int(np.floor(fy)), 0), ny - 1)
        e = lut[(ix, iy, nz - 1 if top else 0)]
        r, s_ = 2 * (fx - ix) - 1, 2 * (fy - iy) - 1
        N = hex_shape(kind, r, s_, 1.0 if top else -1.0)
        keep = np.abs(N) > 1e-14
        res.append((conn[e][keep], N[keep]))
    return res


def _bsp_face_weights(deck, node_off, pts, top, tol=1e-13):
    """(masters, weights) of each point (x, y) on the t = 1 (top) or t = 0
    (bottom) surface of a B-spline block from bspline_box: the surface
    parameters (u, v) of the point by Newton's method, then the tensor
    products N_i(u) N_j(v) of the face's control points (unit weights)."""
    P = deck.patch
    p = P.degree
    nb0, nb1, nb2 = P.grid
    k = nb2 - 1 if top else 0
    Xf = np.array([[deck.coords[node_off + P.cps[i + nb0 * j + nb0 * nb1 * k], :2]
                    for i in range(nb0)] for j in range(nb1)])  # [j][i][2]
    U, V = np.asarray(P.knots[0]), np.asarray(P.knots[1])
    x0 = deck.coords[node_off + P.cps[0]]
    span = np.ptp(deck.coords[node_off + P.cps], axis=0)
    res = []
    for x, y in pts:
        u = U[-1] * (x - x0[0]) / span[0]
        v = V[-1] * (y - x0[1]) / span[1]
        for _ in range(50):
            iu, Nu, dNu = bspline_eval(U, p[0], u)
            iv, Nv, dNv = bspline_eval(V, p[1], v)
            blk = Xf[iv:iv + p[1] + 1, iu:iu + p[0] + 1]        # [j][i][2]
            pos = np.einsum("j,i,jic->c", Nv, Nu, blk)
            Ju = np.einsum("j,i,jic->c", Nv, dNu, blk)
            Jv = np.einsum("j,i,jic->c", dNv, Nu, blk)
            J = np.stack([Ju, Jv], axis=1)
            d = np.linalg.solve(J, np.array([x, y]) - pos)
            u = min(max(u + d[0], U[0]), U[-1])
            v = min(max(v + d[1], V[0]), V[-1])
            if np.abs(d).max() < tol:
                break
        iu, Nu, _ = bspline_eval(U, p[0], u)
        iv, Nv, _ = bspline_eval(V, p[1], v)
        ms, ws = [], []
        for j in range(p[1] + 1):
            for i in range(p[0] + 1):
                w = Nu[i] * Nv[j]
                if abs(w) > 1e-14:
                    ms.append(node_off + P.cps[(iu + i) + nb0 * (iv + j) + nb0 * nb1 * k])
                    ws.append(w)
        res.append((np.asarray(ms), np.asarray(ws)))
    return res


def tied_column(hex8=(40, 40, 20), hex20=(24, 24, 12), p2=(32, 32, 8), p3=(24, 24, 6), width=1.0, jitter=0.05,
                seed=0, E=1000.0, nu=0.3, load=(0.0, 0.0, -1.0)) -> Deck:
    """Four blocks on one width x width footprint, stacked in z and joined by
    tied interfaces: a B-spline p=2 patch (bottom, clamped at z=0), a hex8 box,
    a hex20 box and a B-spline p=3 patch (top, nodal forces summing to
    ``load`` on its top control points).  Each block's height is its element
    count in z times its element size.  Ties: the hex8 box's bottom nodes
    follow the p=2 patch's top surface, its top nodes follow the hex20 box's
    bottom faces, and the hex20 box's top nodes follow the p=3 patch's bottom
    surface (slaves on the finer or interpolating side).  Control points are
    jittered as in bspline_box; the hex boxes are regular."""
    W = float(width)
    z = 0.0
    parts = []
    # p=2 patch
    hz = W / p2[0] * p2[2]
    b2 = bspline_box(2, p2, L=(W, W, hz), origin=(0.0, 0.0, z), jitter=jitter, seed=seed, E=E, nu=nu,
                     clamp_axis=2, load=(0.0, 0.0, 0.0))
    parts.append(b2); z += hz
    h8z = W / hex8[0] * hex8[2]
    c8, k8, _ = box_mesh("hex8", hex8, (W, W, h8z), origin=(0.0, 0.0, z))
    z8 = (z, z + h8z); z += h8z
    h20z = W / hex20[0] * hex20[2]
    c20, k20, _ = box_mesh("hex20", hex20, (W, W, h20z), origin=(0.0, 0.0, z))
    z20 = (z, z + h20z); z += h20z
    h3z = W / p3[0] * p3[2]
    b3 = bspline_box(3, p3, L=(W, W, h3z), origin=(0.0, 0.0, z), jitter=jitter, seed=seed + 1, E=E, nu=nu,
                     clamp_axis=2, load=load)
    z += h3z
    off = np.cumsum([0, b2.num_nodes, len(c8), len(c20), b3.num_nodes])
    coords = np.concatenate([b2.coords, c8, c20, b3.coords])
    nn = len(coords)
    fixed = np.zeros((nn, 3), bool)
    fixed[:b2.num_nodes] = b2.fixed          # p=2 patch: z = 0 face clamped
    nodal = np.zeros((nn, 3))
    far = np.isclose(b3.coords[:, 2], z)     # p=3 patch: load on its top face
    nodal[off[3]:off[4]][far] = np.asarray(load, dtype=np.float64) / int(far.sum())

    def sub(kind, conn, ngp, patch=None):
        ne = len(conn)
        return Deck(kind, coords, conn.astype(np.int32), np.full(ne, float(E)), np.full(ne, float(nu)), ngp,
                    patch=patch)

    p3patch = dataclasses.replace(b3.patch, cps=b3.patch.cps + off[3])
    blocks = [sub("hex8", k8 + off[1], (2, 2, 2)), sub("hex20", k20 + off[2], (3, 3, 3)),
              sub("bsp", b3.conn + off[3], (4, 4, 4), p3patch)]
    main = Deck("bsp", coords, b2.conn.copy(), b2.E.copy(), b2.nu.copy(), (3, 3, 3), fixed, matrix_type="sparse",
                patch=b2.patch, nodal_f=nodal, blocks=blocks, title="tied column")
    # ties
    slaves, masters, weights = [], [], []

    def add(nodes, res):
        for n_, (ms, ws) in zip(nodes, res):
            slaves.append(int(n_)); masters.append(np.asarray(ms, dtype=np.int64)); weights.append(ws)

    bot8 = off[1] + np.nonzero(np.isclose(c8[:, 2], z8[0]))[0]
    add(bot8, _bsp_face_weights(main, 0, coords[bot8, :2], top=True))
    top8 = off[1] + np.nonzero(np.isclose(c8[:, 2], z8[1]))[0]
    add(top8, [(off[2] + ms, ws) for ms, ws in
               _hex_face_weights("hex20", c20, k20, hex20, (W, W, h20z), (0.0, 0.0, z20[0]), coords[top8, :2], top=False)])
    top20 = off[2] + np.nonzero(np.isclose(c20[:, 2], z20[1]))[0]
    add(top20, _bsp_face_weights(dataclasses.replace(b3, coords=coords, patch=p3patch), 0, coords[top20, :2],
                                 top=False))
    ptr = np.concatenate([[0], np.cumsum([len(m) for m in masters])]).astype(np.int64)
    main.ties = Ties(np.asarray(slaves, dtype=np.int64), ptr, np.concatenate(masters).astype(np.int64),
                     np.concatenate(weights).astype(np.float64))
    return main


def nodal_load_vector(deck: Deck) -> np.ndarray:
    """Equation-space vector of the deck's nodal forces (cNodalLoad)."""
    f = np.zeros(deck.num_eq())
    if deck.nodal_f is None:
        return f
    eq = deck.node_eq()
    m = eq > 0
    np.add.at(f, eq[m] - 1, deck.nodal_f[m])
    return f


def read_pos_factors(path: str) -> np.ndarray:
    """Load factor of every printed step of a FAST .pos file
    (%RESULT.CASE.STEP.FACTOR, cControl::PrintResult ctrl/ctrl.cpp:1154-1155)."""
    out = []
    with open(path) as fp:
        lines = fp.read().splitlines()
    for i, ln in enumerate(lines):
        if ln.strip() == "%RESULT.CASE.STEP.FACTOR":
            out.append(float(lines[i + 1].split()[0]))
    return np.asarray(out)


def read_pos_block(path: str, key: str = "NODAL.DISPLACEMENT") -> np.ndarray:
    """Nodal vectors of one result block (``%RESULT.CASE.STEP.<key>``) of every
    printed step of a FAST .pos file: [steps][nnode][3], rows ordered by node
    label.  Keys written by cControl::PrintResult / cCtrlNewmark::PrintVelAcc:
    NODAL.DISPLACEMENT, VELOCITY, ACCELERATION."""
    steps = []
    with open(path) as fp:
        lines = fp.read().splitlines()
    tag = "%RESULT.CASE.STEP." + key
    i = 0
    while i < len(lines):
        if lines[i].strip() == tag:
            n = int(lines[i + 1].split()[0])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            lab = np.array([int(r[0]) for r in rows])
            u = np.array([[float(v) for v in r[1:4]] for r in rows])
            steps.append(u[np.argsort(lab)])
            i += 2 + n
        else:
            i += 1
    return np.asarray(steps)


def read_pos_displacements(path: str, labels=None) -> np.ndarray:
    """Nodal displacements of every printed step of a FAST .pos file: [steps][nnode][3]."""
    return read_pos_block(path, "NODAL.DISPLACEMENT")


# --------------------------------------------------------------------------
# .dat writer / reader

def _fmt(x: float) -> str:
    return repr(float(x))


def write_dat(deck: Deck, base: str) -> str:
    """Write ``base + '.dat'`` readable by FAST; returns the path."""
    path = base + ".dat"
    lab = deck.labels()
    nn = deck.nn
    ne = deck.num_elems
    lines = ["%HEADER", deck.title, ""]
    lines += ["%HEADER.ANALYSIS.ALGORITHM", f"'{deck.algorithm}'", ""]
    lines += ["%HEADER.ANALYSIS.MATRIX.TYPE", f"'{deck.matrix_type}'", ""]
    lines += ["%HEADER.ANALYSIS.TOLERANCE", _fmt(deck.tol), ""]
    if deck.maxit:
        lines += ["%HEADER.ANALYSIS.MAXIMUM.ITERATIONS", str(int(deck.maxit)), ""]
    if deck.maxstep != 1:
        lines += ["%HEADER.ANALYSIS.MAXIMUM.STEPS", str(int(deck.maxstep)), ""]
    if deck.step_factor != 1.0:
        lines += ["%HEADER.ANALYSIS.STEP.FACTOR", _fmt(deck.step_factor), ""]
    if deck.arc_load_coeff is not None:
        lines += ["%HEADER.ANALYSIS.ARC-LENGTH", _fmt(deck.arc_load_coeff), ""]
    if deck.target_iter is not None:
        lines += ["%HEADER.ANALYSIS.TARGET.ITERATIONS", str(int(deck.target_iter)), ""]
    if deck.algorithm.lower() == "newmark":
        lines += ["%HEADER.ANALYSIS.TIME.STEP", _fmt(deck.time_step), ""]
        lines += ["%HEADER.ANALYSIS.NEWMARK.PARAMETERS", f"{_fmt(deck.newmark[0])} {_fmt(deck.newmark[1])}", ""]
        if deck.rayleigh is not None:
            lines += ["%HEADER.ANALYSIS.RAYLEIGH.DAMPING", " ".join(_fmt(v) for v in deck.rayleigh), ""]
        lines += ["%HEADER.ANALYSIS.PRINT.STEPS", str(int(deck.print_step)), ""]
    lines += ["%HEADER.OUTPUT.PRECISION", "15", ""]
    lines += ["%NODE", str(deck.num_nodes), "", "%NODE.COORD", str(deck.num_nodes)]
    lines += [f"{int(l)} {_fmt(x)} {_fmt(y)} {_fmt(z)}" for l, (x, y, z) in zip(lab, deck.coords)]
    lines.append("")
    if deck.solver_rank is not None:
        lines += ["%NODE.SOLVER.ORDER", str(deck.num_nodes)] + [" ".join(str(int(v)) for v in deck.solver_rank), ""]
    if deck.fixed is not None and deck.fixed.any():
        sup = np.nonzero(deck.fixed.any(axis=1))[0]
        lines += ["%NODE.SUPPORT", str(len(sup))]
        lines += [f"{int(lab[i])} {int(deck.fixed[i,0])} {int(deck.fixed[i,1])} {int(deck.fixed[i,2])} 0 0 0" for i in sup]
        lines.append("")
    # one material per distinct (E, nu) pair, one section per material
    pairs = np.stack([deck.E, deck.nu], axis=1)
    uniq, inv = np.unique(pairs, axis=0, return_inverse=True)
    inv = inv.ravel()
    nm = len(uniq)
    lines += ["%MATERIAL", str(nm), "", "%MATERIAL.ISOTROPIC", str(nm)]
    lines += [f"{i+1} {_fmt(E)} {_fmt(nu)}" for i, (E, nu) in enumerate(uniq)]
    lines.append("")
    if deck.rho is not None:
        # density is per material; one density per distinct material is required
        dens = np.zeros(nm)
        dens[inv] = deck.rho
        lines += ["%MATERIAL.DENSITY", str(nm)] + [f"{i+1} {_fmt(d)}" for i, d in enumerate(dens)] + [""]
    lines += ["%SECTION", str(nm), "", "%SECTION.HOMOGENEOUS.ISOTROPIC.3D", str(nm)]
    lines += [f"{i+1} {i+1}" for i in range(nm)]
    lines.append("")
    g = deck.ngp
    lines += ["%INTEGRATION.ORDER", "1", f"1 {g[0]} {g[1]} {g[2]} {g[0]} {g[1]} {g[2]}", ""]
    if deck.kind == "bsp":
        # one B-spline solid patch (cBspPat::Read, geom/patch.cpp:1459-1484): rational
        # flag, then per direction degree 'General' #knots values multiplicities,
        # then the control-point node labels, r fastest
        P = deck.patch
        lines += ["%PATCH", "1", f"1 'bspsol' {int(bool(P.rational))}"]
        for d in range(3):
            vals, mult = np.unique(np.asarray(P.knots[d]), return_counts=True)
            lines.append(f"{P.degree[d]} 'General' {len(vals)} " + " ".join(_fmt(v) for v in vals) + " " +
                         " ".join(str(int(m)) for m in mult))
        lines.append(" ".join(str(int(v)) for v in lab[P.cps]))
        lines.append("")
        if P.weights is not None:
            lines += ["%CONTROL.POINT.WEIGHT", str(deck.num_nodes)]
            lines += [f"{int(l)} {_fmt(w)}" for l, w in zip(lab, P.weights)]
            lines.append("")
        lines += ["%ELEMENT", str(ne), "", "%ELEMENT.BSPLINE.SOLID" + ("TL" if deck.total_lagrangian else ""), str(ne)]
        lines += [f"{e+1} {inv[e]+1} 1 1 {int(P.span[e,0])+1} {int(P.span[e,1])+1} {int(P.span[e,2])+1}"
                  for e in range(ne)]
        lines.append("")
    else:
        key = {"hex8": "BRICK8", "hex20": "BRICK20"}[deck.kind] + ("TL" if deck.total_lagrangian else "")
        lines += ["%ELEMENT", str(ne), "", f"%ELEMENT.{key}", str(ne)]
        cl = lab[deck.conn]
        lines += [f"{e+1} {inv[e]+1} 1 " + " ".join(str(int(v)) for v in cl[e]) for e in range(ne)]
        lines.append("")
    has_face = deck.face_elem is not None and len(deck.face_elem)
    has_nodal = deck.nodal_f is not None and bool(np.any(deck.nodal_f))
    if has_face or has_nodal:
        lines += ["%LOAD", "1", "1 'Load_Case_1'", "%LOAD.CASE", "1"]
    if has_nodal:
        nz = np.nonzero(np.any(deck.nodal_f != 0.0, axis=1))[0]
        lines += ["%LOAD.CASE.NODAL.FORCE", str(len(nz))]
        lines += [f"{int(lab[i])} {_fmt(deck.nodal_f[i,0])} {_fmt(deck.nodal_f[i,1])} {_fmt(deck.nodal_f[i,2])} 0 0 0"
                  for i in nz]
        lines.append("")
    if has_face:
        nf = len(deck.face_elem)
        lines += ["%LOAD.CASE.AREA.UNIFORM", str(nf)]
        for k in range(nf):
            c = lab[deck.face_corners[k]]
            q = deck.face_q[k]
            lines.append(f"{int(deck.face_elem[k])+1} {int(c[0])} {int(c[1])} {int(c[2])} "
                         f"{int(deck.face_local[k])} {_fmt(q[0])} {_fmt(q[1])} {_fmt(q[2])}")
        lines.append("")
    lines += ["%END", ""]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fp:
        fp.write("\n".join(lines))
    return path


def _tokens_by_label(text: str) -> dict:
    blocks, cur, buf = {}, None, []
    for raw in text.splitlines():
        s = raw.strip()
        if s.startswith("%"):
            if cur is not None:
                blocks[cur] = buf
            cur, buf = s[1:].split()[0], []
        elif cur is not None:
            buf.extend(s.split())
    if cur is not None:
        blocks[cur] = buf
    return blocks


def read_dat(path: str) -> Deck:
    """Read the solid hot-path subset of a FAST ``.dat`` deck."""
    with open(path) as fp:
        blk = _tokens_by_label(fp.read())
    t = blk["NODE.COORD"]
    n = int(t[0])
    arr = np.array(t[1:1 + 4 * n], dtype=np.float64).reshape(n, 4)
    labels = arr[:, 0].astype(np.int64)
    order = np.argsort(labels)
    labels = labels[order]
    coords = arr[order, 1:4].copy()
    l2i = {int(l): i for i, l in enumerate(labels)}
    fixed = np.zeros((n, 3), bool)
    if "NODE.SUPPORT" in blk:
        t = blk["NODE.SUPPORT"]
        ns = int(t[0])
        a = np.array(t[1:1 + 7 * ns], dtype=np.int64).reshape(ns, 7)
        for row in a:
            fixed[l2i[int(row[0])]] |= row[1:4].astype(bool)
    mats = {}
    t = blk.get("MATERIAL.ISOTROPIC", ["0"])
    for k in range(int(t[0])):
        mid, E, nu = t[1 + 3 * k: 4 + 3 * k]
        mats[int(mid)] = (float(E), float(nu))
    dens = {}
    if "MATERIAL.DENSITY" in blk:
        t = blk["MATERIAL.DENSITY"]
        for k in range(int(t[0])):
            dens[int(t[1 + 2 * k])] = float(t[2 + 2 * k])
    secs = {}
    t = blk.get("SECTION.HOMOGENEOUS.ISOTROPIC.3D", ["0"])
    for k in range(int(t[0])):
        secs[int(t[1 + 2 * k])] = int(t[2 + 2 * k])
    t = blk["INTEGRATION.ORDER"]
    ords = {}
    for k in range(int(t[0])):
        row = [int(v) for v in t[1 + 7 * k: 8 + 7 * k]]
        ords[row[0]] = tuple(row[1:4])
    if "ELEMENT.BSPLINE.SOLID" in blk or "ELEMENT.BSPLINE.SOLIDTL" in blk:
        return _read_bsp(blk, coords, labels, l2i, fixed, mats, secs, ords, path, dens)
    kind, tl, key = None, False, None
    for k, (kd, t_) in {"ELEMENT.BRICK8": ("hex8", False), "ELEMENT.BRICK20": ("hex20", False),
                        "ELEMENT.BRICK8TL": ("hex8", True), "ELEMENT.BRICK20TL": ("hex20", True)}.items():
        if k in blk:
            if kind is not None:
                raise ValueError("decks with more than one solid element type are not read here")
            kind, tl, key = kd, t_, k
    nn = KINDS[kind][0]
    t = blk[key]
    ne = int(t[0])
    a = np.array(t[1:1 + (3 + nn) * ne], dtype=np.int64).reshape(ne, 3 + nn)
    a = a[np.argsort(a[:, 0])]
    elem_labels = a[:, 0]
    conn = np.vectorize(lambda l: l2i[int(l)])(a[:, 3:]).astype(np.int32)
    E = np.array([mats[secs[int(s)]][0] for s in a[:, 1]])
    nu = np.array([mats[secs[int(s)]][1] for s in a[:, 1]])
    rho = np.array([dens.get(secs[int(s)], 0.0) for s in a[:, 1]]) if dens else None
    ordset = {ords[int(o)] for o in a[:, 2]}
    if len(ordset) != 1:
        raise ValueError("one integration order per deck is read here")
    ngp = ordset.pop()
    e2i = {int(l): i for i, l in enumerate(elem_labels)}
    fe = fc = fq = fl = None
    if "LOAD.CASE.AREA.UNIFORM" in blk:
        t = blk["LOAD.CASE.AREA.UNIFORM"]
        nf = int(t[0])
        rows = [t[1 + 8 * k: 9 + 8 * k] for k in range(nf)]
        fe = np.array([e2i[int(r[0])] for r in rows], np.int32)
        fc = np.array([[l2i[int(v)] for v in r[1:4]] for r in rows], np.int32)
        fl = np.array([int(r[4]) for r in rows], np.int32)
        fq = np.array([[float(v) for v in r[5:8]] for r in rows])

    return Deck(kind, coords, conn, E, nu, ngp, fixed, fe, fc, fq, fl, rho, tl,
                node_labels=labels, title=os.path.basename(path), solver_rank=_solver_rank(blk, n),
                **_analysis_header(blk))


def _analysis_header(blk) -> dict:
    """%HEADER.ANALYSIS.* fields of a deck (defaults as the reference's)."""
    def s1(label, default, cast):
        if label in blk and blk[label]:
            return cast(blk[label][0].strip("'"))
        return default

    return dict(algorithm=s1("HEADER.ANALYSIS.ALGORITHM", "linear", str),
                matrix_type=s1("HEADER.ANALYSIS.MATRIX.TYPE", "skyline", str),
                tol=s1("HEADER.ANALYSIS.TOLERANCE", 1e-5, float),
                maxit=s1("HEADER.ANALYSIS.MAXIMUM.ITERATIONS", 0, int),
                maxstep=s1("HEADER.ANALYSIS.MAXIMUM.STEPS", 1, int),
                step_factor=s1("HEADER.ANALYSIS.STEP.FACTOR", 1.0, float))


def _read_bsp(blk, coords, labels, l2i, fixed, mats, secs, ords, path, dens=None) -> Deck:
    """%PATCH (one 'bspsol' patch, 'General' knot vectors), %CONTROL.POINT.WEIGHT
    and %ELEMENT.BSPLINE.SOLID (cBspPat::Read geom/patch.cpp:1459-1484,
    cKnotVector::ReadKnot/ReadMult geom/knotvec.cpp:91-170, cShapeBsp::ReadIGA
    shp/shpbsp.cpp:57-116)."""
    t = blk["PATCH"]
    if int(t[0]) != 1 or t[2] != "'bspsol'":
        raise ValueError("one 'bspsol' patch per deck is read here")
    rational = bool(int(t[3]))
    pos = 4
    degs, knots, nbas = [], [], []
    for d in range(3):
        deg = int(t[pos]); kind = t[pos + 1]; nk = int(t[pos + 2])
        if kind != "'General'":
            raise ValueError(f"knot vector format {kind} is not read here")
        vals = [float(v) for v in t[pos + 3: pos + 3 + nk]]
        mult = [int(v) for v in t[pos + 3 + nk: pos + 3 + 2 * nk]]
        pos += 3 + 2 * nk
        U = np.repeat(np.asarray(vals), mult)
        degs.append(deg)
        knots.append(U)
        nbas.append(len(U) - deg - 1)
    ncp = nbas[0] * nbas[1] * nbas[2]
    cps = np.array([l2i[int(v)] for v in t[pos: pos + ncp]], dtype=np.int64)
    weights = None
    if "CONTROL.POINT.WEIGHT" in blk:
        w = blk["CONTROL.POINT.WEIGHT"]
        nw = int(w[0])
        weights = np.ones(len(coords))
        for k in range(nw):
            weights[l2i[int(w[1 + 2 * k])]] = float(w[2 + 2 * k])
    # %ELEMENT.BSPLINE.SOLIDTL: the same elements with cElmParamTL
    tl = "ELEMENT.BSPLINE.SOLIDTL" in blk
    t = blk["ELEMENT.BSPLINE.SOLIDTL" if tl else "ELEMENT.BSPLINE.SOLID"]
    ne = int(t[0])
    a = np.array(t[1:1 + 7 * ne], dtype=np.int64).reshape(ne, 7)
    a = a[np.argsort(a[:, 0])]
    span = (a[:, 4:7] - 1).astype(np.int32)
    # first basis function of each non-zero span (cBSplineBasis::getBasInd, geom/bspbasis.cpp:59-62)
    first = []
    for d in range(3):
        U = knots[d]
        left = [i - 1 for i in range(1, len(U)) if U[i] - U[i - 1] > 1e-5]
        first.append(np.asarray(left) - degs[d])
    Qr, Qs, Qt = (v + 1 for v in degs)
    conn = np.zeros((ne, Qr * Qs * Qt), dtype=np.int32)
    for e in range(ne):
        b0, b1, b2 = (int(first[d][span[e, d]]) for d in range(3))
        loc = 0
        for k in range(Qt):
            for j in range(Qs):
                for i in range(Qr):
                    cp = (b0 + i) + nbas[0] * (b1 + j) + nbas[0] * nbas[1] * (b2 + k)
                    conn[e, loc] = cps[cp]
                    loc += 1
    E = np.array([mats[secs[int(s_)]][0] for s_ in a[:, 1]])
    nu = np.array([mats[secs[int(s_)]][1] for s_ in a[:, 1]])
    rho = np.array([dens.get(secs[int(s_)], 0.0) for s_ in a[:, 1]]) if dens else None
    ordset = {ords[int(o)] for o in a[:, 2]}
    if len(ordset) != 1:
        raise ValueError("one integration order per deck is read here")
    patch = Patch(tuple(degs), knots, span, tuple(nbas), cps, weights, rational)
    return Deck("bsp", coords, conn, E, nu, ordset.pop(), fixed, rho=rho, patch=patch, total_lagrangian=tl,
                node_labels=labels, title=os.path.basename(path), solver_rank=_solver_rank(blk, len(coords)),
                **_analysis_header(blk))


def _solver_rank(blk, nnode):
    """%NODE.SOLVER.ORDER: the i-th entry is the solver position of the i-th
    node (cNode::ReadSolverOrder, node/node.cpp:248-284)."""
    if "NODE.SOLVER.ORDER" not in blk:
        return None
    t = blk["NODE.SOLVER.ORDER"]
    if int(t[0]) != nnode:
        raise ValueError("NODE.SOLVER.ORDER must list every node")
    return np.array([int(v) for v in t[1:1 + nnode]], dtype=np.int64)
