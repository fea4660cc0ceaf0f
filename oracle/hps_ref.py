"""Oracle: CPU restatement of robinsolver's HPS factor/solve path (2D, FD leaves).

TEST INFRASTRUCTURE ONLY.  This module is the checker.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline`` leg and its
``--impl reference`` arm) may import it.  The product library never calls it, and
the product has no CPU fallback.

What it restates
----------------
The reference is a serial Fortran 2008 code whose arithmetic all goes through
LAPACK/BLAS ``z*`` routines.  This module follows the reference's operation
sequence call for call, with scipy's LAPACK (OpenBLAS) standing in for the
unpinned BLAS/LAPACK the reference links:

* tree build        -- ``bin_tree``/``node_divide``   robin_tree_module.f90:288-337, 1369-1412
* leaf grid         -- ``get_h``                       fd_module.f90:1060-1084
* index maps        -- ``lin2fgrid``/``fgrid2lin``/``igrid2lin``/``lin2igrid``/``grid2real``
                                                       fd_module.f90:669-975
* leaf matrix       -- ``FD_matrix``/``FD_matrix_row``/``grid_classify``
                                                       fd_module.f90:49-224, 989-1022
* leaf RtR          -- ``FD_solve`` (zgetrf, zgetrs)   fd_module.f90:234-278
                       ``RTR_update``/``RTR_solve``    robin_tree_module.f90:667-799
* merge             -- ``compute_RTR`` merge branch    robin_tree_module.f90:397-647
                       (zgetrf, zgetri with lwork=max(64,m), zgetrs, zgemm)
* solve             -- ``forward_sub``/``backward_sub``/``apply_bc``/``apply_invm``
                                                       robin_tree_module.f90:813-1322
                       ``fd_leaf_solve``/``fd_outgoing_bc``/``fd_leaf_update``/``fd_make_bndry_vec``
                                                       fd_module.f90:390-659
* output            -- ``get_solution``/``get_node_sol`` robin_output_module.f90:48-75, 305-322

Semantics restated, not defects: every solve applies fresh boundary data and
starts from a fresh leaf solution (the reference applies boundary data only on
the first solve of a process, robin_tree_module.f90:1014-1029, and refuses a
second ``leaf_solve``, local_solver_module.f90:229-231).  ``alpha = 0`` blends
overwrite (the reference multiplies uninitialised memory by zero,
robin_tree_module.f90:868-873).

Parity unpinned: the reference ships no tests, fixtures or golden vectors and
cannot be compiled in this container (no Fortran compiler).  The restatement is
cross-checked against an independent global sparse solve of the same FD system
(``fd_global.py``) and against the O(h^2) manufactured solution of
example.f90:107-116, 178-186; neither pins it to the reference's own output.

Callbacks are vectorised: ``fun(X)`` takes an ``(npts, 3)`` float64 array of
points and returns ``npts`` complex values (the reference calls a scalar
``pure function`` once per point with the same coordinates).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import blas, lapack

# ----------------------------------------------------------------------------------------------
# options / operator / rhs containers (derived_type_module.f90:72-115, 285-320)
# ----------------------------------------------------------------------------------------------


@dataclass
class SolveOpts:
    """``solve_opts`` (derived_type_module.f90:309-320)."""
    h_tgt: float = 0.0
    h: np.ndarray = field(default_factory=lambda: np.zeros(3))
    ordering: int = 1
    disc: str = "fd"
    kb: float = 1.0


@dataclass
class EllipticOperator:
    """``elliptic_operator`` (derived_type_module.f90:72-84).  ``coeff`` and
    ``robin_coeff`` are never read on the reference path, so they are absent."""
    d: int
    domain: np.ndarray          # (2, 3): [lo; hi]
    k: object                   # vectorised potential callback


@dataclass
class EllipticRHS:
    """``elliptic_rhs`` (derived_type_module.f90:109-115)."""
    d: int
    f: object                   # vectorised interior source callback
    g: list                     # 2*d vectorised face callbacks, faces x1 x2 y1 y2


# ----------------------------------------------------------------------------------------------
# geometry
# ----------------------------------------------------------------------------------------------


def get_h(h_tgt, box, d=2):
    """fd_module.f90:1060-1084: grid = max(ceiling(w/h_tgt), 3), h = w/grid."""
    h = np.zeros(3)
    grid = [-1, -1, -1]
    for j in range(d):
        w = box[1, j] - box[0, j]
        grid[j] = max(int(math.ceil(w / h_tgt)), 3)
        h[j] = w / grid[j]
    return h, grid


def get_pt_face(ptbox, d=2):
    """fd_module.f90:1033-1049 (2D): faces x1 x2 y1 y2 hold [b, b, a, a] points."""
    a, b = ptbox[0], ptbox[1]
    return [b, b, a, a]


@dataclass
class Node:
    lvl: int
    idx: int                    # index within its level, left to right (child1 first)
    node_id: int = 0            # the reference's pre-order sibling-pair id
    box: np.ndarray = None
    ptbox: list = None
    iface: int = 0              # 1-based face id of the interface with the sibling
    isbndry: list = field(default_factory=lambda: [False] * 6)
    isleaf: bool = False
    child1: "Node" = None
    child2: "Node" = None
    # factor data
    h: np.ndarray = None        # leaf grid spacing
    lu: np.ndarray = None       # leaf LU (LocalOp)
    piv: np.ndarray = None
    rtr: np.ndarray = None      # full nb x nb RtR in face order
    D: tuple = None             # (lu, piv) of zeta*I - T2_ii
    S: tuple = None             # (lu, piv) of zeta*I - T1_ii - nu^2 inv(D)
    nu: complex = 0.0
    # solve data (per call)
    g: dict = None
    hvec: dict = None
    sol: np.ndarray = None


def node_divide(d, node):
    """robin_tree_module.f90:1369-1412: cut the longest side (first on ties)."""
    widths = np.zeros(3)
    widths[:d] = node.box[1, :d] - node.box[0, :d]
    edge = int(np.argmax(widths))       # maxloc: first maximum
    c1, c2 = node.child1, node.child2
    c1.box = node.box.copy()
    c2.box = node.box.copy()
    c1.box[1, edge] = node.box[0, edge] + widths[edge] * 0.5
    c2.box[0, edge] = c1.box[1, edge]
    c1.iface = 2 * (edge + 1)
    c2.iface = 2 * (edge + 1) - 1
    for j in range(2 * d):
        if node.isbndry[j]:
            if j + 1 != c1.iface:
                c1.isbndry[j] = True
            if j + 1 != c2.iface:
                c2.isbndry[j] = True


def build_tree(L, domain, d=2):
    """robin_tree_factor tree setup + bin_tree (robin_tree_module.f90:146-159, 288-337).
    Returns (root, levels) with levels[l] the nodes of level l, left to right."""
    root = Node(lvl=0, idx=0, node_id=0)
    root.box = np.array(domain, dtype=np.float64).copy()
    root.isleaf = (L == 0)
    root.isbndry = [True] * (2 * d) + [False] * (6 - 2 * d)
    levels = [[root]]
    counter = [0]

    def rec(node):
        if node.isleaf:
            return
        node.child1 = Node(lvl=node.lvl + 1, idx=2 * node.idx)
        node.child2 = Node(lvl=node.lvl + 1, idx=2 * node.idx + 1)
        node_divide(d, node)
        for c in (node.child1, node.child2):
            counter[0] += 1
            c.node_id = counter[0]
            c.isleaf = (c.lvl == L)
        rec(node.child1)
        rec(node.child2)

    rec(root)
    # level lists in left-to-right order (child1 first)
    for lv in range(1, L + 1):
        nxt = []
        for p in levels[lv - 1]:
            nxt.extend([p.child1, p.child2])
        levels.append(nxt)
    return root, levels


# ----------------------------------------------------------------------------------------------
# index maps on one cornerless leaf grid (2D)
# ----------------------------------------------------------------------------------------------


def lin2fgrid_all(a, b):
    """fd_module.f90:867-939 for every linear index (0-based here): returns grid indices
    (gi, gj).  Faces x1 (0,j) x2 (a+1,j) y1 (i,0) y2 (i,b+1), then the interior with
    x fastest (igrid2lin ordering 1, fd_module.f90:835-841)."""
    nb = 2 * (a + b)
    n = nb + a * b
    gi = np.zeros(n, dtype=np.int64)
    gj = np.zeros(n, dtype=np.int64)
    jj = np.arange(1, b + 1)
    ii = np.arange(1, a + 1)
    gi[0:b], gj[0:b] = 0, jj
    gi[b:2 * b], gj[b:2 * b] = a + 1, jj
    gi[2 * b:2 * b + a], gj[2 * b:2 * b + a] = ii, 0
    gi[2 * b + a:nb], gj[2 * b + a:nb] = ii, b + 1
    I, J = np.meshgrid(ii, jj, indexing="xy")      # J rows, I fastest
    gi[nb:] = I.ravel()
    gj[nb:] = J.ravel()
    return gi, gj


def fgrid2lin(i, j, a, b):
    """fd_module.f90:717-800 (2D, 0-based result)."""
    nb = 2 * (a + b)
    if i == 0:
        return j - 1
    if i == a + 1:
        return b + j - 1
    if j == 0:
        return 2 * b + i - 1
    if j == b + 1:
        return 2 * b + a + i - 1
    return nb + (j - 1) * a + (i - 1)


def grid2real(gi, gj, a, b, h, box):
    """fd_module.f90:669-700: cell centres lo + g*h - h/2, snapped to the face on the
    boundary.  Returns (npts, 3)."""
    gi = np.asarray(gi)
    gj = np.asarray(gj)
    x = (box[0, 0] + gi * h[0]) - h[0] / 2
    y = (box[0, 1] + gj * h[1]) - h[1] / 2
    z = np.full(gi.shape, (box[0, 2] + 1 * h[2]) - h[2] / 2)
    x = np.where(gi == 0, box[0, 0], np.where(gi == a + 1, box[1, 0], x))
    y = np.where(gj == 0, box[0, 1], np.where(gj == b + 1, box[1, 1], y))
    return np.stack([x, y, z], axis=-1)


def interior_points(a, b, h, box):
    """Interior cell centres in igrid2lin order (the points where the reference calls
    ``ell_op%k`` in FD_matrix_row, fd_module.f90:136,145, and ``f`` in fd_leaf_solve,
    fd_module.f90:427-431)."""
    gi, gj = lin2fgrid_all(a, b)
    nb = 2 * (a + b)
    return grid2real(gi[nb:], gj[nb:], a, b, h, box)


def face_points(a, b, h, box, face):
    """Face-local coordinates handed to ``g_face`` by fd_make_bndry_vec
    (fd_module.f90:636-651).  In 2D x-faces receive (y, 0, 0) and y-faces (x, 0, 0):
    that is what the reference's slice assignment at :648-649 leaves in
    ``face_real_pt``."""
    pf = get_pt_face((a, b))
    off = int(sum(pf[:face - 1]))
    gi, gj = lin2fgrid_all(a, b)
    P = grid2real(gi[off:off + pf[face - 1]], gj[off:off + pf[face - 1]], a, b, h, box)
    out = np.zeros_like(P)
    if face in (1, 2):
        out[:, 0] = P[:, 1]
    else:
        out[:, 0] = P[:, 0]
    return out


def boundary_stencil(a, b):
    """For each boundary row r: (p1, p2) = the first and second interior points along the
    inward normal, and the normal axis (0 = x, 1 = y).  fd_module.f90:187-216 and the
    outgoing stencil of RTR_update (robin_tree_module.f90:686-713)."""
    nb = 2 * (a + b)
    gi, gj = lin2fgrid_all(a, b)
    p1 = np.zeros(nb, dtype=np.int64)
    p2 = np.zeros(nb, dtype=np.int64)
    ax = np.zeros(nb, dtype=np.int64)
    for r in range(nb):
        i, j = gi[r], gj[r]
        if i == 0:
            s, axis = (1, 0), 0
        elif i == a + 1:
            s, axis = (-1, 0), 0
        elif j == 0:
            s, axis = (0, 1), 1
        else:
            s, axis = (0, -1), 1
        p1[r] = fgrid2lin(i + s[0], j + s[1], a, b)
        p2[r] = fgrid2lin(i + 2 * s[0], j + 2 * s[1], a, b)
        ax[r] = axis
    return p1, p2, ax


def fd_matrix(a, b, h, kvals, kb):
    """Dense leaf matrix, FD_matrix/FD_matrix_row (fd_module.f90:49-224).

    Rows and columns in lin2fgrid order.  Interior rows: k(x) on the diagonal (the
    potential as returned, not squared, :145) plus the [1,-2,1]/h^2 stencil, or
    [8/3,-4,4/3]/h^2 next to a face (:150-156), accumulated in the reference's order.
    Boundary rows: i*kb*u + (8/3 u0 - 3 u1 + 1/3 u2)/h (:187-216)."""
    nb = 2 * (a + b)
    n = nb + a * b
    A = np.zeros((n, n), dtype=np.complex128)
    alpha = complex(0.0 * kb, 1.0 * kb)
    p1, p2, ax = boundary_stencil(a, b)
    for r in range(nb):
        hn = h[ax[r]]
        A[r, r] = (A[r, r] + alpha) + (8.0 / 3.0) / hn
        A[r, p1[r]] = A[r, p1[r]] - 3.0 / hn
        A[r, p2[r]] = A[r, p2[r]] + (1.0 / 3.0) / hn
    gi, gj = lin2fgrid_all(a, b)
    shape = (a, b)
    for e in range(nb, n):
        g = (gi[e], gj[e])
        A[e, e] = A[e, e] + kvals[e - nb]
        for dim in range(2):
            if g[dim] == 1:
                w = (8.0 / 3.0, -4.0, 4.0 / 3.0)
            elif g[dim] == shape[dim]:
                w = (4.0 / 3.0, -4.0, 8.0 / 3.0)
            else:
                w = (1.0, -2.0, 1.0)
            h2 = h[dim] ** 2
            A[e, e] = A[e, e] + w[1] / h2
            up = list(g)
            up[dim] += 1
            dn = list(g)
            dn[dim] -= 1
            eu = fgrid2lin(up[0], up[1], a, b)
            ed = fgrid2lin(dn[0], dn[1], a, b)
            A[e, eu] = A[e, eu] + w[2] / h2
            A[e, ed] = A[e, ed] + w[0] / h2
    return A


def outgoing_rows(X, a, b, h, kb):
    """RTR_update (robin_tree_module.f90:667-718) / fd_outgoing_bc (fd_module.f90:449-513):
    rows r < nb of X become sigma*X(r) + tau*(8/3 X(r) - 3 X(p1) + 1/3 X(p2))/h with
    sigma = -i*kb, tau = 1 (:683-684).  Returns the updated boundary rows."""
    nb = 2 * (a + b)
    p1, p2, ax = boundary_stencil(a, b)
    sigma = complex(0.0 * kb, -1.0 * kb)
    tau = 1.0
    out = np.empty((nb,) + X.shape[1:], dtype=np.complex128)
    for r in range(nb):
        hn = h[ax[r]]
        v = sigma * X[r] + ((tau * (8.0 / 3.0)) / hn) * X[r]
        v = v + ((tau * (-3.0)) / hn) * X[p1[r]]
        v = v + ((tau * (1.0 / 3.0)) / hn) * X[p2[r]]
        out[r] = v
    return out


# ----------------------------------------------------------------------------------------------
# LAPACK wrappers with the reference's matrixdata semantics (factorization_module.f90)
# ----------------------------------------------------------------------------------------------

# When a list, every LAPACK/BLAS call adds its wall time to PROFILE[0] and 1 to PROFILE[1]:
# the CPU cost of the reference is its LAPACK/BLAS call sequence (the Python index loops of
# this restatement are compiled loops in the reference and are not counted).
PROFILE = None


def _timed(fn, *a, **kw):
    if PROFILE is None:
        return fn(*a, **kw)
    t0 = time.perf_counter()
    out = fn(*a, **kw)
    PROFILE[0] += time.perf_counter() - t0
    PROFILE[1] += 1
    return out


def _getrf(A):
    lu, piv, info = _timed(lapack.zgetrf, A)
    if info < 0:
        raise RuntimeError(f"zgetrf illegal argument {info}")
    return lu, piv


def _getrs(F, B):
    lu, piv = F
    X, info = _timed(lapack.zgetrs, lu, piv, B)
    if info != 0:
        raise RuntimeError(f"zgetrs info {info}")
    return X


def _getri(F):
    """mtrx_getinv with lwork = max(64, m) (factorization_module.f90:124-129)."""
    lu, piv = F
    m = lu.shape[0]
    inv, info = _timed(lapack.zgetri, lu, piv, lwork=max(64, m))
    return inv


def _gemm(alpha, A, B):
    return _timed(blas.zgemm, alpha, A, B)


# ----------------------------------------------------------------------------------------------
# the tree
# ----------------------------------------------------------------------------------------------


def face_offsets(pf):
    return [0, pf[0], pf[0] + pf[1], pf[0] + pf[1] + pf[2]]


class RobinTree:
    """``robin_tree`` (robin_tree_module.f90:55-77), 2D only.  ``bndry_params`` must be
    set by the caller before ``factor`` (robin_tree_module.f90:61, 135-140)."""

    def __init__(self):
        self.bndry_params = None
        self.factored = False
        self.nlvls = 0
        self.ell_op = None
        self.opts = None
        self.root = None
        self.levels = None

    # --- factor ---------------------------------------------------------------------------
    def factor(self, L, ell_op: EllipticOperator, opts: SolveOpts, keep_leaf=True):
        """robin_tree_factor (robin_tree_module.f90:96-185)."""
        dom = np.asarray(ell_op.domain, dtype=np.float64)
        if np.min(dom[1] - dom[0]) < 0:
            raise ValueError("Error in ROBIN_TREE_FACTOR: Invalid operator domain format.")
        if ell_op.d not in (2, 3):
            raise ValueError("Error in ROBIN_TREE_FACTOR: Dimension must be 2 or 3.")
        if ell_op.d != 2:
            raise NotImplementedError("oracle restates the 2D path only")
        bp = np.asarray(self.bndry_params, dtype=np.complex128)
        if abs(bp[0, 0] * bp[1, 1] - bp[0, 1] * bp[1, 0]) < 10.0 ** (-3.0):
            raise ValueError("Error: Boundary parameter matrix is nearly singular.")
        self.nlvls = L
        self.ell_op = ell_op
        self.opts = SolveOpts(h_tgt=opts.h_tgt, h=np.array(opts.h, dtype=np.float64),
                              ordering=opts.ordering, disc=opts.disc, kb=opts.kb)
        self.root, self.levels = build_tree(L, dom, ell_op.d)
        self.keep_leaf = keep_leaf
        self._compute_rtr(self.root)
        self.factored = True

    def _leaf(self, node):
        """get_h + RTR_solve (robin_tree_module.f90:392-394, 728-799)."""
        h, grid = get_h(self.opts.h_tgt, node.box, 2)
        self.opts.h = h                                   # get_h overwrites T%opts%h
        a, b = grid[0], grid[1]
        node.ptbox = [a, b, -1]
        node.h = h
        pts = interior_points(a, b, h, node.box)
        kvals = np.asarray(self.ell_op.k(pts), dtype=np.complex128)
        A = fd_matrix(a, b, h, kvals, self.opts.kb)
        lu, piv = _getrf(A)
        nb = 2 * (a + b)
        X = np.zeros((A.shape[0], nb), dtype=np.complex128, order="F")
        X[np.arange(nb), np.arange(nb)] = 1.0
        X = _getrs((lu, piv), X)
        node.rtr = np.asfortranarray(outgoing_rows(X, a, b, h, self.opts.kb))
        if self.keep_leaf:
            node.lu, node.piv = lu, piv

    def _compute_rtr(self, node):
        if node.isleaf:
            self._leaf(node)
            return
        self._compute_rtr(node.child1)
        self._compute_rtr(node.child2)
        self._merge(node)

    def _merge(self, node):
        """compute_RTR merge branch (robin_tree_module.f90:397-647)."""
        c1, c2 = node.child1, node.child2
        d = 2
        diffbox = np.abs((node.box[1] - node.box[0]) - (c1.box[1] - c1.box[0]))
        node.ptbox = list(c1.ptbox)
        ax = int(np.argmax(diffbox[:d]))
        node.ptbox[ax] = 2 * node.ptbox[ax]
        pf = get_pt_face(node.ptbox)
        pf1 = get_pt_face(c1.ptbox)
        pf2 = get_pt_face(c2.ptbox)
        o1, o2, op = face_offsets(pf1), face_offsets(pf2), face_offsets(pf)
        i1, i2 = c1.iface, c2.iface

        def blk(rtr, off, pfc, r, c):
            return rtr[off[r - 1]:off[r - 1] + pfc[r - 1], off[c - 1]:off[c - 1] + pfc[c - 1]]

        m = pf1[i1 - 1]
        if m != pf2[i2 - 1]:
            raise ValueError("Error: Interface sizes of node children do not match")
        bp = np.asarray(self.bndry_params, dtype=np.complex128)
        nu = (-bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
        zeta = (bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
        node.nu = nu
        eye = np.arange(m)
        T2ii = -np.array(blk(c2.rtr, o2, pf2, i2, i2), order="F")
        T2ii[eye, eye] += zeta
        node.D = _getrf(T2ii)
        Dinv = _getri(node.D)
        T1ii = -np.array(blk(c1.rtr, o1, pf1, i1, i1), order="F") - (nu * nu) * Dinv
        T1ii[eye, eye] += zeta
        node.S = _getrf(T1ii)

        P = np.zeros((sum(pf), sum(pf)), dtype=np.complex128, order="F")
        for col in range(1, 2 * d + 1):
            C11 = C21 = C12 = C22 = None
            if col != i1:
                C11 = _getrs(node.S, np.asfortranarray(blk(c1.rtr, o1, pf1, i1, col)))
                C21 = nu * _getrs(node.D, C11)
            if col != i2:
                C22 = _getrs(node.D, np.asfortranarray(blk(c2.rtr, o2, pf2, i2, col)))
                C12 = nu * _getrs(node.S, C22)
                C22 = C22 + nu * _getrs(node.D, C12)
            for row in range(1, 2 * d + 1):
                R = np.zeros((pf[row - 1], pf[col - 1]), dtype=np.complex128, order="F")
                prs, pcs = pf[row - 1], pf[col - 1]
                if C11 is not None and row != i1:
                    rs, cs = pf1[row - 1], C11.shape[1]
                    R[0:rs, 0:cs] = _gemm(1.0, np.asfortranarray(blk(c1.rtr, o1, pf1, row, i1)), C11) \
                        + blk(c1.rtr, o1, pf1, row, col)
                if C12 is not None and row != i1:
                    rs, cs = pf1[row - 1], C12.shape[1]
                    R[0:rs, pcs - cs:pcs] = _gemm(-1.0, np.asfortranarray(blk(c1.rtr, o1, pf1, row, i1)), C12)
                if C21 is not None and row != i2:
                    rs, cs = pf2[row - 1], C21.shape[1]
                    R[prs - rs:prs, 0:cs] = _gemm(-1.0, np.asfortranarray(blk(c2.rtr, o2, pf2, row, i2)), C21)
                if C22 is not None and row != i2:
                    rs, cs = pf2[row - 1], C22.shape[1]
                    R[prs - rs:prs, pcs - cs:pcs] = _gemm(1.0, np.asfortranarray(blk(c2.rtr, o2, pf2, row, i2)), C22) \
                        + blk(c2.rtr, o2, pf2, row, col)
                P[op[row - 1]:op[row - 1] + prs, op[col - 1]:op[col - 1] + pcs] = R
        node.rtr = P

    # --- solve ----------------------------------------------------------------------------
    def solve(self, rhs_list):
        """robin_tree_solve (robin_tree_module.f90:198-233) for a batch of right-hand
        sides; column r of every vector belongs to rhs_list[r]."""
        if not self.factored:
            raise RuntimeError("Error: Robin Tree must be factored first.")
        if isinstance(rhs_list, EllipticRHS):
            rhs_list = [rhs_list]
        for r in rhs_list:
            if r.d != self.ell_op.d:
                raise ValueError("Error: Dimensions of Robin Tree and RHS do not match.")
        self._forward(self.root, rhs_list)
        self._apply_bc(self.root, rhs_list)
        self._backward(self.root)

    def _pf(self, node):
        return get_pt_face(node.ptbox)

    def _forward(self, node, rhs_list):
        """forward_sub (robin_tree_module.f90:813-990)."""
        kb = self.opts.kb
        nr = len(rhs_list)
        pf = self._pf(node)
        node.g = {f: np.zeros((pf[f - 1], nr), dtype=np.complex128) for f in range(1, 5)}
        if node.isleaf:
            a, b = node.ptbox[0], node.ptbox[1]
            nb = 2 * (a + b)
            h = self.opts.h                 # T%opts%h: the last leaf's h (fd_module.f90:429)
            pts = interior_points(a, b, h, node.box)
            B = np.zeros((nb + a * b, nr), dtype=np.complex128, order="F")
            for r, rhs in enumerate(rhs_list):
                B[nb:, r] = rhs.f(pts)
            node.sol = _getrs((node.lu, node.piv), B)
            hv = outgoing_rows(node.sol, a, b, h, kb)
            o = face_offsets(pf)
            node.hvec = {f: hv[o[f - 1]:o[f - 1] + pf[f - 1]] for f in range(1, 5)}
            return
        c1, c2 = node.child1, node.child2
        self._forward(c1, rhs_list)
        self._forward(c2, rhs_list)
        y1, y2 = apply_invm(None, None, c1.hvec[c1.iface], c2.hvec[c2.iface], 0.0, node.D, node.S, node.nu)
        c1.g[c1.iface] = y1
        c2.g[c2.iface] = y2
        if node.lvl > 0:
            axis = (c1.iface - 1) // 2
            node.hvec = {}
            for j in range(1, 5):
                if (j - 1) // 2 == axis:
                    if j == c1.iface:
                        node.hvec[j] = c2.hvec[j] + _gemm(1.0, _blk(c2, j, c2.iface), y2)
                    else:
                        node.hvec[j] = c1.hvec[j] + _gemm(1.0, _blk(c1, j, c1.iface), y1)
                else:
                    node.hvec[j] = np.concatenate(
                        [c1.hvec[j] + _gemm(1.0, _blk(c1, j, c1.iface), y1),
                         c2.hvec[j] + _gemm(1.0, _blk(c2, j, c2.iface), y2)], axis=0)
        c1.hvec = None
        c2.hvec = None

    def _apply_bc(self, node, rhs_list):
        """apply_bc (robin_tree_module.f90:1186-1237) with fd_make_bndry_vec
        (fd_module.f90:611-659) at the leaves; evaluated fresh on every solve."""
        if node.isleaf:
            a, b = node.ptbox[0], node.ptbox[1]
            for f in range(1, 5):
                if node.isbndry[f - 1]:
                    pts = face_points(a, b, self.opts.h, node.box, f)
                    node.g[f] = np.stack([np.asarray(r.g[f - 1](pts), dtype=np.complex128)
                                          for r in rhs_list], axis=1)
            return
        if not any(node.isbndry):
            return
        c1, c2 = node.child1, node.child2
        self._apply_bc(c1, rhs_list)
        self._apply_bc(c2, rhs_list)
        for f in range(1, 5):
            if node.isbndry[f - 1]:
                if f == c2.iface:
                    node.g[f] = c1.g[f].copy()
                elif f == c1.iface:
                    node.g[f] = c2.g[f].copy()
                else:
                    node.g[f] = np.concatenate([c1.g[f], c2.g[f]], axis=0)

    def _backward(self, node):
        """backward_sub (robin_tree_module.f90:1002-1146)."""
        if node.isleaf:
            a, b = node.ptbox[0], node.ptbox[1]
            nb = 2 * (a + b)
            nr = node.sol.shape[1]
            B = np.zeros((nb + a * b, nr), dtype=np.complex128, order="F")
            o = face_offsets(self._pf(node))
            for f in range(1, 5):
                B[o[f - 1]:o[f - 1] + node.g[f].shape[0]] = node.g[f]
            node.sol = node.sol + _getrs((node.lu, node.piv), B)
            return
        c1, c2 = node.child1, node.child2
        axis = (c1.iface - 1) // 2
        pf = self._pf(node)
        for f in range(1, 5):
            if not node.isbndry[f - 1]:
                if (f - 1) // 2 != axis:
                    half = pf[f - 1] // 2
                    c1.g[f] = node.g[f][:half].copy()
                    c2.g[f] = node.g[f][half:].copy()
                else:
                    if f == c1.iface:
                        c2.g[f] = node.g[f].copy()
                    elif f == c2.iface:
                        c1.g[f] = node.g[f].copy()
        nr = node.g[1].shape[1]
        m = c1.g[c1.iface].shape[0]
        Tg1 = np.zeros((m, nr), dtype=np.complex128)
        Tg2 = np.zeros((m, nr), dtype=np.complex128)
        for f in range(1, 5):
            if f != c1.iface:
                Tg1 = Tg1 + _gemm(1.0, _blk(c1, c1.iface, f), c1.g[f])
            if f != c2.iface:
                Tg2 = Tg2 + _gemm(1.0, _blk(c2, c2.iface, f), c2.g[f])
        y1, y2 = apply_invm(c1.g[c1.iface], c2.g[c2.iface], Tg1, Tg2, 1.0, node.D, node.S, node.nu)
        c1.g[c1.iface] = y1
        c2.g[c2.iface] = y2
        node.g = None
        self._backward(c1)
        self._backward(c2)

    # --- output ---------------------------------------------------------------------------
    def leaves(self):
        return self.levels[-1]

    def get_solution(self):
        """get_solution/get_node_sol (robin_output_module.f90:48-75, 305-322): leaves in DFS
        order (child1 first) with their box and solution (n x nrhs)."""
        if not self.factored:
            raise RuntimeError("Error in GET_SOLUTION: Robin Tree not factored.")
        return [(lf.box.copy(), lf.sol.copy()) for lf in self.leaves()]


def _blk(node, r, c):
    pf = get_pt_face(node.ptbox)
    o = face_offsets(pf)
    return np.asfortranarray(node.rtr[o[r - 1]:o[r - 1] + pf[r - 1], o[c - 1]:o[c - 1] + pf[c - 1]])


def apply_invm(y1, y2, x1, x2, alpha, D, S, nu):
    """apply_invm (robin_tree_module.f90:1252-1322): y = alpha*y + inv(M) x in the
    reference's five-solve order.  ``alpha == 0`` overwrites."""
    x1 = np.asfortranarray(x1)
    x2 = np.asfortranarray(x2)
    if alpha == 0 or y1 is None:
        y1 = np.zeros_like(x1)
        y2 = np.zeros_like(x2)
    interm = _getrs(S, x1)                          # step 1
    y1 = alpha * y1 + interm                        # step 2
    y2 = alpha * y2 + (-nu) * _getrs(D, interm)     # step 3
    interm = _getrs(D, x2)                          # step 4
    y2 = y2 + interm                                # step 5
    interm = _getrs(S, interm)                      # step 6
    y1 = y1 - nu * interm                           # step 7
    y2 = y2 + (nu * nu) * _getrs(D, interm)         # step 8
    return y1, y2


# ----------------------------------------------------------------------------------------------
# helpers shared by tests and bench: solution layout
# ----------------------------------------------------------------------------------------------


def leaf_all_points(a, b, h, box):
    """Every point of a leaf's u vector (lin2fgrid order), as check_solution's proc2vec
    samples them (robin_output_module.f90:234-273)."""
    gi, gj = lin2fgrid_all(a, b)
    return grid2real(gi, gj, a, b, h, box)
