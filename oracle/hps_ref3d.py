"""Oracle: CPU restatement of robinsolver's HPS factor/solve path in 3D (d = 3, FD leaves).

TEST INFRASTRUCTURE ONLY (same import rule as ``hps_ref.py``: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` may import it; the product never does).

The 3D path of the reference is the 2D path with six faces.  What changes, and where it is
restated here:

* face sizes        -- ``get_pt_face`` with d = 3: faces x1 x2 y1 y2 z1 z2 hold
                       [bc, bc, ac, ac, ab, ab] points          fd_module.f90:1033-1049
* leaf ordering     -- ``lin2fgrid``: the six faces in turn, each in its own 2D lexicographic
                       order (first tangential coordinate fastest, ``lin2igrid`` with d-1),
                       then the interior x fastest, then y, then z (no edges, no corners)
                                                                  fd_module.f90:867-939, 835-841
* leaf matrix       -- ``FD_matrix_row``: k on the diagonal, the 1D stencil in x, y, z
                       ([8/3, -4, 4/3] next to a face), Robin rows i kb u + (8/3 u0 - 3 u1
                       + 1/3 u2)/h along the normal                  fd_module.f90:104-224
* leaf RtR          -- ``RTR_update`` with the shift -1 + 2 mod(face, 2) along the normal
                                                                  robin_tree_module.f90:667-718
* face coordinates  -- ``fd_make_bndry_vec``: the two tangential coordinates in natural order
                       (x faces (y, z), y faces (x, z), z faces (x, y))   fd_module.f90:636-651
* tree, merge, sweeps, apply_invm -- exactly the 2D restatement with 2d = 6 faces: a merged
                       node's face is child1's part then child2's    robin_tree_module.f90:288-1412

The LAPACK/BLAS call sequence (zgetrf, zgetrs, zgetri, zgemm) is the one ``hps_ref`` restates.
Parity unpinned for the same reason as ``hps_ref``; this module is cross-checked against an
assembled global sparse system of the same rows (``global_solve``) and against the O(h^2)
manufactured solution cos(x/sqrt3) cos(y/sqrt3) cos(z/sqrt3) of example.f90:188-196.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import hps_ref as H

D = 3


def get_pt_face(ptbox):
    """fd_module.f90:1033-1049 with d = 3: product of the other two sides."""
    a, b, c = ptbox[0], ptbox[1], ptbox[2]
    return [b * c, b * c, a * c, a * c, a * b, a * b]


def lin2fgrid_all(a, b, c):
    """Grid indices (gi, gj, gk) of every linear index (0-based) of a cornerless, edgeless 3D leaf
    grid: fd_module.f90:867-939 (faces) and igrid2lin ordering 1 (interior, x fastest)."""
    gi, gj, gk = [], [], []

    def face(fix_axis, fix_val, s1, s2):
        # the face's own 2D lexicographic order: first tangential index fastest
        for q in range(1, s2 + 1):
            for p in range(1, s1 + 1):
                g = [0, 0, 0]
                tang = [ax for ax in range(3) if ax != fix_axis]
                g[fix_axis] = fix_val
                g[tang[0]] = p
                g[tang[1]] = q
                gi.append(g[0]); gj.append(g[1]); gk.append(g[2])

    face(0, 0, b, c)
    face(0, a + 1, b, c)
    face(1, 0, a, c)
    face(1, b + 1, a, c)
    face(2, 0, a, b)
    face(2, c + 1, a, b)
    for k in range(1, c + 1):
        for j in range(1, b + 1):
            for i in range(1, a + 1):
                gi.append(i); gj.append(j); gk.append(k)
    return np.array(gi), np.array(gj), np.array(gk)


class LeafIndex:
    """fgrid2lin (fd_module.f90:717-800) for one leaf shape, as a lookup table."""

    def __init__(self, a, b, c):
        self.a, self.b, self.c = a, b, c
        self.gi, self.gj, self.gk = lin2fgrid_all(a, b, c)
        self.n = len(self.gi)
        self.nb = 2 * (b * c + a * c + a * b)
        self.table = -np.ones((a + 2, b + 2, c + 2), dtype=np.int64)
        self.table[self.gi, self.gj, self.gk] = np.arange(self.n)

    def lin(self, i, j, k):
        v = self.table[i, j, k]
        if v < 0:
            raise ValueError("FGRID2LIN: Corner point requested.")
        return int(v)


def grid2real(gi, gj, gk, shape, h, box):
    """fd_module.f90:669-700 in 3D: lo + g h - h/2, snapped to the face on the boundary."""
    g = [np.asarray(gi), np.asarray(gj), np.asarray(gk)]
    out = []
    for ax in range(3):
        v = (box[0, ax] + g[ax] * h[ax]) - h[ax] / 2
        v = np.where(g[ax] == 0, box[0, ax], np.where(g[ax] == shape[ax] + 1, box[1, ax], v))
        out.append(v)
    return np.stack(out, axis=-1)


def interior_points(idx: LeafIndex, h, box):
    nb = idx.nb
    return grid2real(idx.gi[nb:], idx.gj[nb:], idx.gk[nb:], (idx.a, idx.b, idx.c), h, box)


def face_points(idx: LeafIndex, h, box, face):
    """fd_make_bndry_vec (fd_module.f90:636-651): the face's points in its own order, as the
    face-local coordinates handed to g_face (the two tangential coordinates, then 0)."""
    pf = get_pt_face((idx.a, idx.b, idx.c))
    off = int(sum(pf[:face - 1]))
    sl = slice(off, off + pf[face - 1])
    P = grid2real(idx.gi[sl], idx.gj[sl], idx.gk[sl], (idx.a, idx.b, idx.c), h, box)
    ax = (face - 1) // 2
    tang = [t for t in range(3) if t != ax]
    out = np.zeros_like(P)
    out[:, 0] = P[:, tang[0]]
    out[:, 1] = P[:, tang[1]]
    return out


def boundary_stencil(idx: LeafIndex):
    """For each boundary row r: the first and second points along the inward normal, and the
    normal axis (RTR_update's shift, robin_tree_module.f90:694-697)."""
    nb = idx.nb
    p1 = np.zeros(nb, dtype=np.int64)
    p2 = np.zeros(nb, dtype=np.int64)
    ax = np.zeros(nb, dtype=np.int64)
    shape = (idx.a, idx.b, idx.c)
    for r in range(nb):
        g = [idx.gi[r], idx.gj[r], idx.gk[r]]
        for d in range(3):
            if g[d] == 0 or g[d] == shape[d] + 1:
                s = 1 if g[d] == 0 else -1
                g1 = list(g); g1[d] += s
                g2 = list(g); g2[d] += 2 * s
                p1[r] = idx.lin(*g1)
                p2[r] = idx.lin(*g2)
                ax[r] = d
    return p1, p2, ax


def fd_matrix(idx: LeafIndex, h, kvals, kb):
    """FD_matrix/FD_matrix_row (fd_module.f90:49-224) in 3D, rows and columns in lin2fgrid order,
    entries accumulated in the reference's order."""
    nb, n = idx.nb, idx.n
    A = np.zeros((n, n), dtype=np.complex128)
    alpha = complex(0.0 * kb, 1.0 * kb)
    p1, p2, ax = boundary_stencil(idx)
    for r in range(nb):
        hn = h[ax[r]]
        A[r, r] = (A[r, r] + alpha) + (8.0 / 3.0) / hn
        A[r, p1[r]] = A[r, p1[r]] - 3.0 / hn
        A[r, p2[r]] = A[r, p2[r]] + (1.0 / 3.0) / hn
    shape = (idx.a, idx.b, idx.c)
    for e in range(nb, n):
        g = [idx.gi[e], idx.gj[e], idx.gk[e]]
        A[e, e] = A[e, e] + kvals[e - nb]
        for d in range(3):
            if g[d] == 1:
                w = (8.0 / 3.0, -4.0, 4.0 / 3.0)
            elif g[d] == shape[d]:
                w = (4.0 / 3.0, -4.0, 8.0 / 3.0)
            else:
                w = (1.0, -2.0, 1.0)
            h2 = h[d] ** 2
            A[e, e] = A[e, e] + w[1] / h2
            up = list(g); up[d] += 1
            dn = list(g); dn[d] -= 1
            eu = idx.lin(*up)
            ed = idx.lin(*dn)
            A[e, eu] = A[e, eu] + w[2] / h2
            A[e, ed] = A[e, ed] + w[0] / h2
    return A


def outgoing_rows(X, idx: LeafIndex, h, kb):
    """RTR_update (robin_tree_module.f90:667-718): sigma X(r) + tau (8/3 X(r) - 3 X(p1) + 1/3 X(p2))/h
    with sigma = -i kb, tau = 1."""
    p1, p2, ax = boundary_stencil(idx)
    sigma = complex(0.0 * kb, -1.0 * kb)
    tau = 1.0
    out = np.empty((idx.nb,) + X.shape[1:], dtype=np.complex128)
    for r in range(idx.nb):
        hn = h[ax[r]]
        v = sigma * X[r] + ((tau * (8.0 / 3.0)) / hn) * X[r]
        v = v + ((tau * (-3.0)) / hn) * X[p1[r]]
        v = v + ((tau * (1.0 / 3.0)) / hn) * X[p2[r]]
        out[r] = v
    return out


class RobinTree3D:
    """``robin_tree`` (robin_tree_module.f90:55-77) for d = 3."""

    def __init__(self):
        self.bndry_params = None
        self.factored = False

    def factor(self, L, ell_op: H.EllipticOperator, opts: H.SolveOpts):
        """robin_tree_factor (robin_tree_module.f90:96-185)."""
        bp = np.asarray(self.bndry_params, dtype=np.complex128)
        if abs(bp[0, 0] * bp[1, 1] - bp[0, 1] * bp[1, 0]) < 10.0 ** (-3.0):
            raise ValueError("Error: Boundary parameter matrix is nearly singular.")
        self.nlvls = L
        self.ell_op = ell_op
        self.opts = H.SolveOpts(h_tgt=opts.h_tgt, h=np.array(opts.h, dtype=np.float64), ordering=opts.ordering,
                                disc=opts.disc, kb=opts.kb)
        self.root, self.levels = H.build_tree(L, np.asarray(ell_op.domain, dtype=np.float64), D)
        self._idx = {}
        self._compute_rtr(self.root)
        self.factored = True

    def index(self, ptbox):
        key = tuple(ptbox[:3])
        if key not in self._idx:
            self._idx[key] = LeafIndex(*key)
        return self._idx[key]

    def _leaf(self, node):
        h, grid = H.get_h(self.opts.h_tgt, node.box, D)
        self.opts.h = h
        node.ptbox = [grid[0], grid[1], grid[2]]
        node.h = h
        idx = self.index(node.ptbox)
        kvals = np.asarray(self.ell_op.k(interior_points(idx, h, node.box)), dtype=np.complex128)
        A = fd_matrix(idx, h, kvals, self.opts.kb)
        lu, piv = H._getrf(A)
        X = np.zeros((idx.n, idx.nb), dtype=np.complex128, order="F")
        X[np.arange(idx.nb), np.arange(idx.nb)] = 1.0
        X = H._getrs((lu, piv), X)
        node.rtr = np.asfortranarray(outgoing_rows(X, idx, h, self.opts.kb))
        node.lu, node.piv = lu, piv

    def _compute_rtr(self, node):
        if node.isleaf:
            self._leaf(node)
            return
        self._compute_rtr(node.child1)
        self._compute_rtr(node.child2)
        self._merge(node)

    def _merge(self, node):
        """compute_RTR merge branch (robin_tree_module.f90:397-647) with six faces."""
        c1, c2 = node.child1, node.child2
        diffbox = np.abs((node.box[1] - node.box[0]) - (c1.box[1] - c1.box[0]))
        node.ptbox = list(c1.ptbox)
        ax = int(np.argmax(diffbox[:D]))
        node.ptbox[ax] = 2 * node.ptbox[ax]
        pf, pf1, pf2 = get_pt_face(node.ptbox), get_pt_face(c1.ptbox), get_pt_face(c2.ptbox)
        o1, o2, op = _offsets(pf1), _offsets(pf2), _offsets(pf)
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
        node.D = H._getrf(T2ii)
        Dinv = H._getri(node.D)
        T1ii = -np.array(blk(c1.rtr, o1, pf1, i1, i1), order="F") - (nu * nu) * Dinv
        T1ii[eye, eye] += zeta
        node.S = H._getrf(T1ii)
        P = np.zeros((sum(pf), sum(pf)), dtype=np.complex128, order="F")
        for col in range(1, 2 * D + 1):
            C11 = C21 = C12 = C22 = None
            if col != i1:
                C11 = H._getrs(node.S, np.asfortranarray(blk(c1.rtr, o1, pf1, i1, col)))
                C21 = nu * H._getrs(node.D, C11)
            if col != i2:
                C22 = H._getrs(node.D, np.asfortranarray(blk(c2.rtr, o2, pf2, i2, col)))
                C12 = nu * H._getrs(node.S, C22)
                C22 = C22 + nu * H._getrs(node.D, C12)
            for row in range(1, 2 * D + 1):
                R = np.zeros((pf[row - 1], pf[col - 1]), dtype=np.complex128, order="F")
                prs, pcs = pf[row - 1], pf[col - 1]
                if C11 is not None and row != i1:
                    rs, cs = pf1[row - 1], C11.shape[1]
                    R[0:rs, 0:cs] = H._gemm(1.0, np.asfortranarray(blk(c1.rtr, o1, pf1, row, i1)), C11) \
                        + blk(c1.rtr, o1, pf1, row, col)
                if C12 is not None and row != i1:
                    rs, cs = pf1[row - 1], C12.shape[1]
                    R[0:rs, pcs - cs:pcs] = H._gemm(-1.0, np.asfortranarray(blk(c1.rtr, o1, pf1, row, i1)), C12)
                if C21 is not None and row != i2:
                    rs, cs = pf2[row - 1], C21.shape[1]
                    R[prs - rs:prs, 0:cs] = H._gemm(-1.0, np.asfortranarray(blk(c2.rtr, o2, pf2, row, i2)), C21)
                if C22 is not None and row != i2:
                    rs, cs = pf2[row - 1], C22.shape[1]
                    R[prs - rs:prs, pcs - cs:pcs] = H._gemm(1.0, np.asfortranarray(blk(c2.rtr, o2, pf2, row, i2)),
                                                            C22) + blk(c2.rtr, o2, pf2, row, col)
                P[op[row - 1]:op[row - 1] + prs, op[col - 1]:op[col - 1] + pcs] = R
        node.rtr = P

    # --- solve (robin_tree_module.f90:198-233, 813-1237) ----------------------------------------
    def solve(self, rhs_list):
        for r in rhs_list:
            if r.d != self.ell_op.d:
                raise ValueError("Error: Dimensions of Robin Tree and RHS do not match.")
        self._forward(self.root, rhs_list)
        self._apply_bc(self.root, rhs_list)
        self._backward(self.root)

    def _blk(self, node, r, c):
        pf = get_pt_face(node.ptbox)
        o = _offsets(pf)
        return np.asfortranarray(node.rtr[o[r - 1]:o[r - 1] + pf[r - 1], o[c - 1]:o[c - 1] + pf[c - 1]])

    def _forward(self, node, rhs_list):
        kb = self.opts.kb
        nr = len(rhs_list)
        pf = get_pt_face(node.ptbox)
        node.g = {f: np.zeros((pf[f - 1], nr), dtype=np.complex128) for f in range(1, 2 * D + 1)}
        if node.isleaf:
            idx = self.index(node.ptbox)
            h = self.opts.h                 # T%opts%h: the last leaf's h (fd_module.f90:429)
            pts = interior_points(idx, h, node.box)
            B = np.zeros((idx.n, nr), dtype=np.complex128, order="F")
            for r, rhs in enumerate(rhs_list):
                B[idx.nb:, r] = rhs.f(pts)
            node.sol = H._getrs((node.lu, node.piv), B)
            hv = outgoing_rows(node.sol, idx, h, kb)
            o = _offsets(pf)
            node.hvec = {f: hv[o[f - 1]:o[f - 1] + pf[f - 1]] for f in range(1, 2 * D + 1)}
            return
        c1, c2 = node.child1, node.child2
        self._forward(c1, rhs_list)
        self._forward(c2, rhs_list)
        y1, y2 = H.apply_invm(None, None, c1.hvec[c1.iface], c2.hvec[c2.iface], 0.0, node.D, node.S, node.nu)
        c1.g[c1.iface] = y1
        c2.g[c2.iface] = y2
        if node.lvl > 0:
            axis = (c1.iface - 1) // 2
            node.hvec = {}
            for j in range(1, 2 * D + 1):
                if (j - 1) // 2 == axis:
                    if j == c1.iface:
                        node.hvec[j] = c2.hvec[j] + H._gemm(1.0, self._blk(c2, j, c2.iface), y2)
                    else:
                        node.hvec[j] = c1.hvec[j] + H._gemm(1.0, self._blk(c1, j, c1.iface), y1)
                else:
                    node.hvec[j] = np.concatenate(
                        [c1.hvec[j] + H._gemm(1.0, self._blk(c1, j, c1.iface), y1),
                         c2.hvec[j] + H._gemm(1.0, self._blk(c2, j, c2.iface), y2)], axis=0)
        c1.hvec = None
        c2.hvec = None

    def _apply_bc(self, node, rhs_list):
        if node.isleaf:
            idx = self.index(node.ptbox)
            for f in range(1, 2 * D + 1):
                if node.isbndry[f - 1]:
                    pts = face_points(idx, self.opts.h, node.box, f)
                    node.g[f] = np.stack([np.asarray(r.g[f - 1](pts), dtype=np.complex128) for r in rhs_list],
                                         axis=1)
            return
        if not any(node.isbndry):
            return
        c1, c2 = node.child1, node.child2
        self._apply_bc(c1, rhs_list)
        self._apply_bc(c2, rhs_list)
        for f in range(1, 2 * D + 1):
            if node.isbndry[f - 1]:
                if f == c2.iface:
                    node.g[f] = c1.g[f].copy()
                elif f == c1.iface:
                    node.g[f] = c2.g[f].copy()
                else:
                    node.g[f] = np.concatenate([c1.g[f], c2.g[f]], axis=0)

    def _backward(self, node):
        if node.isleaf:
            idx = self.index(node.ptbox)
            nr = node.sol.shape[1]
            B = np.zeros((idx.n, nr), dtype=np.complex128, order="F")
            o = _offsets(get_pt_face(node.ptbox))
            for f in range(1, 2 * D + 1):
                B[o[f - 1]:o[f - 1] + node.g[f].shape[0]] = node.g[f]
            node.sol = node.sol + H._getrs((node.lu, node.piv), B)
            return
        c1, c2 = node.child1, node.child2
        axis = (c1.iface - 1) // 2
        pf = get_pt_face(node.ptbox)
        for f in range(1, 2 * D + 1):
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
        for f in range(1, 2 * D + 1):
            if f != c1.iface:
                Tg1 = Tg1 + H._gemm(1.0, self._blk(c1, c1.iface, f), c1.g[f])
            if f != c2.iface:
                Tg2 = Tg2 + H._gemm(1.0, self._blk(c2, c2.iface, f), c2.g[f])
        y1, y2 = H.apply_invm(c1.g[c1.iface], c2.g[c2.iface], Tg1, Tg2, 1.0, node.D, node.S, node.nu)
        c1.g[c1.iface] = y1
        c2.g[c2.iface] = y2
        node.g = None
        self._backward(c1)
        self._backward(c2)

    def get_solution(self):
        """get_solution/get_node_sol (robin_output_module.f90:48-75, 305-322)."""
        return [(lf.box.copy(), lf.sol.copy()) for lf in self.levels[-1]]


def _offsets(pf):
    out = [0]
    for v in pf[:-1]:
        out.append(out[-1] + v)
    return out


def leaf_all_points(idx: LeafIndex, h, box):
    """Every point of a leaf's u vector (check_solution's proc2vec, robin_output_module.f90:234-273)."""
    return grid2real(idx.gi, idx.gj, idx.gk, (idx.a, idx.b, idx.c), h, box)


def global_solve(L, domain, h_tgt, kb, bndry_params, kfun, f, gfaces):
    """An independent check: the global sparse FD system the 3D tree eliminates, assembled row by
    row (every leaf's PDE rows; Robin rows on the domain boundary; transmission rows
    h_own - zeta g_own - nu g_neighbour = 0 on interfaces) and solved with SuperLU.  Returns the
    per-leaf solutions (nleaves, n) in get_solution order."""
    root, levels = H.build_tree(L, np.asarray(domain, dtype=np.float64), D)
    leaves = levels[-1]
    h, grid = H.get_h(h_tgt, leaves[0].box, D)
    idx = LeafIndex(*grid[:3])
    nb, n = idx.nb, idx.n
    bp = np.asarray(bndry_params, dtype=np.complex128)
    nu = (-bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
    zeta = (bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
    A0 = fd_matrix(idx, h, np.zeros(idx.a * idx.b * idx.c, dtype=np.complex128), kb)
    R = outgoing_rows(np.eye(n, dtype=np.complex128), idx, h, kb)
    w = leaves[0].box[1] - leaves[0].box[0]
    lo = root.box[0]
    pos = {}
    for li, lf in enumerate(leaves):
        key = tuple(int(round((lf.box[0, ax] - lo[ax]) / w[ax])) for ax in range(3))
        pos[key] = li
    where = {li: key for key, li in pos.items()}
    pf = get_pt_face(grid)
    off = _offsets(pf)
    N = len(leaves) * n
    M = sp.lil_matrix((N, N), dtype=np.complex128)
    rhs = np.zeros(N, dtype=np.complex128)
    for li, lf in enumerate(leaves):
        base = li * n
        pts = interior_points(idx, h, lf.box)
        kv = np.asarray(kfun(pts), dtype=np.complex128)
        for e in range(nb, n):
            cols = np.nonzero(A0[e])[0]
            for c in cols:
                M[base + e, base + c] = A0[e, c]
            M[base + e, base + e] = M[base + e, base + e] + kv[e - nb]
        rhs[base + nb:base + n] = f(pts)
        key = where[li]
        for fc in range(1, 2 * D + 1):
            ax = (fc - 1) // 2
            step = -1 if fc % 2 == 1 else 1
            nbr = list(key)
            nbr[ax] += step
            rows = range(off[fc - 1], off[fc - 1] + pf[fc - 1])
            if tuple(nbr) not in pos:
                fpts = face_points(idx, h, lf.box, fc)
                gvals = gfaces[fc - 1](fpts)
                for t, r in enumerate(rows):
                    for c in np.nonzero(A0[r])[0]:
                        M[base + r, base + c] = A0[r, c]
                    rhs[base + r] = gvals[t]
                continue
            lj = pos[tuple(nbr)]
            fo = fc + 1 if fc % 2 == 1 else fc - 1
            for t, r in enumerate(rows):
                rn = off[fo - 1] + t
                for c in np.nonzero(R[r])[0]:
                    M[base + r, base + c] = M[base + r, base + c] + R[r, c]
                for c in np.nonzero(A0[r])[0]:
                    M[base + r, base + c] = M[base + r, base + c] - zeta * A0[r, c]
                for c in np.nonzero(A0[rn])[0]:
                    M[base + r, lj * n + c] = M[base + r, lj * n + c] - nu * A0[rn, c]
    x = spla.spsolve(M.tocsc(), rhs)
    return x.reshape(len(leaves), n)
