"""Oracle: independent global sparse FD system behind robinsolver's HPS factor/solve.

TEST INFRASTRUCTURE ONLY (same import rule as ``hps_ref.py``).

The HPS tree of the reference eliminates, leaf by leaf and merge by merge, one
global finite-difference system.  This module writes that system out directly:

* unknowns: every leaf's cornerless grid (its ``u`` vector in lin2fgrid order,
  fd_module.f90:867-939), leaves in DFS order.  Interface points appear once per
  adjacent leaf, as in the reference;
* per leaf: the interior PDE rows of FD_matrix_row (fd_module.f90:140-181);
* boundary rows on the domain boundary: the Robin row i*kb*u + u_n = g
  (fd_module.f90:187-216);
* boundary rows on an interface: the transmission conditions the merge solves
  (robin_tree_module.f90:425-467 with ``apply_invm`` :1252-1322):
  h1 = zeta*g1 + nu*g2 and h2 = nu*g1 + zeta*g2, where g is a leaf's incoming
  data (its own Robin row) and h = -i*kb*u + u_n its outgoing data
  (RTR_update, robin_tree_module.f90:683-713).

``solve`` factors it with SuperLU (``scipy.sparse.linalg.spsolve``); ``residual``
applies it to a candidate solution, which checks a full-size result without
running the HPS restatement.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import hps_ref as H


def _leaf_rows(a, b, h, kb):
    """COO triplets of one leaf matrix without the potential (structure + constants),
    the diagonal increments of the interior rows, and the outgoing rows R."""
    A0 = H.fd_matrix(a, b, h, np.zeros(a * b, dtype=np.complex128), kb)
    nb = 2 * (a + b)
    n = A0.shape[0]
    R = H.outgoing_rows(np.eye(n, dtype=np.complex128), a, b, h, kb)   # nb x n
    return A0, R, nb, n


class GlobalFD:
    """Assemble the global system for a tree geometry (from ``hps_ref.build_tree``)."""

    def __init__(self, L, domain, h_tgt, kb, bndry_params, kfun):
        self.root, self.levels = H.build_tree(L, np.asarray(domain, dtype=np.float64), 2)
        leaves = self.levels[-1]
        self.leaves = leaves
        h, grid = H.get_h(h_tgt, leaves[0].box, 2)
        a, b = grid[0], grid[1]
        for lf in leaves:
            h2, g2 = H.get_h(h_tgt, lf.box, 2)
            if g2[:2] != grid[:2]:
                raise ValueError("non-uniform leaf grids")
        self.a, self.b, self.h, self.kb = a, b, h, kb
        bp = np.asarray(bndry_params, dtype=np.complex128)
        nu = (-bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
        zeta = (bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
        A0, R, nb, n = _leaf_rows(a, b, h, kb)
        self.nb, self.n = nb, n
        nl = len(leaves)
        # leaf positions on the regular leaf lattice
        w = leaves[0].box[1] - leaves[0].box[0]
        lo = self.root.box[0]
        pos = {}
        where = {}
        for li, lf in enumerate(leaves):
            ix = int(round((lf.box[0, 0] - lo[0]) / w[0]))
            iy = int(round((lf.box[0, 1] - lo[1]) / w[1]))
            pos[(ix, iy)] = li
            where[li] = (ix, iy)
        self.pos = pos
        pf = H.get_pt_face((a, b))
        off = H.face_offsets(pf)
        A0c = sp.coo_matrix(A0)
        Rc = sp.csr_matrix(R)
        rows, cols, vals = [], [], []
        diag_rows = []
        kval = []
        for li, lf in enumerate(leaves):
            base = li * n
            pts = H.interior_points(a, b, h, lf.box)
            kval.append(np.asarray(kfun(pts), dtype=np.complex128))
            # interior rows + boundary Robin rows (interface rows replaced below)
            keep = A0c.row >= nb
            rows.append(base + A0c.row[keep]); cols.append(base + A0c.col[keep]); vals.append(A0c.data[keep])
            diag_rows.append(base + np.arange(nb, n))
            ix, iy = where[li]
            for f in range(1, 5):
                rr = np.arange(off[f - 1], off[f - 1] + pf[f - 1])
                nbr = {1: (ix - 1, iy), 2: (ix + 1, iy), 3: (ix, iy - 1), 4: (ix, iy + 1)}[f]
                if nbr not in pos:
                    sub = sp.coo_matrix(A0[rr])
                    rows.append(base + rr[sub.row]); cols.append(base + sub.col); vals.append(sub.data)
                    continue
                lj = pos[nbr]
                fo = {1: 2, 2: 1, 3: 4, 4: 3}[f]
                rn = np.arange(off[fo - 1], off[fo - 1] + pf[fo - 1])
                # row for (leaf li, face f point p): its own h1 equation
                #   h_li(p) - zeta*g_li(p) - nu*g_lj(p') = 0
                for t in range(len(rr)):
                    r_own, r_nb = rr[t], rn[t]
                    ro = Rc.getrow(r_own).tocoo()
                    go = sp.coo_matrix(A0[r_own:r_own + 1])
                    gn = sp.coo_matrix(A0[r_nb:r_nb + 1])
                    rows.append(np.full(ro.nnz, base + r_own)); cols.append(base + ro.col); vals.append(ro.data)
                    rows.append(np.full(go.nnz, base + r_own)); cols.append(base + go.col); vals.append(-zeta * go.data)
                    rows.append(np.full(gn.nnz, base + r_own)); cols.append(lj * n + gn.col); vals.append(-nu * gn.data)
        rows = np.concatenate(rows); cols = np.concatenate(cols); vals = np.concatenate(vals)
        diag_rows = np.concatenate(diag_rows)
        kval = np.concatenate(kval)
        rows = np.concatenate([rows, diag_rows]); cols = np.concatenate([cols, diag_rows]); vals = np.concatenate([vals, kval])
        N = nl * n
        self.A = sp.csc_matrix((vals, (rows, cols)), shape=(N, N))

    def rhs(self, f, gfaces):
        """Right-hand side for source ``f`` and face data ``gfaces`` (4 callbacks)."""
        a, b, h, nb, n = self.a, self.b, self.h, self.nb, self.n
        pf = H.get_pt_face((a, b))
        off = H.face_offsets(pf)
        out = np.zeros(len(self.leaves) * n, dtype=np.complex128)
        for li, lf in enumerate(self.leaves):
            base = li * n
            out[base + nb:base + n] = f(H.interior_points(a, b, h, lf.box))
            for fc in range(1, 5):
                if lf.isbndry[fc - 1]:
                    pts = H.face_points(a, b, h, lf.box, fc)
                    out[base + off[fc - 1]:base + off[fc - 1] + pf[fc - 1]] = gfaces[fc - 1](pts)
        return out

    def solve(self, f, gfaces):
        """Global solution, split per leaf (DFS order) like get_solution."""
        x = spla.spsolve(self.A, self.rhs(f, gfaces))
        return x.reshape(len(self.leaves), self.n)

    def residual(self, u_leaves, f, gfaces):
        """max|A u - b| / max|b| for a per-leaf solution array (nleaves, n)."""
        b = self.rhs(f, gfaces)
        r = self.A @ np.asarray(u_leaves).reshape(-1) - b
        return float(np.max(np.abs(r)) / max(np.max(np.abs(b)), 1e-300))


def backward_error(L, domain, h_tgt, kb, bndry_params, kvals, U, F, G):
    """Normwise backward error of a candidate solution of the global FD system, vectorised over
    leaves so that it runs at the full benchmark sizes:

        eta = max|A u - b| / (||A||_inf * max|u| + max|b|)

    kvals, F: (nleaves, a*b) potential and source samples (leaf DFS order, x fastest);
    U: (nleaves, n) solution in get_solution order; G: (root_nb,) boundary data in the root's
    face order (faces x1 x2 y1 y2, each ascending).  The rows are the ones ``GlobalFD``
    assembles: leaf PDE rows, Robin rows on the domain boundary, transmission rows
    h1 - zeta*g1 - nu*g2 = 0 on every interface point."""
    root, levels = H.build_tree(L, np.asarray(domain, dtype=np.float64), 2)
    leaves = levels[-1]
    h, grid = H.get_h(h_tgt, leaves[0].box, 2)
    a, b = grid[0], grid[1]
    nb = 2 * (a + b)
    n = nb + a * b
    bp = np.asarray(bndry_params, dtype=np.complex128)
    nu = (-bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
    zeta = (bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
    A0 = sp.csr_matrix(H.fd_matrix(a, b, h, np.zeros(a * b, dtype=np.complex128), kb))
    R = sp.csr_matrix(H.outgoing_rows(np.eye(n, dtype=np.complex128), a, b, h, kb))
    U = np.asarray(U, dtype=np.complex128)
    kvals = np.asarray(kvals, dtype=np.complex128).reshape(len(leaves), a * b)
    F = np.asarray(F, dtype=np.complex128).reshape(len(leaves), a * b)
    G = np.asarray(G, dtype=np.complex128).reshape(-1)
    AU = np.asarray((A0 @ U.T).T)
    AU[:, nb:] += kvals * U[:, nb:]
    hout = np.asarray((R @ U.T).T)
    gin = AU[:, :nb]
    res = np.zeros_like(AU)
    res[:, nb:] = AU[:, nb:] - F
    pf = H.get_pt_face((a, b))
    off = H.face_offsets(pf)
    w = leaves[0].box[1] - leaves[0].box[0]
    lo = root.box[0]
    ix = np.array([int(round((lf.box[0, 0] - lo[0]) / w[0])) for lf in leaves])
    iy = np.array([int(round((lf.box[0, 1] - lo[1]) / w[1])) for lf in leaves])
    nx, ny = ix.max() + 1, iy.max() + 1
    at = -np.ones((nx, ny), dtype=np.int64)
    at[ix, iy] = np.arange(len(leaves))
    rootpf = [ny * b, ny * b, nx * a, nx * a]
    rootoff = H.face_offsets(rootpf)
    for f in range(1, 5):
        sl = slice(off[f - 1], off[f - 1] + pf[f - 1])
        fo = {1: 2, 2: 1, 3: 4, 4: 3}[f]
        so = slice(off[fo - 1], off[fo - 1] + pf[fo - 1])
        jx, jy = {1: (ix - 1, iy), 2: (ix + 1, iy), 3: (ix, iy - 1), 4: (ix, iy + 1)}[f]
        inside = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny)
        li = np.nonzero(inside)[0]
        lj = at[jx[li], jy[li]]
        res[li, sl] = hout[li, sl] - zeta * gin[li, sl] - nu * gin[lj, so]
        lb = np.nonzero(~inside)[0]
        pos = iy[lb] if f in (1, 2) else ix[lb]          # position along the face
        idx = rootoff[f - 1] + pos[:, None] * pf[f - 1] + np.arange(pf[f - 1])[None, :]
        res[lb, sl] = gin[lb, sl] - G[idx]
    A0abs = np.asarray(abs(A0).sum(axis=1)).ravel()
    Rabs = np.asarray(abs(R).sum(axis=1)).ravel()
    normA = max(A0abs[nb:].max() + np.abs(kvals).max(),
                (Rabs + (abs(zeta) + abs(nu)) * A0abs[:nb]).max())
    bmax = max(np.abs(F).max(), np.abs(G).max() if G.size else 0.0)
    return float(np.abs(res).max() / (normA * np.abs(U).max() + bmax))


def _lattice(root, leaves):
    """Leaf positions (ix, iy) on the regular leaf lattice and the inverse table."""
    w = leaves[0].box[1] - leaves[0].box[0]
    lo = root.box[0]
    ix = np.array([int(round((lf.box[0, 0] - lo[0]) / w[0])) for lf in leaves])
    iy = np.array([int(round((lf.box[0, 1] - lo[1]) / w[1])) for lf in leaves])
    nx, ny = ix.max() + 1, iy.max() + 1
    at = -np.ones((nx, ny), dtype=np.int64)
    at[ix, iy] = np.arange(len(leaves))
    return ix, iy, nx, ny, at


class SparseFD:
    """The same global system as ``GlobalFD``, assembled with array operations so that it can be
    built at the full benchmark sizes (1024^2: 1.3 M unknowns), from the potential samples the
    B200 path receives.

    kvals: (nleaves, a*b) potential at the leaves' interior cell centres (leaf DFS order,
    x fastest).  Rows and unknowns: every leaf's u vector in get_solution order.  ``solve``
    factors the matrix once with SuperLU and solves for (F, G) pairs in the B200 path's input
    layout (F: (nleaves, a*b) sources, G: (root_nb,) boundary data in the root's face order)."""

    def __init__(self, L, domain, h_tgt, kb, bndry_params, kvals):
        root, levels = H.build_tree(L, np.asarray(domain, dtype=np.float64), 2)
        leaves = levels[-1]
        h, grid = H.get_h(h_tgt, leaves[0].box, 2)
        a, b = grid[0], grid[1]
        nb = 2 * (a + b)
        n = nb + a * b
        nl = len(leaves)
        self.a, self.b, self.nb, self.n, self.nl = a, b, nb, n, nl
        bp = np.asarray(bndry_params, dtype=np.complex128)
        nu = (-bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
        zeta = (bp[0, 0] * bp[1, 1] + bp[0, 1] * bp[1, 0]) / (2 * bp[0, 0] * bp[0, 1])
        A0 = sp.coo_matrix(H.fd_matrix(a, b, h, np.zeros(a * b, dtype=np.complex128), kb))
        R = sp.coo_matrix(H.outgoing_rows(np.eye(n, dtype=np.complex128), a, b, h, kb))
        kvals = np.asarray(kvals, dtype=np.complex128).reshape(nl, a * b)
        base = (np.arange(nl, dtype=np.int64) * n)[:, None]
        rows, cols, vals = [], [], []

        def put(li_base, lj_base, r, c, v):
            rows.append((li_base + r[None, :]).ravel())
            cols.append((lj_base + c[None, :]).ravel())
            vals.append(np.broadcast_to(v[None, :], (li_base.shape[0], v.size)).ravel())

        keep = A0.row >= nb                                  # interior PDE rows
        put(base, base, A0.row[keep], A0.col[keep], A0.data[keep])
        diag = (base + np.arange(nb, n)[None, :]).ravel()
        rows.append(diag); cols.append(diag); vals.append(kvals.ravel())
        ix, iy, nx, ny, at = _lattice(root, leaves)
        pf = H.get_pt_face((a, b))
        off = H.face_offsets(pf)
        rootpf = [ny * b, ny * b, nx * a, nx * a]
        rootoff = H.face_offsets(rootpf)
        self.g_rows = np.zeros(sum(rootpf), dtype=np.int64)   # root boundary point -> global row
        for f in range(1, 5):
            lo_r, hi_r = off[f - 1], off[f - 1] + pf[f - 1]
            fo = {1: 2, 2: 1, 3: 4, 4: 3}[f]
            jx, jy = {1: (ix - 1, iy), 2: (ix + 1, iy), 3: (ix, iy - 1), 4: (ix, iy + 1)}[f]
            inside = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny)
            li = np.nonzero(inside)[0]
            lj = at[jx[li], jy[li]]
            sel = (A0.row >= lo_r) & (A0.row < hi_r)
            selR = (R.row >= lo_r) & (R.row < hi_r)
            if li.size:
                bi = base[li]
                # transmission row of an interface point: h_own - zeta g_own - nu g_neighbour = 0
                put(bi, bi, R.row[selR], R.col[selR], R.data[selR])
                put(bi, bi, A0.row[sel], A0.col[sel], -zeta * A0.data[sel])
                # the neighbour's row for the same point sits on the opposite face, same position
                selo = (A0.row >= off[fo - 1]) & (A0.row < off[fo - 1] + pf[fo - 1])
                rown = A0.row[selo] - off[fo - 1] + lo_r
                put(bi, base[lj], rown, A0.col[selo], -nu * A0.data[selo])
            lb = np.nonzero(~inside)[0]
            if lb.size:
                put(base[lb], base[lb], A0.row[sel], A0.col[sel], A0.data[sel])
                pos = iy[lb] if f in (1, 2) else ix[lb]
                idx = rootoff[f - 1] + pos[:, None] * pf[f - 1] + np.arange(pf[f - 1])[None, :]
                self.g_rows[idx.ravel()] = (base[lb] + np.arange(lo_r, hi_r)[None, :]).ravel()
        N = nl * n
        self.A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
        self._lu = None

    def rhs(self, F, G):
        out = np.zeros(self.nl * self.n, dtype=np.complex128)
        out.reshape(self.nl, self.n)[:, self.nb:] = np.asarray(F, dtype=np.complex128).reshape(self.nl, -1)
        out[self.g_rows] = np.asarray(G, dtype=np.complex128).reshape(-1)
        return out

    def factor(self):
        if self._lu is None:
            self._lu = spla.splu(self.A, permc_spec="COLAMD")
        return self._lu

    def solve(self, F, G):
        """FP64 solution (nleaves, n) of the system for one right-hand side."""
        return self.factor().solve(self.rhs(F, G)).reshape(self.nl, self.n)

    def residual(self, U, F, G):
        """max|A u - b| / max|b|."""
        b = self.rhs(F, G)
        r = self.A @ np.asarray(U, dtype=np.complex128).reshape(-1) - b
        return float(np.max(np.abs(r)) / max(np.max(np.abs(b)), 1e-300))


def forward_error(U, U_ref):
    """max|u - u_ref| / max|u_ref| over all leaves: the normwise max error every result states."""
    U = np.asarray(U)
    U_ref = np.asarray(U_ref)
    return float(np.max(np.abs(U - U_ref)) / np.max(np.abs(U_ref)))
