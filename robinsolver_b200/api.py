"""Host-side mirror of robinsolver's public API over the B200 C-ABI.

Same type names, fields and calls as the reference:

    T = robin_tree();  T.bndry_params = ...             (robin_tree_module.f90:55-77)
    T.factor(L, op, opts)                               (robin_tree_factor, :96-185)
    T.solve(rhs)                                        (robin_tree_solve, :198-233)
    u = get_solution(T)                                 (robin_output_module.f90:48-75)

Differences that follow from the host/device split:

* callbacks (``elliptic_operator.k``, ``elliptic_rhs.f``, ``bndry_rhs.g_face``) are
  vectorised: they receive an ``(npts, 3)`` float64 array of the points the reference would
  pass one at a time, and return ``npts`` complex values (``scalar_callback`` adapts a
  per-point function);
* ``solve`` also accepts a list of ``elliptic_rhs``: every right-hand side is solved in one
  batched sweep and ``get_solution(T, irhs)`` selects one;
* errors raise ``RobinSolverError`` carrying the reference's ``stop`` message;
* every solve applies its own boundary data (the reference applies boundary data only on the
  first solve of a process).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import lib


class RobinSolverError(RuntimeError):
    """A failed call; ``code`` is the C-ABI status (RB_ERR_*)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def _check(code, handle=None):
    if code != _lib.RB_OK:
        raise RobinSolverError(code, _lib.last_error(handle))


def scalar_callback(fn):
    """Adapts a per-point function ``fn(x) -> complex`` (x of length 3) to the vectorised form."""
    def vec(X):
        return np.array([fn(x) for x in np.asarray(X)], dtype=np.complex128)
    return vec


@dataclass
class debug_opts:
    """derived_type_module.f90:285-290."""
    txt_output: bool = False
    no_delete: bool = False


@dataclass
class solve_opts:
    """derived_type_module.f90:309-320.  ``h`` is overwritten by ``factor`` with the last leaf's
    grid spacing, as get_h does on robin_tree%opts."""
    h_tgt: float = 0.0
    h: np.ndarray = field(default_factory=lambda: np.zeros(3))
    ordering: int = 1
    disc: str = "fd"
    local_mode: str = "LU"
    R_mode: str = "LU"
    kb: float = 1.0
    debug: debug_opts = field(default_factory=debug_opts)


@dataclass
class elliptic_operator:
    """derived_type_module.f90:72-84.  ``coeff`` and ``robin_coeff`` are carried but, as in the
    reference, never read on the factor/solve path."""
    d: int = 2
    domain: np.ndarray = field(default_factory=lambda: np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]))
    coeff: object = None
    k: object = None
    robin_coeff: np.ndarray = field(default_factory=lambda: np.zeros((6, 2), dtype=np.complex128))


@dataclass
class bndry_rhs:
    """derived_type_module.f90:92-96."""
    g_face: object = None


@dataclass
class elliptic_rhs:
    """derived_type_module.f90:109-115."""
    d: int = 2
    f: object = None
    g: list = field(default_factory=lambda: [bndry_rhs() for _ in range(6)])


@dataclass
class leaf_solution:
    """robin_output_module.f90:32-37."""
    box: np.ndarray
    u: np.ndarray


PRECISIONS = {"fp64": _lib.RB_PREC_FP64, "mixed": _lib.RB_PREC_MIXED}


def _face_sizes(d, a, b, c=1):
    """Points per face x1 x2 y1 y2 (z1 z2) of an a x b (x c) grid (get_pt_face, fd_module.f90:1033-1049)."""
    if d == 2:
        return [b, b, a, a]
    return [b * c, b * c, a * c, a * c, a * b, a * b]


def make_geom(L, ell_op, opts, bndry_params, flags=0, budget=0) -> _lib.rb_geom:
    """The C-ABI's rb_geom for robin_tree%factor(L, op, opts) with robin_tree%bndry_params."""
    g = _lib.rb_geom()
    g.d = int(ell_op.d)
    g.L = int(L)
    dom = np.asarray(ell_op.domain, dtype=np.float64)
    for j in range(3):
        g.domain[2 * j] = dom[0, j]
        g.domain[2 * j + 1] = dom[1, j]
    g.h_tgt = float(opts.h_tgt)
    g.kb = float(opts.kb)
    bp = np.asarray(bndry_params, dtype=np.complex128)
    for q, (i, j) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
        g.bndry_params[2 * q] = bp[i, j].real
        g.bndry_params[2 * q + 1] = bp[i, j].imag
    g.ordering = int(opts.ordering)
    g.flags = int(flags)
    g.device_budget = int(budget)
    return g


class robin_tree:
    """robin_tree (robin_tree_module.f90:55-77) backed by a device-resident factorization."""

    def __init__(self, device_budget: int = 0, skip_root_rtr: bool = False, merge_ds: bool = False,
                 async_factor: bool = False, graphs: bool = True, mixed_int8_top: bool = False):
        self.bndry_params = None
        self.nlvls = 0
        self.ell_op = None
        self.opts = None
        self.factored = False
        self.f_time = 0.0
        self.s_time = 0.0
        self._h = None
        self._info = None
        self._budget = int(device_budget)
        self._skip_root = bool(skip_root_rtr)
        self._merge_ds = bool(merge_ds)     # the reference's inv(D), inv(S) interface solve
        self._async = bool(async_factor)    # factor returns when enqueued (RB_FLAG_ASYNC_FACTOR)
        self._graphs = bool(graphs)         # replay factor/solve as CUDA graphs (else RB_FLAG_NO_GRAPHS)
        self._int8_top = bool(mixed_int8_top)   # mixed factor: top two levels' GEMMs on the int8 engine too

    # -- handle ----------------------------------------------------------------------------------
    def close(self):
        if self._h is not None:
            lib.rb_tree_destroy(self._h)
            self._h = None
        self.factored = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _create(self, L, ell_op, opts):
        if self.bndry_params is None:
            raise RobinSolverError(_lib.RB_ERR_BNDRY_PARAMS, "robin_tree%bndry_params is not set")
        self.close()
        flags = (_lib.RB_FLAG_VERBOSE if opts.debug.txt_output else 0) | \
                (_lib.RB_FLAG_SKIP_ROOT_RTR if self._skip_root else 0) | \
                (_lib.RB_FLAG_MERGE_DS if self._merge_ds else 0) | \
                (_lib.RB_FLAG_ASYNC_FACTOR if self._async else 0) | \
                (_lib.RB_FLAG_MIXED_INT8_TOP if self._int8_top else 0) | \
                (0 if self._graphs else _lib.RB_FLAG_NO_GRAPHS)
        g = make_geom(L, ell_op, opts, self.bndry_params, flags, self._budget)
        h = _lib.C.c_void_p()
        _check(lib.rb_tree_create(_lib.C.byref(g), _lib.C.byref(h)))
        self._h = h
        self._info = self.info()

    def info(self) -> _lib.rb_info:
        inf = _lib.rb_info()
        _check(lib.rb_tree_info(self._h, _lib.C.byref(inf)), self._h)
        return inf

    def sample_points(self, which: int) -> np.ndarray:
        inf = self._info
        n = {
            _lib.RB_POINTS_POTENTIAL: inf.n_interior,
            _lib.RB_POINTS_SOURCE: inf.n_interior,
            _lib.RB_POINTS_BOUNDARY: inf.root_nb,
            _lib.RB_POINTS_SOLUTION: inf.nleaves * inf.leaf_n,
        }[which]
        X = np.zeros((n, 3), dtype=np.float64)
        _check(lib.rb_tree_sample_points(self._h, which, _lib.dptr(X)), self._h)
        return X

    # -- factor / solve ----------------------------------------------------------------------------
    def plan(self, L, ell_op, opts):
        """Builds the tree without factoring (host only)."""
        self.nlvls = int(L)
        self.ell_op = ell_op
        self.opts = opts
        self._create(L, ell_op, opts)
        return self._info

    def factor(self, L, ell_op: elliptic_operator, opts: solve_opts, precision: str = "fp64"):
        """robin_tree%factor(L, op, opts)."""
        self.plan(L, ell_op, opts)
        if ell_op.k is None:
            raise RobinSolverError(_lib.RB_ERR_INVALID, "elliptic_operator%k is not associated")
        X = self.sample_points(_lib.RB_POINTS_POTENTIAL)
        kv = np.ascontiguousarray(np.asarray(ell_op.k(X), dtype=np.complex128))
        self.factor_samples(kv, precision)

    def factor_samples(self, kv: np.ndarray, precision: str = "fp64"):
        """Factor with the potential already sampled at RB_POINTS_POTENTIAL."""
        kv = np.ascontiguousarray(kv, dtype=np.complex128)
        if kv.size != self._info.n_interior:
            raise RobinSolverError(_lib.RB_ERR_INVALID, "potential sample count mismatch")
        self.factored = False
        _check(lib.rb_tree_factor(self._h, _lib.dptr(kv), PRECISIONS[precision]), self._h)
        self.factored = True
        self._info = self.info()
        if self.opts is not None:
            self.opts.h = np.array(self._info.h_last[:], dtype=np.float64)
        if not self._async:          # an asynchronous factor's time is taken by the solve
            self._update_times()

    def _update_times(self):
        f = _lib.C.c_double()
        s = _lib.C.c_double()
        _check(lib.rb_tree_times(self._h, _lib.C.byref(f), _lib.C.byref(s)), self._h)
        self.f_time, self.s_time = f.value, s.value

    def sample_rhs(self, rhs_list):
        """(f, g) sample arrays for a list of elliptic_rhs, in the C-ABI layouts."""
        inf = self._info
        Xf = self.sample_points(_lib.RB_POINTS_SOURCE)
        Xg = self.sample_points(_lib.RB_POINTS_BOUNDARY)
        pf = _face_sizes(inf.d, inf.root_a, inf.root_b, inf.root_c)
        bounds = np.concatenate([[0], np.cumsum(pf)])
        F = np.zeros((len(rhs_list), inf.n_interior), dtype=np.complex128)
        G = np.zeros((len(rhs_list), inf.root_nb), dtype=np.complex128)
        for r, rhs in enumerate(rhs_list):
            if rhs.d != self.ell_op.d:
                raise RobinSolverError(_lib.RB_ERR_DIM_MISMATCH, "Error: Dimensions of Robin Tree and RHS do not match.")
            if rhs.f is not None:
                F[r] = rhs.f(Xf)
            for fc in range(len(pf)):
                gf = rhs.g[fc].g_face if isinstance(rhs.g[fc], bndry_rhs) else rhs.g[fc]
                if gf is not None:
                    G[r, bounds[fc]:bounds[fc + 1]] = gf(Xg[bounds[fc]:bounds[fc + 1]])
        return F, G

    def set_refinement(self, tol: float = 1e-10, max_iter: int = 8):
        """Tolerance of the iterative refinement of solves against a mixed-precision factor
        (rb_tree_set_refinement); FP64 factors solve directly."""
        _check(lib.rb_tree_set_refinement(self._h, float(tol), int(max_iter)), self._h)

    def refine_info(self):
        """(corrections, contraction, estimated relative error, relative residual) of the last
        mixed-precision solve."""
        it = _lib.C.c_int32()
        rho = _lib.C.c_double()
        est = _lib.C.c_double()
        res = _lib.C.c_double()
        _check(lib.rb_tree_refine_info(self._h, _lib.C.byref(it), _lib.C.byref(rho), _lib.C.byref(est),
                                       _lib.C.byref(res)), self._h)
        return it.value, rho.value, est.value, res.value

    def solve(self, rhs, tol: float | None = None):
        """robin_tree%solve(rhs); ``rhs`` may be a list for a batched solve.  ``tol``: relative
        error the refinement of a mixed-precision factor reaches (default 1e-10)."""
        if tol is not None:
            self.set_refinement(tol)
        if not self.factored:
            raise RobinSolverError(_lib.RB_ERR_NOT_FACTORED, "Error: Robin Tree must be factored first.")
        rhs_list = rhs if isinstance(rhs, (list, tuple)) else [rhs]
        F, G = self.sample_rhs(rhs_list)
        self.solve_samples(F, G)

    def solve_samples(self, F, G: np.ndarray):
        """Solve with sampled sources F (None: every interior source is zero, nothing is
        uploaded for it) and boundary data G."""
        G = np.ascontiguousarray(G, dtype=np.complex128)
        nr = G.shape[0]
        if F is not None:
            F = np.ascontiguousarray(F, dtype=np.complex128)
            if F.size != nr * self._info.n_interior:
                raise RobinSolverError(_lib.RB_ERR_INVALID, "right-hand side sample count mismatch")
        if G.size != nr * self._info.root_nb:
            raise RobinSolverError(_lib.RB_ERR_INVALID, "right-hand side sample count mismatch")
        _check(lib.rb_tree_solve(self._h, nr, None if F is None else _lib.dptr(F), _lib.dptr(G)), self._h)
        self._info = self.info()
        self._update_times()

    def solution_array(self, irhs: int = 0) -> np.ndarray:
        """Solution of one RHS as an (nleaves, leaf_n) array in get_solution order."""
        inf = self._info
        u = np.zeros((inf.nleaves, inf.leaf_n), dtype=np.complex128)
        _check(lib.rb_get_solution(self._h, irhs, _lib.dptr(u), None), self._h)
        return u

    def get_rtr(self, level: int, node: int) -> np.ndarray:
        """node%RtR of a node as one nb x nb matrix (faces x1 x2 y1 y2, then z1 z2 in 3D)."""
        nb = int(sum(_face_sizes(self._info.d, *self._level_grid(level))))
        out = np.zeros((nb, nb), dtype=np.complex128, order="F")
        _check(lib.rb_tree_get_rtr(self._h, level, node, _lib.dptr(out)), self._h)
        return out

    def _level_grid(self, level: int):
        """(a, b, c) grid of the nodes of a level (c = 1 in 2D)."""
        sh = (_lib.C.c_int32 * 4)()
        _check(lib.rb_tree_level_shape(self._h, level, sh), self._h)
        return sh[1], sh[2], sh[3]

    def stage_times(self, with_flops=False):
        """Timed entries as (name, ms) or (name, ms, flops)."""
        n = lib.rb_tree_stage_times(self._h, None, None, None, 0)
        ms = (_lib.C.c_double * max(n, 1))()
        fl = (_lib.C.c_double * max(n, 1))()
        names = (_lib.C.c_char_p * max(n, 1))()
        lib.rb_tree_stage_times(self._h, ms, fl, names, n)
        if with_flops:
            return [(names[i].decode(), ms[i], fl[i]) for i in range(n)]
        return [(names[i].decode(), ms[i]) for i in range(n)]

    def clear_stage_times(self):
        _check(lib.rb_tree_clear_stage_times(self._h), self._h)

    def set_timing(self, mode=1):
        """0 off, 1 per stage, 2 per kernel launch (accumulating)."""
        _check(lib.rb_tree_set_timing(self._h, int(mode)), self._h)

    def launch_counts(self):
        f = _lib.C.c_int64()
        s = _lib.C.c_int64()
        _check(lib.rb_tree_launch_counts(self._h, _lib.C.byref(f), _lib.C.byref(s)), self._h)
        return f.value, s.value

    # -- beyond the reference: device-side inputs and persistence ------------------------------------
    def sample_device(self, kind: int, count: int, params, d_f: int = 0, d_g: int = 0, sync: bool = True):
        """rb_tree_sample_device: a standard potential / right-hand-side family evaluated on the
        device into the device arrays at addresses d_f, d_g (0 for none)."""
        par = np.ascontiguousarray(np.asarray(params, dtype=np.float64).ravel())
        _check(lib.rb_tree_sample_device(self._h, int(kind), int(count), _lib.dptr(par),
                                         _lib.C.c_void_p(int(d_f) or None), _lib.C.c_void_p(int(d_g) or None),
                                         1 if sync else 0), self._h)

    def save(self, path: str):
        """Writes the factorized tree to `path` (rb_tree_save)."""
        _check(lib.rb_tree_save(self._h, str(path).encode()), self._h)

    @classmethod
    def load(cls, path: str) -> "robin_tree":
        """A factorized tree from a file written by save (rb_tree_load), ready to solve."""
        h = _lib.C.c_void_p()
        _check(lib.rb_tree_load(str(path).encode(), _lib.C.byref(h)))
        T = cls()
        T._h = h
        T._info = T.info()
        T.factored = True
        T.nlvls = 0
        return T


def get_solution(T: robin_tree, irhs: int = 0):
    """get_solution(T, u) (robin_output_module.f90:48-75): leaf_solution per leaf, DFS order."""
    if not T.factored:
        raise RobinSolverError(_lib.RB_ERR_NOT_FACTORED, "Error in GET_SOLUTION: Robin Tree not factored.")
    inf = T._info
    u = np.zeros((inf.nleaves, inf.leaf_n), dtype=np.complex128)
    boxes = np.zeros((inf.nleaves, 6), dtype=np.float64)
    _check(lib.rb_get_solution(T.handle, irhs, _lib.dptr(u), _lib.dptr(boxes)), T.handle)
    out = []
    for i in range(inf.nleaves):
        box = np.array([[boxes[i, 0], boxes[i, 2], boxes[i, 4]], [boxes[i, 1], boxes[i, 3], boxes[i, 5]]])
        out.append(leaf_solution(box=box, u=u[i].copy()))
    return out


def check_solution(T: robin_tree, true_sol, irhs: int = 0, norm: str = "M", rel: bool = False) -> np.ndarray:
    """check_solution(d, leaf_sol, true_sol, opts, error_vec, norm, rel)
    (robin_output_module.f90:84-134) for right-hand side `irhs` of the last solve: per leaf, the
    1-, 2- or max-norm ('1', '2', anything else) of u - u_exact, or of (u - u_exact)/u_exact when
    `rel`.  `true_sol` is vectorised over an (npts, 3) array of points; the solution stays on the
    device."""
    if not T.factored:
        raise RobinSolverError(_lib.RB_ERR_NOT_FACTORED, "Error in GET_SOLUTION: Robin Tree not factored.")
    X = T.sample_points(_lib.RB_POINTS_SOLUTION)
    ue = np.ascontiguousarray(np.asarray(true_sol(X), dtype=np.complex128))
    err = np.zeros(T._info.nleaves, dtype=np.float64)
    code = {"1": 1, "2": 2}.get(str(norm), 0)
    _check(lib.rb_check_solution(T.handle, int(irhs), _lib.dptr(ue), code, 1 if rel else 0, _lib.dptr(err)), T.handle)
    return err


class robin_server:
    """Resident factorized trees behind a continuously batched request loop (rb_server_*; no
    counterpart in the reference, which solves one right-hand side per call).

    Solve requests queued for a tree while its previous sweep runs are merged into one batched
    sweep; trees run concurrently; a tree's first factorization is admitted against the device
    memory budget.  Host arrays handed to ``submit_solve`` are kept referenced here until the
    request is collected with ``wait``."""

    def __init__(self, device_budget: int = 0, max_batch_rhs: int = 64, precision: str = "fp64",
                 tol: float = 1e-10):
        o = _lib.rb_server_opts()
        o.device_budget = int(device_budget)
        o.max_batch_rhs = int(max_batch_rhs)
        o.precision = PRECISIONS[precision]
        o.tol = float(tol)
        h = _lib.C.c_void_p()
        _check(lib.rb_server_create(_lib.C.byref(o), _lib.C.byref(h)))
        self._h = h
        self._keep = {}

    def _err(self, code):
        if code != _lib.RB_OK:
            msg = lib.rb_server_last_error(self._h)
            raise RobinSolverError(code, msg.decode() if msg else "")

    def close(self):
        if self._h is not None:
            lib.rb_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def now(self) -> float:
        return lib.rb_server_now(self._h)

    def add_tree(self, L, ell_op, opts, bndry_params) -> int:
        g = make_geom(L, ell_op, opts, bndry_params)
        tid = _lib.C.c_int32()
        self._err(lib.rb_server_add_tree(self._h, _lib.C.byref(g), _lib.C.byref(tid)))
        return tid.value

    def tree_info(self, tid: int) -> _lib.rb_info:
        inf = _lib.rb_info()
        self._err(lib.rb_server_tree_info(self._h, int(tid), _lib.C.byref(inf)))
        return inf

    def submit_factor(self, tid: int, k=None, bumps=None, arrival: float = -1.0) -> int:
        """k: potential samples at RB_POINTS_POTENTIAL, or bumps = (kb, delta, w, [(cx, cy, a), ...])
        for the bump potential sampled on the device."""
        req = _lib.C.c_int64()
        if k is not None:
            kv = np.ascontiguousarray(k, dtype=np.complex128)
            self._err(lib.rb_server_submit_factor(self._h, int(tid), _lib.dptr(kv), 0, None, float(arrival),
                                                  _lib.C.byref(req)))
        else:
            kb, delta, w, cs = bumps
            par = np.ascontiguousarray(np.concatenate([[kb, delta, w], np.asarray(cs, dtype=np.float64).ravel()]))
            self._err(lib.rb_server_submit_factor(self._h, int(tid), None, len(cs), _lib.dptr(par), float(arrival),
                                                  _lib.C.byref(req)))
        return req.value

    def submit_solve(self, tid: int, nrhs: int, field: int = -1, params=None, f=None, g=None, u=None,
                     arrival: float = -1.0) -> int:
        """field = RB_FIELD_POINT_SOURCE / RB_FIELD_PLANE_WAVE with 3 params per right-hand side,
        or host arrays f (nrhs, n_interior) and g (nrhs, root_nb) (None = zero).  u: complex128
        array of nrhs * nleaves * leaf_n elements receiving the solutions (None: not copied)."""
        req = _lib.C.c_int64()
        keep = []
        par = None
        if params is not None:
            par = np.ascontiguousarray(np.asarray(params, dtype=np.float64).ravel())
            keep.append(par)
        fp = gp = up = None
        for arr in (f, g, u):
            if arr is not None:
                if not (isinstance(arr, np.ndarray) and arr.dtype == np.complex128 and arr.flags.c_contiguous):
                    raise RobinSolverError(_lib.RB_ERR_INVALID, "host arrays must be C-contiguous complex128")
                keep.append(arr)
        fp = f.ctypes.data if f is not None else None
        gp = g.ctypes.data if g is not None else None
        up = u.ctypes.data if u is not None else None
        self._err(lib.rb_server_submit_solve(self._h, int(tid), int(nrhs), int(field),
                                             _lib.dptr(par) if par is not None else None, fp, gp, up,
                                             float(arrival), _lib.C.byref(req)))
        self._keep[req.value] = keep
        return req.value

    def wait(self, req: int, timeout: float = -1.0) -> bool:
        """True once the request completed (raises on its error), False at the timeout."""
        rc = lib.rb_server_wait(self._h, int(req), float(timeout))
        if rc == 1:
            return False
        self._keep.pop(req, None)
        self._err(rc)
        return True

    def stats(self, reset: bool = False) -> dict:
        st = _lib.rb_server_stats()
        self._err(lib.rb_server_get_stats(self._h, _lib.C.byref(st), 1 if reset else 0))
        return {name: getattr(st, name) for name, _ in st._fields_}


class robin_forest:
    """Several robin_tree handles factored together in one level-synchronous schedule with
    autotuned GEMM tile shapes (rb_forest_*; no counterpart in the reference).  The trees must be
    planned (``robin_tree.plan``); after ``factor`` each is factored and solves as usual."""

    def __init__(self, trees):
        self.trees = list(trees)
        arr = (_lib.C.c_void_p * len(self.trees))(*[t.handle for t in self.trees])
        h = _lib.C.c_void_p()
        _check(lib.rb_forest_create(arr, len(self.trees), _lib.C.byref(h)))
        self._h = h

    def _err(self, code):
        if code != _lib.RB_OK:
            msg = lib.rb_forest_last_error(self._h)
            raise RobinSolverError(code, msg.decode() if msg else "")

    def factor(self, d_k_ptrs, autotune: bool = True):
        """d_k_ptrs: device addresses of each tree's potential samples (e.g. tensor.data_ptr())."""
        arr = (_lib.C.c_void_p * len(self.trees))(*[int(p) for p in d_k_ptrs])
        self._err(lib.rb_forest_factor(self._h, arr, 1 if autotune else 0))
        for t in self.trees:
            t.factored = True
            t._info = t.info()

    def info(self):
        f = _lib.C.c_double()
        n = _lib.C.c_int64()
        tu = _lib.C.c_int32()
        self._err(lib.rb_forest_info(self._h, _lib.C.byref(f), _lib.C.byref(n), _lib.C.byref(tu)))
        return {"f_time": f.value, "launches": n.value, "tuned_stages": tu.value}

    def tuning(self):
        n = lib.rb_forest_tuning(self._h, None, None, None, None, 0)
        h = (_lib.C.c_int32 * max(n, 1))()
        st = (_lib.C.c_int32 * max(n, 1))()
        en = (_lib.C.c_int32 * max(n, 1))()
        ms = (_lib.C.c_double * max(n, 1))()
        lib.rb_forest_tuning(self._h, h, st, en, ms, n)
        return [(h[i], st[i], lib.rb_gemm_engine_name(en[i]).decode(), ms[i]) for i in range(n)]

    def close(self):
        if self._h is not None:
            lib.rb_forest_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
