"""B200-native hierarchical Poincare-Steklov (HPS) factor/solve for 2D variable-potential
Helmholtz problems: robinsolver's factor/solve path on sm_100a behind its own API.

The compute path is librobin_b200.so (C-ABI in include/robin_b200.h); this package is the
host-side mirror of the reference's Fortran interface plus the seeded benchmark workloads.
The API names load the shared library on first use (``robinsolver_b200.build`` and
``robinsolver_b200.workloads`` do not need it).
"""
_API = ("RobinSolverError", "bndry_rhs", "check_solution", "debug_opts", "elliptic_operator", "elliptic_rhs",
        "get_solution", "leaf_solution", "robin_forest", "robin_server", "robin_tree", "scalar_callback", "solve_opts")

__all__ = list(_API)


def __getattr__(name):
    if name in _API:
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
