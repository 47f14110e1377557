"""femahoy_b200: the fh-fem iterative solve path of femahoy (global stiffness assembly of
P1/P2 tetrahedral heat and elasticity, PCG with a geometric / p-multigrid V-cycle and a dense
coarse Cholesky) on one B200, behind the C ABI of include/femgpu.h (libfemgpu.so).

The Python names mirror the reference crate: ``Csr`` (sparse.rs), ``Solver``, ``Unknowns``,
``Method``, ``Crossover``, ``Stats`` (solve.rs), ``Level`` (multigrid.rs), ``prolongation``
(pmultigrid.rs), ``Quadratic`` (tet10.rs) and ``reduced_rhs`` (heat.rs); ``Recovery`` and
``Peak`` are the post-solve loop of elastic_tet.rs:367-427; ``prism`` the reference's prism
meshes (prism.rs, mesh2d.rs) and ``grid`` its box grid (grid.rs Grid::build).
"""
from ._lib import (COLOUR, FP64, GATHER, HEX8_ELASTIC, HEX8_HEAT, HEX8_MASS, MIXED, P1_ELASTIC, P1_HEAT, P2_ELASTIC,
                   P2_ELASTIC_ORTHO, P2_MASS, FemError, LIB_PATH, lib)
from .solve import (PCG_MAX_ITER, PCG_TOL, STEADY_DIRECT_LIMIT, TRANSIENT_DIRECT_LIMIT,
                    Cells, Convergence, Crossover, Level, Method, Options, Quadratic, Solver,
                    Stats, Unknowns, coarse_matrix, hex_elements, hex_mass, pcg, prolongation,
                    reduced_rhs, symbolic_counts)
from .recover import Peak, Reactions, Recovery, reactions
from .sparse import Csr, Rect, colour
from . import grid, prism

__all__ = [
    "COLOUR", "FP64", "GATHER", "HEX8_ELASTIC", "HEX8_HEAT", "HEX8_MASS", "MIXED", "P1_ELASTIC", "P1_HEAT", "P2_ELASTIC", "P2_ELASTIC_ORTHO", "P2_MASS",
    "FemError",
    "LIB_PATH", "lib", "PCG_MAX_ITER", "PCG_TOL", "STEADY_DIRECT_LIMIT",
    "TRANSIENT_DIRECT_LIMIT", "Cells", "Crossover", "Level", "Method", "Options", "Quadratic",
    "Solver", "coarse_matrix", "hex_elements", "hex_mass", "symbolic_counts",
    "Stats", "Unknowns", "prolongation", "reduced_rhs", "Csr", "Rect", "colour", "Peak",
    "Recovery", "Reactions", "reactions", "grid", "prism", "pcg", "Convergence",
]
