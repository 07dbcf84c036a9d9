"""grico_b200 — B200-native matrix-free runtime for Grico.jl's hot path.

Host-side mirror of Grico.jl's public API for this path (Domain, HpSpace, AffineProblem,
add_cell_accumulator!, Dirichlet, compile, apply!, solve) on top of the C ABI of
libgrico_b200.so (include/grico_b200.h).  All compute runs in the library's sm_100a kernels.
"""
from ._lib import GricoError, lib
from .mesh import LOWER, UPPER, CartesianGrid, Domain, grid, refine, uniform_refine
from .space import (AxisDegrees, ByLeafDegrees, DegreePlusQuadrature, FullTensorBasis, HpSpace, SpaceOptions,
                    StoredDegrees, TrunkBasis, UniformDegree, active_leaf_count, scalar_dof_count)
from .problem import (SPD, AffineProblem, AssemblyPlan, BoundaryFace, CGSolver, Diffusion, Dirichlet, FGMRESSolver,
                      IdentityPreconditioner, JacobiPreconditioner, Load, Mass, MassDiffusion, Nitsche,
                      NonsymmetricOperator, SIPG, ScalarField, State, VariableDiffusion, add_boundary,
                      add_boundary_accumulator, add_interface,
                      add_cell_accumulator, add_cell_quadrature, add_constraint, add_surface_accumulator,
                      add_surface_quadrature, apply, apply_, compile, expand_reduced, l2_error, reduced_apply,
                      reduced_diagonal, reduced_rhs, relative_l2_error, rhs, solve)
from .regions import (FiniteCellExtension, ImplicitRegion, PhysicalDomain, PhysicalMeasure, SurfaceQuadrature,
                      finite_cell_quadrature, sphere_surface_quadrature)
from .multigrid import GeometricMultigridPreconditioner
from .nonlinear import ExpReaction, ResidualProblem, add_residual_accumulator, newton_solve
from .nonlinear import compile as compile_residual
from .sharded import ShardedOperator, ShardGroup, ShardPlan, sharded_cg
