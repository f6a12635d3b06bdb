"""B200-native drop-in for PyQrackIsing's dense cut-scoring and local-search path.

Public API (same signatures and return tuples as the reference):
  maxcut_tfim(G, quality, shots, is_spin_glass, anneal_t, anneal_h,
              repulsion_base, is_maxcut_gpu, is_nested)
  spin_glass_solver(G, quality, shots, best_guess, is_maxcut_gpu, is_spin_glass,
                    anneal_t, anneal_h, repulsion_base, is_log, gray_iterations,
                    gray_seed_multiple, bp_scale, bp_damping)
  maxcut_tfim_sparse / spin_glass_solver_sparse (CSR or graph input)
  spin_glass_solver_hybrid (dense maxcut_tfim seed, then the sparse solver)
  solve_maxcut_bnb(G, best_guess, quality, shots, is_spin_glass, anneal_t, anneal_h,
                   repulsion_base, is_maxcut_gpu, verbose, time_limit,
                   gray_iterations, gray_seed_multiple[, batch_size])
  solve_maxcut_bnb_sparse (same, CSR or graph input)
  tsp_symmetric / tsp_asymmetric(G, start_node, end_node, quality, shots,
                  anneal_t, anneal_h, repulsion_base, monte_carlo, k_neighbors,
                  is_cyclic, multi_start, is_top_level, is_parallel, parallel_level)
                  (MAXCUT splits on the device for monte_carlo=False)

All arithmetic on the coupling matrix runs in libpqi.so (hand-written sm_100a
CUDA behind the C ABI in include/pqi.h); there is no CPU fallback.
"""

from .maxcut_tfim import maxcut_tfim
from .spin_glass_solver import spin_glass_solver
from .solve_maxcut_bnb import solve_maxcut_bnb, solve_maxcut_bnb_sparse
from .sparse import maxcut_tfim_sparse, spin_glass_solver_hybrid, spin_glass_solver_sparse

__all__ = ["maxcut_tfim", "spin_glass_solver", "maxcut_tfim_sparse", "spin_glass_solver_sparse",
           "spin_glass_solver_hybrid",
           "solve_maxcut_bnb", "solve_maxcut_bnb_sparse", "tsp_symmetric", "tsp_asymmetric"]


def __getattr__(name):
    # the TSP module (numba-compiled path heuristics) loads on first use
    if name in ("tsp_symmetric", "tsp_asymmetric"):
        from . import tsp

        return getattr(tsp, name)
    raise AttributeError(name)
