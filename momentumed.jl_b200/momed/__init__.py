"""momed: B200 backend for MomentumED.jl's matrix-free Hamiltonian map and Lanczos eigensolve.

A drop-in for the path EDsolve(subspace, H::MBOperator; method=:map, device=:gpu):
the host API mirrors the reference's names (EDPara, ED_momentum_subspaces,
ED_scatterlist_onebody/twobody, Scatter, MBOperator, HilbertSubspace,
MBS64Vector, EDsolve) and every compute step runs in libmomed_b200.so (CUDA,
sm_100a) through its C ABI.  There is no CPU fallback.
"""
from ._lib import Handle, MomedError, NotConverged, Server, version
from .analysis import ED_bracket, ED_bracket_threaded, ED_connection_gaugefixing, ED_step_inner_prod, PES_1rdm
from .core import (MBS64, HilbertSubspace, MBOperator, MBS64Vector, Scatter, ScatterList, hermitian_complete,
                   index_fit, make_mask64, occ_list, parity_mask, scat_occ_number, sort_merge_scatlist)
from .methods import (DEFAULT_GPU, GPU_AVAILABLE, EDsolve, LinearMap, activate_b200, activate_gpu_device,
                      create_gpu_linearmap, create_gpu_matrix, krylov_map_solve, krylov_matrix_solve,
                      release_gpu_memory)
from .recipes import KShiftOperator, LandauCoulomb, kshift_sweep
from .preparation import (ED_momentum_subspaces, ED_scatterlist_onebody, ED_scatterlist_twobody,
                          ED_sortedScatterList_onebody, ED_sortedScatterList_twobody, EDPara, MBS_totalmomentum,
                          group_momentum_pairs, momentum_residue)

__all__ = [
    "Handle", "MomedError", "NotConverged", "Server", "version", "ED_bracket", "ED_bracket_threaded", "PES_1rdm",
    "ED_step_inner_prod", "ED_connection_gaugefixing",
    "MBS64", "HilbertSubspace", "MBOperator", "MBS64Vector", "Scatter", "ScatterList", "hermitian_complete",
    "index_fit", "make_mask64", "occ_list", "parity_mask", "scat_occ_number", "sort_merge_scatlist",
    "DEFAULT_GPU", "GPU_AVAILABLE", "EDsolve", "LinearMap", "activate_b200", "activate_gpu_device",
    "create_gpu_linearmap", "create_gpu_matrix", "krylov_map_solve", "krylov_matrix_solve", "release_gpu_memory",
    "ED_momentum_subspaces", "ED_scatterlist_onebody", "ED_scatterlist_twobody", "ED_sortedScatterList_onebody",
    "ED_sortedScatterList_twobody", "EDPara", "MBS_totalmomentum", "group_momentum_pairs", "momentum_residue",
    "KShiftOperator", "LandauCoulomb", "kshift_sweep",
]
