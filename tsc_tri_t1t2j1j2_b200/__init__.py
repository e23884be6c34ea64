"""B200 (sm_100a) superblock engine for the SU(2) DMRG of the t1-t2-J1-J2 model on
triangular cylinders: drop-in for the hot path of hyx15903/TSC_Tri_t1t2J1J2
(Lanczos H.psi, density matrix + truncation, U^dagger O U, wave transformation).
"""
from .dmrg import Context, run_parameter_points  # noqa: F401
from .layout import Basis, Block, Cursor, Model, Wave, pack  # noqa: F401
