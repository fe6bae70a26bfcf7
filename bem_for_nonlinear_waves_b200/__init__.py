"""B200-native (sm_100a) GMRES + fast-multipole Laplace boundary-value solver for BEM-MEL
nonlinear-wave simulation: a drop-in for the GMRES-FMM path of BEM_BVP::solve() of
tomoakihirakawa/BEM_for_Nonlinear_Waves.

    from bem_for_nonlinear_waves_b200 import BEM_BVP, make_tank
"""
from .bvp import BEM_BVP, BatchSolver, MELStage, build_dofs  # noqa: F401
from .tank import CONFIGS, add_box_body, make_tank, known_values, point_normals  # noqa: F401

__all__ = ["BEM_BVP", "BatchSolver", "MELStage", "build_dofs", "make_tank", "add_box_body", "known_values", "point_normals", "CONFIGS"]
