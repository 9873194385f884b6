"""mhdarcy: B200-native mixed-hybrid Darcy flow (Flow123d's MH hot path) over a C ABI."""
from ._lib import (MHError, device_available, lib, MH_BC_NONE, MH_BC_DIRICHLET, MH_BC_NEUMANN,
                   MH_BC_ROBIN, MH_SOLVER_PCG64, MH_SOLVER_IR32, MH_SOLVER_CHEB,
                   MH_SOLVER_FCG_LEARNED, MH_SOLVER_AMG, MH_OK, MH_NOT_CONVERGED, MH_FELL_BACK, LIB_PATH)
from .mesh import Mesh, concat_meshes, cube_mesh, read_element_data, read_gmsh
from .flow import (MHSystem, MH_DofHandler, DarcyFlowMH_Steady, DarcyFlowMH_Unsteady,
                   DarcyFlowLMH_Unsteady, solve_opts, write_raw_output)

__all__ = [n for n in dir() if not n.startswith("_")]
