"""petch_b200 -- B200-native drop-in for petch's per-step 3D etch loop.

The public surface mirrors petch (Domain / SF6O2 / Process / Result, run_etch_3d,
mc_flux_3d_coupled, Flags, PAR); every stage runs as hand-written sm_100a CUDA kernels in
libpetchb200.so, reached through a C ABI (include/petch_b200.h) with ctypes.
"""
from . import _lib
from .params import PAR, Flags, DEFAULT_FLAGS
from .levelset import (reinit_fsm, reinit_gpu, advect_3d_gpu, reinit_fsm_dev, advect_dev, seed_field,
                       grid_shape)
from .threed import (make_trench_3d, run_etch_3d, extract_mesh_3d, extract_mesh_3d_device,
                     mc_flux_3d_coupled, mc_flux_3d_radiosity, mc_flux_3d_dda, mc_flux_3d_knudsen,
                     center_depth_3d, max_depth_3d, DeviceMesh, FluxEngine, EtchEngine)
from .dda import dda_neutral_flux
from .knudsen import knudsen_face_flux

from .api import Domain, SF6O2, Process, Result

__all__ = ["Domain", "SF6O2", "Process", "Result", "PAR", "Flags", "DEFAULT_FLAGS", "run_etch_3d",
           "make_trench_3d", "extract_mesh_3d", "extract_mesh_3d_device", "mc_flux_3d_coupled",
           "mc_flux_3d_radiosity", "mc_flux_3d_dda", "dda_neutral_flux",
           "mc_flux_3d_knudsen", "knudsen_face_flux", "center_depth_3d",
           "max_depth_3d", "reinit_fsm", "reinit_gpu", "advect_3d_gpu", "DeviceMesh", "FluxEngine",
           "EtchEngine"]

__version__ = "0.1.0"
