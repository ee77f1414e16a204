"""haseongpu_b200 -- B200 (sm_100a) implementation of HASEonGPU's adaptive
Monte Carlo phi-ASE computation: the backward, importance-sampled method on
extruded triangle-prism meshes and the forward method on Tet4 meshes.

The compute path is libhase_b200.so (hand-written CUDA behind the C ABI of
include/hase_b200.h and include/hase_b200_forward.h); this package is its host
front end, mirroring the reference's ``PhiASE`` / ``Result`` call surface.
"""

from .batch import MediaBatch
from .forward import TetDeviceMesh
from .mesh import PrismMesh
from .simulation import DeviceMesh, PhiASE, Result
from .spectra import CrossSectionData, interpolate_linear
from .tetmesh import TetMesh

__all__ = ["PrismMesh", "TetMesh", "DeviceMesh", "TetDeviceMesh", "MediaBatch", "PhiASE", "Result", "CrossSectionData",
           "interpolate_linear"]
__version__ = "0.1.0"
