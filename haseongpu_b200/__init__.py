"""haseongpu_b200 -- B200 (sm_100a) implementation of HASEonGPU's adaptive
Monte Carlo phi-ASE computation on extruded triangle-prism meshes.

The compute path is libhase_b200.so (hand-written CUDA behind the C ABI of
include/hase_b200.h); this package is its host front end, mirroring the
reference's ``PhiASE`` / ``Result`` call surface.
"""

from .mesh import PrismMesh
from .simulation import DeviceMesh, PhiASE, Result
from .spectra import CrossSectionData, interpolate_linear

__all__ = ["PrismMesh", "DeviceMesh", "PhiASE", "Result", "CrossSectionData", "interpolate_linear"]
__version__ = "0.1.0"
