"""paragram_b200 -- B200-native (sm_100a) 3D Voronoi and power diagram construction.

Drop-in for ``paragram`` (paragram/__init__.py:1-7): same ``Diagram``,
``voronoi_diagram`` and ``power_diagram``. The work runs in the CUDA library
``libparagram_b200.so`` (C ABI: include/paragram_b200.h); there is no CPU
fallback -- calling the API without the built library raises ImportError.
"""

from ._api import Diagram, power_diagram, voronoi_diagram
from .batch import build_batch
from .geometry import cell_geometry, cell_vertices, face_areas
from .neighbours import knn

__all__ = [
    "Diagram",
    "build_batch",
    "cell_geometry",
    "cell_vertices",
    "face_areas",
    "knn",
    "power_diagram",
    "voronoi_diagram",
]
