"""B200-native dense ZNCC tracker with AutoRIFT.jl's API.

Loaded under the module name ``autorift_b200`` (the directory name is not an identifier);
``__graft_entry__.load_package()`` registers it.
"""

from . import _lib, synthetic
from .methods import (Coherence, GardnerFilter, Highpass, NCC, NoOutlierFilter, NoPreprocess,
                      NoQuantize,
                      NoRefine, NoRotationSearch, Params, PyramidRefine, QuantizeUInt8,
                      RotationSearch, Wallis, ZNCC, angles, chip_sizes, params, upsampling)
from .points import (PointSet, gridpoints, gridpoints_xy, nsearchable, npoints, pointset,
                     sanitize)
from .api import (Ticket, submit, multichip_params, Cache, MultichipResult, autorift, autorift_, build_grid, correlate_multichip,
                  init, reinit_)
from .track import (DisplacementField, ImagePair, PreparedPair, correlate, displacement_field,
                    nmeasured, prepare, prepare_options, refine_patches, track)

__all__ = [
    "GardnerFilter", "Highpass", "NCC", "NoOutlierFilter", "NoPreprocess", "NoQuantize",
    "NoRefine", "Params", "PyramidRefine", "QuantizeUInt8", "Wallis", "ZNCC", "chip_sizes",
    "params", "upsampling", "PointSet", "gridpoints", "gridpoints_xy", "nsearchable", "npoints",
    "pointset", "sanitize", "DisplacementField", "ImagePair", "correlate", "displacement_field",
    "nmeasured", "refine_patches", "track", "PreparedPair", "prepare", "Cache",
    "MultichipResult", "autorift", "autorift_", "build_grid", "correlate_multichip", "init",
    "reinit_", "prepare_options", "multichip_params", "submit", "Ticket", "NoRotationSearch",
    "RotationSearch", "angles", "Coherence",
]
