"""B200-native force path of TREE (hpjeonGIT/TREE): octree build, one-level
multipole upward pass, Barnes-Hut walk with Kelbg-regularised pair laws and a
fused velocity-Verlet step, behind the C ABI of include/tree_gpu.h."""
from . import cloud, units  # noqa: F401
from .api import (Config, Ensemble, TreeForce, TreeGpuError, load_library,  # noqa: F401
                  MAC_FIXED, MAC_LEARNED, PHYS_KELBG, PHYS_REF, PREC_FP64,
                  PREC_MIXED, RDF_BINS)
