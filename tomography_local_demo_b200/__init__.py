"""B200-native (sm_100a) streaming FDK/FBP filter and slice-on-demand back-projection,
a drop-in for minirecast's recon / preprocess / model paths."""
from .geometry import ParallelGeometry, ConeVecGeometry, circular_cone_vectors
from .recon import SliceReconstructor, HAVE_CUDA

HAVE_NUMBA = False      # the reference's flag; this package never uses Numba

__version__ = "0.1.0"
