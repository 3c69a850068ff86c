// kernels for 24 x 24 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(24, 8, 64, 8)
