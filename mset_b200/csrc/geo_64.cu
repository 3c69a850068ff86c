// kernels for 64 x 64 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(64, 8, 256, 2)
