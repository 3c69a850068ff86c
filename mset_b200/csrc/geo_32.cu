// kernels for 32 x 32 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(32, 8, 128, 4)
