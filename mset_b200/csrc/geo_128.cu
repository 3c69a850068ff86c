// kernels for 128 x 128 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(128, 16, 512, 1)
