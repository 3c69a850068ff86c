// kernels for 96 x 96 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(96, 16, 384, 1)
