// alternative shape for 96 x 96 windows: 192 threads, 2 CTAs per SM
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_VARIANT(96v2, 96, 16, 192, 2)
