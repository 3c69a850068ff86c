// alternative shape for 64 x 64 windows: 128 threads, up to 4 CTAs per SM
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_VARIANT(64v2, 64, 8, 128, 4)
