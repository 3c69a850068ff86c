// kernels for 160 x 160 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(160, 16, 640, 1)
