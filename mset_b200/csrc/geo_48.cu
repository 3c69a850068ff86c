// kernels for 48 x 48 windows
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO(48, 16, 192, 2)
