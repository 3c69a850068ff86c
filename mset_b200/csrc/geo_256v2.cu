// alternative shape for 256 x 256 windows: 256 threads per CTA with up to 255 registers
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_CL_VARIANT(256v2, 256, 16, 256, 4, 1)
