// alternative shape for 128 x 128 windows: 256 threads with up to 255 registers
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_VARIANT(128v2, 128, 16, 256, 1)
