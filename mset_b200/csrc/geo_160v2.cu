// alternative shape for 160 x 160 windows: 320 threads with up to 204 registers
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_VARIANT(160v2, 160, 16, 320, 1)
