// alternative for 256 x 256 windows: one field over a cluster of 4 CTAs,
// the saved-wave rows loaded from global memory into registers
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_CL(256, 16, 512, 4)
