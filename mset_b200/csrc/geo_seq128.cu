// 128 x 128 windows for the sequential modes: one field over a cluster of 8 CTAs (16 rows each)
#include "mset_kernels_impl.cuh"
MSET_DEFINE_SEQ_GEO_CL(128c8, 128, 16, 256, 8)
