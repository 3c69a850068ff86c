// the three-phase shape of 128 x 128 windows with 16-byte phase-2 accesses
// (rows padded to 168 elements)
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO3(128w, true)
