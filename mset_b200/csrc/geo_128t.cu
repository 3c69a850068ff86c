// kernels for 128 x 128 windows in the three-phase shape (four shared-memory
// round trips per propagation slab)
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO3(128t, false)
