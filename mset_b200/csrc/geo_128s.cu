// alternative for 128 x 128 windows: the default shape with the adjoint's saved-wave rows staged by bulk copies
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_STAGED(128s, 128, 16, 512, 1)
