// kernels for 256 x 256 windows (the default shape): one field over a 4-CTA
// cluster, the adjoint's saved-wave rows staged by bulk copies
#include "mset_kernels_impl.cuh"
MSET_DEFINE_GEO_CL_STAGED(256s, 256, 16, 512, 4)
