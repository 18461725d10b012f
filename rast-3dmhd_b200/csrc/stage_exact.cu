// Reference-rounding build of the step kernels: compiled with -fmad=false so
// every multiply and add is rounded on its own, in the reference's order.
#define MHD3D_NS exact
#include "stage_impl.cuh"
