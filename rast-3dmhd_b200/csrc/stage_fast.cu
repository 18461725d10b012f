// Fast build of the step kernels: the same source with FMA contraction.
#define MHD3D_NS fast
#include "stage_impl.cuh"
