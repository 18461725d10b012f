// Fast build of the step kernels: FMA contraction, and a right-hand side
// regrouped with pre-multiplied metric factors (same equations, different
// rounding; within 1e-11 of the reference-rounding build after 10 steps).
#define MHD3D_NS fast
#define MHD3D_FAST_BODY 1
#include "stage_impl.cuh"
