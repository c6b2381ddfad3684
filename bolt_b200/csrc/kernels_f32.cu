// FP32 kernels: f and stencil arithmetic in FP32 with FMA and approximate
// reciprocals; moments, the BGK Maxwellian and the divergence check in FP64.
#define BOLT_T float
#define BOLT_EXACT false
#define BOLT_SUFFIX f32
#include "kernels_impl.cuh"
