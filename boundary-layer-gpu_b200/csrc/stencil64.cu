// stencil64.cu -- FP64 instantiation of the stencil kernels (-fmad=false)
#define BLGPU_STENCIL_PRIMARY
#define BLGPU_STENCIL_T double
#include "stencil_impl.cuh"
