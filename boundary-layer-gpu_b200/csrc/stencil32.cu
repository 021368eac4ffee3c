// stencil32.cu -- FP32 (mixed form) instantiation of the stencil kernels
#define BLGPU_STENCIL_T float
#include "stencil_impl.cuh"
