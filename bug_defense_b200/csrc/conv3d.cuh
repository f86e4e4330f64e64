// Internal launch interface of the denoiser's convolution kernels (used by the U-Net driver).
#pragma once

#include <cuda_runtime.h>

#include "../../include/bugdef.h"

namespace bd {

int conv_check(const BdConvCall& c);
// Enqueue one convolution; *err (device) is set if a bounded pipeline wait timed out.
int conv_launch(const BdConvCall& c, cudaStream_t st, int* err);
int wgrad_launch(int nx, int ny, int nz, int cin, int cout, int taps, const void* grad, const void* act, float* dw,
                 cudaStream_t st, int* err);
int pack_weights_launch(int taps, int cin, int cout, int n_off, int n_slice, int transpose, const float* w, void* img,
                        cudaStream_t st);

}  // namespace bd
