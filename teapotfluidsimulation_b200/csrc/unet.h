// Learned-preconditioner U-Net (unet.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace pl {

struct UNetImpl;

UNetImpl* unet_create(uint32_t seed, char* err, size_t errlen, int* rc);
void unet_destroy(UNetImpl* u);
int unet_nparams(const UNetImpl* u);
void unet_set_loss(UNetImpl* u, int kind);
int unet_set_conv_kernel(UNetImpl* u, int kind);
int unet_error(UNetImpl* u);
int unet_get_params(UNetImpl* u, float* host);
int unet_set_params(UNetImpl* u, const float* host);
int unet_prepare(UNetImpl* u, int X, int Y, int Z, int count, char* err, size_t errlen);
int unet_apply(UNetImpl* u, const uint8_t* cell, const float* r, float* z, int X, int Y, int Z, int count,
               cudaStream_t st, char* err, size_t errlen);
int unet_gradient(UNetImpl* u, const uint8_t* cell, const float* r, const float* e, int X, int Y, int Z, int count,
                  float lr, int update, float* loss, float* grad_host, cudaStream_t st, char* err, size_t errlen);

}  // namespace pl
