// The learned denoiser as the serving loop uses it (unet.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "threert_cuda.h"

// The denoise of a device accum (rendered with TRT_RENDER_DEPTH) on the caller's stream, into the network's own RGB
// buffer (h * w * 3 floats, valid until the network's next use): its device pointer, or null when the image is not a
// size the network takes. The network must not be used from elsewhere while a server owns it.
const float* unet_denoise_on_stream(trt_unet* net, const void* accum_device, uint32_t w, uint32_t h, cudaStream_t st);
// Whether the network takes a w x h image (within its size, multiples of 8).
bool unet_fits(const trt_unet* net, uint32_t w, uint32_t h);
