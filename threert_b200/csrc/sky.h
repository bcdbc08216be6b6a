// The atmosphere's sky on the device (renderer/src/sky.rs): the optical-depth and multiple-scattering tables
// (Luts::build, sky.rs:386-433), the equirectangular bake (bake_atmosphere_with, sky.rs:722-819) and the environment's
// importance tables (lib.rs:916-941 build_env_cdf) with its RGBA16F texels. Launched by the C ABI in pathtrace.cu.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "threert_cuda.h"

struct SkyState;

// The bake of `a` into the state's f32 texels (width x height float4, device), the tables built first unless the
// state holds those of the same atmosphere. Results (sun illuminance, horizon_v) land in `out` after a sync; with
// `texels_host` / `tables_host` the arrays are copied back too. 0 or a TRT_E* code with `err` set.
int sky_bake(SkyState** st, int device, cudaStream_t stream, const trt_atmosphere& a, float* texels_host,
             float* tables_host, trt_sky_result* out, std::string* err);

// The last bake as a scene's environment: RGBA16F texels into `env` (width x height), the CDF (height marginal
// entries, then width x height conditional ones) into `cdf`, the brightest luminance into out->brightest. `sin_rows`:
// the host's sin((y + 0.5) / height * pi) for each row, so that the CDF rounds as the host prep's does.
int sky_env(SkyState* st, cudaStream_t stream, const float* sin_rows_host, void* env, float* cdf, trt_sky_result* out,
            std::string* err);

// The f32 texels of the last bake (device).
const float4* sky_texels(const SkyState* st);

void sky_free(SkyState* st);
