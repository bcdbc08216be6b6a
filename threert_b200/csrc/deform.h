// The per-frame deformation of a resident scene (host side, internal to the library): skinning, leaf gather, mesh-tree
// refit, unit boxes and the top tree's rebuild, all on the device. The C entry points (trt_deform_setup, trt_deform in
// threert_cuda.h) are in pathtrace.cu and call these.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "threert_cuda.h"

namespace trt {

struct DeformState;

// What the deformation needs of a trt_scene: its five device buffers (vertices, leaves, nodes, tables, words), their
// sizes, the stream, and the host copies of leaves, nodes and tables kept at upload.
struct SceneBuffers {
    void* buf[5];
    uint64_t bytes[5];
    cudaStream_t stream;
    const std::vector<uint8_t>* host;  // host[5], entries 1-3 filled
};

int deform_setup(DeformState** out, const SceneBuffers& sb, const trt_deform_desc* d, std::string& err);
int deform_run(DeformState* st, const SceneBuffers& sb, const uint32_t* params, const float* palette_rows,
               uint32_t n_matrices, uint32_t flags, trt_deform_stats* stats, std::string& err);
// Errors the device recorded since the last call (bad trees, a top tree deeper than it may be); resets them.
int deform_errors(DeformState* st, cudaStream_t stream, uint32_t* errors);
// The device word the errors are recorded in; DEFORM_E_WIDE is the bit the wide BVH's refit sets in it.
uint32_t* deform_error_word(DeformState* st);
constexpr uint32_t DEFORM_E_WIDE = 16u;
void deform_free(DeformState* st);

}  // namespace trt
