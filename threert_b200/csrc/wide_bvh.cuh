// The wide BVH: the reference's binary trees collapsed to 8-wide nodes with quantised child boxes (declared here;
// built in wide_bvh.cu).
#pragma once
#include "traverse.cuh"

struct trt_ctx;
struct trt_scene_desc_s;

namespace trt {

struct WideView {
    const uint4* nodes;   // 5 uint4s a node
    uint32_t top_root;    // the top tree's root node
    uint32_t valid;
};

struct WideBvh {
    uint4* nodes = nullptr;
    uint64_t n_nodes = 0;
    uint32_t top_root = 0;
    bool built = false;
    bool ready() const { return built; }
    WideView view() const { return WideView{nodes, top_root, built ? 1u : 0u}; }
    int build(trt_ctx*, const DScene&, const void*, cudaStream_t) { built = false; return 0; }
    int refit(trt_ctx*, const DScene&, cudaStream_t) { return 0; }
    void release() {}
};

template <bool COUNT>
__device__ __forceinline__ Hit trace_wide(const DScene& S, const WideView& W, const Sections& X, V3 o, V3 d, float tmax,
                                          uint32_t mode, WalkCount* wc, bool* guard) {
    (void)W;
    return trace_binary<COUNT>(S, X, 0u, 0u, o, d, tmax, mode, wc, guard);
}

}  // namespace trt
