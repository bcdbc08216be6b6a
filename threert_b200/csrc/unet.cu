// The learned denoiser's kernels: a 4-level U-Net (32 / 64 / 96 / 128 channels, 3 x 3 convolutions) over the pass's
// radiance, albedo, normal and depth, its forward pass, its backward pass and its optimiser, all hand-written. It has
// no counterpart in the reference (whose learned denoiser is the external OIDN library, renderer/src/denoise.rs:80-103).
//
// Tensors are NHWC bf16 with channel counts padded to multiples of 32; a convolution is an implicit GEMM (M = pixels,
// N = output channels, K = 9 taps x input channels) on the 5th-generation tensor cores (TMA loads, tcgen05.mma into
// tensor memory, f32 accumulation). The input gradient is the same kernel run on the output gradient with the
// weights flipped and transposed; the weight and bias gradients are one GEMM over pixels on the same tensor cores
// (both operands MN-major, split across CTAs whose f32 partials a second kernel sums in a fixed order, so that training
// is deterministic). Master weights, gradients and Adam's moments are f32.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "threert_cuda.h"
#include "unet.h"

namespace unet {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---- convolution (forward; and the input gradient with flipped, transposed weights) -------------------------------
//
// y[p][n] = bias[n] + sum over taps t and channels c of x[p + off(t)][c] * w[t][c][n], zero outside the image.
// A CTA computes a tile of 128 pixels (a bw x bh rectangle of one image, bw the largest power of two <= 128 that
// divides the width) x N output channels (N 128 where 128 divides co_pad, else 64; blockIdx.y their tile) on the
// 5th-generation tensor cores:
//  - one thread issues the loads: per K stage (one tap, 32 input channels) a TMA box of 32 channels x bw x bh pixels,
//    shifted by the tap (the halo and the image's border read as zeros), and a TMA box of the tap's weights (N
//    output channels x the 32 input channels); both land as 64-byte rows with the 64-byte swizzle, the canonical
//    K-major layout the MMA reads (8-row atoms of 512 bytes);
//  - one thread issues two tcgen05.mma (M 128, N, K 16, bf16 in, f32 accumulate in tensor memory) a stage and
//    commits each stage's buffers back to the loader through an mbarrier; TS stages in flight;
//  - where the layer reads one 32-channel block into one output tile (cin 32, co_pad = N), the nine taps' weight boxes
//    (36 KB) are loaded once a CTA into the weight stages' room, and a stage loads the activations alone;
//  - eight warps read the accumulator out of tensor memory (two a 32-lane quarter = 32 pixels, each half of the
//    columns), add the bias, apply the ReLU and store bf16 (or f32) NHWC.
// Every mbarrier wait is bounded (about a second); a wait that gives up sets the error word, and the CTA waits
// (bounded) for its copies and MMAs in flight and finishes.

struct Conv {
    uint32_t cin;             // channels read (a multiple of 32)
    uint32_t co_pad;          // a multiple of 64 (up to 256)
    uint32_t nt;              // output channels a CTA: 128 where they divide co_pad, else 64 (blockIdx.y the tile)
    const float* bias;        // co_pad, or null
    bf16* y;                  // output, NHWC
    uint32_t y_stride, y_off, cout;
    float* yf;                // or f32 output (stride cout), for the last layer
    uint32_t B, H, W, x_off;
    uint32_t bw, bh, tiles_x, tiles_y;
    int relu;
    uint32_t* err;
    uint32_t resident;        // 1: every tap's weights loaded once a CTA (one 32-channel block, one output tile)
    uint32_t hold;            // 1: CTA 0 withholds its first activation box (trt_unet_hold_next_load: a test of the
                              // bounded waits), so that the stage's wait runs out
    uint32_t stages;          // the halo variant's stages (HALO_TS with resident weights; 2 or 3 streaming them)
};

constexpr uint32_t TS = 5;                  // pipeline stages (82 KB of shared memory: two CTAs an SM)
constexpr uint32_t A_STAGE = 128u * 32u * 2u, B_STAGE = 128u * 32u * 2u;
constexpr uint32_t CONV_SMEM = TS * (A_STAGE + B_STAGE) + 256u + 1024u;  // + room to align the stages to 1 KB
// The halo variant (a row tile of 128 pixels read once with its halo, the taps as shifted descriptors): a stage is a
// 32-channel block as four planes of 8 channels x 3 rows x 130 pixels (16 bytes a pixel, each plane padded to a
// multiple of 128 bytes), the weights resident.
constexpr uint32_t HALO_W = 130u, HALO_ROWS = 3u;
constexpr uint32_t HALO_PLANE = (HALO_ROWS * HALO_W * 16u + 127u) / 128u * 128u;  // 6,272 bytes
constexpr uint32_t HALO_STAGE = 4u * HALO_PLANE, HALO_TS = 3u;
constexpr uint32_t HALO_W_OFF = (HALO_TS * HALO_STAGE + 1023u) / 1024u * 1024u;  // the resident weights, 1 KB aligned
constexpr uint32_t HALO_A_ALIGNED = (HALO_STAGE + 1023u) / 1024u * 1024u;  // a streaming stage's weights start here
constexpr uint32_t SMEM_MAX = 227u * 1024u;                                      // dynamic shared memory a CTA
// The halo variant's shared memory: the stages, then every (32-channel block, tap) weight box of the output tile
// (nt rows of 64 bytes each), then the barriers.
__host__ __device__ constexpr uint32_t halo_weights(uint32_t kc, uint32_t nt) { return 9u * kc * nt * 64u; }
__host__ __device__ constexpr uint32_t conv_smem_halo(uint32_t kc, uint32_t nt) {
    return HALO_W_OFF + halo_weights(kc, nt) + 256u + 1024u;
}
constexpr uint32_t CONV_EPI_THREADS = 256u, CONV_THREADS = 64u + CONV_EPI_THREADS;  // loader, MMA, 8 epilogue warps
constexpr uint32_t CONV_CTAS_PER_SM = 2u;

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0u;
}
// A bounded wait: about 2^31 cycles (a second at the B200's clock), then the error word and the CTA's abort word,
// which ends every other wait of the CTA at once.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, uint32_t* err, volatile uint32_t* abort_flag) {
    long long t0 = clock64();
    while (!mbar_try_wait(a, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > (1ll << 31)) {
            atomicOr(err, 1u);
            *abort_flag = 1u;
            return false;
        }
    }
    return true;
}
// A wait bounded at about 2^31 cycles that ignores the abort word: the drain of a CTA that gave up.
__device__ __forceinline__ bool mbar_wait_drain(uint32_t a, uint32_t parity) {
    long long t0 = clock64();
    while (!mbar_try_wait(a, parity))
        if (clock64() - t0 > (1ll << 31)) return false;
    return true;
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* map, int c0, int c1, int c2, int c3,
                                            uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void* map, int c0, int c1, int c2, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(mbar)
        : "memory");
}
// The canonical K-major shared-memory matrix with the 64-byte swizzle: rows of 64 bytes (32 bf16 of K), atoms of 8
// rows (512 bytes) `sbo` bytes apart along M / N; the leading offset unused (1); descriptor version 1 (sm_100),
// layout type 4 (SWIZZLE_64B). A K step of 16 inside the row advances the start by 32 bytes.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46) | (4ull << 61);
}
// The canonical K-major shared-memory matrix without swizzle: core matrices of 8 rows x 16 bytes, rows 16 bytes
// apart, `sbo` bytes between core matrices along M / N and `lbo` bytes between the two along K (8 elements each);
// descriptor version 1, layout type 0. The start may be any 16-byte boundary.
__device__ __forceinline__ uint64_t umma_desc_plain(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: f32 accumulator, bf16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
__device__ __forceinline__ void umma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 64 accumulator columns of this warp's lanes in one load and one wait.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float* v) {
    uint32_t r[64];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 accumulator columns of this warp's lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// The epilogue of one accumulator row (a pixel) and 16 columns from `c`: bias, ReLU, bf16 NHWC (or the f32 output).
__device__ __forceinline__ void conv_store16(const Conv& a, uint64_t p, uint32_t c, float* v) {
    if (a.bias) {
        const float4* b4 = reinterpret_cast<const float4*>(a.bias + c);  // (16 floats, 64-byte aligned)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float4 bq = __ldg(b4 + q);
            v[4 * q] += bq.x;
            v[4 * q + 1] += bq.y;
            v[4 * q + 2] += bq.z;
            v[4 * q + 3] += bq.w;
        }
    }
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (a.relu) v[i] = fmaxf(v[i], 0.0f);
    if (a.yf) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (c + i < a.cout) a.yf[p * a.cout + c + i] = v[i];
    } else if (c + 16u <= a.cout) {
        uint32_t pk[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
            pk[i] = *reinterpret_cast<uint32_t*>(&h2);
        }
        uint4* dst = reinterpret_cast<uint4*>(a.y + p * a.y_stride + a.y_off + c);
        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    } else {
        for (int i = 0; i < 16; ++i)
            if (c + i < a.cout) a.y[p * a.y_stride + a.y_off + c + i] = __float2bfloat16_rn(v[i]);
    }
}

// HALO: tiles of 128 x 1 pixels, the weights resident (every 32-channel block of one output tile) or, where they do
// not fit, streamed with the activations (a stage then also holds its block's nine weight boxes), and a stage is one
// block of the tile's activations with their halo (four TMA boxes of 8 channels x 130 pixels x 3 rows, no swizzle) from which
// the nine taps' A operands are read by descriptors shifted (dy x 130 + dx) rows of 16 bytes: one load a tile instead
// of nine. The taps' MMAs read rows [dy x 130 + dx, + 128) of each plane, inside the box.
template <bool HALO>
__global__ void __launch_bounds__(CONV_THREADS, 2) k_conv(const __grid_constant__ CUtensorMap xmap,
                                                       const __grid_constant__ CUtensorMap wmap, Conv a) {
    // stages, and a stage's bytes: the halo variant's activations, and where the weights are not resident the nine
    // taps' weight boxes of the stage's 32-channel block after them
    const uint32_t NS = HALO ? a.stages : TS;
    const uint32_t A_BYTES = HALO ? (a.resident ? HALO_STAGE : HALO_A_ALIGNED + 9u * a.nt * 64u) : A_STAGE;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t sraw = smem_addr(smem_raw), sbase = (sraw + 1023u) & ~1023u;
    uint8_t* smem = smem_raw + (sbase - sraw);
    const uint32_t kc = a.cin / 32u, nk = HALO ? kc : 9u * kc;
    constexpr uint32_t B_OFF = HALO ? HALO_W_OFF : TS * A_STAGE;
    const uint32_t BAR_OFF = HALO ? (a.resident ? HALO_W_OFF + halo_weights(kc, a.nt) : NS * A_BYTES)
                                  : TS * (A_STAGE + B_STAGE);
    const uint32_t sA = sbase, sB = sbase + B_OFF, sBar = sbase + BAR_OFF;
    // barriers: full[NS], empty[NS] (the stages), acc_full[2], acc_empty[2] (the accumulators), mma_done (every MMA
    // issued), wfull (the resident weights); the tensor-memory address, the abort word and the counts of stages issued
    // and consumed after them
    auto full = [&](uint32_t s) { return sBar + 8u * s; };
    auto empty = [&](uint32_t s) { return sBar + 8u * (NS + s); };
    auto acc_full = [&](uint32_t i) { return sBar + 8u * (2u * NS + i); };
    auto acc_empty = [&](uint32_t i) { return sBar + 8u * (2u * NS + 2u + i); };
    const uint32_t mma_done = sBar + 8u * (2u * NS + 4u), wfull = sBar + 8u * (2u * NS + 5u);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + BAR_OFF + 8u * (2u * NS + 6u));
    volatile uint32_t* abort_flag = tslot + 1;
    volatile uint32_t* counts = tslot + 2;
    const uint32_t ncols = 2u * a.nt;  // two accumulators of nt columns: 128 or 256
    const uint32_t per_img = a.tiles_x * a.tiles_y, n_ntiles = a.co_pad / a.nt;
    const uint32_t tiles = a.B * per_img * n_ntiles;

    if (tid == 0) {
        for (uint32_t s = 0; s < NS; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (uint32_t i = 0; i < 2u; ++i) {
            mbar_init(acc_full(i), 1);
            mbar_init(acc_empty(i), CONV_EPI_THREADS);
        }
        mbar_init(mma_done, 1);
        mbar_init(wfull, 1);
        *abort_flag = 0u;
        counts[0] = counts[1] = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // A tile: its image, its pixel rectangle, its output-channel slice.
    auto tile_of = [&](uint32_t t, uint32_t& b, int& x0, int& y0, uint32_t& n0) {
        const uint32_t nt_i = t % n_ntiles, pt = t / n_ntiles;
        b = pt / per_img;
        const uint32_t r = pt % per_img;
        x0 = (int)((r % a.tiles_x) * a.bw);
        y0 = (int)((r / a.tiles_x) * a.bh);
        n0 = nt_i * a.nt;
    };

    if (warp == 0) {
        if (lane == 0) {
            // the loader: the resident weights (the nine taps' boxes, one after another), then the stages of every tile
            // of this CTA, in order
            // (halo: every 32-channel block's nine boxes, block-major)
            if (a.resident) {
                const uint32_t blocks = HALO ? kc : 1u;
                mbar_expect_tx(wfull, 9u * blocks * a.nt * 64u);
                for (uint32_t k = 0; k < blocks; ++k)
                    for (uint32_t tap = 0; tap < 9u; ++tap)
                        tma_load_3d(sB + (k * 9u + tap) * a.nt * 64u, &wmap, (int)(k * 32u), 0, (int)tap, wfull);
            }
            uint32_t it = 0;
            bool ok = true;
            for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                uint32_t b, n0;
                int x0, y0;
                tile_of(t, b, x0, y0, n0);
                for (uint32_t k = 0; k < nk; ++k, ++it) {
                    const uint32_t s = it % NS;
                    if (it >= NS && !(ok = mbar_wait(empty(s), ((it / NS) - 1u) & 1u, a.err, abort_flag))) break;
                    const bool withhold = a.hold && blockIdx.x == 0 && it == 0;
                    if constexpr (HALO) {
                        // the tile's rows y0 - 1 .. y0 + 1, pixels x0 - 1 .. x0 + 128, one box a plane of 8 channels
                        mbar_expect_tx(full(s), 4u * HALO_ROWS * HALO_W * 16u + (a.resident ? 0u : 9u * a.nt * 64u));
                        if (!withhold)
                            for (uint32_t pl = 0; pl < 4u; ++pl)
                                tma_load_4d(sA + s * A_BYTES + pl * HALO_PLANE, &xmap, (int)(a.x_off + k * 32u + pl * 8u),
                                            x0 - 1, y0 - 1, (int)b, full(s));
                        if (!a.resident)
                            for (uint32_t tap = 0; tap < 9u; ++tap)
                                tma_load_3d(sA + s * A_BYTES + HALO_A_ALIGNED + tap * a.nt * 64u, &wmap, (int)(k * 32u),
                                            (int)n0, (int)tap, full(s));
                    } else {
                        mbar_expect_tx(full(s), A_STAGE + (a.resident ? 0u : a.nt * 64u));
                        const uint32_t tap = k / kc, c0 = (k % kc) * 32u;
                        const int dy = (int)(tap / 3u) - 1, dx = (int)(tap % 3u) - 1;
                        if (!withhold)
                            tma_load_4d(sA + s * A_STAGE, &xmap, (int)(a.x_off + c0), x0 + dx, y0 + dy, (int)b, full(s));
                        if (!a.resident) tma_load_3d(sB + s * B_STAGE, &wmap, (int)c0, (int)n0, (int)tap, full(s));
                    }
                }
            }
            counts[0] = it;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // the MMA issuer: a tile's stages into accumulator (tile count % 2), then that accumulator to the epilogue
            // (a layer of one 64-column output tile with at most 32 outputs: the MMAs' N covers the outputs only, 32
            // or 16 of the tile's rows of weights; the epilogue reads no column past the outputs)
            const uint32_t n_mma = a.co_pad == a.nt && a.nt == 64u && a.cout <= 32u ? (a.cout <= 16u ? 16u : 32u) : a.nt;
            const uint32_t idesc = umma_idesc(128u, n_mma);
            uint32_t it = 0, ti = 0;
            bool ok = !a.resident || mbar_wait(wfull, 0u, a.err, abort_flag);
            for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++ti) {
                const uint32_t acc = ti & 1u;
                if (ti >= 2u && !(ok = mbar_wait(acc_empty(acc), ((ti / 2u) - 1u) & 1u, a.err, abort_flag))) break;
                tc_fence_after();
                const uint32_t d = tmem + acc * a.nt;
                for (uint32_t k = 0; k < nk; ++k, ++it) {
                    const uint32_t s = it % NS;
                    if (!(ok = mbar_wait(full(s), (it / NS) & 1u, a.err, abort_flag))) break;
                    tc_fence_after();
                    if constexpr (HALO) {
                        // tap (dy, dx): rows from (dy + 1) x 130 + dx + 1 of planes 2j, 2j + 1 (K 16 each MMA)
                        for (uint32_t tap = 0; tap < 9u; ++tap) {
                            const uint32_t row = (tap / 3u) * HALO_W + tap % 3u;
#pragma unroll
                            for (uint32_t j = 0; j < 2u; ++j) {
                                uint64_t ad = umma_desc_plain(sA + s * A_BYTES + 2u * j * HALO_PLANE + row * 16u,
                                                              HALO_PLANE, 128u);
                                const uint32_t wb = a.resident ? sB + (k * 9u + tap) * a.nt * 64u
                                                               : sA + s * A_BYTES + HALO_A_ALIGNED + tap * a.nt * 64u;
                                uint64_t bd = umma_desc_sw64(wb + j * 32u, 512u);
                                umma_f16(d, ad, bd, idesc, (k | tap | j) != 0u ? 1u : 0u);
                            }
                        }
                    } else {
                        // (resident weights: one box a tap, kc = 1)
                        const uint32_t sb = a.resident ? sB + k * a.nt * 64u : sB + s * B_STAGE;
#pragma unroll
                        for (uint32_t j = 0; j < 2u; ++j) {
                            uint64_t ad = umma_desc_sw64(sA + s * A_STAGE + j * 32u, 512u);
                            uint64_t bd = umma_desc_sw64(sb + j * 32u, 512u);
                            umma_f16(d, ad, bd, idesc, (k | j) != 0u ? 1u : 0u);
                        }
                    }
                    umma_commit(empty(s));
                }
                if (ok) umma_commit(acc_full(acc));
            }
            counts[1] = it;
            umma_commit(mma_done);  // every MMA issued is done (after a wait that gave up too)
        }
    } else {
        // the epilogue, eight warps, two a tensor-memory lane quarter: warp w reads lanes 32 (w % 4) ... (its rows:
        // pixels of the tile) and half of the tile's columns, (w - 2) / 4 which
        const uint32_t quarter = warp & 3u, half = (warp - 2u) >> 2;
        const uint32_t m = quarter * 32u + lane, cols = a.nt / 2u, c_first = half * cols;
        uint32_t ti = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++ti) {
            const uint32_t acc = ti & 1u;
            const bool fin = mbar_wait(acc_full(acc), (ti / 2u) & 1u, a.err, abort_flag);
            __syncwarp();
            tc_fence_after();
            uint32_t b, n0;
            int x0, y0;
            tile_of(t, b, x0, y0, n0);
            const int px = x0 + (int)(m % a.bw), py = y0 + (int)(m / a.bw);
            const bool valid = fin && px < (int)a.W && py < (int)a.H;
            const uint64_t p = ((uint64_t)b * a.H + (uint32_t)py) * a.W + (uint32_t)px;
            for (uint32_t cc = c_first; cc < c_first + cols; cc += 32u) {
                if (n0 + cc >= a.cout) break;  // (columns past the layer's outputs: padding, not stored)
                float v[32];
                tmem_ld32(tmem + ((quarter * 32u) << 16) + acc * a.nt + cc, v);
                if (valid) {
                    conv_store16(a, p, n0 + cc, v);
                    conv_store16(a, p, n0 + cc + 16u, v + 16u);
                }
            }
            // this accumulator is read: the MMA issuer may fill it again
            tc_fence_before();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acc_empty(acc)) : "memory");
            if (!fin) break;
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (*abort_flag && lane == 0) {
        // a wait gave up: let the copies and MMAs in flight land before the memory they use is released
        if (warp == 0) {
            if (a.resident) mbar_wait_drain(wfull, 0u);
            for (uint32_t i = counts[1]; i < counts[0]; ++i) mbar_wait_drain(full(i % NS), (i / NS) & 1u);
        } else if (warp == 1) {
            mbar_wait_drain(mma_done, 0u);
        }
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---- weight and bias gradients: dw[t][c][n] += sum over pixels p of x[p + off(t)][c] * dy[p][n]; db[n] += sum dy ---
//
// One GEMM over pixels (K) for every (tap, 32-input-channel block) pair of the layer at once: the pairs fill the
// 32-row slots of a 128-row accumulator (M), four a group, and one more slot holds all ones, so that its rows are the
// bias gradient; N is the layer's output channels (32 to 128). A CTA takes one group of slots (blockIdx.y) over a run
// of 128-pixel tiles (blockIdx.x):
//  - one thread loads a tile's stage: per slot a TMA box of 32 channels x bw x bh pixels of x, shifted by the slot's
//    tap (zeros outside the image), and the output gradient's boxes of 32 channels x the same pixels, unshifted; a
//    box lands as 128 rows (pixels) of 64 bytes with the 64-byte swizzle, which is the canonical MN-major layout
//    (32-element blocks of M or N one box = 8 KB apart, 8-pixel groups of K 512 bytes apart);
//  - one thread issues eight tcgen05.mma (M 128, N, K 16, both operands MN-major, f32 accumulate in tensor memory)
//    a stage and hands the stage back to the loader through an mbarrier;
//  - after the run the four epilogue warps read the accumulator (warp w: slot w % 4, its lanes the slot's 32 input
//    channels) and store it as the CTA's f32 partial; k_wgrad_sum adds the partials of a group's runs, in run order,
//    into dw (and the ones slot's first row into db), so that the sums do not depend on the CTAs' timing.
// Slots that no pair fills hold zeros; they and the ones slot are written once, when the CTA starts. Waits are
// bounded as the convolution's are; after a wait that gave up, the CTA waits (bounded) for its copies and MMAs in
// flight before it frees its tensor memory.

struct WGrad {
    uint32_t cin, x_off;      // input channels (a multiple of 32) and their first channel in x
    uint32_t kc, nb, pairs;   // input blocks of 32, output-gradient blocks of 32 (N = 32 nb), 9 kc (the ones slot's index)
    float* part;              // [group][run][128][32 nb] f32: the CTAs' partials
    uint32_t bw, bh, tiles_x, tiles_y, tiles, chunk;  // 128-pixel tiles (bw x bh) over all images; tiles a CTA
    uint32_t ts;              // pipeline stages
    uint32_t* err;
};
constexpr uint32_t WG_BOX = 128u * 64u;  // one box: 128 pixels x 32 channels of bf16
constexpr uint32_t WG_THREADS = 192u;    // loader, MMA, 4 epilogue warps
constexpr uint32_t WG_SMEM_EXTRA = 1024u + 256u;  // alignment of the stages to 1 KB, the barriers
constexpr uint32_t WG_SMEM_MAX = 227u * 1024u;

// The canonical MN-major shared-memory matrix with the 64-byte swizzle: 32-element blocks of M (or N) `lbo` bytes
// apart, 8-row groups of K (rows of 64 bytes) 512 bytes apart; descriptor version 1, layout type 4 (SWIZZLE_64B).
__device__ __forceinline__ uint64_t umma_desc_mn64(uint32_t saddr, uint32_t lbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(512u >> 4) << 32) | (1ull << 46) | (4ull << 61);
}
__global__ void __launch_bounds__(WG_THREADS) k_wgrad(const __grid_constant__ CUtensorMap xmap,
                                                     const __grid_constant__ CUtensorMap dymap, WGrad a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t sraw = smem_addr(smem_raw), sbase = (sraw + 1023u) & ~1023u;
    uint8_t* smem = smem_raw + (sbase - sraw);
    const uint32_t stage = (4u + a.nb) * WG_BOX, sBar = sbase + a.ts * stage;
    // barriers: full[ts], empty[ts], acc_full; then the tensor-memory address, the abort word and the counts of
    // stages issued and consumed
    auto full = [&](uint32_t s) { return sBar + 8u * s; };
    auto empty = [&](uint32_t s) { return sBar + 8u * (a.ts + s); };
    const uint32_t acc_full = sBar + 16u * a.ts;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + a.ts * stage + 16u * a.ts + 8u);
    volatile uint32_t* abort_flag = tslot + 1;
    volatile uint32_t* counts = tslot + 2;
    const uint32_t n_cols = 32u * a.nb, ncols = a.nb == 1u ? 32u : a.nb == 2u ? 64u : 128u;
    const uint32_t slot0 = blockIdx.y * 4u;
    const uint32_t loaded = slot0 < a.pairs ? min(4u, a.pairs - slot0) : 0u;  // slots 0 .. loaded-1 hold pairs
    const uint32_t k0 = blockIdx.x * a.chunk, k1 = min(a.tiles, k0 + a.chunk);
    const uint32_t per_img = a.tiles_x * a.tiles_y;

    // the slots no pair fills: the ones slot (bf16 1.0) and zeros, in every stage
    for (uint32_t j = loaded; j < 4u; ++j) {
        const uint32_t v = slot0 + j == a.pairs ? 0x3F803F80u : 0u;
        for (uint32_t s = 0; s < a.ts; ++s) {
            uint4* p = reinterpret_cast<uint4*>(smem + s * stage + j * WG_BOX);
            for (uint32_t i = tid; i < WG_BOX / 16u; i += WG_THREADS) p[i] = make_uint4(v, v, v, v);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
    if (tid == 0) {
        for (uint32_t s = 0; s < a.ts; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(acc_full, 1);
        *abort_flag = 0u;
        counts[0] = counts[1] = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            // the loader: a stage a tile
            uint32_t it = 0;
            for (uint32_t t = k0; t < k1; ++t, ++it) {
                const uint32_t s = it % a.ts;
                if (it >= a.ts && !mbar_wait(empty(s), ((it / a.ts) - 1u) & 1u, a.err, abort_flag)) break;
                mbar_expect_tx(full(s), (loaded + a.nb) * WG_BOX);
                const uint32_t b = t / per_img, r = t % per_img;
                const int x0 = (int)((r % a.tiles_x) * a.bw), y0 = (int)((r / a.tiles_x) * a.bh);
                const uint32_t base = sbase + s * stage;
                for (uint32_t j = 0; j < loaded; ++j) {
                    const uint32_t pr = slot0 + j, tap = pr / a.kc, cb = pr % a.kc;
                    tma_load_4d(base + j * WG_BOX, &xmap, (int)(a.x_off + cb * 32u), x0 + (int)(tap % 3u) - 1,
                                y0 + (int)(tap / 3u) - 1, (int)b, full(s));
                }
                for (uint32_t i = 0; i < a.nb; ++i)
                    tma_load_4d(base + (4u + i) * WG_BOX, &dymap, (int)(i * 32u), x0, y0, (int)b, full(s));
            }
            counts[0] = it;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // the MMA issuer: eight K-16 steps a stage into the one accumulator
            const uint32_t idesc = umma_idesc(128u, n_cols) | (1u << 15) | (1u << 16);  // A and B MN-major
            uint32_t it = 0;
            for (uint32_t t = k0; t < k1; ++t, ++it) {
                const uint32_t s = it % a.ts;
                if (!mbar_wait(full(s), (it / a.ts) & 1u, a.err, abort_flag)) break;
                tc_fence_after();
                const uint32_t base = sbase + s * stage;
#pragma unroll
                for (uint32_t j = 0; j < 8u; ++j) {
                    const uint64_t ad = umma_desc_mn64(base + j * 1024u, WG_BOX);
                    const uint64_t bd = umma_desc_mn64(base + 4u * WG_BOX + j * 1024u, WG_BOX);
                    umma_f16(tmem, ad, bd, idesc, (it | j) != 0u ? 1u : 0u);
                }
                umma_commit(empty(s));
            }
            counts[1] = it;
            umma_commit(acc_full);  // every MMA issued is done (after a wait that gave up too)
        }
    } else {
        // the epilogue: warp w reads tensor-memory lanes 32 (w % 4) ..., the rows of slot w % 4
        const uint32_t quarter = warp & 3u, slot = slot0 + quarter;
        const bool fin = mbar_wait(acc_full, 0u, a.err, abort_flag);
        __syncwarp();
        tc_fence_after();
        if (fin && (quarter < loaded || slot == a.pairs)) {
            float* dst = a.part + (((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * 128u + quarter * 32u + lane) * n_cols;
            for (uint32_t cc = 0; cc < n_cols; cc += 32u) {
                float v[32];
                tmem_ld32(tmem + ((quarter * 32u) << 16) + cc, v);
#pragma unroll
                for (uint32_t q = 0; q < 8u; ++q)
                    reinterpret_cast<float4*>(dst + cc)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (*abort_flag && lane == 0) {
        // a wait gave up: let the copies and MMAs in flight land before the memory they use is released
        if (warp == 0)
            for (uint32_t i = counts[1]; i < counts[0]; ++i) mbar_wait_drain(full(i % a.ts), (i / a.ts) & 1u);
        else if (warp == 1)
            mbar_wait_drain(acc_full, 0u);
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// The partials of k_wgrad summed over a group's runs: a block takes 32 outputs (a group's accumulator row and 4
// columns each, of the slots that hold a pair and the first row of the ones slot) x 8 segments of runs (segment j:
// runs j, j + 8, ...), the segments then summed in order; every sum is taken in the same order on every call. Added
// into dw[t][c][n] and db[n].
constexpr uint32_t WS_SEGS = 8u;
__global__ void __launch_bounds__(32u * WS_SEGS) k_wgrad_sum(const float* __restrict__ part, uint32_t runs,
                                                             uint32_t groups, uint32_t n_cols, uint32_t kc,
                                                             uint32_t pairs, uint32_t cin, uint32_t co_pad, float* dw,
                                                             float* db) {
    __shared__ float4 seg[WS_SEGS][32];
    const uint32_t nq = n_cols / 4u, lane = threadIdx.x & 31u, j = threadIdx.x >> 5;
    const uint64_t i = (uint64_t)blockIdx.x * 32u + lane;
    const uint32_t q = (uint32_t)(i % nq), m = (uint32_t)((i / nq) % 128u), g = (uint32_t)(i / (nq * 128u));
    const uint32_t slot = g * 4u + m / 32u, c = m % 32u;
    const bool live = i < (uint64_t)groups * 128u * nq && (slot < pairs || (slot == pairs && c == 0u));
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (live) {
        const float4* p = reinterpret_cast<const float4*>(part + ((uint64_t)g * runs * 128u + m) * n_cols) + q;
        const uint64_t run_stride = 128ull * nq;
        for (uint32_t r = j; r < runs; r += WS_SEGS) {
            const float4 v = __ldg(p + r * run_stride);
            s.x += v.x;
            s.y += v.y;
            s.z += v.z;
            s.w += v.w;
        }
    }
    seg[j][lane] = s;
    __syncthreads();
    if (j != 0u || !live) return;
    for (uint32_t k = 1; k < WS_SEGS; ++k) {
        const float4 v = seg[k][lane];
        s.x += v.x;
        s.y += v.y;
        s.z += v.z;
        s.w += v.w;
    }
    float4* d = reinterpret_cast<float4*>(
                    slot < pairs ? dw + ((uint64_t)(slot / kc) * cin + (slot % kc) * 32u + c) * co_pad : db) + q;
    const float4 o = *d;
    *d = make_float4(o.x + s.x, o.y + s.y, o.z + s.z, o.w + s.w);
}

// ---- the other layers ----------------------------------------------------------------------------------------------

// 2 x 2 average pooling: y[b][y][x][c] = mean of x over the 2 x 2 block (H, W even).
__global__ void k_pool(const bf16* x, uint32_t xs, uint32_t xo, bf16* y, uint32_t ys, uint32_t C, uint32_t B,
                       uint32_t H, uint32_t W) {
    // 8 channels (16 bytes) a thread: C, the strides and the offsets are multiples of 32 channels
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t h2 = H / 2, w2 = W / 2, c8 = C / 8u;
    uint64_t n = (uint64_t)B * h2 * w2 * c8;
    if (i >= n) return;
    uint32_t c = (uint32_t)(i % c8) * 8u;
    uint64_t q = i / c8;
    uint32_t xx = (uint32_t)(q % w2), yy = (uint32_t)((q / w2) % h2), b = (uint32_t)(q / ((uint64_t)w2 * h2));
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            uint4 v = *reinterpret_cast<const uint4*>(x + (((uint64_t)b * H + 2 * yy + j) * W + 2 * xx + k) * xs + xo + c);
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                float2 f = __bfloat1622float2(h[e]);
                s[2 * e] += f.x;
                s[2 * e + 1] += f.y;
            }
        }
    uint4 o;
    __nv_bfloat162* oh = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
    for (int e = 0; e < 4; ++e) oh[e] = __floats2bfloat162_rn(0.25f * s[2 * e], 0.25f * s[2 * e + 1]);
    *reinterpret_cast<uint4*>(y + q * ys + c) = o;
}
// ... its gradient, added: dx[2y + j][2x + k] += dy[y][x] / 4.
__global__ void k_pool_back(const bf16* dy, uint32_t dys, bf16* dx, uint32_t dxs, uint32_t dxo, uint32_t C, uint32_t B,
                            uint32_t H, uint32_t W) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t n = (uint64_t)B * H * W * C;
    if (i >= n) return;
    uint32_t c = (uint32_t)(i % C);
    uint64_t q = i / C;
    uint32_t x = (uint32_t)(q % W), y = (uint32_t)((q / W) % H), b = (uint32_t)(q / ((uint64_t)W * H));
    float g = 0.25f * __bfloat162float(dy[(((uint64_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * dys + c]);
    bf16* d = dx + q * dxs + dxo + c;
    *d = __float2bfloat16_rn(__bfloat162float(*d) + g);
}
// Nearest 2x upsampling into channels [0, C) of y: y[2y + j][2x + k] = x[y][x].
__global__ void k_up(const bf16* x, uint32_t xs, bf16* y, uint32_t ys, uint32_t C, uint32_t B, uint32_t H, uint32_t W) {
    // over the output (H, W: the output's), 8 channels (16 bytes) a thread
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t c8 = C / 8u;
    uint64_t n = (uint64_t)B * H * W * c8;
    if (i >= n) return;
    uint32_t c = (uint32_t)(i % c8) * 8u;
    uint64_t q = i / c8;
    uint32_t px = (uint32_t)(q % W), py = (uint32_t)((q / W) % H), b = (uint32_t)(q / ((uint64_t)W * H));
    *reinterpret_cast<uint4*>(y + q * ys + c) =
        *reinterpret_cast<const uint4*>(x + (((uint64_t)b * (H / 2) + py / 2) * (W / 2) + px / 2) * xs + c);
}
// ... its gradient: dx[y][x] = sum of dy over the 2 x 2 block (channels [0, C) of dy).
__global__ void k_up_back(const bf16* dy, uint32_t dys, bf16* dx, uint32_t dxs, uint32_t C, uint32_t B, uint32_t H,
                          uint32_t W) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // over dx (H, W: dx's)
    uint64_t n = (uint64_t)B * H * W * C;
    if (i >= n) return;
    uint32_t c = (uint32_t)(i % C);
    uint64_t q = i / C;
    uint32_t x = (uint32_t)(q % W), y = (uint32_t)((q / W) % H), b = (uint32_t)(q / ((uint64_t)W * H));
    float s = 0.0f;
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 2; ++k)
            s += __bfloat162float(dy[(((uint64_t)b * 2 * H + 2 * y + j) * 2 * W + 2 * x + k) * dys + c]);
    dx[q * dxs + c] = __float2bfloat16_rn(s);
}
// ReLU's gradient in place: dy = 0 where the layer's output y was 0.
__global__ void k_relu_back(bf16* dy, uint32_t dys, uint32_t dyo, const bf16* y, uint32_t ys, uint32_t yo, uint32_t C,
                            uint64_t P) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * C) return;
    uint64_t p = i / C;
    uint32_t c = (uint32_t)(i % C);
    if (!(__bfloat162float(y[p * ys + yo + c]) > 0.0f)) dy[p * dys + dyo + c] = __float2bfloat16_rn(0.0f);
}
// Copies channels [so, so + C) of a to channels [0, C) of b (the skip part of a concatenation's gradient).
__global__ void k_copy_ch(const bf16* a, uint32_t as, uint32_t so, bf16* b, uint32_t bs, uint32_t bo, uint32_t C,
                          uint64_t P) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * C) return;
    uint64_t p = i / C;
    uint32_t c = (uint32_t)(i % C);
    b[p * bs + bo + c] = a[p * as + so + c];
}
// The L1 loss on log radiance and its gradient (as bf16 into a 32-channel buffer): dpred = sign(pred - t) / count.
__global__ void k_loss(const float* pred, const float* target, uint64_t P, bf16* dpred, float* loss) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < P * 3) {
        float d = pred[i] - target[i];
        l = fabsf(d);
        float g = (d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f)) / (float)(P * 3);
        dpred[(i / 3) * 32 + i % 3] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(~0u, l, o);
    if ((threadIdx.x & 31u) == 0 && l != 0.0f) atomicAdd(loss, l / (float)(P * 3));
}
// Adam (Kingma & Ba 2015) on the f32 master values, then the bf16 forward copy. `args`: the step's learning rate and
// bias corrections 1 - b1^t, 1 - b2^t (device memory, so that a captured step reads each step's values).
__global__ void k_adam(float* w, const float* g, float* m, float* v, uint64_t n, const float* args, float b1, float b2,
                       float eps) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lr = args[0], c1 = args[1], c2 = args[2];
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}
// The bf16 weights of a layer from its f32 masters w[t][c][n], laid out as the convolution's B operand (per tap, the
// output channels' rows of input channels): forward [t][n][c] (n < co_pad rows of cin), and the input gradient's
// [8 - t][c][n] (c < cin of ci_pad64 rows: its output; n < cout32: the output gradient's channels, its input).
__global__ void k_weights(const float* wf, uint32_t cin, uint32_t co_pad, uint32_t cout32, bf16* wfw, bf16* wbw,
                          uint32_t ci_pad64) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t n = 9ull * cin * co_pad;
    if (i >= n) return;
    uint32_t nn = (uint32_t)(i % co_pad), c = (uint32_t)((i / co_pad) % cin), t = (uint32_t)(i / ((uint64_t)co_pad * cin));
    bf16 v = __float2bfloat16_rn(wf[i]);
    wfw[((uint64_t)t * co_pad + nn) * cin + c] = v;
    if (wbw && nn < cout32) wbw[((uint64_t)(8 - t) * ci_pad64 + c) * cout32 + nn] = v;
}

// ---- features from a rendered accum (inference on a scene's result) ----------------------------------------------

constexpr int N_FEAT = 11;  // input channels a pixel

// The image's mean luminance and mean first-hit distance (over pixels that hit): sums into acc[0..2].
// The image's mean luminance and mean first-hit distance (over pixels that hit), in a fixed order so that a denoise
// is the same bit for bit however it is scheduled: each of FEAT_BLOCKS blocks sums its stride of pixels, then one
// block sums the blocks' partials into acc[0..2].
constexpr uint32_t FEAT_BLOCKS = 256, FEAT_THREADS = 256;
__global__ void k_feat_sums(const float4* __restrict__ accum, uint64_t n, float* partial) {
    __shared__ float sh[3][FEAT_THREADS];
    float l = 0.0f, d = 0.0f, dn = 0.0f;
    for (uint64_t i = (uint64_t)blockIdx.x * FEAT_THREADS + threadIdx.x; i < n; i += (uint64_t)FEAT_BLOCKS * FEAT_THREADS) {
        float4 c = accum[5 * i], e = accum[5 * i + 3];
        float cnt = fmaxf(c.w, 1.0f);
        float li = (0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z) / cnt;
        if (isfinite(li)) l += li;
        float dd = e.x / cnt;
        if (dd > 0.0f && isfinite(dd)) {
            d += dd;
            dn += 1.0f;
        }
    }
    sh[0][threadIdx.x] = l;
    sh[1][threadIdx.x] = d;
    sh[2][threadIdx.x] = dn;
    __syncthreads();
    for (uint32_t w = FEAT_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 3) partial[3 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}
__global__ void k_feat_total(const float* __restrict__ partial, float* acc) {
    if (threadIdx.x >= 3) return;
    float t = 0.0f;
    for (uint32_t b = 0; b < FEAT_BLOCKS; ++b) t += partial[3 * b + threadIdx.x];
    acc[threadIdx.x] = t;
}
__device__ __forceinline__ float fin0(float v) { return isfinite(v) ? v : 0.0f; }
// The network's input from the accum: log1p(radiance * s), albedo, normal, log1p(depth * sd) and log1p(the variance of
// the mean luminance * s^2), 32 channels (bf16).
__global__ void k_feat(const float4* __restrict__ accum, uint64_t n, const float* sums, bf16* x) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 1.0f / fmaxf(sums[0] / (float)n, 1e-6f), sd = 1.0f / fmaxf(sums[1] / fmaxf(sums[2], 1.0f), 1e-6f);
    float4 c = accum[5 * i], a = accum[5 * i + 1], nn = accum[5 * i + 2], e = accum[5 * i + 3];
    float cnt = fmaxf(c.w, 1.0f);
    float mean = fin0(a.w) / cnt, var = fmaxf(fin0(nn.w) / cnt - mean * mean, 0.0f) / cnt;
    float f[N_FEAT] = {log1pf(fmaxf(fin0(c.x / cnt) * s, 0.0f)), log1pf(fmaxf(fin0(c.y / cnt) * s, 0.0f)),
                       log1pf(fmaxf(fin0(c.z / cnt) * s, 0.0f)), fin0(a.x / cnt), fin0(a.y / cnt), fin0(a.z / cnt),
                       fin0(nn.x / cnt), fin0(nn.y / cnt), fin0(nn.z / cnt), log1pf(fmaxf(fin0(e.x / cnt) * sd, 0.0f)),
                       log1pf(fmaxf(var * s * s, 0.0f))};
    bf16* row = x + i * 32;
    for (int k = 0; k < 32; ++k) row[k] = __float2bfloat16_rn(k < N_FEAT ? f[k] : 0.0f);
}
// The prediction back to radiance: expm1(pred) / s.
__global__ void k_unfeat(const float* pred, uint64_t n, const float* sums, float* rgb) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 3) return;
    float s = 1.0f / fmaxf(sums[0] / (float)n, 1e-6f);
    rgb[i] = fmaxf(expm1f(pred[i]), 0.0f) / s;
}
// Host features (f32, N_FEAT a pixel) to the network's 32-channel bf16 input.
__global__ void k_feat_host(const float* f, uint64_t n, bf16* x) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 32) return;
    uint64_t p = i / 32;
    uint32_t c = (uint32_t)(i % 32);
    x[i] = __float2bfloat16_rn(c < N_FEAT ? f[p * N_FEAT + c] : 0.0f);
}

// ---- the network ----------------------------------------------------------------------------------------------------

struct Layer { uint32_t cin, cout; int relu; };  // cin: padded to 32 (the input's 10 channels: 32)
constexpr int N_LAYERS = 15;
constexpr Layer LAYERS[N_LAYERS] = {
    {32, 32, 1},  {32, 32, 1},  {32, 64, 1},  {64, 64, 1},  {64, 96, 1},  {96, 96, 1},  {96, 128, 1}, {128, 128, 1},
    {224, 96, 1}, {96, 96, 1},  {160, 64, 1}, {64, 64, 1},  {96, 32, 1},  {32, 32, 1},  {32, 3, 0}};
enum { E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, D0A, D0B, OUT };

inline uint32_t r32(uint32_t v) { return (v + 31u) / 32u * 32u; }
inline uint32_t r64(uint32_t v) { return (v + 63u) / 64u * 64u; }
inline uint64_t w_count(const Layer& l) { return 9ull * l.cin * r64(l.cout); }
inline uint64_t layer_params(const Layer& l) { return w_count(l) + r64(l.cout); }

uint64_t param_count() {
    uint64_t n = 0;
    for (const Layer& l : LAYERS) n += layer_params(l);
    return n;
}

// An activation tensor: pixels x stride channels of bf16.
struct Act { bf16* p = nullptr; uint32_t stride = 0; };

struct Net {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t maxB = 0, maxH = 0, maxW = 0;
    std::string err;
    // f32 masters, gradients, Adam moments (one flat array each, layer after layer: weights then bias)
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    uint64_t n_params = 0, off[N_LAYERS] = {};
    bf16* wf[N_LAYERS] = {};  // forward weights
    bf16* wb[N_LAYERS] = {};  // input-gradient weights
    uint64_t t = 0;           // Adam steps
    // activations and their gradients
    Act in0, a0, cat0, pool0, a1, cat1, pool1, a2, cat2, pool2, a3, b3, t2, u2, t1, u1, t0, u0;
    Act dpred, du0, dt0, dcat0, du1, dt1, dcat1, du2, dt2, dcat2, db3, da3, dpool2, de2b, da2, dpool1, de1b, da1,
        dpool0, de0b, da0;
    float *pred = nullptr, *target = nullptr, *feat = nullptr, *loss = nullptr, *sums = nullptr, *rgb = nullptr;
    std::vector<void*> allocs;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    uint32_t* dev_err = nullptr;  // set by a convolution whose pipeline wait gave up
    bool hold_next = false;       // the next convolution launched outside a graph withholds one copy (a test)
    uint32_t sms = 148;           // the device's SMs (the persistent convolution's grid)
    float* wpart = nullptr;       // the weight gradient's CTA partials (128 x 128 f32 each)
    uint32_t wpart_ctas = 0;      // their room, in CTAs
    // the training step's kernels captured once per batch shape (and with or without the update), replayed after
    float* adam_args = nullptr;       // device: learning rate, 1 - b1^t, 1 - b2^t
    float* adam_host = nullptr;       // pinned: the same, written before each replay
    struct StepGraph { uint32_t B, H, W; int update; cudaGraphExec_t exec; };
    std::vector<StepGraph> graphs;
    float* partial = nullptr;     // the feature sums' block partials
    std::string conv_err;         // a tensor map that could not be made
};

}  // namespace unet

struct trt_unet : unet::Net {};

namespace unet {
namespace {

template <class T>
cudaError_t alloc(Net* n, T** p, uint64_t count) {
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<uint64_t>(count, 1));
    if (e == cudaSuccess) {
        n->allocs.push_back(*p);
        e = cudaMemset(*p, 0, sizeof(T) * std::max<uint64_t>(count, 1));
    }
    return e;
}
cudaError_t act(Net* n, Act& a, uint64_t pixels, uint32_t stride) {
    a.stride = stride;
    return alloc(n, &a.p, pixels * stride);
}

uint32_t blocks(uint64_t n, uint32_t b = 256) { return (uint32_t)((n + b - 1) / b); }

// cuTensorMapEncodeTiled from the driver, found through the runtime (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    });
    return fn;
}

// The 128-pixel tiles of a W x H image: bw the largest power of two <= 128 that divides the width, bh = 128 / bw.
void tile_shape(uint32_t W, uint32_t H, uint32_t& bw, uint32_t& bh, uint32_t& tiles_x, uint32_t& tiles_y) {
    bw = 1;
    while (bw < 128u && W % (bw * 2u) == 0u) bw *= 2u;
    bh = 128u / bw;
    tiles_x = W / bw;
    tiles_y = (H + bh - 1u) / bh;
}

// A tensor map of an activation: (channels, x, y, image) with `stride` channels a pixel, boxes of 32 channels x bw x bh
// pixels landing as 64-byte rows with the 64-byte swizzle (halo: boxes of 8 channels x bw x bh pixels, 16 bytes a
// pixel, no swizzle); reads outside the tensor are zeros.
bool act_map(Net* n, CUtensorMap* m, const bf16* p, uint32_t stride, uint32_t B, uint32_t H, uint32_t W, uint32_t bw,
             uint32_t bh, bool halo = false) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) {
        n->conv_err = "unet: cuTensorMapEncodeTiled is not available";
        return false;
    }
    cuuint64_t d[4] = {stride, W, H, B};
    cuuint64_t st[3] = {(cuuint64_t)stride * 2u, (cuuint64_t)W * stride * 2u, (cuuint64_t)H * W * stride * 2u};
    cuuint32_t box[4] = {halo ? 8u : 32u, bw, bh, 1u}, es[4] = {1u, 1u, 1u, 1u};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(p), d, st, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, halo ? CU_TENSOR_MAP_SWIZZLE_NONE : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        n->conv_err = "unet: an activation's tensor map was refused (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

// One convolution: x (NHWC bf16, x_stride channels a pixel, channels [x_off, x_off + cin) read) into y or yf, with
// w [9][co_pad][cin] (each tap's output channels, their input channels contiguous).
void conv_run(Net* n, const bf16* x, uint32_t x_stride, uint32_t x_off, uint32_t cin, const bf16* w, uint32_t co_pad,
              const float* bias, bf16* y, uint32_t y_stride, uint32_t y_off, uint32_t cout, float* yf, uint32_t B,
              uint32_t H, uint32_t W, int relu) {
    uint32_t bw, bh, tiles_x, tiles_y;
    tile_shape(W, H, bw, bh, tiles_x, tiles_y);
    const uint32_t nt = co_pad % 128u == 0u ? 128u : 64u;  // co_pad: a multiple of 64
    // the nine taps' weights stay in the weight stages' room (9 x nt x 64 bytes <= TS x B_STAGE) where the layer
    // reads one 32-channel block into one output tile
    uint32_t resident = cin == 32u && co_pad == nt && 9u * nt * 64u <= TS * B_STAGE ? 1u : 0u;
    // A layer of one output tile whose weights fit in shared memory beside three halo stages (up to four 32-channel
    // blocks at 64 outputs, two at 128), on an image at least 128 wide, reads its activations once a tile with the
    // halo: row tiles of 128 pixels (the last of a row ragged), boxes of 8 channels x 130 x 3, the weights resident.
    // (Row tiles that would leave more than an eighth of their pixels outside the image keep the 2-D tiles: at
    // 320 x 180 the row tiles measured 24.2 against 20.8 us.)
    const uint32_t kc = cin / 32u, row_tiles = (W + 127u) / 128u;
    const bool rows_ok = cin % 32u == 0u && W >= 128u && row_tiles * 128u - W <= row_tiles * 16u && (x_off % 8u) == 0u;
    const bool halo_res = rows_ok && co_pad == nt && conv_smem_halo(kc, nt) <= SMEM_MAX;
    // Other layers on such levels stream each stage's nine weight boxes beside its activations, one CTA an SM: as
    // many stages (up to three) as fit.
    const uint32_t stream_stage = HALO_A_ALIGNED + 9u * nt * 64u;
    const uint32_t stream_ns = std::min(HALO_TS, (SMEM_MAX - 1280u) / stream_stage);
    const bool halo = halo_res || (rows_ok && stream_ns >= 2u);
    const uint32_t stages = halo_res ? HALO_TS : stream_ns;
    const uint32_t smem = halo_res ? conv_smem_halo(kc, nt) : halo ? stages * stream_stage + 1280u : CONV_SMEM;
    // two CTAs an SM where their shared memory fits (228 KB an SM, 1 KB of it kept a CTA), else one
    const uint32_t per_sm = 2u * (smem + 1024u) <= 228u * 1024u ? CONV_CTAS_PER_SM : 1u;
    if (halo) {
        resident = halo_res ? 1u : 0u;
        bw = 128u;
        bh = 1u;
        tiles_x = (W + 127u) / 128u;
        tiles_y = H;
    }
    // the activations: boxes of 32 channels x bw x bh; the weights: (input channel, output channel, tap), boxes of
    // 32 x nt x 1; both 64-byte rows with the 64-byte swizzle
    CUtensorMap xmap, wmap;
    if (!(halo ? act_map(n, &xmap, x, x_stride, B, H, W, HALO_W, HALO_ROWS, true)
               : act_map(n, &xmap, x, x_stride, B, H, W, bw, bh)))
        return;
    cuuint64_t wd[3] = {cin, co_pad, 9u};
    cuuint64_t ws[2] = {(cuuint64_t)cin * 2u, (cuuint64_t)co_pad * cin * 2u};
    cuuint32_t wb[3] = {32u, nt, 1u}, es[3] = {1u, 1u, 1u};
    CUresult r = encode_tiled()(&wmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(w), wd, ws, wb, es,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        n->conv_err = "unet: a convolution's tensor map was refused (" + std::to_string((int)r) + ")";
        return;
    }
    Conv a{cin, co_pad, nt, bias, y, y_stride, y_off, cout, yf, B, H, W, x_off, bw, bh, tiles_x, tiles_y, relu,
           n->dev_err, resident, n->hold_next ? 1u : 0u, stages};
    n->hold_next = false;
    const uint32_t tiles = B * tiles_x * tiles_y * (co_pad / nt);
    const uint32_t grid = std::min<uint32_t>(tiles, n->sms * per_sm);
    if (halo) k_conv<true><<<grid, CONV_THREADS, smem, n->stream>>>(xmap, wmap, a);
    else k_conv<false><<<grid, CONV_THREADS, CONV_SMEM, n->stream>>>(xmap, wmap, a);
}

void conv(Net* n, int li, const Act& x, uint32_t x_off, const Act& y, uint32_t y_off, uint32_t B, uint32_t H, uint32_t W,
          float* yf = nullptr) {
    const Layer& L = LAYERS[li];
    conv_run(n, x.p, x.stride, x_off, L.cin, n->wf[li], r64(L.cout), n->w + n->off[li] + w_count(L), y.p, y.stride,
             y_off, L.cout, yf, B, H, W, L.relu);
}
// The input gradient of layer li: dx (channels [0, cin_logical)) from dy (cout rounded to 32 channels).
void conv_dx(Net* n, int li, const Act& dy, const Act& dx, uint32_t B, uint32_t H, uint32_t W) {
    const Layer& L = LAYERS[li];
    conv_run(n, dy.p, dy.stride, 0u, r32(L.cout), n->wb[li], r64(L.cin), nullptr, dx.p, dx.stride, 0u, L.cin, nullptr,
             B, H, W, 0);
}
// The weight and bias gradients of layer li from its input x (channels [x_off, x_off + cin)) and its output gradient dy
// (cout rounded to 32 channels), summed into the layer's gradients.
void wgrad(Net* n, int li, const Act& x, uint32_t x_off, const Act& dy, uint32_t B, uint32_t H, uint32_t W) {
    const Layer& L = LAYERS[li];
    uint32_t bw, bh, tiles_x, tiles_y;
    tile_shape(W, H, bw, bh, tiles_x, tiles_y);
    const uint32_t kc = L.cin / 32u, nb = r32(L.cout) / 32u, pairs = 9u * kc, groups = (pairs + 4u) / 4u;
    const uint32_t tiles = B * tiles_x * tiles_y, stage = (4u + nb) * WG_BOX;
    // two stages where two CTAs then fit an SM (228 KB, 1 KB of it reserved a CTA), else as many as one CTA holds
    uint32_t ts = 2u, per_sm = 2u;
    if (2u * (ts * stage + WG_SMEM_EXTRA + 1024u) > 228u * 1024u) {
        ts = std::min<uint32_t>(4u, (WG_SMEM_MAX - WG_SMEM_EXTRA) / stage);
        per_sm = 1u;
    }
    const uint32_t smem = ts * stage + WG_SMEM_EXTRA;
    // one wave: runs of tiles so that the groups x runs fill the SMs
    const uint32_t slots = n->sms * per_sm;
    const uint32_t chunk = std::max<uint32_t>(1u, (tiles * groups + slots - 1u) / slots);
    const uint32_t chunks = (tiles + chunk - 1u) / chunk;
    CUtensorMap xmap, dmap;
    if (!act_map(n, &xmap, x.p, x.stride, B, H, W, bw, bh) || !act_map(n, &dmap, dy.p, dy.stride, B, H, W, bw, bh))
        return;
    if (chunks * groups > n->wpart_ctas) {  // (at most the SMs' slots + groups, which the room holds)
        n->conv_err = "unet: the weight gradient's partials exceed their buffer";
        return;
    }
    WGrad a{L.cin, x_off, kc, nb, pairs, n->wpart, bw, bh, tiles_x, tiles_y, tiles, chunk, ts, n->dev_err};
    k_wgrad<<<dim3(chunks, groups), WG_THREADS, smem, n->stream>>>(xmap, dmap, a);
    float* dw = n->g + n->off[li];
    k_wgrad_sum<<<groups * 128u * nb * 8u / 32u, 32u * WS_SEGS, 0, n->stream>>>(
        n->wpart, chunks, groups, 32u * nb, kc, pairs, L.cin, r64(L.cout), dw, dw + w_count(L));
}
void relu_back(Net* n, const Act& dy, uint32_t dyo, const Act& y, uint32_t yo, uint32_t C, uint64_t P) {
    k_relu_back<<<blocks(P * C), 256, 0, n->stream>>>(dy.p, dy.stride, dyo, y.p, y.stride, yo, C, P);
}

void forward(Net* n, uint32_t B, uint32_t H, uint32_t W) {
    cudaStream_t s = n->stream;
    uint32_t H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
    uint64_t P0 = (uint64_t)B * H * W, P1 = (uint64_t)B * H1 * W1, P2 = (uint64_t)B * H2 * W2, P3 = (uint64_t)B * H3 * W3;
    conv(n, E0A, n->in0, 0, n->a0, 0, B, H, W);
    conv(n, E0B, n->a0, 0, n->cat0, 64, B, H, W);
    k_pool<<<blocks(P1 * 32 / 8), 256, 0, s>>>(n->cat0.p, 96, 64, n->pool0.p, 32, 32, B, H, W);
    conv(n, E1A, n->pool0, 0, n->a1, 0, B, H1, W1);
    conv(n, E1B, n->a1, 0, n->cat1, 96, B, H1, W1);
    k_pool<<<blocks(P2 * 64 / 8), 256, 0, s>>>(n->cat1.p, 160, 96, n->pool1.p, 64, 64, B, H1, W1);
    conv(n, E2A, n->pool1, 0, n->a2, 0, B, H2, W2);
    conv(n, E2B, n->a2, 0, n->cat2, 128, B, H2, W2);
    k_pool<<<blocks(P3 * 96 / 8), 256, 0, s>>>(n->cat2.p, 224, 128, n->pool2.p, 96, 96, B, H2, W2);
    conv(n, E3A, n->pool2, 0, n->a3, 0, B, H3, W3);
    conv(n, E3B, n->a3, 0, n->b3, 0, B, H3, W3);
    k_up<<<blocks(P2 * 128 / 8), 256, 0, s>>>(n->b3.p, 128, n->cat2.p, 224, 128, B, H2, W2);
    conv(n, D2A, n->cat2, 0, n->t2, 0, B, H2, W2);
    conv(n, D2B, n->t2, 0, n->u2, 0, B, H2, W2);
    k_up<<<blocks(P1 * 96 / 8), 256, 0, s>>>(n->u2.p, 96, n->cat1.p, 160, 96, B, H1, W1);
    conv(n, D1A, n->cat1, 0, n->t1, 0, B, H1, W1);
    conv(n, D1B, n->t1, 0, n->u1, 0, B, H1, W1);
    k_up<<<blocks(P0 * 64 / 8), 256, 0, s>>>(n->u1.p, 64, n->cat0.p, 96, 64, B, H, W);
    conv(n, D0A, n->cat0, 0, n->t0, 0, B, H, W);
    conv(n, D0B, n->t0, 0, n->u0, 0, B, H, W);
    conv(n, OUT, n->u0, 0, Act{}, 0, B, H, W, n->pred);
    (void)P0;
}

void backward(Net* n, uint32_t B, uint32_t H, uint32_t W) {
    cudaStream_t s = n->stream;
    uint32_t H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
    uint64_t P0 = (uint64_t)B * H * W, P1 = (uint64_t)B * H1 * W1, P2 = (uint64_t)B * H2 * W2, P3 = (uint64_t)B * H3 * W3;
    // output layer (linear)
    wgrad(n, OUT, n->u0, 0, n->dpred, B, H, W);
    conv_dx(n, OUT, n->dpred, n->du0, B, H, W);
    // level 0 decoder
    relu_back(n, n->du0, 0, n->u0, 0, 32, P0);
    wgrad(n, D0B, n->t0, 0, n->du0, B, H, W);
    conv_dx(n, D0B, n->du0, n->dt0, B, H, W);
    relu_back(n, n->dt0, 0, n->t0, 0, 32, P0);
    wgrad(n, D0A, n->cat0, 0, n->dt0, B, H, W);
    conv_dx(n, D0A, n->dt0, n->dcat0, B, H, W);
    k_up_back<<<blocks(P1 * 64), 256, 0, s>>>(n->dcat0.p, 96, n->du1.p, 64, 64, B, H1, W1);
    k_copy_ch<<<blocks(P0 * 32), 256, 0, s>>>(n->dcat0.p, 96, 64, n->de0b.p, 32, 0, 32, P0);
    // level 1 decoder
    relu_back(n, n->du1, 0, n->u1, 0, 64, P1);
    wgrad(n, D1B, n->t1, 0, n->du1, B, H1, W1);
    conv_dx(n, D1B, n->du1, n->dt1, B, H1, W1);
    relu_back(n, n->dt1, 0, n->t1, 0, 64, P1);
    wgrad(n, D1A, n->cat1, 0, n->dt1, B, H1, W1);
    conv_dx(n, D1A, n->dt1, n->dcat1, B, H1, W1);
    k_up_back<<<blocks(P2 * 96), 256, 0, s>>>(n->dcat1.p, 160, n->du2.p, 96, 96, B, H2, W2);
    k_copy_ch<<<blocks(P1 * 64), 256, 0, s>>>(n->dcat1.p, 160, 96, n->de1b.p, 64, 0, 64, P1);
    // level 2 decoder
    relu_back(n, n->du2, 0, n->u2, 0, 96, P2);
    wgrad(n, D2B, n->t2, 0, n->du2, B, H2, W2);
    conv_dx(n, D2B, n->du2, n->dt2, B, H2, W2);
    relu_back(n, n->dt2, 0, n->t2, 0, 96, P2);
    wgrad(n, D2A, n->cat2, 0, n->dt2, B, H2, W2);
    conv_dx(n, D2A, n->dt2, n->dcat2, B, H2, W2);
    k_up_back<<<blocks(P3 * 128), 256, 0, s>>>(n->dcat2.p, 224, n->db3.p, 128, 128, B, H3, W3);
    k_copy_ch<<<blocks(P2 * 96), 256, 0, s>>>(n->dcat2.p, 224, 128, n->de2b.p, 96, 0, 96, P2);
    // bottleneck
    relu_back(n, n->db3, 0, n->b3, 0, 128, P3);
    wgrad(n, E3B, n->a3, 0, n->db3, B, H3, W3);
    conv_dx(n, E3B, n->db3, n->da3, B, H3, W3);
    relu_back(n, n->da3, 0, n->a3, 0, 128, P3);
    wgrad(n, E3A, n->pool2, 0, n->da3, B, H3, W3);
    conv_dx(n, E3A, n->da3, n->dpool2, B, H3, W3);
    // level 2 encoder (its output's gradient: the skip's and the pooling's)
    k_pool_back<<<blocks(P2 * 96), 256, 0, s>>>(n->dpool2.p, 96, n->de2b.p, 96, 0, 96, B, H2, W2);
    relu_back(n, n->de2b, 0, n->cat2, 128, 96, P2);
    wgrad(n, E2B, n->a2, 0, n->de2b, B, H2, W2);
    conv_dx(n, E2B, n->de2b, n->da2, B, H2, W2);
    relu_back(n, n->da2, 0, n->a2, 0, 96, P2);
    wgrad(n, E2A, n->pool1, 0, n->da2, B, H2, W2);
    conv_dx(n, E2A, n->da2, n->dpool1, B, H2, W2);
    // level 1 encoder
    k_pool_back<<<blocks(P1 * 64), 256, 0, s>>>(n->dpool1.p, 64, n->de1b.p, 64, 0, 64, B, H1, W1);
    relu_back(n, n->de1b, 0, n->cat1, 96, 64, P1);
    wgrad(n, E1B, n->a1, 0, n->de1b, B, H1, W1);
    conv_dx(n, E1B, n->de1b, n->da1, B, H1, W1);
    relu_back(n, n->da1, 0, n->a1, 0, 64, P1);
    wgrad(n, E1A, n->pool0, 0, n->da1, B, H1, W1);
    conv_dx(n, E1A, n->da1, n->dpool0, B, H1, W1);
    // level 0 encoder
    k_pool_back<<<blocks(P0 * 32), 256, 0, s>>>(n->dpool0.p, 32, n->de0b.p, 32, 0, 32, B, H, W);
    relu_back(n, n->de0b, 0, n->cat0, 64, 32, P0);
    wgrad(n, E0B, n->a0, 0, n->de0b, B, H, W);
    conv_dx(n, E0B, n->de0b, n->da0, B, H, W);
    relu_back(n, n->da0, 0, n->a0, 0, 32, P0);
    wgrad(n, E0A, n->in0, 0, n->da0, B, H, W);
}

void refresh_weights(Net* n) {
    for (int li = 0; li < N_LAYERS; ++li) {
        const Layer& L = LAYERS[li];
        uint64_t cnt = w_count(L);
        k_weights<<<blocks(cnt), 256, 0, n->stream>>>(n->w + n->off[li], L.cin, r64(L.cout), r32(L.cout), n->wf[li],
                                                       li == E0A ? nullptr : n->wb[li], r64(L.cin));
    }
}

int check_size(Net* n, uint32_t B, uint32_t H, uint32_t W) {
    if (B == 0 || H == 0 || W == 0 || B > n->maxB || H > n->maxH || W > n->maxW || H % 8 || W % 8) {
        n->err = "unet: batch and image must be within the sizes given at creation, the image a multiple of 8";
        return TRT_EINVAL;
    }
    return TRT_OK;
}

int cuda_check(Net* n, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TRT_OK;
    n->err = std::string(what) + ": " + cudaGetErrorString(e);
    return TRT_ECUDA;
}

// The denoise of a device accum (rendered with TRT_RENDER_DEPTH) into the network's RGB buffer, on the network's
// current stream: the features, the forward pass, the radiance back.
void denoise_device(Net* n, const void* accum_device, uint32_t W, uint32_t H) {
    uint64_t P = (uint64_t)H * W;
    cudaStream_t s = n->stream;
    k_feat_sums<<<FEAT_BLOCKS, FEAT_THREADS, 0, s>>>((const float4*)accum_device, P, n->partial);
    k_feat_total<<<1, 32, 0, s>>>(n->partial, n->sums);
    k_feat<<<blocks(P), 256, 0, s>>>((const float4*)accum_device, P, n->sums, n->in0.p);
    forward(n, 1, H, W);
    k_unfeat<<<blocks(P * 3), 256, 0, s>>>(n->pred, P, n->sums, n->rgb);
}

// A training step's kernels, from the staged features and targets to the refreshed weights (Adam's scalars read from
// adam_args).
void train_kernels(Net* n, uint32_t B, uint32_t H, uint32_t W, int update) {
    uint64_t P = (uint64_t)B * H * W;
    cudaStream_t s = n->stream;
    k_feat_host<<<blocks(P * 32), 256, 0, s>>>(n->feat, P, n->in0.p);
    forward(n, B, H, W);
    cudaMemsetAsync(n->loss, 0, 4, s);
    cudaMemsetAsync(n->dpred.p, 0, 2 * 32 * P, s);
    cudaMemsetAsync(n->g, 0, 4 * n->n_params, s);
    k_loss<<<blocks(P * 3), 256, 0, s>>>(n->pred, n->target, P, n->dpred.p, n->loss);
    backward(n, B, H, W);
    if (update) {
        k_adam<<<blocks(n->n_params), 256, 0, s>>>(n->w, n->g, n->m, n->v, n->n_params, n->adam_args, 0.9f, 0.999f,
                                                    1e-8f);
        refresh_weights(n);
    }
}

// The training step's graph for this shape: captured from train_kernels on first use (a tensor map refused during
// the capture leaves no graph and the error in conv_err); at most MAX_STEP_GRAPHS shapes are kept.
constexpr size_t MAX_STEP_GRAPHS = 16;
cudaError_t step_graph(Net* n, uint32_t B, uint32_t H, uint32_t W, int update, cudaGraphExec_t* out) {
    for (const Net::StepGraph& g : n->graphs)
        if (g.B == B && g.H == H && g.W == W && g.update == update) {
            *out = g.exec;
            return cudaSuccess;
        }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(n->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    train_kernels(n, B, H, W, update);
    e = cudaStreamEndCapture(n->stream, &graph);
    if (e == cudaSuccess && !n->conv_err.empty()) e = cudaErrorInvalidValue;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return e;
    if (n->graphs.size() >= MAX_STEP_GRAPHS) {  // the oldest shape's graph makes room (its launches have finished:
        cudaGraphExecDestroy(n->graphs.front().exec);  // every call ends with the stream drained)
        n->graphs.erase(n->graphs.begin());
    }
    n->graphs.push_back({B, H, W, update, exec});
    *out = exec;
    return cudaSuccess;
}

// The end of a call: its stream drained, then what its convolutions reported (a refused tensor map on the host, a
// pipeline wait that gave up on the device).
int finish(Net* n, const char* what) {
    int rc = cuda_check(n, cudaStreamSynchronize(n->stream), what);
    if (!rc) rc = cuda_check(n, cudaGetLastError(), what);
    if (rc) return rc;
    if (!n->conv_err.empty()) {
        n->err = n->conv_err;
        n->conv_err.clear();
        return TRT_ECUDA;
    }
    uint32_t e = 0;
    rc = cuda_check(n, cudaMemcpy(&e, n->dev_err, 4, cudaMemcpyDeviceToHost), what);
    if (rc) return rc;
    if (e) {
        cudaMemset(n->dev_err, 0, 4);
        n->err = std::string(what) + ": a convolution's pipeline wait gave up";
        return TRT_ECUDA;
    }
    return TRT_OK;
}

}  // namespace
}  // namespace unet

using namespace unet;

extern "C" {

uint64_t trt_unet_param_count(void) { return param_count(); }

int trt_unet_create(int device, uint32_t max_batch, uint32_t max_h, uint32_t max_w, trt_unet** out) {
    if (!out || max_batch == 0 || max_h < 8 || max_w < 8 || max_h % 8 || max_w % 8) return TRT_EINVAL;
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return TRT_ECUDA;
    auto* n = new trt_unet();
    n->device = device;
    n->maxB = max_batch;
    n->maxH = max_h;
    n->maxW = max_w;
    n->n_params = param_count();
    uint64_t o = 0;
    for (int li = 0; li < N_LAYERS; ++li) {
        n->off[li] = o;
        o += layer_params(LAYERS[li]);
    }
    uint64_t P0 = (uint64_t)max_batch * max_h * max_w, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
    e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
    auto A = [&](Act& a, uint64_t px, uint32_t st) { if (e == cudaSuccess) e = act(n, a, px, st); };
    if (e == cudaSuccess) e = alloc(n, &n->w, n->n_params);
    if (e == cudaSuccess) e = alloc(n, &n->g, n->n_params);
    if (e == cudaSuccess) e = alloc(n, &n->m, n->n_params);
    if (e == cudaSuccess) e = alloc(n, &n->v, n->n_params);
    for (int li = 0; li < N_LAYERS && e == cudaSuccess; ++li) {
        const Layer& L = LAYERS[li];
        e = alloc(n, &n->wf[li], w_count(L));
        if (e == cudaSuccess) e = alloc(n, &n->wb[li], 9ull * r32(L.cout) * r64(L.cin));
    }
    A(n->in0, P0, 32); A(n->a0, P0, 32); A(n->cat0, P0, 96); A(n->pool0, P1, 32); A(n->a1, P1, 64);
    A(n->cat1, P1, 160); A(n->pool1, P2, 64); A(n->a2, P2, 96); A(n->cat2, P2, 224); A(n->pool2, P3, 96);
    A(n->a3, P3, 128); A(n->b3, P3, 128); A(n->t2, P2, 96); A(n->u2, P2, 96); A(n->t1, P1, 64); A(n->u1, P1, 64);
    A(n->t0, P0, 32); A(n->u0, P0, 32);
    A(n->dpred, P0, 32); A(n->du0, P0, 32); A(n->dt0, P0, 32); A(n->dcat0, P0, 96); A(n->du1, P1, 64);
    A(n->dt1, P1, 64); A(n->dcat1, P1, 160); A(n->du2, P2, 96); A(n->dt2, P2, 96); A(n->dcat2, P2, 224);
    A(n->db3, P3, 128); A(n->da3, P3, 128); A(n->dpool2, P3, 96); A(n->de2b, P2, 96); A(n->da2, P2, 96);
    A(n->dpool1, P2, 64); A(n->de1b, P1, 64); A(n->da1, P1, 64); A(n->dpool0, P1, 32); A(n->de0b, P0, 32);
    A(n->da0, P0, 32);
    if (e == cudaSuccess) e = alloc(n, &n->pred, P0 * 3);
    if (e == cudaSuccess) e = alloc(n, &n->target, P0 * 3);
    if (e == cudaSuccess) e = alloc(n, &n->feat, P0 * N_FEAT);
    if (e == cudaSuccess) e = alloc(n, &n->rgb, P0 * 3);
    if (e == cudaSuccess) e = alloc(n, &n->loss, 4);
    if (e == cudaSuccess) e = alloc(n, &n->sums, 4);
    if (e == cudaSuccess) e = alloc(n, &n->dev_err, 1);
    if (e == cudaSuccess) e = alloc(n, &n->partial, 3 * FEAT_BLOCKS);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_conv<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WG_SMEM_MAX);
    if (e == cudaSuccess) {
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (sms > 0) n->sms = (uint32_t)sms;
        n->wpart_ctas = 2u * n->sms + 16u;
        e = alloc(n, &n->wpart, (uint64_t)n->wpart_ctas * 128u * 128u);
    }
    if (e == cudaSuccess) e = alloc(n, &n->adam_args, 4);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&n->adam_host, 16);
    if (e == cudaSuccess) e = cudaEventCreate(&n->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&n->e1);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "trt_unet_create: %s\n", cudaGetErrorString(e));
        trt_unet_destroy(n);
        return TRT_ECUDA;
    }
    *out = n;
    return TRT_OK;
}

void trt_unet_destroy(trt_unet* n) {
    if (!n) return;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    for (const Net::StepGraph& g : n->graphs) cudaGraphExecDestroy(g.exec);
    if (n->adam_host) cudaFreeHost(n->adam_host);
    for (void* p : n->allocs) cudaFree(p);
    if (n->e0) cudaEventDestroy(n->e0);
    if (n->e1) cudaEventDestroy(n->e1);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

const char* trt_unet_last_error(const trt_unet* n) { return n ? n->err.c_str() : "no network"; }

int trt_unet_set_params(trt_unet* n, const float* params) {
    if (!n || !params) return TRT_EINVAL;
    cudaSetDevice(n->device);
    int rc = cuda_check(n, cudaMemcpyAsync(n->w, params, 4 * n->n_params, cudaMemcpyHostToDevice, n->stream), "params");
    if (rc) return rc;
    cudaMemsetAsync(n->m, 0, 4 * n->n_params, n->stream);
    cudaMemsetAsync(n->v, 0, 4 * n->n_params, n->stream);
    n->t = 0;
    refresh_weights(n);
    return cuda_check(n, cudaStreamSynchronize(n->stream), "params");
}

int trt_unet_get_params(trt_unet* n, float* params) {
    if (!n || !params) return TRT_EINVAL;
    cudaSetDevice(n->device);
    cudaMemcpyAsync(params, n->w, 4 * n->n_params, cudaMemcpyDeviceToHost, n->stream);
    return cuda_check(n, cudaStreamSynchronize(n->stream), "params");
}

int trt_unet_forward(trt_unet* n, const float* features, uint32_t B, uint32_t H, uint32_t W, float* pred, float* ms) {
    if (!n || !features || !pred) return TRT_EINVAL;
    cudaSetDevice(n->device);
    int rc = check_size(n, B, H, W);
    if (rc) return rc;
    uint64_t P = (uint64_t)B * H * W;
    cudaMemcpyAsync(n->feat, features, 4ull * N_FEAT * P, cudaMemcpyHostToDevice, n->stream);
    cudaEventRecord(n->e0, n->stream);
    k_feat_host<<<blocks(P * 32), 256, 0, n->stream>>>(n->feat, P, n->in0.p);
    forward(n, B, H, W);
    cudaEventRecord(n->e1, n->stream);
    cudaMemcpyAsync(pred, n->pred, 12 * P, cudaMemcpyDeviceToHost, n->stream);
    rc = finish(n, "trt_unet_forward");
    if (!rc && ms) cudaEventElapsedTime(ms, n->e0, n->e1);
    return rc;
}

int trt_unet_hold_next_load(trt_unet* n) {
    if (!n) return TRT_EINVAL;
    n->hold_next = true;
    return TRT_OK;
}

int trt_unet_train_step(trt_unet* n, const float* features, const float* targets, uint32_t B, uint32_t H, uint32_t W,
                        float lr, int update, float* loss, float* grads, float* ms) {
    if (!n || !features || !targets) return TRT_EINVAL;
    n->hold_next = false;  // (the step is captured in a graph: a withheld copy is for direct launches only)
    cudaSetDevice(n->device);
    int rc = check_size(n, B, H, W);
    if (rc) return rc;
    uint64_t P = (uint64_t)B * H * W;
    cudaStream_t s = n->stream;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = step_graph(n, B, H, W, update ? 1 : 0, &exec);
    if (e != cudaSuccess) {
        if (!n->conv_err.empty()) {
            n->err = n->conv_err;
            n->conv_err.clear();
            return TRT_ECUDA;
        }
        return cuda_check(n, e, "trt_unet_train_step: the step's graph");
    }
    if (update) {
        n->t++;
        n->adam_host[0] = lr;
        n->adam_host[1] = 1.0f - std::pow(0.9f, (float)n->t);
        n->adam_host[2] = 1.0f - std::pow(0.999f, (float)n->t);
        cudaMemcpyAsync(n->adam_args, n->adam_host, 12, cudaMemcpyHostToDevice, s);
    }
    cudaMemcpyAsync(n->feat, features, 4ull * N_FEAT * P, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(n->target, targets, 12 * P, cudaMemcpyHostToDevice, s);
    cudaEventRecord(n->e0, s);
    cudaGraphLaunch(exec, s);
    cudaEventRecord(n->e1, s);
    if (loss) cudaMemcpyAsync(loss, n->loss, 4, cudaMemcpyDeviceToHost, s);
    if (grads) cudaMemcpyAsync(grads, n->g, 4 * n->n_params, cudaMemcpyDeviceToHost, s);
    rc = finish(n, "trt_unet_train_step");
    if (!rc && ms) cudaEventElapsedTime(ms, n->e0, n->e1);
    return rc;
}

int trt_unet_denoise_accum(trt_unet* n, const void* accum_device, uint32_t W, uint32_t H, float* rgb_host, float* ms) {
    if (!n || !accum_device || !rgb_host) return TRT_EINVAL;
    cudaSetDevice(n->device);
    int rc = check_size(n, 1, H, W);
    if (rc) return rc;
    uint64_t P = (uint64_t)H * W;
    cudaStream_t s = n->stream;
    cudaEventRecord(n->e0, s);
    denoise_device(n, accum_device, W, H);
    cudaEventRecord(n->e1, s);
    cudaMemcpyAsync(rgb_host, n->rgb, 12 * P, cudaMemcpyDeviceToHost, s);
    rc = finish(n, "trt_unet_denoise_accum");
    if (!rc && ms) cudaEventElapsedTime(ms, n->e0, n->e1);
    return rc;
}

}  // extern "C"

// The serving loop's denoise: on its stream, into the network's RGB buffer (returned; null when the image is not a
// size the network takes, or a convolution's tensor map was refused). The network belongs to the server meanwhile.
const float* unet_denoise_on_stream(trt_unet* n, const void* accum_device, uint32_t w, uint32_t h, cudaStream_t st) {
    if (!n || !accum_device || w == 0 || h == 0 || h > n->maxH || w > n->maxW || h % 8 || w % 8) return nullptr;
    cudaStream_t own = n->stream;
    n->stream = st;
    denoise_device(n, accum_device, w, h);
    n->stream = own;
    if (!n->conv_err.empty()) return nullptr;
    return n->rgb;
}

bool unet_fits(const trt_unet* n, uint32_t w, uint32_t h) {
    return n && w > 0 && h > 0 && h <= n->maxH && w <= n->maxW && h % 8 == 0 && w % 8 == 0;
}
