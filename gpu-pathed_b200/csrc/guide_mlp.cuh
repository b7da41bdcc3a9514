// Guide network inference on the tensor cores: one warp evaluates 16 samples through the
// four layers with BF16 mma.sync (m16n8k16, FP32 accumulate). Each layer's FP32
// accumulators are ReLU'd and re-packed in registers as the next layer's A fragments (the
// m16n8 accumulator layout coincides with the m16k16 operand layout), so activations never
// leave registers; weights are read from shared memory in B-fragment order.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "guide.cuh"

namespace pt {

// Shared-memory layout of the packed weights (32-bit words). Rows hold BF16 pairs of two
// consecutive input rows (k, k+1); row strides are padded (72 and 40 words) so that the
// B-fragment loads of a warp hit 32 distinct banks.
constexpr int kSW1 = 0;                          // 40 rows x 72
constexpr int kSW2 = kSW1 + 40 * 72;             // 32 rows x 72
constexpr int kSW3 = kSW2 + 32 * 72;             // 32 rows x 72
constexpr int kSW4 = kSW3 + 32 * 72;             // 32 rows x 40
constexpr int kSB = kSW4 + 32 * 40;              // biases (FP32 bits): b1 64, b2 64, b3 64, b4 40
constexpr int kSWords = kSB + 3 * 64 + 40;       // 9000 words = 36000 bytes
constexpr int kSXStride = 44;                    // words per input row of a warp's 16 x 80 tile
// Shared-memory copy of the transposed weights for the backward pass (dA = dZ W^T): one row
// per layer input k, each word a BF16 pair of two consecutive outputs (n, n + 1); rows of 32
// words (W4: 40 outputs zero-padded to 48, 24 words) at a stride of 36 words, so that the
// B-fragment loads of a warp cover 32 distinct banks.
constexpr int kSTStride = 36;
constexpr int kST2 = 0, kST3 = kST2 + 64 * kSTStride, kST4 = kST3 + 64 * kSTStride;
constexpr int kSTWords = kST4 + 64 * kSTStride;  // 6912 words
// The packed weights in global memory are the two shared-memory images back to back
// (forward, then transposed), so that a block loads them with plain 16-byte copies.
constexpr int kPackT = kSWords;
constexpr int kPackWords = kSWords + kSTWords;  // 15912 words
static_assert(kSWords % 4 == 0 && kSTWords % 4 == 0, "16-byte copies");

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void copy_words16(const uint32_t* __restrict__ src, uint32_t* dst, int words) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int i = threadIdx.x; i < words / 4; i += blockDim.x) d[i] = s[i];
}

// Copy the forward weight image into shared memory (all threads of the block).
__device__ __forceinline__ void guide_load_weights(const uint32_t* __restrict__ gw, uint32_t* sw) {
    copy_words16(gw, sw, kSWords);
}

// Copy the transposed weight image into shared memory (all threads of the block).
__device__ __forceinline__ void guide_load_weights_t(const uint32_t* __restrict__ gw, uint32_t* swt) {
    copy_words16(gw + kPackT, swt, kSTWords);
}

// ldmatrix of four (two) 8x8 BF16 tiles, transposed on the way into registers.
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const uint32_t* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t& r0, uint32_t& r1, const uint32_t* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}

// Store a warp's 16 x 64 BF16 activation tile (A-fragment registers) into shared memory,
// row-major with `stride` words per row.
__device__ __forceinline__ void guide_store_frag(uint32_t* dst, int stride, const uint32_t (&h)[4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
        dst[g * stride + kt * 8 + t] = h[kt][0];
        dst[(g + 8) * stride + kt * 8 + t] = h[kt][1];
        dst[g * stride + kt * 8 + 4 + t] = h[kt][2];
        dst[(g + 8) * stride + kt * 8 + 4 + t] = h[kt][3];
    }
}

// Hidden layer: 64 outputs from K = 16 * KT inputs held as A fragments.
template <int KT>
__device__ __forceinline__ void guide_hidden(const uint32_t* sw, int w_off, int b_off, const uint32_t (&a)[KT][4],
                                             uint32_t (&out)[4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = __uint_as_float(sw[b_off + nt * 8 + 2 * t]);
        const float b1 = __uint_as_float(sw[b_off + nt * 8 + 2 * t + 1]);
        acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < KT; kt++) {
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint32_t b0 = sw[w_off + (kt * 8 + t) * 72 + nt * 8 + g];
            const uint32_t b1 = sw[w_off + (kt * 8 + 4 + t) * 72 + nt * 8 + g];
            mma16816(acc[nt], a[kt][0], a[kt][1], a[kt][2], a[kt][3], b0, b1);
        }
    }
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
        out[kt][0] = pack_bf16(fmaxf(acc[2 * kt][0], 0.f), fmaxf(acc[2 * kt][1], 0.f));
        out[kt][1] = pack_bf16(fmaxf(acc[2 * kt][2], 0.f), fmaxf(acc[2 * kt][3], 0.f));
        out[kt][2] = pack_bf16(fmaxf(acc[2 * kt + 1][0], 0.f), fmaxf(acc[2 * kt + 1][1], 0.f));
        out[kt][3] = pack_bf16(fmaxf(acc[2 * kt + 1][2], 0.f), fmaxf(acc[2 * kt + 1][3], 0.f));
    }
}

// Full network for the warp's 16 samples. sx: 16 rows x kSXStride words (BF16 input pairs);
// sy: 16 rows x 40 floats of raw outputs.
__device__ __forceinline__ void guide_mlp_warp16(const uint32_t* sw, const uint32_t* sx, float* sy) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a1[5][4];
#pragma unroll
    for (int kt = 0; kt < 5; kt++) {
        a1[kt][0] = sx[g * kSXStride + kt * 8 + t];
        a1[kt][1] = sx[(g + 8) * kSXStride + kt * 8 + t];
        a1[kt][2] = sx[g * kSXStride + kt * 8 + 4 + t];
        a1[kt][3] = sx[(g + 8) * kSXStride + kt * 8 + 4 + t];
    }
    uint32_t h1[4][4], h2[4][4], h3[4][4];
    guide_hidden<5>(sw, kSW1, kSB, a1, h1);
    guide_hidden<4>(sw, kSW2, kSB + 64, h1, h2);
    guide_hidden<4>(sw, kSW3, kSB + 128, h2, h3);
    float acc[5][4];
#pragma unroll
    for (int nt = 0; nt < 5; nt++) {
        const float b0 = __uint_as_float(sw[kSB + 192 + nt * 8 + 2 * t]);
        const float b1 = __uint_as_float(sw[kSB + 192 + nt * 8 + 2 * t + 1]);
        acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
#pragma unroll
        for (int nt = 0; nt < 5; nt++) {
            const uint32_t b0 = sw[kSW4 + (kt * 8 + t) * 40 + nt * 8 + g];
            const uint32_t b1 = sw[kSW4 + (kt * 8 + 4 + t) * 40 + nt * 8 + g];
            mma16816(acc[nt], h3[kt][0], h3[kt][1], h3[kt][2], h3[kt][3], b0, b1);
        }
    }
#pragma unroll
    for (int nt = 0; nt < 5; nt++) {
        sy[g * kGuideOut + nt * 8 + 2 * t] = acc[nt][0];
        sy[g * kGuideOut + nt * 8 + 2 * t + 1] = acc[nt][1];
        sy[(g + 8) * kGuideOut + nt * 8 + 2 * t] = acc[nt][2];
        sy[(g + 8) * kGuideOut + nt * 8 + 2 * t + 1] = acc[nt][3];
    }
}

// Hidden layer for R groups of 16 rows: each B fragment is loaded once for all groups.
template <int KT, int R>
__device__ __forceinline__ void guide_hidden_rows(const uint32_t* sw, int w_off, int b_off,
                                                  const uint32_t (&a)[R][KT][4], uint32_t (&out)[R][4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[R][8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = __uint_as_float(sw[b_off + nt * 8 + 2 * t]);
        const float b1 = __uint_as_float(sw[b_off + nt * 8 + 2 * t + 1]);
#pragma unroll
        for (int r = 0; r < R; r++) {
            acc[r][nt][0] = b0; acc[r][nt][1] = b1; acc[r][nt][2] = b0; acc[r][nt][3] = b1;
        }
    }
#pragma unroll
    for (int kt = 0; kt < KT; kt++) {
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint32_t b0 = sw[w_off + (kt * 8 + t) * 72 + nt * 8 + g];
            const uint32_t b1 = sw[w_off + (kt * 8 + 4 + t) * 72 + nt * 8 + g];
#pragma unroll
            for (int r = 0; r < R; r++) mma16816(acc[r][nt], a[r][kt][0], a[r][kt][1], a[r][kt][2], a[r][kt][3], b0, b1);
        }
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            out[r][kt][0] = pack_bf16(fmaxf(acc[r][2 * kt][0], 0.f), fmaxf(acc[r][2 * kt][1], 0.f));
            out[r][kt][1] = pack_bf16(fmaxf(acc[r][2 * kt][2], 0.f), fmaxf(acc[r][2 * kt][3], 0.f));
            out[r][kt][2] = pack_bf16(fmaxf(acc[r][2 * kt + 1][0], 0.f), fmaxf(acc[r][2 * kt + 1][1], 0.f));
            out[r][kt][3] = pack_bf16(fmaxf(acc[r][2 * kt + 1][2], 0.f), fmaxf(acc[r][2 * kt + 1][3], 0.f));
        }
    }
}

// Full network for 32 samples (two 16-row groups sharing the weight fragments). sx: 32 rows x
// kSXStride words; the raw outputs of group r (16 rows x 40 floats) overwrite the first 640
// words of its 16 input rows.
__device__ __forceinline__ void guide_mlp_warp32(const uint32_t* sw, uint32_t* sx) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a1[2][5][4];
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const uint32_t* x = sx + r * 16 * kSXStride;
#pragma unroll
        for (int kt = 0; kt < 5; kt++) {
            a1[r][kt][0] = x[g * kSXStride + kt * 8 + t];
            a1[r][kt][1] = x[(g + 8) * kSXStride + kt * 8 + t];
            a1[r][kt][2] = x[g * kSXStride + kt * 8 + 4 + t];
            a1[r][kt][3] = x[(g + 8) * kSXStride + kt * 8 + 4 + t];
        }
    }
    uint32_t h1[2][4][4], h2[2][4][4];
    guide_hidden_rows<5, 2>(sw, kSW1, kSB, a1, h1);
    guide_hidden_rows<4, 2>(sw, kSW2, kSB + 64, h1, h2);
    guide_hidden_rows<4, 2>(sw, kSW3, kSB + 128, h2, h1);
    float acc[2][5][4];
#pragma unroll
    for (int nt = 0; nt < 5; nt++) {
        const float b0 = __uint_as_float(sw[kSB + 192 + nt * 8 + 2 * t]);
        const float b1 = __uint_as_float(sw[kSB + 192 + nt * 8 + 2 * t + 1]);
#pragma unroll
        for (int r = 0; r < 2; r++) {
            acc[r][nt][0] = b0; acc[r][nt][1] = b1; acc[r][nt][2] = b0; acc[r][nt][3] = b1;
        }
    }
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
#pragma unroll
        for (int nt = 0; nt < 5; nt++) {
            const uint32_t b0 = sw[kSW4 + (kt * 8 + t) * 40 + nt * 8 + g];
            const uint32_t b1 = sw[kSW4 + (kt * 8 + 4 + t) * 40 + nt * 8 + g];
#pragma unroll
            for (int r = 0; r < 2; r++)
                mma16816(acc[r][nt], h1[r][kt][0], h1[r][kt][1], h1[r][kt][2], h1[r][kt][3], b0, b1);
        }
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
        float* sy = reinterpret_cast<float*>(sx + r * 16 * kSXStride);
#pragma unroll
        for (int nt = 0; nt < 5; nt++) {
            sy[g * kGuideOut + nt * 8 + 2 * t] = acc[r][nt][0];
            sy[g * kGuideOut + nt * 8 + 2 * t + 1] = acc[r][nt][1];
            sy[(g + 8) * kGuideOut + nt * 8 + 2 * t] = acc[r][nt][2];
            sy[(g + 8) * kGuideOut + nt * 8 + 2 * t + 1] = acc[r][nt][3];
        }
    }
}

// Write one sample's 80 inputs as BF16 pairs into row `row` of the warp's input tile.
__device__ __forceinline__ void guide_store_input(uint32_t* sx, int row, const float x[kGuideIn]) {
#pragma unroll
    for (int k = 0; k < kGuideIn / 2; k++) sx[row * kSXStride + k] = pack_bf16(x[2 * k], x[2 * k + 1]);
}

}  // namespace pt
