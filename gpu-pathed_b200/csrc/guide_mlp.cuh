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
// Global packed layout (unpadded): W1 40x64, W2 32x64, W3 32x64, W4 32x40, biases.
constexpr int kGP1 = 0, kGP2 = 2560, kGP3 = 4608, kGP4 = 6656, kGPB = 7936;

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

// Copy the packed global weights into shared memory with the padded strides (all threads).
__device__ __forceinline__ void guide_load_weights(const uint32_t* __restrict__ gw, uint32_t* sw) {
    for (int i = threadIdx.x; i < kSWords; i += blockDim.x) {
        uint32_t v;
        if (i < kSW2) {
            const int r = i / 72, c = i % 72;
            v = c < 64 ? gw[kGP1 + r * 64 + c] : 0u;
        } else if (i < kSW3) {
            const int j = i - kSW2, r = j / 72, c = j % 72;
            v = c < 64 ? gw[kGP2 + r * 64 + c] : 0u;
        } else if (i < kSW4) {
            const int j = i - kSW3, r = j / 72, c = j % 72;
            v = c < 64 ? gw[kGP3 + r * 64 + c] : 0u;
        } else if (i < kSB) {
            const int j = i - kSW4;
            v = gw[kGP4 + j];
        } else {
            v = gw[kGPB + (i - kSB)];
        }
        sw[i] = v;
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

// Write one sample's 80 inputs as BF16 pairs into row `row` of the warp's input tile.
__device__ __forceinline__ void guide_store_input(uint32_t* sx, int row, const float x[kGuideIn]) {
#pragma unroll
    for (int k = 0; k < kGuideIn / 2; k++) sx[row * kSXStride + k] = pack_bf16(x[2 * k], x[2 * k + 1]);
}

}  // namespace pt
