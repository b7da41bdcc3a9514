// Guide network training on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One CTA of 256 threads (8 warps) per SM walks tiles of 256 samples, two sub-tiles of 128
// (the MMA's M), one thread per sample. Per tile:
//   1. every thread encodes its sample into row `row` of its sub-tile's X tile (BF16);
//   2. forward: for each layer one thread issues the MMAs of both sub-tiles into their FP32
//      scratch accumulators in tensor memory and commits; the epilogue (bias, ReLU, BF16)
//      writes the layer's activations A1, A2, A3 into their own tiles, kept for backward;
//   3. every thread computes its sample's loss gradient dY (FP32, stored as BF16);
//   4. backward, per layer l = 4, 3, 2: the weight-gradient product W_l' += A_{l-1}^T dZ_l
//      and the data product dZ_{l-1} = (dZ_l W_l) [A_{l-1} > 0] issued together; the masked
//      dZ_{l-1} overwrites A_{l-1} in place once both have completed; then W_1' += X^T dZ_1.
// The weight-gradient products contract over the samples: D'[i][o] = sum_s A[s][i] dZ[s][o]
// with M' = 128 rows of layer inputs i and K' = the tile's samples. Both operands are the
// sample-major activation tiles read through MN-major descriptors (the inputs i, resp. the
// outputs o, contiguous), so nothing is transposed. The four gradient accumulators (240 of
// the 512 TMEM columns) stay in tensor memory across every tile the CTA processes and are
// added to the global gradient once at the end. The bias gradients ride on a ones column:
// input 78 of X (b1, as in the mma.sync kernel) and feature 64 of A1-A3 (b2-b4). The
// backward data products read the forward weight images (K-major in the inputs) through
// MN-major descriptors as well: B[i][o] = W[o][i].
//
// Every wait on the mbarrier is bounded: one that gives up counts a failure in the
// network's sums (word 2), waits (bounded) for the MMAs in flight, frees tensor memory and
// returns without adding its partial gradient.
#pragma once

#include "guide_tc.cuh"

namespace pt {

constexpr int kTtSub = 2;                     // 128-sample sub-tiles per CTA tile
constexpr int kTtThreads = kTcRows * kTtSub;  // 256
constexpr int kTtRows = kTcRows * kTtSub;     // samples per CTA tile
constexpr int kTtFeatBytes = 10 * kTcLboA;    // a 128 x 80 BF16 tile: 20,480 B
constexpr int kTtDyBytes = 6 * kTcLboA;       // 128 x 48 (40 output gradients + 8 zeros)
// TMEM columns: the gradient accumulators, then one scratch accumulator per sub-tile
constexpr uint32_t kTtColW1 = 0, kTtColW2 = 64, kTtColW3 = 128, kTtColW4 = 192;  // W4: 48 columns
constexpr uint32_t kTtColScratch = 256;  // + 64 per sub-tile
constexpr uint32_t kTtTmemCols = 512;

struct TtSubTile {
    uint8_t x[kTtFeatBytes];   // inputs (80; input 78 set to one before the W1 product)
    uint8_t a1[kTtFeatBytes];  // activations (64) + ones column (64) + zeros; then dZ1
    uint8_t a2[kTtFeatBytes];  // then dZ2
    uint8_t a3[kTtFeatBytes];  // then dZ3
    uint8_t dy[kTtDyBytes];    // loss gradient of the raw outputs
};
// A weight-gradient product reads 128 feature rows (16 groups of 8 at the tile's 2,048-byte
// chunk stride: 32 KB) from the start of a 20 KB tile: rows past the tile's own features
// read the next tile (garbage rows of the accumulator, never used). The tiles of a sub-tile
// are consecutive, and the last over-read (A3's) ends exactly at the end of dY.
static_assert(sizeof(TtSubTile) == 4 * kTtFeatBytes + kTtDyBytes, "packed sub-tile");
static_assert(3 * kTtFeatBytes + 16 * kTcLboA <= (int)sizeof(TtSubTile), "A3 over-read inside its sub-tile");

struct TtSmem {
    uint8_t w[kTcWBytes];        // forward weight images (K-major in the inputs)
    TtSubTile sub[kTtSub];
    float bias[64 * 3 + 48];     // b1, b2, b3, b4 (b4 zero-padded to 48)
    unsigned long long mbar;
    uint32_t tmem_slot;
};

// Instruction descriptor with MN-major (transposed) A and/or B operands (bits 15, 16).
__host__ __device__ constexpr uint32_t tc_idesc_t(int m, int n, bool a_mn, bool b_mn) {
    return tc_idesc(m, n) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u);
}
// MN-major no-swizzle descriptor of a tile laid out by tc_offset (chunk stride `chunk` along
// the contiguous dimension): groups of 8 contiguous elements `chunk` bytes apart (SBO), K
// groups of 8 rows 128 bytes apart (LBO).
__device__ __forceinline__ uint64_t tc_desc_mn(uint32_t saddr, uint32_t chunk) {
    return tc_smem_desc(saddr, 128u, chunk);
}

// Weight-gradient product of one sub-tile: D'[i][o] (+)= sum over its 128 samples of
// A[s][i] dZ[s][o]; `a` the activations (MN-major, 128 rows i), `b` the output gradients
// (MN-major, n columns o), both with the 2,048-byte chunk stride.
__device__ __forceinline__ void tt_wgrad(uint32_t tmem_d, uint32_t a, uint32_t b, int n, bool first) {
    const uint32_t idesc = tc_idesc_t(kTcRows, n, true, true);
    for (int s = 0; s < kTcRows / 16; s++)  // 16 samples per MMA: two 8-row groups, 256 B
        tc_mma(tmem_d, tc_desc_mn(a + s * 256, kTcLboA), tc_desc_mn(b + s * 256, kTcLboA), idesc,
               (first && s == 0) ? 0u : 1u);
}
// Backward data product of one sub-tile: D[s][i] = sum_o dZ[s][o] W[o][i]; `a` the output
// gradients (K-major, k columns), `w` the layer's forward image read MN-major (64 inputs i,
// chunk stride `wchunk`).
__device__ __forceinline__ void tt_bdata(uint32_t tmem_d, uint32_t a, uint32_t w, int k, uint32_t wchunk) {
    const uint32_t idesc = tc_idesc_t(kTcRows, 64, false, true);
    for (int s = 0; s < k / 16; s++)
        tc_mma(tmem_d, tc_smem_desc(a + s * 2 * kTcLboA, kTcLboA, 128), tc_desc_mn(w + s * 256, wchunk), idesc,
               s > 0 ? 1u : 0u);
}

// This thread's 64 accumulator columns masked by its row of the ReLU input A (BF16, > 0),
// written back as BF16 over A (the row's own elements only).
__device__ __forceinline__ void tt_epilogue_mask(uint32_t tmem_row, uint8_t* tile, int row) {
#pragma unroll
    for (int c = 0; c < 64; c += 16) {
        float v[16];
        tc_ld16(tmem_row + c, v);
        tc_wait_ld();
        uint4* p0 = reinterpret_cast<uint4*>(tile + tc_offset(row, c, kTcLboA));
        uint4* p1 = reinterpret_cast<uint4*>(tile + tc_offset(row, c + 8, kTcLboA));
        const uint4 a0 = *p0, a1 = *p1;
        const uint32_t av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        uint32_t w[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            // BF16 > 0: sign bit clear and not zero
            const bool lo = (av[j] & 0x8000u) == 0u && (av[j] & 0x7FFFu) != 0u;
            const bool hi = (av[j] & 0x80000000u) == 0u && (av[j] & 0x7FFF0000u) != 0u;
            w[j] = pack_bf16(lo ? v[2 * j] : 0.f, hi ? v[2 * j + 1] : 0.f);
        }
        *p0 = make_uint4(w[0], w[1], w[2], w[3]);
        *p1 = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// Wait for the commit of phase `phase`; false (with the MMAs in flight drained) when it gave up.
__device__ __forceinline__ bool tt_wait(uint32_t mbar, uint32_t& phase) {
    const int kLimit = 1 << 22;
    const bool done = mbar_wait(mbar, phase, kLimit);
    if (!__syncthreads_and(done ? 1 : 0)) {
        mbar_wait(mbar, phase, kLimit);
        return false;
    }
    phase ^= 1u;
    tc_fence_after();
    return true;
}

}  // namespace pt
