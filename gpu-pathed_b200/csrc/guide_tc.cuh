// Guide network inference on the 5th-generation tensor cores (tcgen05, sm_100a): one CTA of
// 256 threads evaluates tiles of 256 samples, two sub-tiles of 128 (the MMA's M), one thread
// per sample; one thread issues both sub-tiles' MMAs of a layer before a single commit, so
// each commit-and-wait round serves 256 samples and one weight copy serves the whole CTA.
//
// Per layer: the activations (M x K, BF16) and the transposed weights (N x K, BF16) sit in
// shared memory in the canonical K-major, no-swizzle layout of the UMMA descriptors (core
// matrices of 8 rows x 16 bytes; LBO = byte stride between 8-element K chunks, SBO = byte
// stride between 8-row groups); one thread issues K/16 `tcgen05.mma.kind::f16` into an FP32
// accumulator of N columns in tensor memory and commits them to an mbarrier; every warp then
// reads its 32 rows back with `tcgen05.ld.32x32b`, adds the bias, applies ReLU and writes the
// BF16 row into the next layer's A tile. Waits are bounded: a wait that gives up raises an
// error flag and the tile's outputs are not used.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "guide_mlp.cuh"

namespace pt {

// ---- shared-memory images (bytes) -------------------------------------------------------
// B operands: N rows (layer outputs) x K (layer inputs); chunk c holds k in [8c, 8c + 8).
constexpr int kTcW1 = 0;                       // N 64, K 80: 10 chunks x 8 row groups x 128 B
constexpr int kTcW2 = kTcW1 + 10 * 8 * 128;    // N 64, K 64
constexpr int kTcW3 = kTcW2 + 8 * 8 * 128;     // N 64, K 64
constexpr int kTcW4 = kTcW3 + 8 * 8 * 128;     // N 48 (40 outputs + 8 zero rows), K 64
constexpr int kTcWBytes = kTcW4 + 8 * 6 * 128; // 32,768 B
constexpr int kTcLboW = 8 * 128;               // chunk stride of W1-W3 (8 row groups)
constexpr int kTcLboW4 = 6 * 128;              // chunk stride of W4 (6 row groups)
// A operand: 128 rows x K (80 for layer 1, 64 after), chunk stride 16 row groups x 128 B
constexpr int kTcRows = 128;
constexpr int kTcLboA = (kTcRows / 8) * 128;   // 2048 B
constexpr int kTcABytes = 10 * kTcLboA;        // 20,480 B
constexpr int kTcPackWords = kTcWBytes / 4;    // 8,192 words in the packed global image

// Byte offset of element (row, k) in a K-major no-swizzle image with chunk stride `lbo`.
__host__ __device__ __forceinline__ int tc_offset(int row, int k, int lbo) {
    return (k >> 3) * lbo + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// ---- descriptors -------------------------------------------------------------------------
// Shared-memory matrix descriptor (tcgen05 form): start >> 4 in bits [0, 14), LBO >> 4 in
// [16, 30), SBO >> 4 in [32, 46), version 1 in [46, 48), layout 0 (no swizzle) in [61, 64).
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor for kind::f16: FP32 accumulate (bits 4-5 = 1), BF16 A and B
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 in bits [17, 23), M >> 4 in [24, 29).
__host__ __device__ constexpr uint32_t tc_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Non-blocking test of the mbarrier's phase `parity`.
__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for the mbarrier's phase `parity` to complete; gives up after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 accumulator columns of this thread's row (TMEM lane).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMEM allocation by one warp (the address is written to shared memory) and release.
__device__ __forceinline__ void tc_alloc(uint32_t slot_saddr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Issue one layer: D[128 x n] = A[128 x k] . B[n x k]^T (k / 16 MMAs), then commit.
__device__ __forceinline__ void tc_layer(uint32_t tmem, uint32_t a_saddr, uint32_t b_saddr, int k, int n, int b_lbo,
                                         uint32_t mbar) {
    const uint32_t idesc = tc_idesc(kTcRows, n);
    for (int s = 0; s < k / 16; s++) {
        const uint64_t ad = tc_smem_desc(a_saddr + s * 2 * kTcLboA, kTcLboA, 128);
        const uint64_t bd = tc_smem_desc(b_saddr + s * 2 * b_lbo, b_lbo, 128);
        tc_mma(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
    }
    tc_commit(mbar);
}

// This thread's row of a 64-column accumulator -> bias + ReLU -> BF16 row `row` of the A tile.
__device__ __forceinline__ void tc_epilogue_hidden(uint32_t tmem_row, const float* bias, uint8_t* a_tile, int row) {
#pragma unroll
    for (int c = 0; c < 64; c += 16) {
        float v[16];
        tc_ld16(tmem_row + c, v);
        tc_wait_ld();
        uint32_t w[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
            w[j] = pack_bf16(fmaxf(v[2 * j] + bias[c + 2 * j], 0.f), fmaxf(v[2 * j + 1] + bias[c + 2 * j + 1], 0.f));
        *reinterpret_cast<uint4*>(a_tile + tc_offset(row, c, kTcLboA)) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(a_tile + tc_offset(row, c + 8, kTcLboA)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// Write one sample's 80 inputs (inputs 78 and 79 read as zero) as BF16 row `row` of the A tile.
__device__ __forceinline__ void tc_store_input(uint8_t* a_tile, int row, const float x[kGuideIn]) {
#pragma unroll
    for (int c = 0; c < kGuideIn / 8; c++) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = 8 * c + 2 * j;
            w[j] = pack_bf16(x[k], k + 1 < kGuideIn - 2 ? x[k + 1] : 0.f);
        }
        if (c == kGuideIn / 8 - 1) w[3] = 0u;  // inputs 78, 79
        *reinterpret_cast<uint4*>(a_tile + tc_offset(row, 8 * c, kTcLboA)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Shared memory of a tensor-core inference CTA.
constexpr int kTcSub = 2;                     // sub-tiles per CTA
constexpr int kTcThreads = kTcRows * kTcSub;  // 256 threads, 256 samples per tile
struct TcSmem {
    uint8_t w[kTcWBytes];        // transposed weight images (B operands)
    uint8_t a[kTcSub][kTcABytes];  // activation tiles (A operands), one per sub-tile
    float bias[64 * 3 + 48];     // b1, b2, b3, b4 (b4 zero-padded to 48)
    unsigned long long mbar;
    uint32_t tmem_slot;
    int failed;
};
__device__ __forceinline__ int tc_sub() { return (int)threadIdx.x / kTcRows; }  // this thread's sub-tile
__device__ __forceinline__ int tc_row() { return (int)threadIdx.x % kTcRows; }  // its row (TMEM lane)

// The whole network for the CTA's current tile (inputs already in s.a, fenced and
// synchronised). Leaves each thread's 40 raw outputs in `raw`. Returns false when a wait
// gave up (outputs invalid). All threads of the CTA call it; sub-tile b accumulates in TMEM
// columns [64 b, 64 b + 64). test_polls > 0 (a test hook) limits the first wait of each
// layer to that many non-blocking polls, so it gives up while the layer's MMA is still
// running; the bounded drain that follows still waits for that MMA to finish.
__device__ __forceinline__ bool tc_network(TcSmem& s, uint32_t tmem, uint32_t& phase, float raw[kGuideOut],
                                           int test_polls = 0) {
    const int t = threadIdx.x, warp = t >> 5, sub = tc_sub(), row = tc_row();
    const uint32_t mbar = smem_u32(&s.mbar);
    const uint32_t w_saddr = smem_u32(s.w);
    const uint32_t tmem_row = tmem + 64u * sub + ((uint32_t)((warp & 3) * 32) << 16);
    const int kLimit = 1 << 22;
    for (int layer = 0; layer < 4; layer++) {
        if (t == 0) {
            tc_fence_after();
            const int k = layer == 0 ? kGuideIn : kGuideHidden;
            const int n = layer == 3 ? 48 : 64;
            const int woff = layer == 0 ? kTcW1 : layer == 1 ? kTcW2 : layer == 2 ? kTcW3 : kTcW4;
            const int lbo = layer == 3 ? kTcLboW4 : kTcLboW;
            const uint32_t idesc = tc_idesc(kTcRows, n);
            for (int b = 0; b < kTcSub; b++) {  // both sub-tiles, then one commit
                const uint32_t a_saddr = smem_u32(s.a[b]);
                for (int st = 0; st < k / 16; st++)
                    tc_mma(tmem + 64u * b, tc_smem_desc(a_saddr + st * 2 * kTcLboA, kTcLboA, 128),
                           tc_smem_desc(w_saddr + woff + st * 2 * lbo, lbo, 128), idesc, st > 0 ? 1u : 0u);
            }
            tc_commit(mbar);
        }
        bool done = false;
        if (test_polls > 0) {
            for (int i = 0; i < test_polls && !done; i++) done = mbar_test(mbar, phase);
        } else {
            done = mbar_wait(mbar, phase, kLimit);
        }
        if (!__syncthreads_and(done ? 1 : 0)) {
            // give up: wait once more (bounded) for the layer in flight before the caller
            // releases tensor memory; the phase bookkeeping is lost, so the caller stops
            mbar_wait(mbar, phase, kLimit);
            return false;
        }
        phase ^= 1u;
        tc_fence_after();
        if (layer < 3) {
            tc_epilogue_hidden(tmem_row, s.bias + 64 * layer, s.a[sub], row);
            tc_fence_before();
            fence_async_smem();
            __syncthreads();
        } else {
#pragma unroll
            for (int c = 0; c < 48; c += 16) {
                float v[16];
                tc_ld16(tmem_row + c, v);
                tc_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (c + j < kGuideOut) raw[c + j] = v[j] + s.bias[192 + c + j];
            }
        }
    }
    return true;
}

// CTA setup: weight images and biases into shared memory, mbarrier, 64 TMEM columns per
// sub-tile.
__device__ __forceinline__ uint32_t tc_setup(TcSmem& s, const uint32_t* __restrict__ wpack_fwd,
                                             const uint32_t* __restrict__ wpack_tc) {
    copy_words16(wpack_tc, reinterpret_cast<uint32_t*>(s.w), kTcPackWords);
    for (int i = threadIdx.x; i < 64 * 3 + 48; i += blockDim.x)
        s.bias[i] = i < 192 + kGuideOut ? __uint_as_float(wpack_fwd[kSB + i]) : 0.f;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&s.mbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) tc_alloc(smem_u32(&s.tmem_slot), 64 * kTcSub);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return s.tmem_slot;
}

__device__ __forceinline__ void tc_teardown(uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32) tc_dealloc(tmem, 64 * kTcSub);
}

}  // namespace pt
