// Path-guiding network kernels: weight packing, tensor-core inference on explicit inputs,
// the fused tensor-core training kernel (forward + loss + backward + weight gradients) and
// the Adam update.
//
// Loss (neural importance sampling, Mueller et al. 2019): for samples wi_i drawn with
// density p_i, F_i the integrand value and w_i = F_i / p_i, minimise
//     L = - sum_i min(w_i / sum_j w_j, 500 / n) log q(wi_i | x_i),
// a Monte Carlo estimate of the KL divergence from the normalised integrand to q (up to a
// constant). Every matrix product of training runs on BF16 mma.sync tiles with FP32
// accumulation, with the same BF16 weights and FP32 biases as the inference kernel, so the
// trained and the evaluated network are the same function.
#include "guide.h"

#include <cuda_bf16.h>

#include <algorithm>

#include "guide_mlp.cuh"
#include "guide_tc.cuh"
#include "guide_train_tc.cuh"

namespace pt {

static_assert(kPackWords + kTcPackWords == kGuidePackWords, "packed weight layout");

namespace {

// FP32 master parameters -> the two shared-memory images (forward, transposed).
__global__ void k_guide_pack(const float* __restrict__ w, uint32_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGuidePackWords) return;
    w += (size_t)blockIdx.y * kGuideParams;  // network blockIdx.y
    out += (size_t)blockIdx.y * kGuidePackWords;
    // forward: pair of rows (2 kp, 2 kp + 1) at column n
    auto pair = [&](int base, int ncol, int kp, int n) {
        return pack_bf16(w[base + (2 * kp) * ncol + n], w[base + (2 * kp + 1) * ncol + n]);
    };
    // backward: pair of columns (2 c, 2 c + 1) of row k, zero past the last column
    auto tpair = [&](int base, int ncol, int k, int c) {
        const float lo = 2 * c < ncol ? w[base + k * ncol + 2 * c] : 0.f;
        const float hi = 2 * c + 1 < ncol ? w[base + k * ncol + 2 * c + 1] : 0.f;
        return pack_bf16(lo, hi);
    };
    uint32_t v = 0u;
    if (i < kSW2) {
        const int r = i / 72, c = i % 72;
        if (c < 64) v = pair(kGW1, 64, r, c);
    } else if (i < kSW3) {
        const int r = (i - kSW2) / 72, c = (i - kSW2) % 72;
        if (c < 64) v = pair(kGW2, 64, r, c);
    } else if (i < kSW4) {
        const int r = (i - kSW3) / 72, c = (i - kSW3) % 72;
        if (c < 64) v = pair(kGW3, 64, r, c);
    } else if (i < kSB) {
        v = pair(kGW4, 40, (i - kSW4) / 40, (i - kSW4) % 40);
    } else if (i < kSWords) {
        const int j = i - kSB;  // b1 64, b2 64, b3 64, b4 40
        const float b = j < 64 ? w[kGB1 + j] : j < 128 ? w[kGB2 + j - 64] : j < 192 ? w[kGB3 + j - 128] : w[kGB4 + j - 192];
        v = __float_as_uint(b);
    } else if (i < kPackWords) {
        const int j = i - kPackT, layer = j / (64 * kSTStride), r = (j % (64 * kSTStride)) / kSTStride,
                  c = j % kSTStride;
        if (layer == 0 && c < 32) v = tpair(kGW2, 64, r, c);
        else if (layer == 1 && c < 32) v = tpair(kGW3, 64, r, c);
        else if (layer == 2 && c < 24) v = tpair(kGW4, 40, r, c);
    } else {
        // K-major operand images of the tensor-memory inference: element (n, k) = W[k][n]
        const int b = 4 * (i - kPackWords);
        int base, ncol, lbo, off;
        if (b < kTcW2) { base = kGW1; ncol = 64; lbo = kTcLboW; off = b - kTcW1; }
        else if (b < kTcW3) { base = kGW2; ncol = 64; lbo = kTcLboW; off = b - kTcW2; }
        else if (b < kTcW4) { base = kGW3; ncol = 64; lbo = kTcLboW; off = b - kTcW3; }
        else { base = kGW4; ncol = 40; lbo = kTcLboW4; off = b - kTcW4; }
        const int kc = off / lbo, rem = off % lbo;
        const int n = (rem / 128) * 8 + (rem % 128) / 16, k = kc * 8 + (rem % 16) / 2;
        if (n < ncol) v = pack_bf16(w[base + k * ncol + n], w[base + (k + 1) * ncol + n]);
    }
    out[i] = v;
}

// Inference on explicit input vectors (tests, tools): 4 warps per block, 16 rows per warp.
// Inputs 78 and 79 are padding and read as zero.
__global__ void k_guide_forward_x(const uint32_t* __restrict__ wpack, const float* __restrict__ x, int n,
                                  float* __restrict__ raw) {
    __shared__ __align__(16) uint32_t sw[kSWords];
    __shared__ uint32_t sx[4][16 * kSXStride];
    // outputs overwrite the inputs (all input fragments are in registers before the stores)
    float(*sy)[16 * kSXStride] = reinterpret_cast<float(*)[16 * kSXStride]>(sx);
    guide_load_weights(wpack, sw);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int groups = (n + 15) / 16;
    for (int grp = blockIdx.x * 4 + warp; grp < groups; grp += gridDim.x * 4) {
        const int row0 = grp * 16;
        for (int e = lane; e < 16 * (kGuideIn / 2); e += 32) {
            const int r = e / (kGuideIn / 2), k = e % (kGuideIn / 2);
            const int gi = row0 + r;
            const bool ok = gi < n && k < kGuideIn / 2 - 1;
            const float a = ok ? x[(size_t)gi * kGuideIn + 2 * k] : 0.f;
            const float b = ok ? x[(size_t)gi * kGuideIn + 2 * k + 1] : 0.f;
            sx[warp][r * kSXStride + k] = pack_bf16(a, b);
        }
        __syncwarp();
        guide_mlp_warp16(sw, sx[warp], sy[warp]);
        __syncwarp();
        for (int e = lane; e < 16 * kGuideOut; e += 32) {
            const int r = e / kGuideOut, j = e % kGuideOut;
            if (row0 + r < n) raw[(size_t)(row0 + r) * kGuideOut + j] = sy[warp][e];
        }
        __syncwarp();
    }
}

// Inference on explicit input vectors on the tensor cores (tcgen05, TMEM accumulators):
// kTcThreads inputs per tile, one thread each. Raw outputs like k_guide_forward_x.
__global__ void __launch_bounds__(kTcThreads) k_guide_forward_x_tc(const uint32_t* __restrict__ wpack,
                                                                const float* __restrict__ x, int n,
                                                                float* __restrict__ raw, int* error,
                                                                int test_polls) {
    extern __shared__ __align__(1024) uint8_t tsm[];
    TcSmem& s = *reinterpret_cast<TcSmem*>(tsm);
    const int tiles = (n + kTcThreads - 1) / kTcThreads;
    if ((int)blockIdx.x >= tiles) return;
    const uint32_t tmem = tc_setup(s, wpack, wpack + kPackWords);
    uint32_t phase = 0;
    const int t = threadIdx.x;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int row = tile * kTcThreads + t;
        float xi[kGuideIn];
        for (int k = 0; k < kGuideIn; k++) xi[k] = row < n ? x[(size_t)row * kGuideIn + k] : 0.f;
        tc_store_input(s.a[tc_sub()], tc_row(), xi);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        float out[kGuideOut];
        if (!tc_network(s, tmem, phase, out, test_polls)) {
            if (t == 0) atomicOr(error, 2);
            break;
        }
        if (row < n)
            for (int j = 0; j < kGuideOut; j++) raw[(size_t)row * kGuideOut + j] = out[j];
    }
    tc_teardown(tmem);
}

// Sample source of the training kernel: explicit inputs, or a ring of GuideSamples.
struct TrainSource {
    const float* x;        // explicit: n x 80
    const float* wi;       // explicit: n x 3
    const float* w;        // explicit: n
    const GuideSample* ring;
    int cap;
    const int* count;      // ring: number of samples written so far (monotone)
    int n;                 // explicit count, or the batch size for the ring
};

// The sample source of network `net` (its own ring and counter).
__device__ __forceinline__ TrainSource source_of_net(TrainSource s, int net) {
    if (s.ring) {
        s.ring += (size_t)net * s.cap;
        s.count += net;
    }
    return s;
}

__device__ __forceinline__ void source_range(const TrainSource& s, int& first, int& n) {
    if (s.ring) {
        // the counter only grows (and may wrap past 2^31): unsigned arithmetic, newest n samples
        const unsigned c = (unsigned)*s.count;
        unsigned m = c < (unsigned)s.n ? c : (unsigned)s.n;
        m = m < (unsigned)s.cap ? m : (unsigned)s.cap;
        n = (int)m;
        first = (int)(c - m);
    } else {
        first = 0;
        n = s.n;
    }
}

// Fetch sample `i` of the range: inputs, direction, weight.
__device__ __forceinline__ void source_sample(const TrainSource& s, const GuideFrame& gf, int first, int i,
                                              float* xrow, float wi[3], float& w) {
    if (s.ring) {
        const GuideSample sm = s.ring[(unsigned)(first + i) % (unsigned)s.cap];
        guide_encode(gf, sm.p, sm.n, sm.wo, xrow);
        wi[0] = sm.wi[0]; wi[1] = sm.wi[1]; wi[2] = sm.wi[2];
        w = sm.weight;
    } else {
        const float4* xr = reinterpret_cast<const float4*>(s.x + (size_t)i * kGuideIn);  // 320-byte rows
#pragma unroll
        for (int k = 0; k < kGuideIn / 4; k++) {
            const float4 v = __ldg(xr + k);
            xrow[4 * k] = v.x;
            xrow[4 * k + 1] = v.y;
            xrow[4 * k + 2] = v.z;
            xrow[4 * k + 3] = v.w;
        }
        wi[0] = s.wi[3 * i]; wi[1] = s.wi[3 * i + 1]; wi[2] = s.wi[3 * i + 2];
        w = s.w[i];
    }
    xrow[kGuideIn - 2] = 0.f;  // padding inputs
    xrow[kGuideIn - 1] = 0.f;
}

__global__ void k_guide_wsum(TrainSource s0, float* wsum) {
    const TrainSource s = source_of_net(s0, blockIdx.y);
    wsum += 4 * blockIdx.y;
    int first, n;
    source_range(s, first, n);
    float acc = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += s.ring ? s.ring[(unsigned)(first + i) % (unsigned)s.cap].weight : s.w[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(wsum, acc);
}

// Gradient of -w log q(wi) with respect to the 40 raw outputs of one sample; returns the loss.
__device__ __forceinline__ float loss_grad(const float* raw, const float wi[3], float w, float* dy) {
    if (w == 0.f) {
        for (int j = 0; j < kGuideOut; j++) dy[j] = 0.f;
        return 0.f;
    }
    float mx = -1e30f;
    for (int j = 0; j < kGuideLobes; j++) mx = fmaxf(mx, raw[5 * j + 4]);
    float se = 0.f, pi[kGuideLobes], lf[kGuideLobes], kap[kGuideLobes], len[kGuideLobes], mu[kGuideLobes][3],
          dot_[kGuideLobes];
    for (int j = 0; j < kGuideLobes; j++) {
        pi[j] = expf(raw[5 * j + 4] - mx);
        se += pi[j];
    }
    float lmax = -1e30f;
    for (int j = 0; j < kGuideLobes; j++) {
        pi[j] /= se;
        const float m0 = raw[5 * j], m1 = raw[5 * j + 1], m2 = raw[5 * j + 2];
        len[j] = sqrtf(m0 * m0 + m1 * m1 + m2 * m2) + 1e-12f;
        mu[j][0] = m0 / len[j]; mu[j][1] = m1 / len[j]; mu[j][2] = m2 / len[j];
        kap[j] = expf(fminf(kKappaLogMax, fmaxf(kKappaLogMin, raw[5 * j + 3])));
        dot_[j] = mu[j][0] * wi[0] + mu[j][1] * wi[1] + mu[j][2] * wi[2];
        lf[j] = logf(pi[j] + 1e-30f) + vmf_log_norm(kap[j]) + kap[j] * (dot_[j] - 1.f);
        lmax = fmaxf(lmax, lf[j]);
    }
    float sq = 0.f;
    for (int j = 0; j < kGuideLobes; j++) sq += expf(lf[j] - lmax);
    const float logq = lmax + logf(sq);
    for (int j = 0; j < kGuideLobes; j++) {
        const float s = expf(lf[j] - logq);  // responsibility of lobe j
        dy[5 * j + 4] = -w * (s - pi[j]);
        const float kr = raw[5 * j + 3];
        const float k = kap[j];
        const float dlogc = 1.f / k - 2.f * expf(-2.f * k) / (-expm1f(-2.f * k));
        dy[5 * j + 3] = (kr > kKappaLogMin && kr < kKappaLogMax) ? -w * s * (dlogc + dot_[j] - 1.f) * k : 0.f;
        const float c = -w * s * k / len[j];
        for (int a = 0; a < 3; a++) dy[5 * j + a] = c * (wi[a] - dot_[j] * mu[j][a]);
    }
    return -w * logq;
}

// ---- fused training kernel -------------------------------------------------------------
//
// One block of 8 warps per SM walks tiles of 128 samples (16 per warp). Per tile:
//   1. each warp stages its 16 samples (encoded inputs, direction, normalised weight);
//   2. forward through the four layers on mma.sync (the inference code path), storing the
//      BF16 activations X, A1, A2, A3 in the warp's shared-memory tiles;
//   3. the loss gradient dY of each sample (FP32), stored as BF16;
//   4. backward dZ3 = (dY W4^T) . [A3 > 0], dZ2 = (dZ3 W3^T) . [A2 > 0],
//      dZ1 = (dZ2 W2^T) . [A1 > 0] on mma.sync, chained in registers, each stored as BF16;
//   5. weight gradients G = A^T dZ over the block's 128 samples as 16x8 output tiles on
//      mma.sync (operands transposed by ldmatrix.trans): 145 tiles (W1 40, W2 32, W3 32,
//      W4 20, and bias tiles b2 8, b3 8, b4 5 computed as ones^T dZ), 19 per warp, each held
//      in FP32 registers across every tile the block processes. The bias of layer 1 rides on
//      W1's padding input 78, set to one in the stored X tile after the forward pass.
// At the end each block adds its register accumulators to the global gradient.

// No sample's normalised weight exceeds kWeightCap times the batch average: the rare paths
// that carry a sun or the slit's sky (weights 10^3-10^5 times the mean) otherwise dominate
// each step's gradient. (Measured on the slit room: time-to-relMSE 1.71x instead of 1.58x
// at a 256-spp budget; caps of 20 and 2000 were worse.)
constexpr float kWeightCap = 500.f;
constexpr int kTrainWarps = 8;
constexpr int kTrainThreads = 32 * kTrainWarps;
constexpr int kBlockRows = 16 * kTrainWarps;  // samples per block tile
// per-warp tile row strides in 32-bit words (rows are multiples of 16 bytes for ldmatrix and
// spread 8 consecutive rows over distinct 16-byte bank groups)
constexpr int kXW = kSXStride;  // 44: 80 BF16 inputs
constexpr int kAW = 36;         // 64 BF16 activations
constexpr int kYW = 28;         // 48 BF16 (40 output gradients, zero-padded)
constexpr int kRawW = 41;       // FP32 raw outputs
constexpr int kWX = 0;
constexpr int kWA1 = kWX + 16 * kXW;
constexpr int kWA2 = kWA1 + 16 * kAW;
constexpr int kWA3 = kWA2 + 16 * kAW;
constexpr int kWD1 = kWA3 + 16 * kAW;
constexpr int kWD2 = kWD1 + 16 * kAW;
constexpr int kWD3 = kWD2 + 16 * kAW;
constexpr int kWDY = kWD3 + 16 * kAW;
constexpr int kWWi = kWDY + 16 * kYW;  // 16 x (wi.xyz, normalised weight)
constexpr int kWarpWords = kWWi + 16 * 4;
constexpr int kWRaw = kWD2;  // raw outputs alias dZ2/dZ3, consumed before either is written
static_assert(16 * kRawW <= 2 * 16 * kAW, "raw outputs must fit the dZ2/dZ3 tiles");
static_assert((kSWords + kSTWords) % 4 == 0 && kWarpWords % 4 == 0, "16-byte aligned warp tiles");
constexpr int kTrainSmemWords = kSWords + kSTWords + kTrainWarps * kWarpWords;
constexpr int kGradTiles = 145;
constexpr int kOwnTiles = (kGradTiles + kTrainWarps - 1) / kTrainWarps;  // 19

// Operands and destination of weight-gradient tile `id`.
struct GradTile {
    int a_off, a_stride, a_col;  // A^T source tile (a_off < 0: ones, a bias tile)
    int b_off, b_stride, b_col;  // dZ source tile
    int out, out_stride;         // parameter index of element (0, 0), row stride
};

__device__ __forceinline__ GradTile grad_tile(int id) {
    GradTile t;
    if (id < 40) {  // W1 = X^T dZ1 (row 78 is b1, row 79 unused)
        t = {kWX, kXW, (id / 8) * 16, kWD1, kAW, (id % 8) * 8, kGW1 + (id / 8) * 16 * 64 + (id % 8) * 8, 64};
    } else if (id < 72) {  // W2 = A1^T dZ2
        const int j = id - 40;
        t = {kWA1, kAW, (j / 8) * 16, kWD2, kAW, (j % 8) * 8, kGW2 + (j / 8) * 16 * 64 + (j % 8) * 8, 64};
    } else if (id < 104) {  // W3 = A2^T dZ3
        const int j = id - 72;
        t = {kWA2, kAW, (j / 8) * 16, kWD3, kAW, (j % 8) * 8, kGW3 + (j / 8) * 16 * 64 + (j % 8) * 8, 64};
    } else if (id < 124) {  // W4 = A3^T dY
        const int j = id - 104;
        t = {kWA3, kAW, (j / 5) * 16, kWDY, kYW, (j % 5) * 8, kGW4 + (j / 5) * 16 * 40 + (j % 5) * 8, 40};
    } else if (id < 132) {  // b2 = 1^T dZ2
        const int j = id - 124;
        t = {-1, 0, 0, kWD2, kAW, j * 8, kGB2 + j * 8, 0};
    } else if (id < 140) {  // b3 = 1^T dZ3
        const int j = id - 132;
        t = {-1, 0, 0, kWD3, kAW, j * 8, kGB3 + j * 8, 0};
    } else {  // b4 = 1^T dY
        const int j = id - 140;
        t = {-1, 0, 0, kWDY, kYW, j * 8, kGB4 + j * 8, 0};
    }
    return t;
}

// Backward through one layer: dA = dZ W^T (KT k-steps of 16 over the layer's outputs, 64
// inputs), masked by the layer input's ReLU ([A > 0], read from the stored BF16 tile) and
// re-packed as BF16 A fragments.
template <int KT>
__device__ __forceinline__ void guide_backward(const uint32_t* swt_layer, const uint32_t (&dz)[KT][4],
                                               const uint32_t* a_tile, uint32_t (&out)[4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float c[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.f;
#pragma unroll
    for (int kt = 0; kt < KT; kt++) {
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint32_t b0 = swt_layer[(nt * 8 + g) * kSTStride + kt * 8 + t];
            const uint32_t b1 = swt_layer[(nt * 8 + g) * kSTStride + kt * 8 + 4 + t];
            mma16816(c[nt], dz[kt][0], dz[kt][1], dz[kt][2], dz[kt][3], b0, b1);
        }
    }
    auto masked = [&](float lo, float hi, uint32_t a) {
        return pack_bf16((a & 0x7FFFu) ? lo : 0.f, (a & 0x7FFF0000u) ? hi : 0.f);
    };
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
        out[kt][0] = masked(c[2 * kt][0], c[2 * kt][1], a_tile[g * kAW + kt * 8 + t]);
        out[kt][1] = masked(c[2 * kt][2], c[2 * kt][3], a_tile[(g + 8) * kAW + kt * 8 + t]);
        out[kt][2] = masked(c[2 * kt + 1][0], c[2 * kt + 1][1], a_tile[g * kAW + kt * 8 + 4 + t]);
        out[kt][3] = masked(c[2 * kt + 1][2], c[2 * kt + 1][3], a_tile[(g + 8) * kAW + kt * 8 + 4 + t]);
    }
}

__global__ void __launch_bounds__(kTrainThreads, 1) k_guide_train(GuideDevice g, TrainSource src0) {
    extern __shared__ __align__(16) uint32_t smem[];
    // network blockIdx.y: its weights, gradient, sums and samples
    const int net = blockIdx.y;
    g.wpack += (size_t)net * kGuidePackWords;
    g.grad += (size_t)net * kGuideParams;
    g.wsum += 4 * net;
    const TrainSource src = source_of_net(src0, net);
    uint32_t* sw = smem;               // forward weights and biases (inference layout)
    uint32_t* swt = sw + kSWords;      // transposed weights
    uint32_t* tiles = swt + kSTWords;  // per-warp tiles
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g8 = lane >> 2, t4 = lane & 3;
    uint32_t* my = tiles + warp * kWarpWords;
    float* myf = reinterpret_cast<float*>(my);
    guide_load_weights(g.wpack, sw);
    guide_load_weights_t(g.wpack, swt);
    int first, n;
    source_range(src, first, n);
    const float wsum = g.wsum[0];
    const float inv_wsum = wsum > 0.f ? 1.f / wsum : 0.f;
    float acc[kOwnTiles][4];
#pragma unroll
    for (int j = 0; j < kOwnTiles; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    float loss = 0.f;
    __syncthreads();
    for (int tile = blockIdx.x; tile * kBlockRows < n; tile += gridDim.x) {
        // 1. stage this warp's 16 samples
        if (lane < 16) {
            const int i = tile * kBlockRows + warp * 16 + lane;
            float x[kGuideIn], wi[3] = {0.f, 0.f, 1.f}, w = 0.f;
            if (i < n) {
                source_sample(src, g.frames ? g.frames[net] : g.frame, first, i, x, wi, w);
            } else {
#pragma unroll
                for (int k = 0; k < kGuideIn; k++) x[k] = 0.f;
            }
            guide_store_input(my + kWX, lane, x);
            float* f = myf + kWWi + 4 * lane;
            f[0] = wi[0]; f[1] = wi[1]; f[2] = wi[2];
            f[3] = fminf(w * inv_wsum, kWeightCap / (float)n);
        }
        __syncwarp();
        // 2. forward
        {
            uint32_t a1[5][4];
#pragma unroll
            for (int kt = 0; kt < 5; kt++) {
                a1[kt][0] = my[kWX + g8 * kXW + kt * 8 + t4];
                a1[kt][1] = my[kWX + (g8 + 8) * kXW + kt * 8 + t4];
                a1[kt][2] = my[kWX + g8 * kXW + kt * 8 + 4 + t4];
                a1[kt][3] = my[kWX + (g8 + 8) * kXW + kt * 8 + 4 + t4];
            }
            __syncwarp();
            if (lane < 16) my[kWX + lane * kXW + kGuideIn / 2 - 1] = pack_bf16(1.f, 0.f);  // b1 rides on input 78
            uint32_t h[4][4], h2[4][4];
            guide_hidden<5>(sw, kSW1, kSB, a1, h);
            guide_store_frag(my + kWA1, kAW, h);
            guide_hidden<4>(sw, kSW2, kSB + 64, h, h2);
            guide_store_frag(my + kWA2, kAW, h2);
            guide_hidden<4>(sw, kSW3, kSB + 128, h2, h);
            guide_store_frag(my + kWA3, kAW, h);
            float y[5][4];
#pragma unroll
            for (int nt = 0; nt < 5; nt++) {
                const float b0 = __uint_as_float(sw[kSB + 192 + nt * 8 + 2 * t4]);
                const float b1 = __uint_as_float(sw[kSB + 192 + nt * 8 + 2 * t4 + 1]);
                y[nt][0] = b0; y[nt][1] = b1; y[nt][2] = b0; y[nt][3] = b1;
            }
#pragma unroll
            for (int kt = 0; kt < 4; kt++) {
#pragma unroll
                for (int nt = 0; nt < 5; nt++) {
                    const uint32_t b0 = sw[kSW4 + (kt * 8 + t4) * 40 + nt * 8 + g8];
                    const uint32_t b1 = sw[kSW4 + (kt * 8 + 4 + t4) * 40 + nt * 8 + g8];
                    mma16816(y[nt], h[kt][0], h[kt][1], h[kt][2], h[kt][3], b0, b1);
                }
            }
#pragma unroll
            for (int nt = 0; nt < 5; nt++) {
                myf[kWRaw + g8 * kRawW + nt * 8 + 2 * t4] = y[nt][0];
                myf[kWRaw + g8 * kRawW + nt * 8 + 2 * t4 + 1] = y[nt][1];
                myf[kWRaw + (g8 + 8) * kRawW + nt * 8 + 2 * t4] = y[nt][2];
                myf[kWRaw + (g8 + 8) * kRawW + nt * 8 + 2 * t4 + 1] = y[nt][3];
            }
        }
        __syncwarp();
        // 3. loss gradient per sample
        if (lane < 16) {
            float raw[kGuideOut], dy[kGuideOut];
#pragma unroll
            for (int j = 0; j < kGuideOut; j++) raw[j] = myf[kWRaw + lane * kRawW + j];
            const float* f = myf + kWWi + 4 * lane;
            const float wi[3] = {f[0], f[1], f[2]};
            loss += loss_grad(raw, wi, f[3], dy);
#pragma unroll
            for (int j = 0; j < kGuideOut / 2; j++) my[kWDY + lane * kYW + j] = pack_bf16(dy[2 * j], dy[2 * j + 1]);
#pragma unroll
            for (int j = kGuideOut / 2; j < 24; j++) my[kWDY + lane * kYW + j] = 0u;
        }
        __syncwarp();
        // 4. backward, chained in registers
        {
            uint32_t ay[3][4];
#pragma unroll
            for (int kt = 0; kt < 3; kt++) {
                ay[kt][0] = my[kWDY + g8 * kYW + kt * 8 + t4];
                ay[kt][1] = my[kWDY + (g8 + 8) * kYW + kt * 8 + t4];
                ay[kt][2] = my[kWDY + g8 * kYW + kt * 8 + 4 + t4];
                ay[kt][3] = my[kWDY + (g8 + 8) * kYW + kt * 8 + 4 + t4];
            }
            uint32_t d[4][4], d2[4][4];
            guide_backward<3>(swt + kST4, ay, my + kWA3, d);
            guide_store_frag(my + kWD3, kAW, d);
            guide_backward<4>(swt + kST3, d, my + kWA2, d2);
            guide_store_frag(my + kWD2, kAW, d2);
            guide_backward<4>(swt + kST2, d2, my + kWA1, d);
            guide_store_frag(my + kWD1, kAW, d);
        }
        __syncthreads();
        // 5. weight gradients over the block's 128 samples
        {
            // ldmatrix row addresses: A^T from four 8x8 tiles (samples 0-7 / 8-15 x columns
            // a_col + 0-7 / 8-15), dZ from two (samples 0-7 / 8-15)
            const int mi = lane >> 3, mr = lane & 7;
            const int a_row = mr + ((mi >> 1) << 3), a_half = (mi & 1) << 2;
            const int b_row = lane & 15;
#pragma unroll
            for (int j = 0; j < kOwnTiles; j++) {
                const int id = warp * kOwnTiles + j;
                if (id < kGradTiles) {
                    const GradTile gt = grad_tile(id);
                    const int a_addr = gt.a_off + a_row * gt.a_stride + (gt.a_col >> 1) + a_half;
                    const int b_addr = gt.b_off + b_row * gt.b_stride + (gt.b_col >> 1);
#pragma unroll 2
                    for (int s = 0; s < kTrainWarps; s++) {
                        const uint32_t* base = tiles + s * kWarpWords;
                        uint32_t a[4] = {0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u};  // BF16 ones
                        if (gt.a_off >= 0) ldsm_x4_t(a, base + a_addr);
                        uint32_t b0, b1;
                        ldsm_x2_t(b0, b1, base + b_addr);
                        mma16816(acc[j], a[0], a[1], a[2], a[3], b0, b1);
                    }
                }
            }
        }
        __syncthreads();
    }
    // 6. add this block's partial gradients
#pragma unroll
    for (int j = 0; j < kOwnTiles; j++) {
        const int id = warp * kOwnTiles + j;
        if (id < kGradTiles) {
            const GradTile gt = grad_tile(id);
            if (gt.a_off < 0) {  // bias tile: every row holds the column sums
                if (g8 == 0) {
                    if (acc[j][0] != 0.f) atomicAdd(&g.grad[gt.out + 2 * t4], acc[j][0]);
                    if (acc[j][1] != 0.f) atomicAdd(&g.grad[gt.out + 2 * t4 + 1], acc[j][1]);
                }
            } else {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = gt.a_col + g8 + 8 * h;
                    int o = gt.out + (g8 + 8 * h) * gt.out_stride + 2 * t4;
                    bool skip = false;
                    if (id < 40 && row >= kGuideIn - 2) {
                        skip = row == kGuideIn - 1;          // padding input
                        o = kGB1 + gt.b_col + 2 * t4;        // the ones column: b1
                    }
                    if (!skip && acc[j][2 * h] != 0.f) atomicAdd(&g.grad[o], acc[j][2 * h]);
                    if (!skip && acc[j][2 * h + 1] != 0.f) atomicAdd(&g.grad[o + 1], acc[j][2 * h + 1]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0 && loss != 0.f) atomicAdd(g.wsum + 1, loss);  // batch loss, for monitoring
}

// The training step of k_guide_train on tcgen05 (guide_train_tc.cuh): the same loss,
// weight cap and gradient layout, every product on the tensor cores with the accumulators in
// tensor memory.
__global__ void __launch_bounds__(kTtThreads, 1) k_guide_train_tc(GuideDevice g, TrainSource src0) {
    extern __shared__ __align__(1024) uint8_t ttsm[];
    TtSmem& s = *reinterpret_cast<TtSmem*>(ttsm);
    const int net = blockIdx.y;
    g.wpack += (size_t)net * kGuidePackWords;
    g.grad += (size_t)net * kGuideParams;
    g.wsum += 4 * net;
    const TrainSource src = source_of_net(src0, net);
    const int t = threadIdx.x, warp = t >> 5, sub = t / kTcRows, row = t % kTcRows;
    TtSubTile& my = s.sub[sub];
    int first, n;
    source_range(src, first, n);
    if ((int)blockIdx.x * kTtRows >= n) return;  // no tile for this CTA: no setup, no TMEM
    // ---- setup: weight images, biases, the ones columns, mbarrier, tensor memory
    copy_words16(g.wpack + kPackWords, reinterpret_cast<uint32_t*>(s.w), kTcPackWords);
    for (int i = t; i < 64 * 3 + 48; i += blockDim.x)
        s.bias[i] = i < 192 + kGuideOut ? __uint_as_float(g.wpack[kSB + i]) : 0.f;
    {
        const uint4 ones = make_uint4(pack_bf16(1.f, 0.f), 0u, 0u, 0u), zero = make_uint4(0u, 0u, 0u, 0u);
        uint8_t* tiles[3] = {my.a1, my.a2, my.a3};
        for (int k = 0; k < 3; k++) {  // features 64 (one) and 65-79 (zero) of the row
            *reinterpret_cast<uint4*>(tiles[k] + tc_offset(row, 64, kTcLboA)) = ones;
            *reinterpret_cast<uint4*>(tiles[k] + tc_offset(row, 72, kTcLboA)) = zero;
        }
    }
    if (t == 0) {
        mbar_init(smem_u32(&s.mbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc_alloc(smem_u32(&s.tmem_slot), kTtTmemCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem_slot;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;  // this warp's TMEM lanes
    const uint32_t scratch = tmem + kTtColScratch + 64u * sub;
    const uint32_t mbar = smem_u32(&s.mbar);
    const uint32_t w_s = smem_u32(s.w);
    uint32_t sx[kTtSub], sa1[kTtSub], sa2[kTtSub], sa3[kTtSub], sdy[kTtSub];
#pragma unroll
    for (int k = 0; k < kTtSub; k++) {
        sx[k] = smem_u32(s.sub[k].x);
        sa1[k] = smem_u32(s.sub[k].a1);
        sa2[k] = smem_u32(s.sub[k].a2);
        sa3[k] = smem_u32(s.sub[k].a3);
        sdy[k] = smem_u32(s.sub[k].dy);
    }
    const float wsum = g.wsum[0];
    const float inv_wsum = wsum > 0.f ? 1.f / wsum : 0.f;
    uint32_t phase = 0;
    bool ok = true, first_tile = true;
    float loss = 0.f;
    for (int tile = blockIdx.x; tile * kTtRows < n && ok; tile += gridDim.x) {
        // 1. stage this thread's sample
        float wi[3] = {0.f, 0.f, 1.f}, w = 0.f;
        {
            const int i = tile * kTtRows + t;
            float x[kGuideIn];
            if (i < n) {
                source_sample(src, g.frames ? g.frames[net] : g.frame, first, i, x, wi, w);
            } else {
#pragma unroll
                for (int k = 0; k < kGuideIn; k++) x[k] = 0.f;
            }
            w = fminf(w * inv_wsum, kWeightCap / (float)n);
            tc_store_input(my.x, row, x);  // inputs 78, 79 read as zero in the forward pass
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // 2. forward
        float raw[kGuideOut];
        for (int layer = 0; layer < 4 && ok; layer++) {
            if (t == 0) {
                tc_fence_after();
                const int k = layer == 0 ? kGuideIn : kGuideHidden;
                const int nn = layer == 3 ? 48 : 64;
                const int woff = layer == 0 ? kTcW1 : layer == 1 ? kTcW2 : layer == 2 ? kTcW3 : kTcW4;
                const int lbo = layer == 3 ? kTcLboW4 : kTcLboW;
                const uint32_t idesc = tc_idesc(kTcRows, nn);
                for (int b = 0; b < kTtSub; b++) {
                    const uint32_t a = layer == 0 ? sx[b] : layer == 1 ? sa1[b] : layer == 2 ? sa2[b] : sa3[b];
                    for (int st = 0; st < k / 16; st++)
                        tc_mma(tmem + kTtColScratch + 64u * b, tc_smem_desc(a + st * 2 * kTcLboA, kTcLboA, 128),
                               tc_smem_desc(w_s + woff + st * 2 * lbo, lbo, 128), idesc, st > 0 ? 1u : 0u);
                }
                tc_commit(mbar);
            }
            if (!(ok = tt_wait(mbar, phase))) break;
            if (layer < 3) {
                uint8_t* dst = layer == 0 ? my.a1 : layer == 1 ? my.a2 : my.a3;
                tc_epilogue_hidden(scratch + lane_base, s.bias + 64 * layer, dst, row);
                tc_fence_before();
                fence_async_smem();
                __syncthreads();
            } else {
#pragma unroll
                for (int c = 0; c < 48; c += 16) {
                    float v[16];
                    tc_ld16(scratch + lane_base + c, v);
                    tc_wait_ld();
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        if (c + j < kGuideOut) raw[c + j] = v[j] + s.bias[192 + c + j];
                }
            }
        }
        if (!ok) break;
        // 3. loss gradient of the raw outputs, BF16 into dY (columns 40-47 zero)
        {
            float dy[kGuideOut];
            loss += loss_grad(raw, wi, w, dy);
#pragma unroll
            for (int c = 0; c < 48; c += 8) {
                uint32_t q[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int k = c + 2 * j;
                    q[j] = pack_bf16(k < kGuideOut ? dy[k] : 0.f, k + 1 < kGuideOut ? dy[k + 1] : 0.f);
                }
                *reinterpret_cast<uint4*>(my.dy + tc_offset(row, c, kTcLboA)) = make_uint4(q[0], q[1], q[2], q[3]);
            }
        }
        tc_fence_before();
        fence_async_smem();
        __syncthreads();
        // 4. backward: layer 4 (W4' += A3^T dY, dZ3 = dY W4), 3, 2, then W1' += X^T dZ1
        for (int layer = 3; layer >= 1 && ok; layer--) {
            if (t == 0) {
                tc_fence_after();
                const uint32_t gcol = layer == 3 ? kTtColW4 : layer == 2 ? kTtColW3 : kTtColW2;
                const int nn = layer == 3 ? 48 : 64;
                const int woff = layer == 3 ? kTcW4 : layer == 2 ? kTcW3 : kTcW2;
                const uint32_t wchunk = layer == 3 ? kTcLboW4 : kTcLboW;
                for (int b = 0; b < kTtSub; b++) {
                    const uint32_t act = layer == 3 ? sa3[b] : layer == 2 ? sa2[b] : sa1[b];  // A_{l-1}
                    const uint32_t dz = layer == 3 ? sdy[b] : layer == 2 ? sa3[b] : sa2[b];   // dZ_l
                    tt_wgrad(tmem + gcol, act, dz, nn, first_tile && b == 0);
                    tt_bdata(tmem + kTtColScratch + 64u * b, dz, w_s + woff, nn, wchunk);
                }
                tc_commit(mbar);
            }
            if (!(ok = tt_wait(mbar, phase))) break;
            // dZ_{l-1} = D [A_{l-1} > 0], over A_{l-1}
            tt_epilogue_mask(scratch + lane_base, layer == 3 ? my.a3 : layer == 2 ? my.a2 : my.a1, row);
            tc_fence_before();
            fence_async_smem();
            __syncthreads();
        }
        if (!ok) break;
        // b1 rides on input 78 of X for the W1 product
        *reinterpret_cast<uint32_t*>(my.x + tc_offset(row, kGuideIn - 2, kTcLboA)) = pack_bf16(1.f, 0.f);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            for (int b = 0; b < kTtSub; b++) tt_wgrad(tmem + kTtColW1, sx[b], sa1[b], 64, first_tile && b == 0);
            tc_commit(mbar);
        }
        if (!(ok = tt_wait(mbar, phase))) break;
        first_tile = false;
    }
    if (!ok) {
        if (t == 0) atomicAdd(g.wsum + 2, 1.f);  // a wait gave up: no partial gradient
    } else if (!first_tile && t < 2 * kTcRows) {
        // 5. the accumulators to the global gradient: warps 0-3 add W1 and W2, warps 4-7 W3
        //    and W4; the thread's TMEM lane is input row i
        const int i = row;
        for (int m = 0; m < 2; m++) {
            const int layer = sub == 0 ? m : 2 + m;  // 0..3 = W1..W4
            const uint32_t col = layer == 0 ? kTtColW1 : layer == 1 ? kTtColW2 : layer == 2 ? kTtColW3 : kTtColW4;
            const int nout = layer == 3 ? kGuideOut : 64;
            const int wbase = layer == 0 ? kGW1 : layer == 1 ? kGW2 : layer == 2 ? kGW3 : kGW4;
            const int bbase = layer == 0 ? kGB1 : layer == 1 ? kGB2 : layer == 2 ? kGB3 : kGB4;
            const int ones = layer == 0 ? kGuideIn - 2 : 64;  // the row of the ones input
            const int nin = layer == 0 ? kGuideIn - 2 : 64;   // real input rows
            // rows of padding inputs and past the layer's inputs add nothing (every lane of the
            // warp still takes part in the warp-wide tcgen05.ld)
            const bool use = i < nin || i == ones;
            float* dst = i < nin ? g.grad + wbase + i * nout : g.grad + bbase;  // 16-byte aligned rows
            for (int c = 0; c < 64; c += 16) {
                if (layer == 3 && c >= 48) break;
                float v[16];
                tc_ld16(tmem + lane_base + col + c, v);
                tc_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; j += 4)  // one 16-byte reduction per four outputs
                    if (use && c + j < nout)
                        atomicAdd(reinterpret_cast<float4*>(dst + c + j), make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((t & 31) == 0 && loss != 0.f) atomicAdd(g.wsum + 1, loss);  // batch loss, for monitoring
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, kTtTmemCols);
}

__global__ void k_guide_adam(GuideDevice g, float lr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGuideParams) return;
    const size_t off = (size_t)blockIdx.y * kGuideParams;  // network blockIdx.y
    g.w += off;
    g.grad += off;
    g.adam_m += off;
    g.adam_v += off;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float t = (float)(*(g.step + 4 * blockIdx.y) + 1);
    const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
    float gr = g.grad[i];
    if (!isfinite(gr)) gr = 0.f;
    gr = fminf(10.f, fmaxf(-10.f, gr));
    const float m = b1 * g.adam_m[i] + (1.f - b1) * gr;
    const float v = b2 * g.adam_v[i] + (1.f - b2) * gr * gr;
    g.adam_m[i] = m;
    g.adam_v[i] = v;
    g.w[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    g.grad[i] = 0.f;
}

__global__ void k_guide_step(int* step, int nets) {
    if (threadIdx.x < nets) step[4 * threadIdx.x] += 1;  // one counter per network, 4 words apart
}

constexpr size_t kTrainSmemBytes = (size_t)kTrainSmemWords * sizeof(uint32_t);

__global__ void k_guide_clear_sums(float* wsum, int nets) {
    if (threadIdx.x < nets) {  // weight sum, batch loss, failed waits of each network
        wsum[4 * threadIdx.x] = 0.f;
        wsum[4 * threadIdx.x + 1] = 0.f;
        wsum[4 * threadIdx.x + 2] = 0.f;
    }
}

cudaError_t launch_train(const GuideDevice& g, const TrainSource& src, cudaStream_t s) {
    const int nets = g.nets > 0 ? g.nets : 1;
    k_guide_clear_sums<<<1, 64, 0, s>>>(g.wsum, nets);
    // about one block per SM in total, at least 4 per network
    const int per = std::max(4, g.num_sms / nets);
    k_guide_wsum<<<dim3(per, nets), 256, 0, s>>>(src, g.wsum);
    if (g.train_tc)
        k_guide_train_tc<<<dim3(per, nets), kTtThreads, sizeof(TtSmem), s>>>(g, src);
    else
        k_guide_train<<<dim3(per, nets), kTrainThreads, kTrainSmemBytes, s>>>(g, src);
    return cudaGetLastError();
}

}  // namespace

cudaError_t guide_configure() {
    cudaError_t e =
        cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmemBytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TtSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_guide_forward_x_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TcSmem));
}

cudaError_t guide_forward_features_tc(const GuideDevice& g, const float* x, int n, float* raw, int* error,
                                      cudaStream_t s, int test_polls) {
    if (n <= 0) return cudaSuccess;
    const int tiles = (n + kTcThreads - 1) / kTcThreads;
    const int grid = tiles < g.num_sms * 2 ? tiles : g.num_sms * 2;
    k_guide_forward_x_tc<<<grid, kTcThreads, sizeof(TcSmem), s>>>(g.wpack, x, n, raw, error, test_polls);
    return cudaGetLastError();
}

cudaError_t guide_pack(const GuideDevice& g, cudaStream_t s) {
    k_guide_pack<<<dim3((kGuidePackWords + 255) / 256, g.nets > 0 ? g.nets : 1), 256, 0, s>>>(g.w, g.wpack);
    return cudaGetLastError();
}

cudaError_t guide_forward_features(const GuideDevice& g, const float* x, int n, float* raw, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int groups = (n + 15) / 16;
    const int blocks = (groups + 3) / 4 < 1184 ? (groups + 3) / 4 : 1184;
    k_guide_forward_x<<<blocks, 128, 0, s>>>(g.wpack, x, n, raw);
    return cudaGetLastError();
}

cudaError_t guide_gradients_features(const GuideDevice& g, const float* x, const float* wi, const float* w, int n,
                                     cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(g.grad, 0, kGuideParams * sizeof(float), s);
    if (e != cudaSuccess) return e;
    TrainSource src{x, wi, w, nullptr, 0, nullptr, n};
    GuideDevice g1 = g;  // explicit samples train network 0
    g1.nets = 1;
    return launch_train(g1, src, s);
}

cudaError_t guide_train_step(const GuideDevice& g, const GuideSample* ring, int cap, const int* count, int batch,
                             float lr, cudaStream_t s) {
    TrainSource src{nullptr, nullptr, nullptr, ring, cap, count, batch};
    cudaError_t e = launch_train(g, src, s);
    if (e != cudaSuccess) return e;
    const int nets = g.nets > 0 ? g.nets : 1;
    k_guide_adam<<<dim3((kGuideParams + 255) / 256, nets), 256, 0, s>>>(g, lr);
    k_guide_step<<<1, 64, 0, s>>>(g.step, nets);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return guide_pack(g, s);
}

}  // namespace pt
