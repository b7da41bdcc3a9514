// Path-guiding network kernels: weight packing, tensor-core inference on explicit inputs,
// the fused training kernel (forward + loss + backward + per-block gradient accumulation)
// and the Adam update.
//
// Loss (neural importance sampling, Mueller et al. 2019): for samples wi_i drawn with
// density p_i, F_i the integrand value and w_i = F_i / p_i, minimise
//     L = - sum_i w_i log q(wi_i | x_i) / sum_i w_i,
// a Monte Carlo estimate of the KL divergence from the normalised integrand to q (up to a
// constant). Training arithmetic is FP32 with the BF16-rounded weights the inference kernel
// uses, so the trained and the evaluated network are the same function.
#include "guide.h"

#include <cuda_bf16.h>

#include "guide_mlp.cuh"

namespace pt {

namespace {

constexpr int kTile = 64;      // samples per training tile
constexpr int kTrainThreads = 256;
constexpr int kOwned = (kGuideParams + kTrainThreads - 1) / kTrainThreads;  // 63 parameters per thread
// padded row strides (odd) so that column-wise walks hit distinct banks
constexpr int kXS = 81, kAS = 65, kYS = 41;
constexpr int kSmemFloats = kGuideParams + kTile * kXS + 3 * kTile * kAS + kTile * kYS + 2 * kTile * kAS +
                            kTile * 3 + kTile;

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__global__ void k_guide_pack(const float* __restrict__ w, uint32_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGuidePackWords) return;
    auto pair = [&](int base, int ncol, int kp, int n) {
        return pack_bf16(w[base + (2 * kp) * ncol + n], w[base + (2 * kp + 1) * ncol + n]);
    };
    uint32_t v;
    if (i < kGP2) v = pair(kGW1, 64, i / 64, i % 64);
    else if (i < kGP3) v = pair(kGW2, 64, (i - kGP2) / 64, (i - kGP2) % 64);
    else if (i < kGP4) v = pair(kGW3, 64, (i - kGP3) / 64, (i - kGP3) % 64);
    else if (i < kGPB) v = pair(kGW4, 40, (i - kGP4) / 40, (i - kGP4) % 40);
    else {
        const int j = i - kGPB;  // b1 64, b2 64, b3 64, b4 40
        const float b = j < 64 ? w[kGB1 + j] : j < 128 ? w[kGB2 + j - 64] : j < 192 ? w[kGB3 + j - 128] : w[kGB4 + j - 192];
        v = __float_as_uint(b);
    }
    out[i] = v;
}

// Inference on explicit input vectors (tests, tools): 4 warps per block, 16 rows per warp.
__global__ void k_guide_forward_x(const uint32_t* __restrict__ wpack, const float* __restrict__ x, int n,
                                  float* __restrict__ raw) {
    __shared__ uint32_t sw[kSWords];
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
            const float a = gi < n ? x[(size_t)gi * kGuideIn + 2 * k] : 0.f;
            const float b = gi < n ? x[(size_t)gi * kGuideIn + 2 * k + 1] : 0.f;
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
        float x[kGuideIn];
        guide_encode(gf, sm.p, sm.n, sm.wo, x);
        for (int k = 0; k < kGuideIn; k++) xrow[k] = x[k];
        wi[0] = sm.wi[0]; wi[1] = sm.wi[1]; wi[2] = sm.wi[2];
        w = sm.weight;
    } else {
        for (int k = 0; k < kGuideIn; k++) xrow[k] = s.x[(size_t)i * kGuideIn + k];
        wi[0] = s.wi[3 * i]; wi[1] = s.wi[3 * i + 1]; wi[2] = s.wi[3 * i + 2];
        w = s.w[i];
    }
}

__global__ void k_guide_wsum(TrainSource s, float* wsum) {
    int first, n;
    source_range(s, first, n);
    float acc = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += s.ring ? s.ring[(unsigned)(first + i) % (unsigned)s.cap].weight : s.w[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(wsum, acc);
}

// out[t][n] = act(b[n] + sum_k in[t][k] W[k][n]) for a tile of kTile rows.
template <bool RELU>
__device__ __forceinline__ void dense_fwd(const float* in, int in_stride, int K, const float* W, const float* b, int N,
                                          float* out, int out_stride) {
    for (int o = threadIdx.x; o < kTile * N; o += blockDim.x) {
        const int t = o % kTile, n = o / kTile;
        float acc = b[n];
        for (int k = 0; k < K; k++) acc = fmaf(in[t * in_stride + k], W[k * N + n], acc);
        out[t * out_stride + n] = RELU ? fmaxf(acc, 0.f) : acc;
    }
}

// dA[t][k] = (sum_n dZ[t][n] W[k][n]) * (A[t][k] > 0): backward through a dense layer and the
// ReLU of its input.
__device__ __forceinline__ void dense_bwd(const float* dz, int dz_stride, int N, const float* W, int K, const float* a,
                                          float* da) {
    for (int o = threadIdx.x; o < kTile * K; o += blockDim.x) {
        const int t = o % kTile, k = o / kTile;
        float acc = 0.f;
        for (int n = 0; n < N; n++) acc = fmaf(dz[t * dz_stride + n], W[k * N + n], acc);
        da[t * kAS + k] = a[t * kAS + k] > 0.f ? acc : 0.f;
    }
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

__global__ void __launch_bounds__(kTrainThreads) k_guide_train(GuideDevice g, TrainSource src) {
    extern __shared__ float sm[];
    float* sW = sm;
    float* sX = sW + kGuideParams;
    float* sA1 = sX + kTile * kXS;
    float* sA2 = sA1 + kTile * kAS;
    float* sA3 = sA2 + kTile * kAS;
    float* sY = sA3 + kTile * kAS;
    float* sD0 = sY + kTile * kYS;
    float* sD1 = sD0 + kTile * kAS;
    float* sWi = sD1 + kTile * kAS;
    float* sWt = sWi + kTile * 3;
    for (int i = threadIdx.x; i < kGuideParams; i += blockDim.x) sW[i] = bf16_round(g.w[i]);
    int first, n;
    source_range(src, first, n);
    const float wsum = g.wsum[0];
    const float inv_wsum = wsum > 0.f ? 1.f / wsum : 0.f;
    float gacc[kOwned];
#pragma unroll
    for (int i = 0; i < kOwned; i++) gacc[i] = 0.f;
    __syncthreads();
    // accumulate the gradients of the parameters this thread owns that lie in [lo, hi)
    auto own = [&](int lo, int hi, const float* a, int a_stride, int K, const float* dz, int dz_stride, int N,
                   int blo) {
#pragma unroll
        for (int i = 0; i < kOwned; i++) {
            const int gi = threadIdx.x + kTrainThreads * i;
            if (gi >= lo && gi < hi) {
                const int k = (gi - lo) / N, nn = (gi - lo) % N;
                float acc = 0.f;
                for (int t = 0; t < kTile; t++) acc = fmaf(a[t * a_stride + k], dz[t * dz_stride + nn], acc);
                gacc[i] += acc;
            } else if (gi >= blo && gi < blo + N) {
                const int nn = gi - blo;
                float acc = 0.f;
                for (int t = 0; t < kTile; t++) acc += dz[t * dz_stride + nn];
                gacc[i] += acc;
            }
        }
        (void)K;
    };
    for (int tile = blockIdx.x; tile * kTile < n; tile += gridDim.x) {
        if (threadIdx.x < kTile) {
            const int t = threadIdx.x, i = tile * kTile + t;
            float wi[3] = {0.f, 0.f, 1.f}, w = 0.f;
            if (i < n) {
                source_sample(src, g.frame, first, i, sX + t * kXS, wi, w);
            } else {
                for (int k = 0; k < kGuideIn; k++) sX[t * kXS + k] = 0.f;
            }
            sWi[3 * t] = wi[0]; sWi[3 * t + 1] = wi[1]; sWi[3 * t + 2] = wi[2];
            sWt[t] = w * inv_wsum;
        }
        __syncthreads();
        dense_fwd<true>(sX, kXS, kGuideIn, sW + kGW1, sW + kGB1, kGuideHidden, sA1, kAS);
        __syncthreads();
        dense_fwd<true>(sA1, kAS, kGuideHidden, sW + kGW2, sW + kGB2, kGuideHidden, sA2, kAS);
        __syncthreads();
        dense_fwd<true>(sA2, kAS, kGuideHidden, sW + kGW3, sW + kGB3, kGuideHidden, sA3, kAS);
        __syncthreads();
        dense_fwd<false>(sA3, kAS, kGuideHidden, sW + kGW4, sW + kGB4, kGuideOut, sY, kYS);
        __syncthreads();
        if (threadIdx.x < kTile) {
            const int t = threadIdx.x;
            float raw[kGuideOut], dy[kGuideOut];
            for (int j = 0; j < kGuideOut; j++) raw[j] = sY[t * kYS + j];
            const float wi[3] = {sWi[3 * t], sWi[3 * t + 1], sWi[3 * t + 2]};
            const float l = loss_grad(raw, wi, sWt[t], dy);
            if (l != 0.f) atomicAdd(g.wsum + 1, l);  // batch loss, for monitoring
            for (int j = 0; j < kGuideOut; j++) sY[t * kYS + j] = dy[j];
        }
        __syncthreads();
        // layer 4: dW4 = A3^T dY, db4 = sum dY; dZ3 = (dY W4^T) * relu'(Z3)
        own(kGW4, kGB4, sA3, kAS, kGuideHidden, sY, kYS, kGuideOut, kGB4);
        dense_bwd(sY, kYS, kGuideOut, sW + kGW4, kGuideHidden, sA3, sD0);
        __syncthreads();
        own(kGW3, kGB3, sA2, kAS, kGuideHidden, sD0, kAS, kGuideHidden, kGB3);
        dense_bwd(sD0, kAS, kGuideHidden, sW + kGW3, kGuideHidden, sA2, sD1);
        __syncthreads();
        own(kGW2, kGB2, sA1, kAS, kGuideHidden, sD1, kAS, kGuideHidden, kGB2);
        __syncthreads();  // sD0 is overwritten next
        dense_bwd(sD1, kAS, kGuideHidden, sW + kGW2, kGuideHidden, sA1, sD0);
        __syncthreads();
        own(kGW1, kGB1, sX, kXS, kGuideIn, sD0, kAS, kGuideHidden, kGB1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < kOwned; i++) {
        const int gi = threadIdx.x + kTrainThreads * i;
        if (gi < kGuideParams && gacc[i] != 0.f) atomicAdd(&g.grad[gi], gacc[i]);
    }
}

__global__ void k_guide_adam(GuideDevice g, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGuideParams) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
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

cudaError_t launch_train(const GuideDevice& g, const TrainSource& src, cudaStream_t s) {
    static bool configured = false;
    const size_t smem = (size_t)kSmemFloats * sizeof(float);
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    cudaError_t e = cudaMemsetAsync(g.wsum, 0, 2 * sizeof(float), s);  // weight sum, batch loss
    if (e != cudaSuccess) return e;
    k_guide_wsum<<<148, 256, 0, s>>>(src, g.wsum);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_guide_train<<<sms, kTrainThreads, smem, s>>>(g, src);
    return cudaGetLastError();
}

}  // namespace

cudaError_t guide_pack(const GuideDevice& g, cudaStream_t s) {
    k_guide_pack<<<(kGuidePackWords + 255) / 256, 256, 0, s>>>(g.w, g.wpack);
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
    return launch_train(g, src, s);
}

cudaError_t guide_adam(const GuideDevice& g, float lr, int t, cudaStream_t s) {
    const float c1 = 1.f - powf(0.9f, (float)t), c2 = 1.f - powf(0.999f, (float)t);
    k_guide_adam<<<(kGuideParams + 255) / 256, 256, 0, s>>>(g, lr, c1, c2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return guide_pack(g, s);
}

cudaError_t guide_train_step(const GuideDevice& g, const GuideSample* ring, int cap, const int* count, int batch,
                             float lr, int t, cudaStream_t s) {
    TrainSource src{nullptr, nullptr, nullptr, ring, cap, count, batch};
    cudaError_t e = launch_train(g, src, s);
    if (e != cudaSuccess) return e;
    return guide_adam(g, lr, t, s);
}

}  // namespace pt
