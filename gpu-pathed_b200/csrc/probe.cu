// Measurement support: the read bandwidth of an L2-resident buffer on this GPU, the
// denominator of the traversal roofline on scenes whose BVH and leaf entries fit in L2.
//
// Every thread of a full persistent grid (resident CTAs x SMs) walks the buffer with a grid
// stride, 16-byte loads cached in L2 only (ld.global.cg: the buffer is re-read from L2, never
// from L1), `reps` times per launch. The sum feeds a data-dependent store, so no load is
// dropped. A first launch brings the buffer into L2; the best of `trials` timed launches
// (CUDA events on one stream) gives the figure.
#include <cuda_runtime.h>
#include <stdint.h>

#include "wavefront.h"

namespace pt {
namespace {

constexpr int kProbeBlock = 256;

__global__ void __launch_bounds__(kProbeBlock) k_l2_read(const float4* __restrict__ buf, long long n4, int reps,
                                                         float* __restrict__ sink) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    for (int r = 0; r < reps; r++) {
        long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        // four independent loads in flight per thread
        for (; i + 3 * stride < n4; i += 4 * stride) {
            const float4 v0 = __ldcg(buf + i);
            const float4 v1 = __ldcg(buf + i + stride);
            const float4 v2 = __ldcg(buf + i + 2 * stride);
            const float4 v3 = __ldcg(buf + i + 3 * stride);
            a0 += v0.x + v0.y + v0.z + v0.w;
            a1 += v1.x + v1.y + v1.z + v1.w;
            a2 += v2.x + v2.y + v2.z + v2.w;
            a3 += v3.x + v3.y + v3.z + v3.w;
        }
        for (; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            a0 += v.x + v.y + v.z + v.w;
        }
    }
    const float s = a0 + a1 + a2 + a3;
    if (s != 0.f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // the buffer holds zeros
}

}  // namespace

cudaError_t measure_l2_read(size_t bytes, int reps, int trials, double* gbs, double* ms) {
    if (bytes < (1u << 20) || bytes % 16 != 0 || reps <= 0 || trials <= 0) return cudaErrorInvalidValue;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_l2_read, kProbeBlock, 0);
    if (e != cudaSuccess) return e;
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    float4* buf = nullptr;
    float* sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double best = 0.0;
    e = cudaMalloc(&buf, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&sink, (size_t)grid * kProbeBlock * sizeof(float));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, bytes, st);
    const long long n4 = (long long)(bytes / 16);
    if (e == cudaSuccess) {
        k_l2_read<<<grid, kProbeBlock, 0, st>>>(buf, n4, 1, sink);  // bring the buffer into L2
        e = cudaGetLastError();
    }
    for (int t = 0; t < trials && e == cudaSuccess; t++) {
        e = cudaEventRecord(ev0, st);
        if (e == cudaSuccess) {
            k_l2_read<<<grid, kProbeBlock, 0, st>>>(buf, n4, reps, sink);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev1, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev1);
        float m = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&m, ev0, ev1);
        if (e == cudaSuccess && m > 0.f) {
            const double g = (double)bytes * reps / (m * 1e-3) / 1e9;
            if (g > best) {
                best = g;
                if (ms) *ms = m;
            }
        }
    }
    if (st) cudaStreamSynchronize(st);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
    if (sink) cudaFree(sink);
    if (buf) cudaFree(buf);
    if (e == cudaSuccess && gbs) *gbs = best;
    return e;
}

}  // namespace pt
