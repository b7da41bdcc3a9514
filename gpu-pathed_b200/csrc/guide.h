// Host-visible interface of the path-guiding kernels (guide.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "guide.cuh"
#include "pt_types.h"

namespace pt {

// Device buffers of the guide networks and their training state. With nets > 1 (batched
// frames, one network per guided scene) every array holds `nets` consecutive copies: per net
// kGuideParams parameters, kGuidePackWords packed words, 4 words of sums (weight sum, loss,
// unused, step counter) and its own sample ring.
struct GuideDevice {
    float* w;            // FP32 master parameters [kGuideParams]
    uint32_t* wpack;     // [kGuidePackWords] shared-memory images of the BF16 weights
    float* grad;         // [kGuideParams]
    float* adam_m;       // [kGuideParams]
    float* adam_v;       // [kGuideParams]
    float* wsum;         // [2] sum of sample weights of the current batch, batch loss
    int* step;           // Adam steps taken (device counter, so training launches replay in graphs)
    int num_sms;         // training grid: one block per SM
    int nets;            // networks trained together (1 for a single scene)
    int train_tc;        // 1: the training kernel on tcgen05 (k_guide_train_tc), 0: on mma.sync
    const GuideFrame* frames;  // per-network encoding frames (nets > 1), else `frame`
    GuideFrame frame;
};

// One training sample: where, which direction was sampled, and its weight F / p.
struct GuideSample {
    float p[3], n[3], wo[3], wi[3];
    float weight;
    float pad[3];
};
static_assert(sizeof(GuideSample) == 64, "GuideSample layout");

// Vertex record written while shading a training path; resolved into a GuideSample once the
// path's later contributions are known.
struct GuideRecord {
    float p[3], n[3], wo[3], wi[3];
    float fcos_over_p;   // luminance of f |cos| / p_mix at the vertex
    float beta_next;     // luminance of the throughput after the vertex
    int tpath;           // training-path index within the wave
    int depth;           // vertex depth
};
static_assert(sizeof(GuideRecord) == 64, "GuideRecord layout");

// 32-bit words of the packed weights: the shared-memory images of the forward weights (BF16
// pairs of consecutive inputs, padded rows, FP32 biases; 9000 words), of the transposed
// backward weights (BF16 pairs of consecutive outputs, padded rows; 6912 words) and of the
// tensor-memory inference's K-major operand images (8192 words).
constexpr int kGuidePackWords = 24104;

// Opt the training kernel into its dynamic shared memory (once per device, before capture).
cudaError_t guide_configure();
// Repack the FP32 master weights into the packed images.
cudaError_t guide_pack(const GuideDevice& g, cudaStream_t s);
// Raw network outputs for n explicit input vectors (inference kernel, tensor cores).
cudaError_t guide_forward_features(const GuideDevice& g, const float* x, int n, float* raw, cudaStream_t s);
// The same on the 5th-generation tensor cores (tcgen05.mma into tensor memory); a wait that
// gives up sets bit 1 of *error (device int). test_polls > 0: the test hook of tc_network.
cudaError_t guide_forward_features_tc(const GuideDevice& g, const float* x, int n, float* raw, int* error,
                                      cudaStream_t s, int test_polls = 0);
// Gradient of the batch loss -sum_i w_i log q(wi_i | x_i) / sum_i w_i with respect to all
// parameters, for explicit input vectors (training kernel); grad is overwritten.
cudaError_t guide_gradients_features(const GuideDevice& g, const float* x, const float* wi, const float* w, int n,
                                     cudaStream_t s);
// Training on the newest `batch` samples of a ring of capacity `cap` (`count` samples written
// so far): gradients, then one Adam step (lr, betas 0.9 / 0.999, eps 1e-8) whose bias
// correction uses the device step counter, then the repack. Graph-capturable: no argument
// changes from step to step.
cudaError_t guide_train_step(const GuideDevice& g, const GuideSample* ring, int cap, const int* count, int batch,
                             float lr, cudaStream_t s);
// Per-net views of a multi-net GuideDevice.
inline float* guide_net_params(const GuideDevice& g, int net) { return g.w + (size_t)net * kGuideParams; }

}  // namespace pt
