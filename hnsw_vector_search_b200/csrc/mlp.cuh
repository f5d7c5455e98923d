#pragma once

// The learned early-termination network (mlp.cu): training on the GPU, its device copy for the
// search kernel.

#include <cstddef>
#include <cstdint>
#include <memory>

#include "search.cuh"

namespace vdx::dev {

constexpr int kStopFeatures = 12;
constexpr int kStopHidden = 64;
// Parameter offsets in the 5,057-float vector: W1 [64][12], b1, W2 [64][64], b2, W3, b3.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kStopHidden * kStopFeatures;
constexpr int kOffW2 = kOffB1 + kStopHidden;
constexpr int kOffB2 = kOffW2 + kStopHidden * kStopHidden;
constexpr int kOffW3 = kOffB2 + kStopHidden;
constexpr int kOffB3 = kOffW3 + kStopHidden;
constexpr int kStopParams = kOffB3 + 1;
static_assert(kStopParams == 5057, "12 -> 64 -> 64 -> 1");

struct MlpTrainConfig {
    int epochs = 8;
    std::size_t batch = 4096;
    float lr = 1e-3F;
    float beta1 = 0.9F;
    float beta2 = 0.999F;
    std::uint64_t seed = 7;
};

// Trains on raw features x [n][12] and labels y [n] (0 or 1); returns the FP32 weights, the
// standardization (mean, 1/std, computed from x) and the mean loss of each epoch.
void mlp_train(const float* x, const float* y, std::size_t n, const MlpTrainConfig& cfg,
               float* weights, float* mean, float* inv_std, float* loss_per_epoch);

// One forward and backward pass over already standardized x: the gradient of the mean loss with
// respect to the (bfloat16-rounded) weights, and that loss.
void mlp_gradient(const float* x, const float* y, std::size_t n, const float* weights, float* grad,
                  float* loss);

// P(converged) for raw features x [n][12].
void mlp_probabilities(const float* x, std::size_t n, const float* weights, const float* mean,
                       const float* inv_std, float* prob);

struct DeviceStopNet {
    StopNetView view{};
    void* alloc = nullptr;
    int device = 0;
    ~DeviceStopNet();
};

// proj: 4 rows of `dim` floats (the random projection directions of features 8..11).
std::unique_ptr<DeviceStopNet> upload_stop_net(const float* weights, const float* mean,
                                               const float* inv_std, const float* proj,
                                               std::uint32_t dim, std::uint32_t row32, int device);

}  // namespace vdx::dev
