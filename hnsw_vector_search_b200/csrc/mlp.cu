// The learned early-termination network: training kernels (forward, backward, Adam), the host
// training loop, and the device copy the search kernel evaluates.
//
// Network: 12 standardized features -> 64 ReLU -> 64 ReLU -> 1 logit, sigmoid = P(converged).
// Parameters (5,057, FP32 masters, this order): W1 [64][12], b1 [64], W2 [64][64], b2 [64],
// W3 [64], b3. Weights are used rounded to bfloat16 (round to nearest even) in every forward
// pass, in training as in the search kernel, with FP32 accumulation; gradients are those of the
// rounded weights applied to the FP32 masters. Loss: binary cross-entropy with logits, mean
// over the batch.
//
// Kernels: mlp_forward_kernel (one block of 64 threads per 32 samples: thread j owns hidden unit
// j of both layers), mlp_backward_kernel (same shape; each thread accumulates its rows of dW1 and
// dW2 in registers over the block's samples, then one atomicAdd per parameter per block),
// adam_kernel (elementwise). All FP32.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "gpu_runtime.cuh"
#include "mlp.cuh"

namespace vdx::dev {
namespace {

constexpr int F = kStopFeatures;
constexpr int H = kStopHidden;
constexpr int kSamplesPerBlock = 32;

__device__ __forceinline__ float bf16_round(float x) {
    // Round to nearest even at 8 significant bits; inputs are finite.
    const std::uint32_t u = __float_as_uint(x);
    const std::uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
    return __uint_as_float(r & 0xFFFF0000u);
}

// Rounded copy of the weights (biases stay FP32).
__global__ void round_weights_kernel(const float* w, float* wq) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kStopParams; i += gridDim.x * blockDim.x) {
        const bool bias = (i >= kOffB1 && i < kOffW2) || (i >= kOffB2 && i < kOffW3) || i == kOffB3;
        wq[i] = bias ? w[i] : bf16_round(w[i]);
    }
}

// Forward: h1, h2 (post-ReLU) and the logit of each sample; loss summed into *loss.
__global__ void __launch_bounds__(H) mlp_forward_kernel(const float* __restrict__ x,
                                                        const float* __restrict__ y,
                                                        const float* __restrict__ wq, int n,
                                                        float* __restrict__ h1,
                                                        float* __restrict__ h2,
                                                        float* __restrict__ logit, float* loss) {
    __shared__ float sw2[H * H];
    __shared__ float sh1[H];
    __shared__ float red[H];
    const int j = threadIdx.x;
    for (int i = j; i < H * H; i += H) {
        sw2[i] = wq[kOffW2 + i];
    }
    float w1[F];
#pragma unroll
    for (int c = 0; c < F; ++c) {
        w1[c] = wq[kOffW1 + j * F + c];
    }
    const float b1 = wq[kOffB1 + j];
    const float b2 = wq[kOffB2 + j];
    const float w3 = wq[kOffW3 + j];
    const float b3 = wq[kOffB3];
    __syncthreads();
    float block_loss = 0.0F;
    const int first = blockIdx.x * kSamplesPerBlock;
    for (int s = first; s < min(first + kSamplesPerBlock, n); ++s) {
        float a = b1;
#pragma unroll
        for (int c = 0; c < F; ++c) {
            a = fmaf(w1[c], x[static_cast<std::size_t>(s) * F + c], a);
        }
        a = fmaxf(a, 0.0F);
        sh1[j] = a;
        h1[static_cast<std::size_t>(s) * H + j] = a;
        __syncthreads();
        float z = b2;
        for (int i = 0; i < H; ++i) {
            z = fmaf(sw2[j * H + i], sh1[i], z);
        }
        z = fmaxf(z, 0.0F);
        h2[static_cast<std::size_t>(s) * H + j] = z;
        red[j] = w3 * z;
        __syncthreads();
        for (int o = H / 2; o > 0; o >>= 1) {
            if (j < o) {
                red[j] += red[j + o];
            }
            __syncthreads();
        }
        if (j == 0) {
            const float l = red[0] + b3;
            logit[s] = l;
            // BCE with logits: max(l, 0) - l y + log(1 + exp(-|l|))
            block_loss += fmaxf(l, 0.0F) - l * y[s] + log1pf(expf(-fabsf(l)));
        }
        __syncthreads();
    }
    if (j == 0 && loss != nullptr) {
        atomicAdd(loss, block_loss);
    }
}

// Backward for the mean loss over `n_total` samples: gradients of the rounded weights summed
// into `grad` (zeroed by the caller).
__global__ void __launch_bounds__(H) mlp_backward_kernel(
    const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ wq, int n,
    float inv_n, const float* __restrict__ h1, const float* __restrict__ h2,
    const float* __restrict__ logit, float* __restrict__ grad) {
    __shared__ float sw2[H * H];
    __shared__ float sdh2[H];
    __shared__ float sh1[H];
    __shared__ float sx[F];
    const int j = threadIdx.x;
    for (int i = j; i < H * H; i += H) {
        sw2[i] = wq[kOffW2 + i];
    }
    const float w3 = wq[kOffW3 + j];
    __syncthreads();
    float gw2[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        gw2[i] = 0.0F;
    }
    float gw1[F];
#pragma unroll
    for (int c = 0; c < F; ++c) {
        gw1[c] = 0.0F;
    }
    float gb1 = 0.0F, gb2 = 0.0F, gw3 = 0.0F, gb3 = 0.0F;
    const int first = blockIdx.x * kSamplesPerBlock;
    for (int s = first; s < min(first + kSamplesPerBlock, n); ++s) {
        const float l = logit[s];
        const float dl = (1.0F / (1.0F + expf(-l)) - y[s]) * inv_n;
        const float z = h2[static_cast<std::size_t>(s) * H + j];
        const float a = h1[static_cast<std::size_t>(s) * H + j];
        gw3 = fmaf(dl, z, gw3);
        gb3 += dl;
        const float dz = z > 0.0F ? dl * w3 : 0.0F;  // d loss / d (pre-ReLU layer 2), unit j
        sdh2[j] = dz;
        sh1[j] = a;
        if (j < F) {
            sx[j] = x[static_cast<std::size_t>(s) * F + j];
        }
        __syncthreads();
        // Layer 2 weights, row j: dz_j * h1_i.
#pragma unroll
        for (int i = 0; i < H; ++i) {
            gw2[i] = fmaf(dz, sh1[i], gw2[i]);
        }
        gb2 += dz;
        // Layer 1, unit j: sum over layer-2 units m of dz_m * W2[m][j], through the ReLU.
        float da = 0.0F;
        for (int m = 0; m < H; ++m) {
            da = fmaf(sdh2[m], sw2[m * H + j], da);
        }
        da = a > 0.0F ? da : 0.0F;
#pragma unroll
        for (int c = 0; c < F; ++c) {
            gw1[c] = fmaf(da, sx[c], gw1[c]);
        }
        gb1 += da;
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < H; ++i) {
        atomicAdd(grad + kOffW2 + j * H + i, gw2[i]);
    }
#pragma unroll
    for (int c = 0; c < F; ++c) {
        atomicAdd(grad + kOffW1 + j * F + c, gw1[c]);
    }
    atomicAdd(grad + kOffB1 + j, gb1);
    atomicAdd(grad + kOffB2 + j, gb2);
    atomicAdd(grad + kOffW3 + j, gw3);
    if (j == 0) {
        atomicAdd(grad + kOffB3, gb3);
    }
}

__global__ void adam_kernel(float* w, const float* g, float* m, float* v, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kStopParams; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0F - b1) * gi;
        const float vi = b2 * v[i] + (1.0F - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void gather_rows_kernel(const float* x, const float* y, const std::uint32_t* idx, int n,
                                   float* bx, float* by) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        const std::uint32_t r = idx[s];
        for (int c = 0; c < F; ++c) {
            bx[static_cast<std::size_t>(s) * F + c] = x[static_cast<std::size_t>(r) * F + c];
        }
        by[s] = y[r];
    }
}

__global__ void standardize_kernel(float* x, std::size_t n, const float* mean, const float* inv_std) {
    for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < n * F;
         i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i % F);
        x[i] = (x[i] - mean[c]) * inv_std[c];
    }
}

__global__ void sigmoid_kernel(const float* logit, float* p, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        p[s] = 1.0F / (1.0F + expf(-logit[s]));
    }
}

struct DeviceBuffer {
    void* p = nullptr;
    explicit DeviceBuffer(std::size_t bytes) { gpu::check(cudaMalloc(&p, bytes ? bytes : 16), "mlp buffer"); }
    ~DeviceBuffer() { cudaFree(p); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// He-uniform initialization from a seeded 64-bit LCG (deterministic on every host).
std::vector<float> initial_weights(std::uint64_t seed) {
    std::vector<float> w(kStopParams, 0.0F);
    std::uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
    const auto uniform = [&s]() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return static_cast<float>((s >> 11) * 0x1.0p-53) * 2.0F - 1.0F;
    };
    const float a1 = std::sqrt(6.0F / F), a2 = std::sqrt(6.0F / H), a3 = std::sqrt(6.0F / H);
    for (int i = 0; i < H * F; ++i) w[kOffW1 + i] = a1 * uniform();
    for (int i = 0; i < H * H; ++i) w[kOffW2 + i] = a2 * uniform();
    for (int i = 0; i < H; ++i) w[kOffW3 + i] = a3 * uniform() * 0.1F;
    return w;
}

void forward_backward(const float* dx, const float* dy, int n, const float* dwq, float* dh1,
                      float* dh2, float* dlogit, float* dgrad, float* dloss, cudaStream_t s) {
    const int blocks = (n + kSamplesPerBlock - 1) / kSamplesPerBlock;
    mlp_forward_kernel<<<blocks, H, 0, s>>>(dx, dy, dwq, n, dh1, dh2, dlogit, dloss);
    gpu::check(cudaGetLastError(), "mlp forward");
    if (dgrad != nullptr) {
        mlp_backward_kernel<<<blocks, H, 0, s>>>(dx, dy, dwq, n, 1.0F / static_cast<float>(n), dh1,
                                                  dh2, dlogit, dgrad);
        gpu::check(cudaGetLastError(), "mlp backward");
    }
}

}  // namespace

void mlp_gradient(const float* x, const float* y, std::size_t n, const float* weights, float* grad,
                  float* loss) {
    cudaStream_t s = gpu::workspace(0).stream;
    DeviceBuffer dx(n * F * 4), dy(n * 4), dw(kStopParams * 4), dwq(kStopParams * 4),
        dg(kStopParams * 4), dh1(n * H * 4), dh2(n * H * 4), dl(n * 4), dloss(4);
    gpu::check(cudaMemcpyAsync(dx.p, x, n * F * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(dy.p, y, n * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(dw.p, weights, kStopParams * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemsetAsync(dg.p, 0, kStopParams * 4, s), "memset");
    gpu::check(cudaMemsetAsync(dloss.p, 0, 4, s), "memset");
    round_weights_kernel<<<8, 256, 0, s>>>(dw.as<float>(), dwq.as<float>());
    forward_backward(dx.as<float>(), dy.as<float>(), static_cast<int>(n), dwq.as<float>(),
                     dh1.as<float>(), dh2.as<float>(), dl.as<float>(), dg.as<float>(),
                     dloss.as<float>(), s);
    gpu::check(cudaMemcpyAsync(grad, dg.p, kStopParams * 4, cudaMemcpyDeviceToHost, s), "copy");
    float total = 0.0F;
    gpu::check(cudaMemcpyAsync(&total, dloss.p, 4, cudaMemcpyDeviceToHost, s), "copy");
    gpu::check(cudaStreamSynchronize(s), "mlp gradient");
    *loss = total / static_cast<float>(n);
}

void mlp_probabilities(const float* x, std::size_t n, const float* weights, const float* mean,
                       const float* inv_std, float* prob) {
    cudaStream_t s = gpu::workspace(0).stream;
    DeviceBuffer dx(n * F * 4), dy(n * 4), dw(kStopParams * 4), dwq(kStopParams * 4),
        dh1(n * H * 4), dh2(n * H * 4), dl(n * 4), dm(F * 4), ds(F * 4);
    gpu::check(cudaMemcpyAsync(dx.p, x, n * F * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemsetAsync(dy.p, 0, n * 4, s), "memset");
    gpu::check(cudaMemcpyAsync(dw.p, weights, kStopParams * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(dm.p, mean, F * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(ds.p, inv_std, F * 4, cudaMemcpyHostToDevice, s), "copy");
    standardize_kernel<<<256, 256, 0, s>>>(dx.as<float>(), n, dm.as<float>(), ds.as<float>());
    round_weights_kernel<<<8, 256, 0, s>>>(dw.as<float>(), dwq.as<float>());
    forward_backward(dx.as<float>(), dy.as<float>(), static_cast<int>(n), dwq.as<float>(),
                     dh1.as<float>(), dh2.as<float>(), dl.as<float>(), nullptr, nullptr, s);
    sigmoid_kernel<<<(static_cast<int>(n) + 255) / 256, 256, 0, s>>>(dl.as<float>(), dy.as<float>(),
                                                                     static_cast<int>(n));
    gpu::check(cudaMemcpyAsync(prob, dy.p, n * 4, cudaMemcpyDeviceToHost, s), "copy");
    gpu::check(cudaStreamSynchronize(s), "mlp forward");
}

void mlp_train(const float* x, const float* y, std::size_t n, const MlpTrainConfig& cfg,
               float* weights, float* mean, float* inv_std, float* loss_per_epoch) {
    if (n == 0) {
        throw std::invalid_argument("mlp_train: no samples");
    }
    // Standardization statistics (FP64 on the host).
    for (int c = 0; c < F; ++c) {
        double m = 0.0, v = 0.0;
        for (std::size_t i = 0; i < n; ++i) {
            m += x[i * F + c];
        }
        m /= static_cast<double>(n);
        for (std::size_t i = 0; i < n; ++i) {
            const double d = x[i * F + c] - m;
            v += d * d;
        }
        v /= static_cast<double>(n);
        mean[c] = static_cast<float>(m);
        inv_std[c] = static_cast<float>(1.0 / std::sqrt(v + 1e-12));
    }
    cudaStream_t s = gpu::workspace(0).stream;
    const int batch = static_cast<int>(std::min<std::size_t>(cfg.batch, n));
    DeviceBuffer dx(n * F * 4), dy(n * 4), dm(F * 4), ds(F * 4), dw(kStopParams * 4),
        dwq(kStopParams * 4), dg(kStopParams * 4), dmom(kStopParams * 4), dvar(kStopParams * 4),
        dbx(static_cast<std::size_t>(batch) * F * 4), dby(batch * 4ull),
        dh1(static_cast<std::size_t>(batch) * H * 4), dh2(static_cast<std::size_t>(batch) * H * 4),
        dl(batch * 4ull), dloss(4), didx(n * 4);
    gpu::check(cudaMemcpyAsync(dx.p, x, n * F * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(dy.p, y, n * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(dm.p, mean, F * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemcpyAsync(ds.p, inv_std, F * 4, cudaMemcpyHostToDevice, s), "copy");
    standardize_kernel<<<1024, 256, 0, s>>>(dx.as<float>(), n, dm.as<float>(), ds.as<float>());
    const std::vector<float> w0 = initial_weights(cfg.seed);
    gpu::check(cudaMemcpyAsync(dw.p, w0.data(), kStopParams * 4, cudaMemcpyHostToDevice, s), "copy");
    gpu::check(cudaMemsetAsync(dmom.p, 0, kStopParams * 4, s), "memset");
    gpu::check(cudaMemsetAsync(dvar.p, 0, kStopParams * 4, s), "memset");
    std::vector<std::uint32_t> order(n);
    for (std::size_t i = 0; i < n; ++i) {
        order[i] = static_cast<std::uint32_t>(i);
    }
    std::uint64_t rng = cfg.seed ^ 0x9E3779B97F4A7C15ull;
    int step = 0;
    for (int epoch = 0; epoch < cfg.epochs; ++epoch) {
        for (std::size_t i = n - 1; i > 0; --i) {  // Fisher-Yates with a 64-bit LCG
            rng = rng * 6364136223846793005ull + 1442695040888963407ull;
            std::swap(order[i], order[(rng >> 33) % (i + 1)]);
        }
        gpu::check(cudaMemcpyAsync(didx.p, order.data(), n * 4, cudaMemcpyHostToDevice, s), "copy");
        gpu::check(cudaMemsetAsync(dloss.p, 0, 4, s), "memset");
        for (std::size_t start = 0; start + batch <= n; start += batch) {
            gather_rows_kernel<<<(batch + 255) / 256, 256, 0, s>>>(
                dx.as<float>(), dy.as<float>(), didx.as<std::uint32_t>() + start, batch,
                dbx.as<float>(), dby.as<float>());
            round_weights_kernel<<<8, 256, 0, s>>>(dw.as<float>(), dwq.as<float>());
            gpu::check(cudaMemsetAsync(dg.p, 0, kStopParams * 4, s), "memset");
            forward_backward(dbx.as<float>(), dby.as<float>(), batch, dwq.as<float>(),
                             dh1.as<float>(), dh2.as<float>(), dl.as<float>(), dg.as<float>(),
                             dloss.as<float>(), s);
            ++step;
            const float c1 = 1.0F - std::pow(cfg.beta1, static_cast<float>(step));
            const float c2 = 1.0F - std::pow(cfg.beta2, static_cast<float>(step));
            adam_kernel<<<8, 256, 0, s>>>(dw.as<float>(), dg.as<float>(), dmom.as<float>(),
                                          dvar.as<float>(), cfg.lr, cfg.beta1, cfg.beta2, 1e-8F, c1, c2);
            gpu::check(cudaGetLastError(), "adam");
        }
        float total = 0.0F;
        gpu::check(cudaMemcpyAsync(&total, dloss.p, 4, cudaMemcpyDeviceToHost, s), "copy");
        gpu::check(cudaStreamSynchronize(s), "mlp train");
        if (loss_per_epoch != nullptr) {
            const std::size_t used = (n / batch) * static_cast<std::size_t>(batch);
            loss_per_epoch[epoch] = total / static_cast<float>(used);
        }
    }
    gpu::check(cudaMemcpyAsync(weights, dw.p, kStopParams * 4, cudaMemcpyDeviceToHost, s), "copy");
    gpu::check(cudaStreamSynchronize(s), "mlp train");
}

// ---------------------------------------------------------------------------------------------
// The device copy the search kernel reads.

DeviceStopNet::~DeviceStopNet() {
    if (alloc != nullptr) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaFree(alloc);
        cudaSetDevice(prev);
    }
}

std::unique_ptr<DeviceStopNet> upload_stop_net(const float* weights, const float* mean,
                                               const float* inv_std, const float* proj,
                                               std::uint32_t dim, std::uint32_t row32, int device) {
    gpu::use_device(device);
    auto net = std::make_unique<DeviceStopNet>();
    net->device = device;
    // Layout, for a warp whose lane L owns hidden units L and L + 32 of both layers: bf16 pairs
    // (unit L in the low half, unit L + 32 in the high half) — w1 as [32 lanes][12 features],
    // w2 as [16 groups of 4 inputs][32 lanes][4 inputs] (one 16-byte load per lane per group),
    // w3 as [32 lanes] — then FP32 b1, b2, b3, mean, inv_std, proj.
    const std::size_t n16 = H * F + H * H + H;
    const std::size_t off32 = (n16 * 2 + 255) / 256 * 256;
    const std::size_t n32 = H + H + 1 + F + F;
    const std::size_t offp = off32 + (n32 * 4 + 255) / 256 * 256;
    const std::size_t bytes = offp + 4ull * row32 * 4;
    std::vector<unsigned char> host(bytes, 0);
    auto* h16 = reinterpret_cast<std::uint16_t*>(host.data());
    const auto bf = [](float v) {
        std::uint32_t u;
        std::memcpy(&u, &v, 4);
        const std::uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
        return static_cast<std::uint16_t>(r >> 16);
    };
    const int half = H / 2;
    for (int l = 0; l < half; ++l) {
        for (int c = 0; c < F; ++c) {
            h16[2 * (l * F + c)] = bf(weights[kOffW1 + l * F + c]);
            h16[2 * (l * F + c) + 1] = bf(weights[kOffW1 + (l + half) * F + c]);
        }
        for (int i = 0; i < H; ++i) {
            const std::size_t at = H * F + 2 * ((static_cast<std::size_t>(i / 4) * half + l) * 4 + i % 4);
            h16[at] = bf(weights[kOffW2 + l * H + i]);
            h16[at + 1] = bf(weights[kOffW2 + (l + half) * H + i]);
        }
        h16[H * F + H * H + 2 * l] = bf(weights[kOffW3 + l]);
        h16[H * F + H * H + 2 * l + 1] = bf(weights[kOffW3 + l + half]);
    }
    auto* h32 = reinterpret_cast<float*>(host.data() + off32);
    std::memcpy(h32, weights + kOffB1, H * 4);
    std::memcpy(h32 + H, weights + kOffB2, H * 4);
    h32[2 * H] = weights[kOffB3];
    std::memcpy(h32 + 2 * H + 1, mean, F * 4);
    std::memcpy(h32 + 2 * H + 1 + F, inv_std, F * 4);
    auto* hp = reinterpret_cast<float*>(host.data() + offp);
    for (int i = 0; i < 4; ++i) {
        std::memcpy(hp + i * row32, proj + static_cast<std::size_t>(i) * dim, dim * 4);
    }
    gpu::check(cudaMalloc(&net->alloc, bytes), "stop net");
    gpu::check(cudaMemcpy(net->alloc, host.data(), bytes, cudaMemcpyHostToDevice), "upload stop net");
    auto* base = static_cast<unsigned char*>(net->alloc);
    auto* d16 = reinterpret_cast<const std::uint16_t*>(base);
    auto* d32 = reinterpret_cast<const float*>(base + off32);
    net->view.w1 = d16;
    net->view.w2 = d16 + H * F;
    net->view.w3 = d16 + H * F + H * H;
    net->view.b1 = d32;
    net->view.b2 = d32 + H;
    net->view.b3 = d32 + 2 * H;
    net->view.mean = d32 + 2 * H + 1;
    net->view.inv_std = d32 + 2 * H + 1 + F;
    net->view.proj = reinterpret_cast<const float*>(base + offp);
    return net;
}

}  // namespace vdx::dev
