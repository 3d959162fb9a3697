// rrb_mlp.cu — the learned cost model: an FP32 MLP 24 -> 64 -> 64 -> 1 (ReLU)
// trained with its own CUDA kernels (forward, backward, Adam). It predicts the
// log render time of a page for a tile shape from host-computed page
// features; it never touches pixels.
//
// Parameter vector layout (RRB_MLP_PARAMS floats):
//   W1[64][24], b1[64], W2[64][64], b2[64], W3[64], b3[1]
// Loss: mean squared error on the log time.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/rrb.h"
#include "rrb_device_scope.h"

namespace {

constexpr int IN = RRB_MLP_IN, H = RRB_MLP_HIDDEN;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * IN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H, NPARAM = OFF_B3 + 1;
static_assert(NPARAM == RRB_MLP_PARAMS, "parameter layout");
constexpr int SAMPLES_PER_CTA = 64;

// One CTA of H threads per chunk of samples; thread j owns hidden unit j.
// With `grad`, the CTA accumulates d(loss)/d(params) in shared memory and
// adds it to grad with one atomic per parameter; loss gets the summed
// squared error. Without it, out[] receives the predictions.
__global__ void __launch_bounds__(H) k_mlp(const float* __restrict__ params, const float* __restrict__ X,
                                           const float* __restrict__ y, int n, float inv_n, float* __restrict__ out,
                                           float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float p[NPARAM];
    __shared__ float g[NPARAM];
    __shared__ float x[IN], h1[H], h2[H], dh2[H], red[2];
    const int j = threadIdx.x;
    for (int k = j; k < NPARAM; k += H) {
        p[k] = params[k];
        g[k] = 0.f;
    }
    __syncthreads();
    float lsum = 0.f;
    const int s0 = blockIdx.x * SAMPLES_PER_CTA, s1 = min(n, s0 + SAMPLES_PER_CTA);
    for (int s = s0; s < s1; ++s) {
        if (j < IN) x[j] = X[static_cast<size_t>(s) * IN + j];
        __syncthreads();
        float a = p[OFF_B1 + j];
        for (int k = 0; k < IN; ++k) a = fmaf(p[OFF_W1 + j * IN + k], x[k], a);
        const float z1 = a;
        h1[j] = fmaxf(z1, 0.f);
        __syncthreads();
        a = p[OFF_B2 + j];
        for (int k = 0; k < H; ++k) a = fmaf(p[OFF_W2 + j * H + k], h1[k], a);
        const float z2 = a;
        h2[j] = fmaxf(z2, 0.f);
        // output: sum over the two warps
        float o = p[OFF_W3 + j] * h2[j];
        for (int d = 16; d; d >>= 1) o += __shfl_xor_sync(0xffffffffu, o, d);
        if ((j & 31) == 0) red[j >> 5] = o;
        __syncthreads();
        const float yhat = red[0] + red[1] + p[OFF_B3];
        if (!grad) {
            if (j == 0) out[s] = yhat;
            __syncthreads();
            continue;
        }
        const float err = yhat - y[s];
        if (j == 0) lsum += err * err;
        const float dout = 2.f * err * inv_n;
        g[OFF_W3 + j] += dout * h2[j];
        if (j == 0) g[OFF_B3] += dout;
        const float d2 = z2 > 0.f ? dout * p[OFF_W3 + j] : 0.f;
        dh2[j] = d2;
        g[OFF_B2 + j] += d2;
        for (int k = 0; k < H; ++k) g[OFF_W2 + j * H + k] += d2 * h1[k];
        __syncthreads();
        // thread j now owns hidden unit j of layer 1
        float d1 = 0.f;
        for (int i = 0; i < H; ++i) d1 = fmaf(dh2[i], p[OFF_W2 + i * H + j], d1);
        d1 = z1 > 0.f ? d1 : 0.f;
        g[OFF_B1 + j] += d1;
        for (int k = 0; k < IN; ++k) g[OFF_W1 + j * IN + k] += d1 * x[k];
        __syncthreads();
    }
    if (!grad) return;
    __syncthreads();
    for (int k = j; k < NPARAM; k += H)
        if (g[k] != 0.f) atomicAdd(&grad[k], g[k]);
    if (j == 0 && lsum != 0.f) atomicAdd(loss, lsum);
}

// Adam (Kingma & Ba 2015) with bias correction; clears the gradient.
__global__ void k_adam(float* __restrict__ params, float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float gk = grad[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        params[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
        grad[k] = 0.f;
    }
}

}  // namespace

struct rrb_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float* d_params = nullptr;
    float* d_grad = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_loss = nullptr;
    float* d_x = nullptr;
    float* d_y = nullptr;
    float* d_out = nullptr;
    size_t cap = 0;
    int step = 0;
};

namespace {

int ensure_io(rrb_mlp* m, size_t n) {
    if (n <= m->cap) return RRB_OK;
    cudaFree(m->d_x);
    cudaFree(m->d_y);
    cudaFree(m->d_out);
    m->d_x = m->d_y = m->d_out = nullptr;
    m->cap = 0;
    if (cudaMalloc(&m->d_x, n * IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&m->d_y, n * sizeof(float)) != cudaSuccess || cudaMalloc(&m->d_out, n * sizeof(float)) != cudaSuccess)
        return RRB_ERR_OUT_OF_MEMORY;
    m->cap = n;
    return RRB_OK;
}

// He-normal initialisation from a SplitMix64 stream (Box-Muller).
void init_params(std::vector<float>& w, uint64_t seed) {
    uint64_t st = seed;
    auto next = [&] {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto u01 = [&] { return (static_cast<double>(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
    auto normal = [&] { return std::sqrt(-2.0 * std::log(u01())) * std::cos(6.283185307179586 * u01()); };
    w.assign(NPARAM, 0.f);
    for (int k = 0; k < H * IN; ++k) w[OFF_W1 + k] = static_cast<float>(normal() * std::sqrt(2.0 / IN));
    for (int k = 0; k < H * H; ++k) w[OFF_W2 + k] = static_cast<float>(normal() * std::sqrt(2.0 / H));
    for (int k = 0; k < H; ++k) w[OFF_W3 + k] = static_cast<float>(normal() * std::sqrt(1.0 / H));
}

}  // namespace

extern "C" {

int rrb_mlp_create(int device, uint64_t seed, rrb_mlp** out) {
    if (!out) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(device);
    if (dev_scope.status() != cudaSuccess) return RRB_ERR_DEVICE;
    rrb_mlp* m = new rrb_mlp();
    m->device = device;
    bool ok = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&m->d_params, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&m->d_grad, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&m->d_m, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&m->d_v, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&m->d_loss, sizeof(float)) == cudaSuccess;
    if (!ok) {
        rrb_mlp_destroy(m);
        return RRB_ERR_DEVICE;
    }
    std::vector<float> w;
    init_params(w, seed);
    int rc = rrb_mlp_set_params(m, w.data());
    if (rc) {
        rrb_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return RRB_OK;
}

int rrb_mlp_destroy(rrb_mlp* m) {
    if (!m) return RRB_OK;
    const rrb_host::DeviceScope dev_scope(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    float* bufs[] = {m->d_params, m->d_grad, m->d_m, m->d_v, m->d_loss, m->d_x, m->d_y, m->d_out};
    for (float* b : bufs) cudaFree(b);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return RRB_OK;
}

int rrb_mlp_set_params(rrb_mlp* m, const float* params) {
    if (!m || !params) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(m->device);
    if (cudaMemcpyAsync(m->d_params, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_grad, 0, NPARAM * sizeof(float), m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_m, 0, NPARAM * sizeof(float), m->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_v, 0, NPARAM * sizeof(float), m->stream) != cudaSuccess)
        return RRB_ERR_DEVICE;
    m->step = 0;
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? RRB_OK : RRB_ERR_DEVICE;
}

int rrb_mlp_get_params(rrb_mlp* m, float* params) {
    if (!m || !params) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(m->device);
    if (cudaMemcpyAsync(params, m->d_params, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess)
        return RRB_ERR_DEVICE;
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? RRB_OK : RRB_ERR_DEVICE;
}

int rrb_mlp_loss_grad(rrb_mlp* m, const float* X, const float* y, uint32_t n, float* grad_out, float* loss_out) {
    if (!m || !X || !y || !n) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(m->device);
    int rc = ensure_io(m, n);
    if (rc) return rc;
    cudaMemcpyAsync(m->d_x, X, static_cast<size_t>(n) * IN * sizeof(float), cudaMemcpyHostToDevice, m->stream);
    cudaMemcpyAsync(m->d_y, y, n * sizeof(float), cudaMemcpyHostToDevice, m->stream);
    cudaMemsetAsync(m->d_grad, 0, NPARAM * sizeof(float), m->stream);
    cudaMemsetAsync(m->d_loss, 0, sizeof(float), m->stream);
    k_mlp<<<(n + SAMPLES_PER_CTA - 1) / SAMPLES_PER_CTA, H, 0, m->stream>>>(m->d_params, m->d_x, m->d_y, static_cast<int>(n),
                                                                          1.f / n, nullptr, m->d_grad, m->d_loss);
    if (grad_out) cudaMemcpyAsync(grad_out, m->d_grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    float l = 0.f;
    cudaMemcpyAsync(&l, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    cudaMemsetAsync(m->d_grad, 0, NPARAM * sizeof(float), m->stream);
    if (cudaStreamSynchronize(m->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) return RRB_ERR_DEVICE;
    if (loss_out) *loss_out = l / n;
    return RRB_OK;
}

int rrb_mlp_train(rrb_mlp* m, const float* X, const float* y, uint32_t n, uint32_t epochs, uint32_t batch,
                  float lr, uint64_t seed, float* final_loss) {
    if (!m || !X || !y || !n || !epochs) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(m->device);
    int rc = ensure_io(m, n);
    if (rc) return rc;
    if (!batch || batch > n) batch = n;
    // Shuffle once per epoch on the host (SplitMix64 Fisher-Yates) and upload.
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    std::vector<float> xs(static_cast<size_t>(n) * IN), ys(n);
    uint64_t st = seed;
    auto next = [&] {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    float last = 0.f;
    for (uint32_t e = 0; e < epochs; ++e) {
        for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[next() % (i + 1)]);
        for (uint32_t i = 0; i < n; ++i) {
            std::memcpy(&xs[static_cast<size_t>(i) * IN], &X[static_cast<size_t>(perm[i]) * IN], IN * sizeof(float));
            ys[i] = y[perm[i]];
        }
        cudaMemcpyAsync(m->d_x, xs.data(), xs.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream);
        cudaMemcpyAsync(m->d_y, ys.data(), n * sizeof(float), cudaMemcpyHostToDevice, m->stream);
        cudaMemsetAsync(m->d_loss, 0, sizeof(float), m->stream);
        for (uint32_t b0 = 0; b0 < n; b0 += batch) {
            const uint32_t nb = std::min(batch, n - b0);
            k_mlp<<<(nb + SAMPLES_PER_CTA - 1) / SAMPLES_PER_CTA, H, 0, m->stream>>>(
                m->d_params, m->d_x + static_cast<size_t>(b0) * IN, m->d_y + b0, static_cast<int>(nb), 1.f / nb,
                nullptr, m->d_grad, m->d_loss);
            m->step += 1;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, static_cast<float>(m->step));
            const float c2 = 1.f - std::pow(b2, static_cast<float>(m->step));
            k_adam<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->d_params, m->d_grad, m->d_m, m->d_v, NPARAM, lr, b1,
                                                               b2, 1e-8f, c1, c2);
        }
        cudaMemcpyAsync(&last, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
        if (cudaStreamSynchronize(m->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) return RRB_ERR_DEVICE;
    }
    if (final_loss) *final_loss = last / n;
    return RRB_OK;
}

int rrb_mlp_predict(rrb_mlp* m, const float* X, uint32_t n, float* out) {
    if (!m || !X || !out || !n) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(m->device);
    int rc = ensure_io(m, n);
    if (rc) return rc;
    cudaMemcpyAsync(m->d_x, X, static_cast<size_t>(n) * IN * sizeof(float), cudaMemcpyHostToDevice, m->stream);
    k_mlp<<<(n + SAMPLES_PER_CTA - 1) / SAMPLES_PER_CTA, H, 0, m->stream>>>(m->d_params, m->d_x, nullptr, static_cast<int>(n),
                                                                          1.f, m->d_out, nullptr, nullptr);
    cudaMemcpyAsync(out, m->d_out, n * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (cudaStreamSynchronize(m->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) return RRB_ERR_DEVICE;
    return RRB_OK;
}

// The same forward pass on the host, operation for operation (fmaf chains in
// the kernel's order, the output summed as the kernel's two-warp butterfly),
// so its predictions equal rrb_mlp_predict's bit for bit. For callers that
// must not wait on the device (a scheduler deciding while kernels run).
int rrb_mlp_predict_host(const float* params, const float* X, uint32_t n, float* out) {
    if (!params || (!X && n) || (!out && n)) return RRB_ERR_INVARIANT;
    float h1[H], h2[H], o[H];
    for (uint32_t s = 0; s < n; ++s) {
        const float* x = X + static_cast<size_t>(s) * IN;
        for (int j = 0; j < H; ++j) {
            float a = params[OFF_B1 + j];
            for (int k = 0; k < IN; ++k) a = std::fmaf(params[OFF_W1 + j * IN + k], x[k], a);
            h1[j] = std::fmax(a, 0.f);
        }
        for (int j = 0; j < H; ++j) {
            float a = params[OFF_B2 + j];
            for (int k = 0; k < H; ++k) a = std::fmaf(params[OFF_W2 + j * H + k], h1[k], a);
            h2[j] = std::fmax(a, 0.f);
            o[j] = params[OFF_W3 + j] * h2[j];
        }
        // __shfl_xor_sync butterfly within each warp of 32 lanes.
        for (int w = 0; w < H / 32; ++w) {
            float* v = o + 32 * w;
            for (int d = 16; d; d >>= 1) {
                float t[32];
                for (int l = 0; l < 32; ++l) t[l] = v[l] + v[l ^ d];
                for (int l = 0; l < 32; ++l) v[l] = t[l];
            }
        }
        out[s] = (o[0] + o[32]) + params[OFF_B3];
    }
    return RRB_OK;
}

}  // extern "C"
