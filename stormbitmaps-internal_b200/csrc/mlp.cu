// mlp.cu -- forward/backward and Adam kernels of the learned cell selector,
// and the host training loop.  Loss: mean softmax cross-entropy of the
// logits against the index of the fastest measured cell.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/storm_rows.h"
#include "mlp.cuh"

namespace sb200 {

// One thread per sample; gradients accumulate in shared memory, then once
// per block into `grads` (mean over the batch).
__global__ void mlp_fwd_bwd_kernel(const float* __restrict__ p, MlpShape sh, const float* __restrict__ x,
                                   const int32_t* __restrict__ y, uint32_t batch, float* __restrict__ logits_out,
                                   float* __restrict__ loss, float* __restrict__ grads) {
    extern __shared__ float sg[];
    const uint32_t np = sh.n_params();
    for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) sg[i] = 0.f;
    __shared__ float sloss;
    if (threadIdx.x == 0) sloss = 0.f;
    __syncthreads();
    const float* W1 = p;
    const float* b1 = W1 + sh.H * sh.F;
    const float* W2 = b1 + sh.H;
    const float* b2 = W2 + sh.C * sh.H;
    float* gW1 = sg;
    float* gb1 = gW1 + sh.H * sh.F;
    float* gW2 = gb1 + sh.H;
    float* gb2 = gW2 + sh.C * sh.H;
    const float inv_b = 1.0f / (float)batch;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < batch; s += gridDim.x * blockDim.x) {
        const float* xs = x + (uint64_t)s * sh.F;
        float pre[MLP_MAX_H], h[MLP_MAX_H], lg[MLP_MAX_C];
        for (uint32_t j = 0; j < sh.H; ++j) {
            float acc = b1[j];
            for (uint32_t f = 0; f < sh.F; ++f) acc += W1[j * sh.F + f] * xs[f];
            pre[j] = acc;
            h[j] = acc > 0.f ? acc : 0.f;
        }
        float mx = -3.0e38f;
        for (uint32_t c = 0; c < sh.C; ++c) {
            float acc = b2[c];
            for (uint32_t j = 0; j < sh.H; ++j) acc += W2[c * sh.H + j] * h[j];
            lg[c] = acc;
            mx = fmaxf(mx, acc);
            if (logits_out) logits_out[(uint64_t)s * sh.C + c] = acc;
        }
        float z = 0.f;
        for (uint32_t c = 0; c < sh.C; ++c) z += expf(lg[c] - mx);
        const int32_t lab = y[s];
        float dl[MLP_MAX_C];
        for (uint32_t c = 0; c < sh.C; ++c) dl[c] = (expf(lg[c] - mx) / z - (c == (uint32_t)lab ? 1.f : 0.f)) * inv_b;
        atomicAdd(&sloss, (logf(z) + mx - lg[lab]) * inv_b);
        float dh[MLP_MAX_H];
        for (uint32_t j = 0; j < sh.H; ++j) dh[j] = 0.f;
        for (uint32_t c = 0; c < sh.C; ++c) {
            atomicAdd(&gb2[c], dl[c]);
            for (uint32_t j = 0; j < sh.H; ++j) {
                atomicAdd(&gW2[c * sh.H + j], dl[c] * h[j]);
                dh[j] += W2[c * sh.H + j] * dl[c];
            }
        }
        for (uint32_t j = 0; j < sh.H; ++j) {
            if (pre[j] <= 0.f) continue;
            atomicAdd(&gb1[j], dh[j]);
            for (uint32_t f = 0; f < sh.F; ++f) atomicAdd(&gW1[j * sh.F + f], dh[j] * xs[f]);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < np; i += blockDim.x)
        if (sg[i] != 0.f) atomicAdd(&grads[i], sg[i]);
    if (threadIdx.x == 0 && loss) atomicAdd(loss, sloss);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, uint32_t np, float lr, float b1, float b2, float eps, float c1,
                            float c2, float wd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i] + wd * p[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void mlp_init(Mlp& m, uint64_t seed) {
    const MlpShape& sh = m.shape;
    m.params.assign(sh.n_params(), 0.f);
    uint64_t s = seed ? seed : 1;
    auto uni = [&](float a) { return a * (2.0f * (float)((splitmix(s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0f); };
    const float a1 = std::sqrt(6.0f / (sh.F + sh.H)), a2 = std::sqrt(6.0f / (sh.H + sh.C));
    for (uint32_t i = 0; i < sh.H * sh.F; ++i) m.params[i] = uni(a1);
    for (uint32_t i = 0; i < sh.C * sh.H; ++i) m.params[sh.H * sh.F + sh.H + i] = uni(a2);
    m.dirty = true;
}

// Full-batch Adam on (X [n x F], Y [n]).  Returns the final loss.
float mlp_train(Mlp& m, const std::vector<float>& X, const std::vector<int32_t>& Y, uint32_t epochs, cudaStream_t st) {
    const MlpShape sh = m.shape;
    const uint32_t np = sh.n_params();
    const uint32_t n = (uint32_t)Y.size();
    if (n == 0) return 0.f;
    DevBuf<float> dx, dg, dm, dv, dloss;
    DevBuf<int32_t> dy;
    dx.reserve(X.size());
    dy.reserve(Y.size());
    dg.reserve(np);
    dm.reserve(np);
    dv.reserve(np);
    dloss.reserve(1);
    m.ensure_device(st);
    SB_CUDA(cudaMemcpyAsync(dx.p, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(dy.p, Y.data(), Y.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemsetAsync(dm.p, 0, np * sizeof(float), st));
    SB_CUDA(cudaMemsetAsync(dv.p, 0, np * sizeof(float), st));
    const uint32_t grid = std::min<uint32_t>((n + 127) / 128, 64);
    const float b1 = 0.9f, b2 = 0.999f;
    float p1 = 1.f, p2 = 1.f, last = 0.f;
    for (uint32_t e = 0; e < epochs; ++e) {
        SB_CUDA(cudaMemsetAsync(dg.p, 0, np * sizeof(float), st));
        SB_CUDA(cudaMemsetAsync(dloss.p, 0, sizeof(float), st));
        mlp_fwd_bwd_kernel<<<grid, 128, np * sizeof(float), st>>>(m.d_params.p, sh, dx.p, dy.p, n, nullptr, dloss.p,
                                                                  dg.p);
        p1 *= b1;
        p2 *= b2;
        adam_kernel<<<(np + 255) / 256, 256, 0, st>>>(m.d_params.p, dg.p, dm.p, dv.p, np, 0.01f, b1, b2, 1e-8f,
                                                      1.f - p1, 1.f - p2, 1e-4f);
    }
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaMemcpyAsync(&last, dloss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    m.params.resize(np);
    SB_CUDA(cudaMemcpyAsync(m.params.data(), m.d_params.p, np * sizeof(float), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    m.dirty = false;
    return last;
}

}  // namespace sb200

using namespace sb200;

extern "C" int STORM_mlp_forward_backward(const float* params, uint32_t F, uint32_t H, uint32_t Cn, const float* x,
                                          const int32_t* labels, uint32_t batch, float* logits, float* loss,
                                          float* grads) {
    if (!params || !x || !labels) return STORM_B200_EVALUES;
    if (F == 0 || H == 0 || Cn == 0 || F > MLP_MAX_F || H > MLP_MAX_H || Cn > MLP_MAX_C) return STORM_B200_ELIMIT;
    return guard([&]() -> int {
        require_device();
        for (uint32_t i = 0; i < batch; ++i)
            if (labels[i] < 0 || (uint32_t)labels[i] >= Cn) return STORM_B200_EARG;
        MlpShape sh;
        sh.F = F;
        sh.H = H;
        sh.C = Cn;
        const uint32_t np = sh.n_params();
        cudaStream_t st;
        SB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DevBuf<float> dp, dx, dl, dloss, dg;
        DevBuf<int32_t> dy;
        dp.reserve(np);
        dx.reserve((size_t)batch * F + 1);
        dl.reserve((size_t)batch * Cn + 1);
        dy.reserve(batch + 1);
        dg.reserve(np);
        dloss.reserve(1);
        SB_CUDA(cudaMemcpyAsync(dp.p, params, np * sizeof(float), cudaMemcpyHostToDevice, st));
        SB_CUDA(cudaMemcpyAsync(dx.p, x, (size_t)batch * F * sizeof(float), cudaMemcpyHostToDevice, st));
        SB_CUDA(cudaMemcpyAsync(dy.p, labels, batch * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        SB_CUDA(cudaMemsetAsync(dg.p, 0, np * sizeof(float), st));
        SB_CUDA(cudaMemsetAsync(dloss.p, 0, sizeof(float), st));
        const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>((batch + 127) / 128, 64));
        mlp_fwd_bwd_kernel<<<grid, 128, np * sizeof(float), st>>>(dp.p, sh, dx.p, dy.p, batch, dl.p, dloss.p, dg.p);
        SB_CUDA(cudaGetLastError());
        if (logits) SB_CUDA(cudaMemcpyAsync(logits, dl.p, (size_t)batch * Cn * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (loss) SB_CUDA(cudaMemcpyAsync(loss, dloss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
        if (grads) SB_CUDA(cudaMemcpyAsync(grads, dg.p, np * sizeof(float), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
        return 0;
    });
}
