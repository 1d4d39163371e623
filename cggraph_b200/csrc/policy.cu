// Learned per-iteration scheduler: inference and training kernels.
//
// The network is tiny (6,345 FP32 parameters), so every kernel here is
// plain CUDA-core code: one 64-thread CTA per sample for the forward and the
// activation backward pass, one thread per parameter for the gradient
// (summing over the batch in a fixed order, so training is deterministic for
// a given seed), one thread per parameter for Adam.
#include <cmath>
#include <mutex>
#include <random>
#include <vector>

#include "../../include/cgb200.h"
#include "policy.cuh"

namespace cgb {

constexpr int kF = kPolicyFeatures, kH = kPolicyHidden, kO = kPolicyOutputs;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kF * kH, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH * kO;
static_assert(kOffB3 + kO == kPolicyParams, "layout");

// ------------------------------------------------------------ registry
struct Policy {
    float* params = nullptr;  // device copy
};

static std::mutex g_pol_mu;
static Policy g_pol[64];

Policy* policy_get()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_pol_mu);
    return g_pol[dev].params ? &g_pol[dev] : nullptr;
}

const float* policy_params_device(Policy* p) { return p ? p->params : nullptr; }

Policy* policy_for(const cgb_graph* g)
{
    return g->E >= kPolicyMinEdges ? policy_get() : nullptr;
}

// ------------------------------------------------------------ kernels
// One sample through the network with the CTA's 64 threads.  f: 24 features
// in shared memory; h1, h2: 64 floats each in shared memory.
__device__ __forceinline__ void mlp_forward_cta(const float* __restrict__ P, const float* f, float* h1, float* h2,
                                                float* out)
{
    const int j = threadIdx.x;
    float a = P[kOffB1 + j];
#pragma unroll 8
    for (int i = 0; i < kF; i++) a += f[i] * P[kOffW1 + i * kH + j];
    h1[j] = a > 0.f ? a : 0.f;
    __syncthreads();
    float b = P[kOffB2 + j];
#pragma unroll 8
    for (int i = 0; i < kH; i++) b += h1[i] * P[kOffW2 + i * kH + j];
    h2[j] = b > 0.f ? b : 0.f;
    __syncthreads();
    if (j < kO) {
        float c = P[kOffB3 + j];
#pragma unroll 8
        for (int i = 0; i < kH; i++) c += h2[i] * P[kOffW3 + i * kO + j];
        out[j] = c;
    }
}

// Inference fused into the engine's iteration: patches the counters of the
// level just run into the raw quantities, builds the features, runs the
// network and leaves the outputs in the counters.
__global__ void __launch_bounds__(kH) k_policy_step(const float* __restrict__ P, FeatIn in, DevCounters* ctr,
                                                    int patch, int was_pull, int out_q)
{
    __shared__ float f[kF], h1[kH], h2[kH];
    if (threadIdx.x == 0) {
        if (patch == 2) {
            // SSSP near round just queued: the next near queue and the far set
            in.prev_nf = in.nf;
            in.nf = ctr->qlen[out_q];
            in.mf = (double)ctr->medges;
            in.max_deg = ctr->max_deg;
            in.far_count = ctr->far_len[0];
            in.iteration += 1;
        }
        if (patch == 1) {
            const double n_next = ctr->qlen[out_q];
            in.prev_nf = in.nf;
            in.nf = n_next;
            in.mf = (double)ctr->medges;
            in.max_deg = ctr->max_deg;
            in.unvisited_v -= was_pull ? (double)ctr->found : n_next;
            if (in.unvisited_v < 0) in.unvisited_v = 0;
            in.prev_dir = was_pull;
            in.iteration += 1;
        }
        policy_features(in, f);
    }
    __syncthreads();
    mlp_forward_cta(P, f, h1, h2, ctr->policy_out);
}

// Batched forward: keeps the activations for the backward pass.
__global__ void __launch_bounds__(kH) k_mlp_fwd(const float* __restrict__ P, const float* __restrict__ X, uint32_t n,
                                                float* H1, float* H2, float* Y)
{
    __shared__ float f[kF], h1[kH], h2[kH], y[kO];
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        if (threadIdx.x < kF) f[threadIdx.x] = X[(size_t)s * kF + threadIdx.x];
        __syncthreads();
        mlp_forward_cta(P, f, h1, h2, y);
        __syncthreads();
        if (H1) H1[(size_t)s * kH + threadIdx.x] = h1[threadIdx.x];
        if (H2) H2[(size_t)s * kH + threadIdx.x] = h2[threadIdx.x];
        if (threadIdx.x < kO) Y[(size_t)s * kO + threadIdx.x] = y[threadIdx.x];
        __syncthreads();
    }
}

// dY = 2 * mask * (Y - T) / count; per-sample squared error into err[s].
__global__ void k_mlp_loss(const float* __restrict__ Y, const float* __restrict__ T, const uint8_t* __restrict__ M,
                           uint32_t n, float inv_count, float* dY, float* err)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float e = 0.f;
        for (int k = 0; k < kO; k++) {
            const size_t i = (size_t)s * kO + k;
            const float d = M[i] ? Y[i] - T[i] : 0.f;
            dY[i] = 2.f * d * inv_count;
            e += d * d;
        }
        err[s] = e;
    }
}

// Activation gradients of one sample per CTA.
__global__ void __launch_bounds__(kH) k_mlp_bwd_act(const float* __restrict__ P, const float* __restrict__ H1,
                                                    const float* __restrict__ H2, const float* __restrict__ dY,
                                                    uint32_t n, float* dH1, float* dH2)
{
    __shared__ float dy[kO], dh2[kH];
    const int j = threadIdx.x;
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        if (j < kO) dy[j] = dY[(size_t)s * kO + j];
        __syncthreads();
        float a = 0.f;
        for (int k = 0; k < kO; k++) a += dy[k] * P[kOffW3 + j * kO + k];
        a = H2[(size_t)s * kH + j] > 0.f ? a : 0.f;
        dh2[j] = a;
        dH2[(size_t)s * kH + j] = a;
        __syncthreads();
        float b = 0.f;
        for (int k = 0; k < kH; k++) b += dh2[k] * P[kOffW2 + j * kH + k];
        dH1[(size_t)s * kH + j] = H1[(size_t)s * kH + j] > 0.f ? b : 0.f;
        __syncthreads();
    }
}

// Parameter gradients, one thread per parameter, summed over the batch in
// sample order.
__global__ void k_mlp_param_grad(const float* __restrict__ X, const float* __restrict__ H1,
                                 const float* __restrict__ H2, const float* __restrict__ dH1,
                                 const float* __restrict__ dH2, const float* __restrict__ dY, uint32_t n, float* G)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kPolicyParams) return;
    float g = 0.f;
    if (p < kOffB1) {
        const int i = p / kH, j = p % kH;
        for (uint32_t s = 0; s < n; s++) g += X[(size_t)s * kF + i] * dH1[(size_t)s * kH + j];
    } else if (p < kOffW2) {
        const int j = p - kOffB1;
        for (uint32_t s = 0; s < n; s++) g += dH1[(size_t)s * kH + j];
    } else if (p < kOffB2) {
        const int i = (p - kOffW2) / kH, j = (p - kOffW2) % kH;
        for (uint32_t s = 0; s < n; s++) g += H1[(size_t)s * kH + i] * dH2[(size_t)s * kH + j];
    } else if (p < kOffW3) {
        const int j = p - kOffB2;
        for (uint32_t s = 0; s < n; s++) g += dH2[(size_t)s * kH + j];
    } else if (p < kOffB3) {
        const int i = (p - kOffW3) / kO, k = (p - kOffW3) % kO;
        for (uint32_t s = 0; s < n; s++) g += H2[(size_t)s * kH + i] * dY[(size_t)s * kO + k];
    } else {
        const int k = p - kOffB3;
        for (uint32_t s = 0; s < n; s++) g += dY[(size_t)s * kO + k];
    }
    G[p] = g;
}

// Adam (Kingma and Ba 2015) with bias correction folded into the step size.
__global__ void k_adam(float* P, const float* __restrict__ G, float* m, float* v, float lr_t, float b1, float b2,
                       float eps)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kPolicyParams) return;
    const float g = G[p];
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    P[p] -= lr_t * mm / (sqrtf(vv) + eps);
}

// ------------------------------------------------------------ host side
void policy_enqueue(Policy* p, cgb_graph* g, const FeatIn& in, int patch, bool was_pull, int out_q)
{
    ++g->stats.launches;
    k_policy_step<<<1, kH, 0, g->stream>>>(p->params, in, g->ctr, patch, was_pull ? 1 : 0, out_q);
}

void policy_log_sample(cgb_graph* g, const FeatIn& in, const float* ms, const bool* have)
{
    PolicySamples* c = g->collect;
    if (!c || c->count >= c->max) return;
    const size_t i = c->count++;
    policy_features(in, c->features + i * kF);
    for (int k = 0; k < kO; k++) {
        c->mask[i * kO + k] = have[k] ? 1 : 0;
        c->targets[i * kO + k] = have[k] ? std::log(std::max(ms[k], 1e-4f)) : 0.f;
    }
}

// A choice is taken only when the network predicts a clear gain (5 % in
// cost); otherwise the heuristic decides.
// An override needs a predicted gain of 20 % (log-cost 0.2): most choices
// the traces time are near-ties (the two sparse expansions of a round, the
// delta on RMAT), where the network's error (RMS about 5 % on its training
// samples) would pick at random; with a 10 % margin it lost 3-12 % on
// held-out RMAT runs.
constexpr float kMargin = 0.20f;

// The cheapest of n choices (outputs out[idx[i]]), or -1 when it does not
// beat the heuristic's choice `heur` by the margin.
static int pick_among(const float* out, const int* idx, int n, int heur)
{
    int best = -1;
    float bv = 0.f;
    for (int i = 0; i < n; i++) {
        const float v = out[idx[i]];
        if (!std::isfinite(v)) return -1;
        if (best < 0 || v < bv) {
            best = i;
            bv = v;
        }
    }
    if (best == heur || out[idx[heur]] - bv < kMargin) return -1;
    return best;
}

int policy_pick_bfs_level(const float* out, int heur)
{
    const int idx[3] = {kOutPush, kOutPull, kOutPushChunked};
    return pick_among(out, idx, 3, heur);
}

// The network may move a round between the two sparse-frontier expansions,
// or keep the heuristic's dense or pull round; it never starts a dense or
// pull round itself.  Those are rarely the cheapest in the traces (a pull
// round on RMAT-24 costs 3-6 ms against 0.05-4 ms pushed), and on graphs
// beyond the training range the network chose them where they cost 5x.
int policy_pick_round(const float* out, int heur)
{
    const int idx[kNumRoundChoices] = {kOutRound0, kOutRound0 + 1, kOutRound0 + 2, kOutRound0 + 3};
    if (heur != kRoundPush && heur != kRoundPushChunked) {
        const int pair[2] = {heur, kRoundPush};
        const int k[2] = {idx[heur], idx[kRoundPush]};
        const int c = pick_among(out, k, 2, 0);
        return c < 0 ? -1 : pair[c];
    }
    return pick_among(out, idx, 2, heur);
}

int policy_pick_delta(const float* out)
{
    int best = -1;
    float bv = 0.f;
    for (int i = 0; i < kNumDeltaChoices; i++) {
        const float v = out[kOutDelta0 + i];
        if (!std::isfinite(v)) return -1;
        if (best < 0 || v < bv) {
            best = i;
            bv = v;
        }
    }
    // keep the heuristic delta unless another choice is clearly cheaper
    if (best != kDeltaUnit && out[kOutDelta0 + kDeltaUnit] - bv < kMargin) return -1;
    return best;
}

// Scratch of one training / evaluation call.
struct TrainBufs {
    float *P = nullptr, *X = nullptr, *T = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr, *dY = nullptr,
          *dH1 = nullptr, *dH2 = nullptr, *G = nullptr, *m = nullptr, *v = nullptr, *err = nullptr;
    uint8_t* M = nullptr;
    ~TrainBufs()
    {
        float* fs[] = {P, X, T, H1, H2, Y, dY, dH1, dH2, G, m, v, err};
        for (float* f : fs)
            if (f) cudaFree(f);
        if (M) cudaFree(M);
    }
};

template <typename T>
static void balloc(T*& p, size_t n)
{
    CGB_CUDA_TRY(cudaMalloc((void**)&p, (n ? n : 1) * sizeof(T)));
}

static void alloc_batch(TrainBufs& b, uint32_t n)
{
    balloc(b.X, (size_t)n * kF);
    balloc(b.T, (size_t)n * kO);
    balloc(b.M, (size_t)n * kO);
    balloc(b.H1, (size_t)n * kH);
    balloc(b.H2, (size_t)n * kH);
    balloc(b.Y, (size_t)n * kO);
    balloc(b.dY, (size_t)n * kO);
    balloc(b.dH1, (size_t)n * kH);
    balloc(b.dH2, (size_t)n * kH);
    balloc(b.err, n);
    balloc(b.G, kPolicyParams);
}

// loss and gradient of P on the n samples already in b.X/b.T/b.M
static float loss_grad_device(TrainBufs& b, uint32_t n, float inv_count, cudaStream_t st)
{
    const uint32_t grid = std::min<uint32_t>(n ? n : 1, 4096);
    k_mlp_fwd<<<grid, kH, 0, st>>>(b.P, b.X, n, b.H1, b.H2, b.Y);
    k_mlp_loss<<<div_up(n ? n : 1, 256), 256, 0, st>>>(b.Y, b.T, b.M, n, inv_count, b.dY, b.err);
    k_mlp_bwd_act<<<grid, kH, 0, st>>>(b.P, b.H1, b.H2, b.dY, n, b.dH1, b.dH2);
    k_mlp_param_grad<<<div_up(kPolicyParams, 128), 128, 0, st>>>(b.X, b.H1, b.H2, b.dH1, b.dH2, b.dY, n, b.G);
    CGB_CUDA_TRY(cudaGetLastError());
    std::vector<float> err(n);
    if (n) CGB_CUDA_TRY(cudaMemcpyAsync(err.data(), b.err, n * 4ull, cudaMemcpyDeviceToHost, st));
    CGB_CUDA_TRY(cudaStreamSynchronize(st));
    double e = 0;
    for (float x : err) e += x;
    return (float)(e * inv_count);
}

static void init_params(std::vector<float>& P, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int fan_out) {
        const float a = std::sqrt(6.f / (float)(fan_in + fan_out));  // Glorot uniform
        std::uniform_real_distribution<float> d(-a, a);
        for (int i = 0; i < fan_in * fan_out; i++) P[off + i] = d(rng);
    };
    P.assign(kPolicyParams, 0.f);
    fill(kOffW1, kF, kH);
    fill(kOffW2, kH, kH);
    fill(kOffW3, kH, kO);
}

}  // namespace cgb

using namespace cgb;

template <typename F>
static cgb_status pol_guard(F&& f)
{
    try {
        f();
        return CGB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CGB_ECUDA;
    }
}

extern "C" cgb_status cgb_policy_load(const float* params)
{
    return pol_guard([&] {
        int dev = 0;
        CGB_CUDA_TRY(cudaGetDevice(&dev));
        CGB_REQUIRE(dev >= 0 && dev < 64, CGB_EUNSUPPORTED, "device ordinal out of range");
        std::lock_guard<std::mutex> lock(g_pol_mu);
        Policy& p = g_pol[dev];
        if (!params) {
            if (p.params) cudaFree(p.params);
            p.params = nullptr;
            return;
        }
        for (int i = 0; i < kPolicyParams; i++)
            CGB_REQUIRE(std::isfinite(params[i]), CGB_EINVAL, "policy parameters must be finite");
        if (!p.params) CGB_CUDA_TRY(cudaMalloc((void**)&p.params, kPolicyParams * sizeof(float)));
        CGB_CUDA_TRY(cudaMemcpy(p.params, params, kPolicyParams * sizeof(float), cudaMemcpyHostToDevice));
    });
}

extern "C" cgb_status cgb_policy_forward(const float* params, const float* features, uint32_t n, float* outputs)
{
    return pol_guard([&] {
        CGB_REQUIRE(params && features && outputs, CGB_EINVAL, "NULL argument");
        TrainBufs b;
        balloc(b.P, kPolicyParams);
        balloc(b.X, (size_t)n * kF);
        balloc(b.Y, (size_t)n * kO);
        CGB_CUDA_TRY(cudaMemcpy(b.P, params, kPolicyParams * 4ull, cudaMemcpyHostToDevice));
        if (n) CGB_CUDA_TRY(cudaMemcpy(b.X, features, (size_t)n * kF * 4, cudaMemcpyHostToDevice));
        if (n) k_mlp_fwd<<<std::min<uint32_t>(n, 4096), kH>>>(b.P, b.X, n, nullptr, nullptr, b.Y);
        CGB_CUDA_TRY(cudaGetLastError());
        if (n) CGB_CUDA_TRY(cudaMemcpy(outputs, b.Y, (size_t)n * kO * 4, cudaMemcpyDeviceToHost));
    });
}

extern "C" cgb_status cgb_policy_loss_grad(const float* params, const float* features, const float* targets,
                                           const uint8_t* mask, uint32_t n, float* loss, float* grad)
{
    return pol_guard([&] {
        CGB_REQUIRE(params && features && targets && mask && loss && grad, CGB_EINVAL, "NULL argument");
        uint64_t count = 0;
        for (size_t i = 0; i < (size_t)n * kO; i++) count += mask[i] ? 1 : 0;
        CGB_REQUIRE(count > 0, CGB_EINVAL, "mask selects no target");
        TrainBufs b;
        alloc_batch(b, n);
        balloc(b.P, kPolicyParams);
        CGB_CUDA_TRY(cudaMemcpy(b.P, params, kPolicyParams * 4ull, cudaMemcpyHostToDevice));
        CGB_CUDA_TRY(cudaMemcpy(b.X, features, (size_t)n * kF * 4, cudaMemcpyHostToDevice));
        CGB_CUDA_TRY(cudaMemcpy(b.T, targets, (size_t)n * kO * 4, cudaMemcpyHostToDevice));
        CGB_CUDA_TRY(cudaMemcpy(b.M, mask, (size_t)n * kO, cudaMemcpyHostToDevice));
        *loss = loss_grad_device(b, n, 1.f / (float)count, 0);
        CGB_CUDA_TRY(cudaMemcpy(grad, b.G, kPolicyParams * 4ull, cudaMemcpyDeviceToHost));
    });
}

extern "C" cgb_status cgb_policy_train(const float* features, const float* targets, const uint8_t* mask, uint32_t n,
                                       uint32_t epochs, uint32_t batch, float lr, uint64_t seed, const float* init,
                                       float* params_out, float* final_loss)
{
    return pol_guard([&] {
        CGB_REQUIRE(features && targets && mask && params_out && n > 0, CGB_EINVAL, "bad training arguments");
        if (batch == 0 || batch > n) batch = n;
        if (lr <= 0) lr = 1e-3f;
        std::vector<float> P;
        if (init) P.assign(init, init + kPolicyParams);
        else init_params(P, seed);
        TrainBufs b;
        alloc_batch(b, batch);
        balloc(b.P, kPolicyParams);
        balloc(b.m, kPolicyParams);
        balloc(b.v, kPolicyParams);
        CGB_CUDA_TRY(cudaMemcpy(b.P, P.data(), kPolicyParams * 4ull, cudaMemcpyHostToDevice));
        CGB_CUDA_TRY(cudaMemset(b.m, 0, kPolicyParams * 4ull));
        CGB_CUDA_TRY(cudaMemset(b.v, 0, kPolicyParams * 4ull));
        std::vector<uint32_t> order(n);
        for (uint32_t i = 0; i < n; i++) order[i] = i;
        std::mt19937_64 rng(seed ^ 0x5EEDull);
        std::vector<float> bx((size_t)batch * kF), bt((size_t)batch * kO);
        std::vector<uint8_t> bm((size_t)batch * kO);
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        uint64_t t = 0;
        double epoch_loss = 0;
        for (uint32_t ep = 0; ep < epochs; ep++) {
            std::shuffle(order.begin(), order.end(), rng);
            epoch_loss = 0;
            uint64_t epoch_count = 0;
            for (uint32_t s0 = 0; s0 < n; s0 += batch) {
                const uint32_t nb = std::min(batch, n - s0);
                uint64_t count = 0;
                for (uint32_t i = 0; i < nb; i++) {
                    const uint32_t s = order[s0 + i];
                    std::copy(features + (size_t)s * kF, features + (size_t)(s + 1) * kF, bx.begin() + (size_t)i * kF);
                    std::copy(targets + (size_t)s * kO, targets + (size_t)(s + 1) * kO, bt.begin() + (size_t)i * kO);
                    std::copy(mask + (size_t)s * kO, mask + (size_t)(s + 1) * kO, bm.begin() + (size_t)i * kO);
                    for (int k = 0; k < kO; k++) count += mask[(size_t)s * kO + k] ? 1 : 0;
                }
                if (!count) continue;
                CGB_CUDA_TRY(cudaMemcpy(b.X, bx.data(), (size_t)nb * kF * 4, cudaMemcpyHostToDevice));
                CGB_CUDA_TRY(cudaMemcpy(b.T, bt.data(), (size_t)nb * kO * 4, cudaMemcpyHostToDevice));
                CGB_CUDA_TRY(cudaMemcpy(b.M, bm.data(), (size_t)nb * kO, cudaMemcpyHostToDevice));
                const float l = loss_grad_device(b, nb, 1.f / (float)count, 0);
                epoch_loss += (double)l * (double)count;
                epoch_count += count;
                t++;
                const float lr_t = lr * std::sqrt(1.f - std::pow(b2, (float)t)) / (1.f - std::pow(b1, (float)t));
                k_adam<<<div_up(kPolicyParams, 256), 256>>>(b.P, b.G, b.m, b.v, lr_t, b1, b2, eps);
                CGB_CUDA_TRY(cudaGetLastError());
            }
            if (epoch_count) epoch_loss /= (double)epoch_count;
        }
        CGB_CUDA_TRY(cudaMemcpy(params_out, b.P, kPolicyParams * 4ull, cudaMemcpyDeviceToHost));
        if (final_loss) *final_loss = (float)epoch_loss;
    });
}
