// model.cu -- forward, backward and Adam kernels of the cost-model MLP.
// Inputs are the per-query features of k_features (batch.cu) scaled by 1/8;
// the two outputs times 8 are log-rates r of the per-query counts (candidates
// to verify, result pairs), trained with the Poisson loss exp(r) - y r, whose
// optimum matches the summed counts of the training joins (the output bias's
// gradient is sum(exp(r) - y)).  Plain FP32 SIMT: the network is 354
// parameters, far too small for tensor cores to matter.
#include <math.h>
#include <string.h>

#include <random>

#include "model.h"
#include "prims.cuh"

namespace fgss {

namespace {

constexpr float kInScale = 0.125f;
constexpr float kOutScale = 8.0f;
constexpr float kRateClamp = 30.0f;  // log-rates are clamped to [-30, 30] (zero gradient outside)

__device__ __forceinline__ void mlp_fwd(const float* P, const float* x, float* hpre, float* o) {
    const float* W1 = P;
    const float* b1 = W1 + kHidden * kFeatM;
    const float* W2 = b1 + kHidden;
    const float* b2 = W2 + kOut * kHidden;
#pragma unroll
    for (int k = 0; k < kHidden; k++) {
        float s = b1[k];
#pragma unroll
        for (int f = 0; f < kFeatM; f++) s = fmaf(W1[k * kFeatM + f], x[f], s);
        hpre[k] = s;
    }
#pragma unroll
    for (int j = 0; j < kOut; j++) {
        float s = b2[j];
#pragma unroll
        for (int k = 0; k < kHidden; k++) s = fmaf(W2[j * kHidden + k], fmaxf(hpre[k], 0.f), s);
        o[j] = s;
    }
}

__global__ void __launch_bounds__(256) k_mlp_grad(const float* __restrict__ feat, const float* __restrict__ target,
                                                  uint64_t n, const float* __restrict__ Pg, float* __restrict__ G,
                                                  float* __restrict__ loss) {
    __shared__ float P[kParams];
    __shared__ float acc[kParams + 1];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        P[i] = Pg[i];
        acc[i] = 0.f;
    }
    if (threadIdx.x == 0) acc[kParams] = 0.f;
    __syncthreads();
    const uint32_t lane = lane_id();
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const float inv_n = n ? 1.0f / (float)n : 0.f;
    for (uint64_t base = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += warps * 32) {
        uint64_t i = base + lane;
        bool valid = i < n;
        float x[kFeatM], hpre[kHidden], o[kOut], dO[kOut];
#pragma unroll
        for (int f = 0; f < kFeatM; f++) x[f] = valid ? feat[i * kFeatM + f] * kInScale : 0.f;
        mlp_fwd(P, x, hpre, o);
        float l = 0.f;
#pragma unroll
        for (int j = 0; j < kOut; j++) {
            const float y = valid ? target[i * kOut + j] : 0.f;
            const float r = o[j] * kOutScale;
            const float rc = fminf(fmaxf(r, -kRateClamp), kRateClamp);
            const float e = expf(rc);
            l += valid ? e - y * rc : 0.f;
            dO[j] = (valid && r > -kRateClamp && r < kRateClamp) ? (e - y) * kOutScale * inv_n : 0.f;
        }
        float ls = warp_sum(l);
        if (lane == 0) atomicAdd(&acc[kParams], ls * inv_n);
        // output layer
        float* gW1 = acc;
        float* gb1 = gW1 + kHidden * kFeatM;
        float* gW2 = gb1 + kHidden;
        float* gb2 = gW2 + kOut * kHidden;
        const float* W2 = P + kHidden * kFeatM + kHidden;
#pragma unroll
        for (int j = 0; j < kOut; j++) {
            float g = warp_sum(dO[j]);
            if (lane == 0) atomicAdd(&gb2[j], g);
        }
#pragma unroll 4
        for (int k = 0; k < kHidden; k++) {
            float h = fmaxf(hpre[k], 0.f);
            float dh = 0.f;
#pragma unroll
            for (int j = 0; j < kOut; j++) {
                float g = warp_sum(dO[j] * h);
                if (lane == 0) atomicAdd(&gW2[j * kHidden + k], g);
                dh = fmaf(W2[j * kHidden + k], dO[j], dh);
            }
            dh = hpre[k] > 0.f ? dh : 0.f;
            float gb = warp_sum(dh);
            if (lane == 0) atomicAdd(&gb1[k], gb);
#pragma unroll
            for (int f = 0; f < kFeatM; f++) {
                float g = warp_sum(dh * x[f]);
                if (lane == 0) atomicAdd(&gW1[k * kFeatM + f], g);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
        if (acc[i] != 0.f) atomicAdd(&G[i], acc[i]);
    if (threadIdx.x == 0) atomicAdd(loss, acc[kParams]);
}

// Adam step; the step number lives on the device so a captured graph of many
// steps can be replayed.
__global__ void k_mlp_adam(float* P, const float* G, float* m, float* v, int* d_step, float lr) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int step = *d_step + 1;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        float g = G[i];
        float mi = b1 * m[i] + (1.f - b1) * g;
        float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
    __syncthreads();
    if (threadIdx.x == 0) *d_step = step;
}

__global__ void k_zero(float* p, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 0.f;
}

// Predicted candidates per query and the sum of predicted results (rounded up).
__global__ void __launch_bounds__(256) k_mlp_predict(const float* __restrict__ feat, uint64_t n,
                                                     const float* __restrict__ Pg, uint32_t* __restrict__ pred,
                                                     unsigned long long* res_sum, unsigned long long* cand_sum) {
    __shared__ float P[kParamsAll];
    for (int i = threadIdx.x; i < kParamsAll; i += blockDim.x) P[i] = Pg[i];
    __syncthreads();
    const float calib = P[kParams + 1] > 0.f ? P[kParams + 1] : 1.f;
    unsigned long long cs = 0;
    double rs = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float x[kFeatM], hpre[kHidden], o[kOut];
#pragma unroll
        for (int f = 0; f < kFeatM; f++) x[f] = feat[i * kFeatM + f] * kInScale;
        mlp_fwd(P, x, hpre, o);
        const float ec = expf(fminf(fmaxf(o[0] * kOutScale, -kRateClamp), kRateClamp));
        const float er = expf(fminf(fmaxf(o[1] * kOutScale, -kRateClamp), kRateClamp));
        pred[i] = (uint32_t)fminf(ec + 0.5f, 1.0e9f);
        cs += pred[i];
        rs += (double)er;
    }
    // expected results: summed per warp, then rounded up once
    rs = warp_sum(rs);
    if (lane_id() == 0 && rs > 0.0) atomicAdd(res_sum, (unsigned long long)ceil(rs * (double)calib));
    if (cand_sum) {
        cs = warp_sum(cs);
        if (lane_id() == 0 && cs) atomicAdd(cand_sum, cs);
    }
}

// The same prediction for every join of a batch: rows are the batch's
// records, one per thread of a tile (tiles.cuh; blockDim == tile), the sums
// per join (one atomic per block each).
__global__ void __launch_bounds__(256) k_mlp_predict_tiles(const float* __restrict__ feat, TileMap m,
                                                           const float* __restrict__ Pg, uint32_t* __restrict__ pred,
                                                           unsigned long long* res_sums,
                                                           unsigned long long* cand_sums) {
    __shared__ float P[kParamsAll];
    __shared__ double s_rs[8];
    __shared__ unsigned long long s_cs[8];
    for (int i = threadIdx.x; i < kParamsAll; i += blockDim.x) P[i] = Pg[i];
    __syncthreads();
    const float calib = P[kParams + 1] > 0.f ? P[kParams + 1] : 1.f;
    for (uint32_t b = blockIdx.x; b < m.ntiles; b += gridDim.x) {
        const TileRange t = tile_range(m, b);
        const uint64_t g = __ldg(m.roff + t.j) + t.r0 + threadIdx.x;
        unsigned long long cs = 0;
        double rs = 0.0;
        if (t.r0 + threadIdx.x < t.r1) {
            float x[kFeatM], hpre[kHidden], o[kOut];
#pragma unroll
            for (int f = 0; f < kFeatM; f++) x[f] = feat[g * kFeatM + f] * kInScale;
            mlp_fwd(P, x, hpre, o);
            const float ec = expf(fminf(fmaxf(o[0] * kOutScale, -kRateClamp), kRateClamp));
            const float er = expf(fminf(fmaxf(o[1] * kOutScale, -kRateClamp), kRateClamp));
            pred[g] = (uint32_t)fminf(ec + 0.5f, 1.0e9f);
            cs = pred[g];
            rs = (double)er;
        }
        rs = warp_sum(rs);
        cs = warp_sum(cs);
        if (lane_id() == 0) {
            s_rs[threadIdx.x >> 5] = rs;
            s_cs[threadIdx.x >> 5] = cs;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            unsigned long long c = 0;
            for (uint32_t w = 0; w < (blockDim.x >> 5); w++) {
                r += s_rs[w];
                c += s_cs[w];
            }
            // expected results: summed per tile, then rounded up once
            if (r > 0.0) atomicAdd(res_sums + t.j, (unsigned long long)ceil(r * (double)calib));
            if (c) atomicAdd(cand_sums + t.j, c);
        }
        __syncthreads();
    }
}

__global__ void k_sum_cost(const uint32_t* __restrict__ c, uint64_t n, unsigned long long* out) {
    unsigned long long s = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += c[i];
    s = warp_sum(s);
    if (lane_id() == 0 && s) atomicAdd(out, s);
}

}  // namespace

void model_sum_cost(Ctx& c, const uint32_t* cost, uint64_t n, uint64_t* out) {
    k_sum_cost<<<grid_for(n, 256, c.num_sms * 8), 256, 0, c.stream>>>(cost, n, (unsigned long long*)out);
    FGSS_LAUNCH_CK();
}

void model_predict(Ctx& c, const float* feat, uint64_t n, uint32_t* pred, uint64_t* res_sum, uint64_t* cand_sum) {
    if (!c.model || !c.model->dev) fail(FGSS_ERR_INVALID, "no cost model loaded");
    k_mlp_predict<<<grid_for(n, 256, c.num_sms * 8), 256, 0, c.stream>>>(
        feat, n, c.model->dev, pred, (unsigned long long*)res_sum, (unsigned long long*)cand_sum);
    FGSS_LAUNCH_CK();
}

void model_predict_tiles(Ctx& c, const float* feat, const TileMap& m, uint32_t* pred, uint64_t* res_sums,
                         uint64_t* cand_sums) {
    if (!c.model || !c.model->dev) fail(FGSS_ERR_INVALID, "no cost model loaded");
    if (m.ntiles == 0) return;
    k_mlp_predict_tiles<<<std::min<uint32_t>(m.ntiles, (uint32_t)c.num_sms * 8), 256, 0, c.stream>>>(
        feat, m, c.model->dev, pred, (unsigned long long*)res_sums, (unsigned long long*)cand_sums);
    FGSS_LAUNCH_CK();
}

float model_grad(Ctx& c, const float* feat, const float* target, uint64_t n, const float* params, float* grads) {
    float* P = c.devT<float>("m.P.grad", kParamsAll);
    float* G = c.devT<float>("m.G.grad", kParams + 1);
    FGSS_CK(cudaMemcpyAsync(P, params, kParams * 4, cudaMemcpyHostToDevice, c.stream));
    FGSS_CK(cudaMemsetAsync(G, 0, (kParams + 1) * 4, c.stream));
    k_mlp_grad<<<grid_for(n, 256, c.num_sms * 4), 256, 0, c.stream>>>(feat, target, n, P, G, G + kParams);
    FGSS_LAUNCH_CK();
    std::vector<float> h(kParams + 1);
    FGSS_CK(cudaMemcpyAsync(h.data(), G, (kParams + 1) * 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    memcpy(grads, h.data(), kParams * 4);
    return h[kParams];
}

float model_fit(Ctx& c, const float* feat, const float* target, uint64_t n, int epochs, float lr, uint64_t seed) {
    if (!c.model) c.model = new fgss_model();
    fgss_model& M = *c.model;
    M.host.assign(kParamsAll, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    const float s1 = sqrtf(2.f / kFeatM), s2 = sqrtf(1.f / kHidden);
    for (int i = 0; i < kHidden * kFeatM; i++) M.host[i] = nd(rng) * s1;
    float* W2 = M.host.data() + kHidden * kFeatM + kHidden;
    for (int i = 0; i < kOut * kHidden; i++) W2[i] = nd(rng) * s2 * 0.1f;
    {
        // output biases start at the log of the mean count of each head
        std::vector<float> ht((size_t)n * kOut);
        FGSS_CK(cudaMemcpyAsync(ht.data(), target, ht.size() * 4, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        float* b2 = W2 + kOut * kHidden;
        for (int j = 0; j < kOut; j++) {
            double m = 0.0;
            for (uint64_t i = 0; i < n; i++) m += ht[i * kOut + j];
            m = n ? m / (double)n : 0.0;
            b2[j] = (float)(log(std::max(m, 1e-3)) / kOutScale);
        }
    }
    M.host[kParams] = 1.f;
    M.host[kParams + 1] = 1.f;
    M.dev = c.devT<float>("m.P", kParamsAll);
    float* G = c.devT<float>("m.G", kParams + 1);
    float* mo = c.devT<float>("m.m", kParams);
    float* ve = c.devT<float>("m.v", kParams);
    FGSS_CK(cudaMemcpyAsync(M.dev, M.host.data(), kParamsAll * 4, cudaMemcpyHostToDevice, c.stream));
    FGSS_CK(cudaMemsetAsync(mo, 0, kParams * 4, c.stream));
    FGSS_CK(cudaMemsetAsync(ve, 0, kParams * 4, c.stream));
    int* d_step = c.devT<int>("m.step", 1);
    FGSS_CK(cudaMemsetAsync(d_step, 0, 4, c.stream));
    const unsigned grid = grid_for(n, 256, c.num_sms * 4);
    // the epoch loop is captured once into a CUDA graph and replayed
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const int chunk = 50;
    int step = 0;
    float* loss_h = c.pinnedT<float>("m.loss", 1);
    for (int e = 0; e < epochs; e += chunk) {
        int m = std::min(chunk, epochs - e);
        if (m != chunk || !exec) {
            if (exec) {
                FGSS_CK(cudaGraphExecDestroy(exec));
                exec = nullptr;
            }
            if (graph) {
                FGSS_CK(cudaGraphDestroy(graph));
                graph = nullptr;
            }
            FGSS_CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < m; k++) {
                k_zero<<<1, 512, 0, c.stream>>>(G, kParams + 1);
                k_mlp_grad<<<grid, 256, 0, c.stream>>>(feat, target, n, M.dev, G, G + kParams);
                k_mlp_adam<<<1, 512, 0, c.stream>>>(M.dev, G, mo, ve, d_step, lr);
            }
            FGSS_CK(cudaStreamEndCapture(c.stream, &graph));
            FGSS_CK(cudaGraphInstantiate(&exec, graph, 0));
        }
        FGSS_CK(cudaGraphLaunch(exec, c.stream));
        step += m;
    }
    FGSS_CK(cudaMemcpyAsync(loss_h, G + kParams, 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (exec) FGSS_CK(cudaGraphExecDestroy(exec));
    if (graph) FGSS_CK(cudaGraphDestroy(graph));
    FGSS_CK(cudaMemcpyAsync(M.host.data(), M.dev, kParamsAll * 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    M.last_loss = *loss_h;
    M.trained = 1;
    return M.last_loss;
}

}  // namespace fgss
