// model_api.cu -- training, saving and loading of the cost model through the
// C ABI.  Training data come from the exact count pass of the plain method:
// per query the window entries its filter reads and the result pairs it
// emits, next to the features k_features computes.
#include <stdio.h>
#include <string.h>

#include <memory>
#include <vector>

#include "join.h"
#include "model.h"
#include "prims.cuh"

using namespace fgss;

namespace fgss {
__global__ void k_features(JoinArgs a, float* __restrict__ feat);
}

namespace {

__global__ void k_res_hist(const uint32_t* __restrict__ oq, uint64_t R, uint32_t* __restrict__ rcnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < R; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&rcnt[oq[i]], 1u);
}

__global__ void k_targets(const uint32_t* __restrict__ vcnt, const uint32_t* __restrict__ rcnt, uint64_t n,
                          float* __restrict__ target) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        target[2 * i] = (float)vcnt[i];
        target[2 * i + 1] = (float)rcnt[i];
    }
}

const uint32_t kMagic = 0x4d535346u;  // "FSSM"
const uint32_t kFormat = 2;  // 2: Poisson log-rate outputs (1 held log1p outputs)

}  // namespace

extern "C" {

fgss_status fgss_model_train(fgss_ctx* ctx, const fgss_sets_view* sets, const float* thresholds, int n, int epochs,
                             float lr, uint64_t seed, float* final_loss) {
    if (!ctx || !sets || !thresholds || n <= 0 || epochs <= 0) return FGSS_ERR_INVALID;
    try {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        uint64_t total = 0;
        for (int i = 0; i < n; i++) total += sets[i].n_sets;
        float* feat = c.devT<float>("mt.feat", (total + 1) * kFeat);
        float* target = c.devT<float>("mt.target", (total + 1) * 2);
        uint64_t off = 0, res_total = 0;
        for (int i = 0; i < n; i++) {
            JoinState J;
            fgss_join_opts o;
            fgss_join_opts_default(&o);
            o.threshold = thresholds[i];
            join_setup(c, J, sets[i], o, 100);
            join_index(c, J);
            join_plain_filter_verify(c, J, false);
            join_finish_status(c, J);
            const uint64_t m = J.in.n_sets;
            if (!m) continue;
            uint32_t* rcnt = c.devT<uint32_t>("mt.rcnt", m + 1);
            FGSS_CK(cudaMemsetAsync(rcnt, 0, m * 4, c.stream));
            if (J.n_res) {
                k_res_hist<<<grid_for(J.n_res, 256, c.num_sms * 8), 256, 0, c.stream>>>(J.oq, J.n_res, rcnt);
                FGSS_LAUNCH_CK();
            }
            k_features<<<grid_for(m * 32, 256, c.num_sms * 32), 256, 0, c.stream>>>(J.args, feat + off * kFeat);
            FGSS_LAUNCH_CK();
            k_targets<<<grid_for(m, 256, c.num_sms * 8), 256, 0, c.stream>>>(J.args.vcnt, rcnt, m, target + off * 2);
            FGSS_LAUNCH_CK();
            off += m;
            res_total += J.n_res;
        }
        c.sync();
        clear_graphs(c);  // captured batches presized with the previous model
        float loss = model_fit(c, feat, target, off, epochs, lr, seed);
        // calibration of the summed result estimate against the truth
        uint32_t* cost = c.devT<uint32_t>("mt.cost2", off + 1);
        uint64_t* rs = c.devT<uint64_t>("mt.rs", 1);
        FGSS_CK(cudaMemsetAsync(rs, 0, 8, c.stream));
        c.model->host[kParams + 1] = 1.f;
        FGSS_CK(cudaMemcpyAsync(c.model->dev, c.model->host.data(), kParamsAll * 4, cudaMemcpyHostToDevice, c.stream));
        model_predict(c, feat, off, cost, rs);
        uint64_t pred = 0;
        FGSS_CK(cudaMemcpyAsync(&pred, rs, 8, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        float calib = pred ? (float)((double)res_total / (double)pred) : 1.f;
        if (calib < 1.f) calib = 1.f;
        if (calib > 64.f) calib = 64.f;
        c.model->host[kParams + 1] = calib;
        FGSS_CK(cudaMemcpyAsync(c.model->dev, c.model->host.data(), kParamsAll * 4, cudaMemcpyHostToDevice, c.stream));
        c.sync();
        if (final_loss) *final_loss = loss;
        c.last_error.clear();
        return FGSS_OK;
    } catch (const Error& e) {
        ctx->c.last_error = e.msg;
        return e.st;
    }
}

int fgss_model_num_params(void) { return kParams; }

fgss_status fgss_model_grad(fgss_ctx* ctx, const float* feat, const float* target, uint64_t n, const float* params,
                            float* grads, float* loss) {
    if (!ctx || !feat || !target || !params || !grads || n == 0) return FGSS_ERR_INVALID;
    try {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        float* df = c.devT<float>("mg.feat", n * kFeat);
        float* dt = c.devT<float>("mg.target", n * 2);
        FGSS_CK(cudaMemcpyAsync(df, feat, n * kFeat * 4, cudaMemcpyHostToDevice, c.stream));
        FGSS_CK(cudaMemcpyAsync(dt, target, n * 2 * 4, cudaMemcpyHostToDevice, c.stream));
        float l = model_grad(c, df, dt, n, params, grads);
        if (loss) *loss = l;
        return FGSS_OK;
    } catch (const Error& e) {
        ctx->c.last_error = e.msg;
        return e.st;
    }
}

fgss_status fgss_model_save(fgss_ctx* ctx, const char* path) {
    if (!ctx || !path) return FGSS_ERR_INVALID;
    if (!ctx->c.model || !ctx->c.model->trained) return FGSS_ERR_INVALID;
    FILE* f = fopen(path, "wb");
    if (!f) return FGSS_ERR_IO;
    uint32_t hdr[4] = {kMagic, kFormat, (uint32_t)kParamsAll, (uint32_t)kHidden};
    bool ok = fwrite(hdr, 4, 4, f) == 4 &&
              fwrite(ctx->c.model->host.data(), 4, kParamsAll, f) == (size_t)kParamsAll;
    if (fclose(f) != 0) ok = false;
    return ok ? FGSS_OK : FGSS_ERR_IO;
}

fgss_status fgss_model_load(fgss_ctx* ctx, const char* path) {
    if (!ctx || !path) return FGSS_ERR_INVALID;
    FILE* f = fopen(path, "rb");
    if (!f) return FGSS_ERR_IO;
    uint32_t hdr[4];
    std::vector<float> p(kParamsAll);
    bool ok = fread(hdr, 4, 4, f) == 4 && hdr[0] == kMagic && hdr[1] == kFormat && hdr[2] == (uint32_t)kParamsAll &&
              hdr[3] == (uint32_t)kHidden && fread(p.data(), 4, kParamsAll, f) == (size_t)kParamsAll;
    fclose(f);
    if (!ok) return FGSS_ERR_FORMAT;
    for (float x : p)
        if (!(x == x) || x > 1e30f || x < -1e30f) return FGSS_ERR_FORMAT;  // NaN / inf weights are rejected
    try {
        Ctx& c = ctx->c;
        FGSS_CK(cudaSetDevice(c.device));
        clear_graphs(c);
        if (!c.model) c.model = new fgss_model();
        c.model->host = p;
        c.model->dev = c.devT<float>("m.P", kParamsAll);
        FGSS_CK(cudaMemcpyAsync(c.model->dev, p.data(), kParamsAll * 4, cudaMemcpyHostToDevice, c.stream));
        c.sync();
        c.model->trained = 1;
        return FGSS_OK;
    } catch (const Error& e) {
        ctx->c.last_error = e.msg;
        return e.st;
    }
}

}  // extern "C"
