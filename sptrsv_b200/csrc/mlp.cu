// mlp.cu — the schedule selector: a 12 -> 64 -> 64 -> 24 MLP, trained and
// evaluated with the hand-written CUDA kernels below.
//
// Inputs: the 12 analysis features (features.cu), normalised on the device
// with a stored mean/std.  Outputs: for each of the 24 schedule classes
// (4 variants x 6 parameter presets, schedule_from_class) the predicted
// log2(time / best time); the selector picks the argmin.  Training
// minimises the masked mean-squared error against autotuner timings with
// Adam.  Parameter layout (flat FP32, 6552 values), weights [in][out]:
//   W1[12][64] b1[64] W2[64][64] b2[64] W3[64][24] b3[24]
// At these sizes (a few thousand rows, 64-wide layers) the work is a few
// MFLOP per step: plain FP32 CUDA-core kernels, one thread per output,
// deterministic reductions (gradients are bit-reproducible).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "internal.h"

namespace sptrsv {

constexpr int NI = 12, NH = 64, NO = 24;
constexpr int O_W1 = 0, O_B1 = O_W1 + NI * NH, O_W2 = O_B1 + NH, O_B2 = O_W2 + NH * NH, O_W3 = O_B2 + NH,
              O_B3 = O_W3 + NH * NO, NPARAM = O_B3 + NO;
static_assert(NPARAM == 6552, "parameter count");

namespace {

__global__ void k_normalise(const float* __restrict__ X, const float* __restrict__ mean, const float* __restrict__ sd,
                            int B, float* __restrict__ Xn)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < B * NI; t += gridDim.x * blockDim.x) {
        int i = t % NI;
        Xn[t] = (X[t] - mean[i]) / sd[i];
    }
}

// Y[b][o] = act(sum_i X[b][i] W[i][o] + bias[o]); Z keeps the pre-activation
__global__ void k_dense_fwd(const float* __restrict__ X, const float* __restrict__ W, const float* __restrict__ bias,
                            int B, int I, int O, int relu, float* __restrict__ Z, float* __restrict__ Y)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < B * O; t += gridDim.x * blockDim.x) {
        int b = t / O, o = t % O;
        float s = bias[o];
        for (int i = 0; i < I; i++) s = fmaf(X[b * I + i], W[i * O + o], s);
        if (Z) Z[t] = s;
        Y[t] = relu ? fmaxf(s, 0.f) : s;
    }
}

// dY = 2 M (Y - T) / max(1, sum M); loss terms per element into L
__global__ void k_out_grad(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ M,
                           int n, float inv_denom, float* __restrict__ dY, float* __restrict__ L)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        float d = Y[t] - T[t];
        dY[t] = 2.f * M[t] * d * inv_denom;
        L[t] = M[t] * d * d * inv_denom;
    }
}

// dW[i][o] = sum_b X[b][i] dY[b][o]; db[o] = sum_b dY[b][o] (thread per weight)
__global__ void k_dense_bwd_w(const float* __restrict__ X, const float* __restrict__ dY, int B, int I, int O,
                              float* __restrict__ dW, float* __restrict__ db)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < (I + 1) * O; t += gridDim.x * blockDim.x) {
        int i = t / O, o = t % O;
        float s = 0.f;
        if (i < I) {
            for (int b = 0; b < B; b++) s = fmaf(X[b * I + i], dY[b * O + o], s);
            dW[i * O + o] = s;
        } else {
            for (int b = 0; b < B; b++) s += dY[b * O + o];
            db[o] = s;
        }
    }
}

// dX[b][i] = sum_o dY[b][o] W[i][o], times relu'(Z[b][i])
__global__ void k_dense_bwd_x(const float* __restrict__ dY, const float* __restrict__ W, const float* __restrict__ Z,
                              int B, int I, int O, float* __restrict__ dX)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < B * I; t += gridDim.x * blockDim.x) {
        int b = t / I, i = t % I;
        float s = 0.f;
        for (int o = 0; o < O; o++) s = fmaf(dY[b * O + o], W[i * O + o], s);
        dX[t] = Z[t] > 0.f ? s : 0.f;
    }
}

__global__ void k_sum(const float* __restrict__ a, int n, float* __restrict__ out)
{
    // one block, deterministic
    __shared__ float sh[256];
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += a[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.f - b1) * gi;
        float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void k_gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int B, int W,
                              float* __restrict__ dst)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < B * W; t += gridDim.x * blockDim.x) {
        int b = t / W, c = t % W;
        dst[t] = src[(size_t)idx[b] * W + c];
    }
}

int g1(long long n) { return (int)((n + 255) / 256 > 1024 ? 1024 : (n + 255) / 256 < 1 ? 1 : (n + 255) / 256); }

}  // namespace

// Workspace for a batch of up to `cap` rows.
struct MlpWork {
    int cap = 0;
    float *xn = nullptr, *z1 = nullptr, *h1 = nullptr, *z2 = nullptr, *h2 = nullptr, *y = nullptr;
    float *dy = nullptr, *dh2 = nullptr, *dh1 = nullptr, *lt = nullptr, *loss = nullptr;
    float *bx = nullptr, *bt = nullptr, *bm = nullptr;
    int* idx = nullptr;
    void release()
    {
        float* a[] = {xn, z1, h1, z2, h2, y, dy, dh2, dh1, lt, loss, bx, bt, bm};
        for (float* q : a) cudaFree(q);
        cudaFree(idx);
        *this = MlpWork();
    }
    int ensure(int B)
    {
        if (B <= cap) return 0;
        release();
        SPT_CUDA(dalloc(&xn, (long long)B * NI));
        SPT_CUDA(dalloc(&z1, (long long)B * NH));
        SPT_CUDA(dalloc(&h1, (long long)B * NH));
        SPT_CUDA(dalloc(&z2, (long long)B * NH));
        SPT_CUDA(dalloc(&h2, (long long)B * NH));
        SPT_CUDA(dalloc(&y, (long long)B * NO));
        SPT_CUDA(dalloc(&dy, (long long)B * NO));
        SPT_CUDA(dalloc(&dh2, (long long)B * NH));
        SPT_CUDA(dalloc(&dh1, (long long)B * NH));
        SPT_CUDA(dalloc(&lt, (long long)B * NO));
        SPT_CUDA(dalloc(&loss, 1));
        SPT_CUDA(dalloc(&bx, (long long)B * NI));
        SPT_CUDA(dalloc(&bt, (long long)B * NO));
        SPT_CUDA(dalloc(&bm, (long long)B * NO));
        SPT_CUDA(dalloc(&idx, B));
        cap = B;
        return 0;
    }
};

}  // namespace sptrsv

struct sptrsv_mlp_s {
    float* p = nullptr;     // params
    float* g = nullptr;     // gradient
    float* m = nullptr;     // Adam moments
    float* v = nullptr;
    float* mean = nullptr;  // feature normalisation
    float* sd = nullptr;
    long long step = 0;
    sptrsv::MlpWork w;
};

namespace sptrsv {

namespace {

// forward on normalised inputs already in w.xn
void forward(sptrsv_mlp_s* M, int B)
{
    MlpWork& w = M->w;
    k_dense_fwd<<<g1((long long)B * NH), 256>>>(w.xn, M->p + O_W1, M->p + O_B1, B, NI, NH, 1, w.z1, w.h1);
    k_dense_fwd<<<g1((long long)B * NH), 256>>>(w.h1, M->p + O_W2, M->p + O_B2, B, NH, NH, 1, w.z2, w.h2);
    k_dense_fwd<<<g1((long long)B * NO), 256>>>(w.h2, M->p + O_W3, M->p + O_B3, B, NH, NO, 0, nullptr, w.y);
}

// loss + gradient into M->g for targets/mask already on the device
void backward(sptrsv_mlp_s* M, int B, const float* T, const float* Mk, float inv_denom)
{
    MlpWork& w = M->w;
    k_out_grad<<<g1((long long)B * NO), 256>>>(w.y, T, Mk, B * NO, inv_denom, w.dy, w.lt);
    k_sum<<<1, 256>>>(w.lt, B * NO, w.loss);
    k_dense_bwd_w<<<g1((long long)(NH + 1) * NO), 256>>>(w.h2, w.dy, B, NH, NO, M->g + O_W3, M->g + O_B3);
    k_dense_bwd_x<<<g1((long long)B * NH), 256>>>(w.dy, M->p + O_W3, w.z2, B, NH, NO, w.dh2);
    k_dense_bwd_w<<<g1((long long)(NH + 1) * NH), 256>>>(w.h1, w.dh2, B, NH, NH, M->g + O_W2, M->g + O_B2);
    k_dense_bwd_x<<<g1((long long)B * NH), 256>>>(w.dh2, M->p + O_W2, w.z1, B, NH, NH, w.dh1);
    k_dense_bwd_w<<<g1((long long)(NI + 1) * NH), 256>>>(w.xn, w.dh1, B, NI, NH, M->g + O_W1, M->g + O_B1);
}

float mask_denom(const float* Mh, long long n)
{
    double s = 0;
    for (long long i = 0; i < n; i++) s += Mh[i];
    return (float)(s > 1 ? s : 1);
}

}  // namespace

}  // namespace sptrsv

using namespace sptrsv;

extern "C" {

int sptrsv_mlp_create(uint64_t seed, sptrsv_mlp_t* out)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!out) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_create: NULL");
        if (!ctx()) return set_error(SPTRSV_ERR_CUDA, "mlp_create: no CUDA device");
        sptrsv_mlp_s* M = new sptrsv_mlp_s();
        auto fail = [&](int code) {
            cudaFree(M->p); cudaFree(M->g); cudaFree(M->m); cudaFree(M->v); cudaFree(M->mean); cudaFree(M->sd);
            delete M;
            return code;
        };
        if (dalloc(&M->p, NPARAM) || dalloc(&M->g, NPARAM) || dalloc(&M->m, NPARAM) || dalloc(&M->v, NPARAM) ||
            dalloc(&M->mean, NI) || dalloc(&M->sd, NI))
            return fail(set_error(SPTRSV_ERR_ALLOC, "mlp_create: allocation failed"));
        // He-uniform weights, zero biases
        std::vector<float> h(NPARAM, 0.f);
        std::mt19937_64 g(seed);
        auto init = [&](int off, int fan_in, int count) {
            float a = std::sqrt(6.f / (float)fan_in);
            std::uniform_real_distribution<float> u(-a, a);
            for (int i = 0; i < count; i++) h[off + i] = u(g);
        };
        init(O_W1, NI, NI * NH);
        init(O_W2, NH, NH * NH);
        init(O_W3, NH, NH * NO);
        std::vector<float> mean(NI, 0.f), sd(NI, 1.f);
        if (cudaMemcpy(M->p, h.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(M->m, 0, sizeof(float) * NPARAM) != cudaSuccess ||
            cudaMemset(M->v, 0, sizeof(float) * NPARAM) != cudaSuccess ||
            cudaMemcpy(M->mean, mean.data(), sizeof(float) * NI, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(M->sd, sd.data(), sizeof(float) * NI, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(set_error(SPTRSV_ERR_CUDA, "mlp_create: upload failed"));
        *out = M;
        return ok();
    });
}

int sptrsv_mlp_destroy(sptrsv_mlp_t M)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M) return ok();
        M->w.release();
        cudaFree(M->p); cudaFree(M->g); cudaFree(M->m); cudaFree(M->v); cudaFree(M->mean); cudaFree(M->sd);
        delete M;
        return ok();
    });
}

int sptrsv_mlp_get_params(sptrsv_mlp_t M, float* host)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !host) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_get_params: NULL");
        SPT_CUDA(cudaMemcpy(host, M->p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
        return ok();
    });
}

int sptrsv_mlp_set_params(sptrsv_mlp_t M, const float* host)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !host) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_set_params: NULL");
        SPT_CUDA(cudaMemcpy(M->p, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
        SPT_CUDA(cudaMemset(M->m, 0, sizeof(float) * NPARAM));
        SPT_CUDA(cudaMemset(M->v, 0, sizeof(float) * NPARAM));
        M->step = 0;
        return ok();
    });
}

int sptrsv_mlp_set_normalization(sptrsv_mlp_t M, const float* mean12, const float* std12)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !mean12 || !std12) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_set_normalization: NULL");
        for (int i = 0; i < NI; i++)
            if (!(std12[i] > 0.f)) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_set_normalization: std must be > 0");
        SPT_CUDA(cudaMemcpy(M->mean, mean12, sizeof(float) * NI, cudaMemcpyHostToDevice));
        SPT_CUDA(cudaMemcpy(M->sd, std12, sizeof(float) * NI, cudaMemcpyHostToDevice));
        return ok();
    });
}

int sptrsv_mlp_get_normalization(sptrsv_mlp_t M, float* mean12, float* std12)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !mean12 || !std12) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_get_normalization: NULL");
        SPT_CUDA(cudaMemcpy(mean12, M->mean, sizeof(float) * NI, cudaMemcpyDeviceToHost));
        SPT_CUDA(cudaMemcpy(std12, M->sd, sizeof(float) * NI, cudaMemcpyDeviceToHost));
        return ok();
    });
}

int sptrsv_mlp_forward_host(sptrsv_mlp_t M, const float* X, int B, float* Y)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !X || !Y || B < 1) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_forward: bad arguments");
        int e = M->w.ensure(B);
        if (e) return e;
        SPT_CUDA(cudaMemcpy(M->w.bx, X, sizeof(float) * (size_t)B * NI, cudaMemcpyHostToDevice));
        k_normalise<<<g1((long long)B * NI), 256>>>(M->w.bx, M->mean, M->sd, B, M->w.xn);
        forward(M, B);
        SPT_CUDA(cudaGetLastError());
        SPT_CUDA(cudaMemcpy(Y, M->w.y, sizeof(float) * (size_t)B * NO, cudaMemcpyDeviceToHost));
        return ok();
    });
}

int sptrsv_mlp_gradient_host(sptrsv_mlp_t M, const float* X, const float* T, const float* Mk, int B, float* grad,
                             float* loss)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !X || !T || !Mk || B < 1) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_gradient: bad arguments");
        int e = M->w.ensure(B);
        if (e) return e;
        MlpWork& w = M->w;
        SPT_CUDA(cudaMemcpy(w.bx, X, sizeof(float) * (size_t)B * NI, cudaMemcpyHostToDevice));
        SPT_CUDA(cudaMemcpy(w.bt, T, sizeof(float) * (size_t)B * NO, cudaMemcpyHostToDevice));
        SPT_CUDA(cudaMemcpy(w.bm, Mk, sizeof(float) * (size_t)B * NO, cudaMemcpyHostToDevice));
        k_normalise<<<g1((long long)B * NI), 256>>>(w.bx, M->mean, M->sd, B, w.xn);
        forward(M, B);
        backward(M, B, w.bt, w.bm, 1.f / mask_denom(Mk, (long long)B * NO));
        SPT_CUDA(cudaGetLastError());
        if (grad) SPT_CUDA(cudaMemcpy(grad, M->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
        if (loss) SPT_CUDA(cudaMemcpy(loss, w.loss, sizeof(float), cudaMemcpyDeviceToHost));
        return ok();
    });
}

// Minibatch Adam over a dataset of N rows held on the device for the call.
// loss_curve[e] = mean minibatch loss of epoch e (may be NULL).
int sptrsv_mlp_train_host(sptrsv_mlp_t M, const float* X, const float* T, const float* Mk, int N, int epochs,
                          int batch, float lr, uint64_t seed, float* loss_curve)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !X || !T || !Mk || N < 1 || epochs < 0 || batch < 1 || !(lr > 0.f))
            return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_train: bad arguments");
        if (batch > N) batch = N;
        int e = M->w.ensure(batch);
        if (e) return e;
        float *dX = nullptr, *dT = nullptr, *dM = nullptr;
        auto cleanup = [&]() { cudaFree(dX); cudaFree(dT); cudaFree(dM); };
        if (dalloc(&dX, (long long)N * NI) || dalloc(&dT, (long long)N * NO) || dalloc(&dM, (long long)N * NO)) {
            cleanup();
            return set_error(SPTRSV_ERR_ALLOC, "mlp_train: allocation failed");
        }
        cudaMemcpy(dX, X, sizeof(float) * (size_t)N * NI, cudaMemcpyHostToDevice);
        cudaMemcpy(dT, T, sizeof(float) * (size_t)N * NO, cudaMemcpyHostToDevice);
        cudaMemcpy(dM, Mk, sizeof(float) * (size_t)N * NO, cudaMemcpyHostToDevice);
        std::mt19937_64 g(seed);
        std::vector<int> perm(N);
        for (int i = 0; i < N; i++) perm[i] = i;
        MlpWork& w = M->w;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        std::vector<float> mh((size_t)batch * NO);
        for (int ep = 0; ep < epochs; ep++) {
            std::shuffle(perm.begin(), perm.end(), g);
            double lsum = 0;
            int nb = 0;
            for (int s = 0; s < N; s += batch) {
                int B = std::min(batch, N - s);
                cudaMemcpy(w.idx, perm.data() + s, sizeof(int) * B, cudaMemcpyHostToDevice);
                k_gather_rows<<<g1((long long)B * NI), 256>>>(dX, w.idx, B, NI, w.bx);
                k_gather_rows<<<g1((long long)B * NO), 256>>>(dT, w.idx, B, NO, w.bt);
                k_gather_rows<<<g1((long long)B * NO), 256>>>(dM, w.idx, B, NO, w.bm);
                double msum = 0;
                for (int b = 0; b < B; b++)
                    for (int c = 0; c < NO; c++) msum += Mk[(size_t)perm[s + b] * NO + c];
                k_normalise<<<g1((long long)B * NI), 256>>>(w.bx, M->mean, M->sd, B, w.xn);
                forward(M, B);
                backward(M, B, w.bt, w.bm, 1.f / (float)(msum > 1 ? msum : 1));
                M->step++;
                float c1 = 1.f - std::pow(b1, (float)M->step), c2 = 1.f - std::pow(b2, (float)M->step);
                k_adam<<<g1(NPARAM), 256>>>(M->p, M->g, M->m, M->v, NPARAM, lr, b1, b2, eps, c1, c2);
                float lh = 0;
                cudaMemcpy(&lh, w.loss, sizeof(float), cudaMemcpyDeviceToHost);
                lsum += lh;
                nb++;
            }
            if (loss_curve) loss_curve[ep] = (float)(lsum / (nb ? nb : 1));
        }
        cleanup();
        cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) return cuda_fail(ce, "mlp_train");
        return ok();
    });
}

}  // extern "C"
