// Training, gradient and inference kernels of the row-size predictor, and its
// checkpoint registry. C ABI in include/rvsp_cuda.h (rvsp_cuda_mlp_*).
//
// Training runs entirely on the GPU: one CTA of MLP_TPB threads takes
// MLP_TPB samples of the mini-batch, runs the forward pass one sample per
// thread with the activations kept in shared memory, forms the output
// gradient, back-propagates, and reduces the weight gradients over its
// samples in shared memory before adding them to the global gradient; a
// second kernel applies Adam. The gradient of the mean batch loss is what the
// tests check against an FP64 restatement of the same network.

#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "mlp.cuh"
#include "spgemm_types.cuh"
#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"

using namespace rvsp;

namespace rvsp {

constexpr int MLP_TPB = 64;
constexpr int MLP_LD = MLP_H + 1;  // padded row stride of activation tiles

// Forward + backward over samples idx[blockIdx.x*TPB + t] (or the identity
// when idx is null). X holds normalised features [n][4]; y the targets
// log2(1 + nnz); w the per-sample loss weights. Gradients of
// scale * sum(loss) are added to grad; scale * sum(loss) to *loss.
__global__ void __launch_bounds__(MLP_TPB)
    k_mlp_fwd_bwd(const float* __restrict__ P, const float* __restrict__ X,
                  const float* __restrict__ Y, const float* __restrict__ W,
                  const int32_t* __restrict__ idx, int32_t nb, float scale,
                  float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float sP[MLP_NPARAM];
    __shared__ float sX[MLP_TPB][MLP_IN];
    __shared__ float sH1[MLP_TPB][MLP_LD];
    __shared__ float sH2[MLP_TPB][MLP_LD];
    __shared__ float sD2[MLP_TPB][MLP_LD];  // dL/dz2
    __shared__ float sD1[MLP_TPB][MLP_LD];  // dL/dz1
    __shared__ float sDO[MLP_TPB][MLP_OUT];
    __shared__ float sLoss[MLP_TPB];
    const int t = threadIdx.x;
    for (int i = t; i < MLP_NPARAM; i += MLP_TPB) sP[i] = P[i];
    const int j = blockIdx.x * MLP_TPB + t;
    const bool live = j < nb;
    const int s = live ? (idx ? idx[j] : j) : 0;
    for (int i = 0; i < MLP_IN; ++i) sX[t][i] = live ? X[(size_t)s * MLP_IN + i] : 0.0f;
    __syncthreads();
    // forward
    for (int h = 0; h < MLP_H; ++h) {
        float z = sP[MLP_B1 + h];
        for (int i = 0; i < MLP_IN; ++i) z += sP[MLP_W1 + h * MLP_IN + i] * sX[t][i];
        sH1[t][h] = z;  // pre-activation, ReLU applied on use
    }
    for (int h = 0; h < MLP_H; ++h) {
        float z = sP[MLP_B2 + h];
        for (int k = 0; k < MLP_H; ++k) z += sP[MLP_W2 + h * MLP_H + k] * fmaxf(sH1[t][k], 0.0f);
        sH2[t][h] = z;
    }
    float o[MLP_OUT];
    for (int c = 0; c < MLP_OUT; ++c) {
        float z = sP[MLP_B3 + c];
        for (int k = 0; k < MLP_H; ++k) z += sP[MLP_W3 + c * MLP_H + k] * fmaxf(sH2[t][k], 0.0f);
        o[c] = z;
    }
    // Gaussian NLL on y, sigma = softplus(s) + 1e-3
    float dmu = 0.0f, ds = 0.0f, l = 0.0f;
    if (live) {
        const float y = Y[s], w = W ? W[s] : 1.0f;
        const float sig = mlp_softplus(o[1]) + 1e-3f;
        const float r = (y - o[0]) / sig;
        l = w * (0.5f * r * r + logf(sig));
        dmu = w * (-r / sig) * scale;
        const float dsig = w * (-r * r / sig + 1.0f / sig) * scale;
        ds = dsig / (1.0f + expf(-o[1]));
    }
    sDO[t][0] = dmu;
    sDO[t][1] = ds;
    sLoss[t] = l * scale;
    // backward through layer 3 and the second ReLU
    for (int h = 0; h < MLP_H; ++h) {
        const float g = dmu * sP[MLP_W3 + h] + ds * sP[MLP_W3 + MLP_H + h];
        sD2[t][h] = sH2[t][h] > 0.0f ? g : 0.0f;
    }
    for (int k = 0; k < MLP_H; ++k) {
        float g = 0.0f;
        for (int h = 0; h < MLP_H; ++h) g += sD2[t][h] * sP[MLP_W2 + h * MLP_H + k];
        sD1[t][k] = sH1[t][k] > 0.0f ? g : 0.0f;
    }
    __syncthreads();
    // weight gradients: reduce over the block's samples
    for (int e = t; e < MLP_NPARAM; e += MLP_TPB) {
        float g = 0.0f;
        if (e < MLP_B1) {  // W1[h][i]
            const int h = e / MLP_IN, i = e % MLP_IN;
            for (int q = 0; q < MLP_TPB; ++q) g += sD1[q][h] * sX[q][i];
        } else if (e < MLP_W2) {  // b1[h]
            const int h = e - MLP_B1;
            for (int q = 0; q < MLP_TPB; ++q) g += sD1[q][h];
        } else if (e < MLP_B2) {  // W2[h][k]
            const int h = (e - MLP_W2) / MLP_H, k = (e - MLP_W2) % MLP_H;
            for (int q = 0; q < MLP_TPB; ++q) g += sD2[q][h] * fmaxf(sH1[q][k], 0.0f);
        } else if (e < MLP_W3) {  // b2[h]
            const int h = e - MLP_B2;
            for (int q = 0; q < MLP_TPB; ++q) g += sD2[q][h];
        } else if (e < MLP_B3) {  // W3[c][k]
            const int c = (e - MLP_W3) / MLP_H, k = (e - MLP_W3) % MLP_H;
            for (int q = 0; q < MLP_TPB; ++q) g += sDO[q][c] * fmaxf(sH2[q][k], 0.0f);
        } else {  // b3[c]
            const int c = e - MLP_B3;
            for (int q = 0; q < MLP_TPB; ++q) g += sDO[q][c];
        }
        atomicAdd(&grad[e], g);
    }
    if (t == 0) {
        float sum = 0.0f;
        for (int q = 0; q < MLP_TPB; ++q) sum += sLoss[q];
        atomicAdd(loss, sum);
    }
}

__global__ void k_adam(float* __restrict__ P, float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_NPARAM) return;
    const float g = grad[i];
    m[i] = b1 * m[i] + (1.0f - b1) * g;
    v[i] = b2 * v[i] + (1.0f - b2) * g * g;
    P[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
    grad[i] = 0.0f;
}

// Inference on raw features: capacity per row (see mlp.cuh). Rows with
// ub <= 0 get capacity 0. With bin given, only rows above the tiny bin are
// predicted (the others never use a prediction).
__global__ void __launch_bounds__(256)
    k_mlp_infer(MlpModel model, const float4* __restrict__ feat, const int32_t* __restrict__ ub,
                const uint8_t* __restrict__ bin, int32_t n, float* __restrict__ mu_out,
                float* __restrict__ sig_out, int32_t* __restrict__ cap_out) {
    __shared__ float sP[MLP_NPARAM];
    // a block none of whose rows needs a prediction (all tiny or empty, as in
    // stencil products) leaves before loading the parameters
    bool any = bin == nullptr;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n && !any; r += gridDim.x * blockDim.x)
        any = bin[r] >= BIN_WARP0;
    if (!__syncthreads_or(any)) return;
    for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) sP[i] = model.params[i];
    __syncthreads();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        if (bin && bin[r] < BIN_WARP0) continue;
        const float4 f = feat[r];
        const float raw[MLP_IN] = {f.x, f.y, f.z, f.w};
        float x[MLP_IN];
        for (int i = 0; i < MLP_IN; ++i)
            x[i] = (log2f(1.0f + raw[i]) - model.mean[i]) * model.inv_std[i];
        float h1[MLP_H];
        for (int h = 0; h < MLP_H; ++h) {
            float z = sP[MLP_B1 + h];
            for (int i = 0; i < MLP_IN; ++i) z += sP[MLP_W1 + h * MLP_IN + i] * x[i];
            h1[h] = fmaxf(z, 0.0f);
        }
        float o0 = sP[MLP_B3], o1 = sP[MLP_B3 + 1];
        for (int h = 0; h < MLP_H; ++h) {
            float z = sP[MLP_B2 + h];
            for (int k = 0; k < MLP_H; ++k) z += sP[MLP_W2 + h * MLP_H + k] * h1[k];
            z = fmaxf(z, 0.0f);
            o0 += sP[MLP_W3 + h] * z;
            o1 += sP[MLP_W3 + MLP_H + h] * z;
        }
        const float sig = mlp_softplus(o1) + 1e-3f;
        const int32_t u = ub[r];
        const float e = fminf(o0 + model.z * sig, 30.0f);
        int32_t cap = (int32_t)ceilf(exp2f(e) - 1.0f);
        cap = u <= 0 ? 0 : min(max(cap, 1), u);
        if (mu_out) mu_out[r] = o0;
        if (sig_out) sig_out[r] = sig;
        cap_out[r] = cap;
    }
}

// ---------------------------------------------------------------------------
// model registry: the checkpoint in use, loaded lazily
// ---------------------------------------------------------------------------
static std::mutex g_model_mu;
static bool g_model_ok = false;
static bool g_model_tried = false;
static MlpModel g_model;

static const char kMagic[8] = {'R', 'V', 'S', 'P', 'M', 'L', 'P', 0};
constexpr uint32_t kVersion = 1;
constexpr int kModelFloats = 2 * MLP_IN + 1 + MLP_NPARAM;

static uint32_t fnv1a(const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    uint32_t h = 2166136261u;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 16777619u;
    return h;
}

static void unpack(const float* f, MlpModel* m) {
    memcpy(m->mean, f, sizeof(m->mean));
    memcpy(m->inv_std, f + MLP_IN, sizeof(m->inv_std));
    m->z = f[2 * MLP_IN];
    memcpy(m->params, f + 2 * MLP_IN + 1, sizeof(m->params));
}

static int load_file(const char* path, MlpModel* m) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return RVSP_ERROR_INVALID_ARGUMENT;
    char magic[8];
    uint32_t ver = 0, cnt = 0, sum = 0;
    std::vector<float> f(kModelFloats);
    bool ok = fread(magic, 1, 8, fp) == 8 && memcmp(magic, kMagic, 8) == 0 &&
              fread(&ver, 4, 1, fp) == 1 && ver == kVersion && fread(&cnt, 4, 1, fp) == 1 &&
              cnt == (uint32_t)kModelFloats &&
              fread(f.data(), 4, kModelFloats, fp) == (size_t)kModelFloats &&
              fread(&sum, 4, 1, fp) == 1 && sum == fnv1a(f.data(), f.size() * 4);
    fclose(fp);
    if (!ok) return RVSP_ERROR_INVALID_ARGUMENT;
    unpack(f.data(), m);
    return RVSP_SUCCESS;
}

// The default checkpoint: $RVSP_MLP_WEIGHTS, else weights/row_mlp_v1.bin
// next to the directory holding this library.
static std::string default_path() {
    if (const char* e = getenv("RVSP_MLP_WEIGHTS")) return e;
    Dl_info info;
    if (dladdr((void*)&default_path, &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        const size_t cut = so.find_last_of('/');
        const std::string dir = cut == std::string::npos ? "." : so.substr(0, cut);
        return dir + "/../weights/row_mlp_v1.bin";
    }
    return "weights/row_mlp_v1.bin";
}

void launch_mlp_infer(const MlpModel& m, const float4* feat, const int32_t* ub, const uint8_t* bin,
                      int32_t n, int32_t* cap, cudaStream_t st) {
    // grid-stride over the rows: the weights are staged once per CTA
    k_mlp_infer<<<std::min((n + 255) / 256, 148 * 8), 256, 0, st>>>(m, feat, ub, bin, n, nullptr,
                                                                   nullptr, cap);
}

bool current_model(MlpModel* out) {
    std::lock_guard<std::mutex> lk(g_model_mu);
    if (!g_model_ok && !g_model_tried) {
        g_model_tried = true;
        g_model_ok = load_file(default_path().c_str(), &g_model) == RVSP_SUCCESS;
    }
    if (g_model_ok && out) *out = g_model;
    return g_model_ok;
}

}  // namespace rvsp

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int rvsp_cuda_mlp_load(const char* path) {
    MlpModel m;
    const int st = load_file(path ? path : default_path().c_str(), &m);
    if (st) return st;
    std::lock_guard<std::mutex> lk(g_model_mu);
    g_model = m;
    g_model_ok = true;
    g_model_tried = true;
    return RVSP_SUCCESS;
}

int rvsp_cuda_mlp_set(const float* model, int32_t nfloats) {
    if (!model) return RVSP_ERROR_NULL_POINTER;
    if (nfloats != kModelFloats) return RVSP_ERROR_INVALID_ARGUMENT;
    MlpModel m;
    unpack(model, &m);
    std::lock_guard<std::mutex> lk(g_model_mu);
    g_model = m;
    g_model_ok = true;
    g_model_tried = true;
    return RVSP_SUCCESS;
}

int rvsp_cuda_mlp_save(const char* path, const float* model, int32_t nfloats) {
    if (!path || !model) return RVSP_ERROR_NULL_POINTER;
    if (nfloats != kModelFloats) return RVSP_ERROR_INVALID_ARGUMENT;
    FILE* fp = fopen(path, "wb");
    if (!fp) return RVSP_ERROR_INVALID_ARGUMENT;
    const uint32_t ver = kVersion, cnt = kModelFloats, sum = fnv1a(model, (size_t)nfloats * 4);
    bool ok = fwrite(kMagic, 1, 8, fp) == 8 && fwrite(&ver, 4, 1, fp) == 1 &&
              fwrite(&cnt, 4, 1, fp) == 1 &&
              fwrite(model, 4, (size_t)nfloats, fp) == (size_t)nfloats && fwrite(&sum, 4, 1, fp) == 1;
    ok = (fclose(fp) == 0) && ok;
    return ok ? RVSP_SUCCESS : RVSP_ERROR_INVALID_ARGUMENT;
}

int rvsp_cuda_mlp_get(float* model_out, int32_t nfloats) {
    if (!model_out) return RVSP_ERROR_NULL_POINTER;
    if (nfloats != kModelFloats) return RVSP_ERROR_INVALID_ARGUMENT;
    MlpModel m;
    if (!current_model(&m)) return RVSP_ERROR_UNSUPPORTED_BACKEND;
    memcpy(model_out, m.mean, sizeof(m.mean));
    memcpy(model_out + MLP_IN, m.inv_std, sizeof(m.inv_std));
    model_out[2 * MLP_IN] = m.z;
    memcpy(model_out + 2 * MLP_IN + 1, m.params, sizeof(m.params));
    return RVSP_SUCCESS;
}

int rvsp_cuda_learned_available(void) { return current_model(nullptr) ? 1 : 0; }

int rvsp_cuda_mlp_grad(const float* params, const float* X, const float* y, const float* w,
                       int32_t n, float* loss_out, float* grad_out) {
    if (!params || !X || !y || !loss_out || !grad_out) return RVSP_ERROR_NULL_POINTER;
    if (n <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
    float *dP = nullptr, *dX = nullptr, *dY = nullptr, *dW = nullptr, *dG = nullptr;
    cudaError_t e = cudaMalloc(&dP, MLP_NPARAM * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * MLP_IN * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dY, (size_t)n * 4);
    if (e == cudaSuccess && w) e = cudaMalloc(&dW, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dG, (MLP_NPARAM + 1) * 4);
    if (e == cudaSuccess) e = cudaMemcpy(dP, params, MLP_NPARAM * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dX, X, (size_t)n * MLP_IN * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dY, y, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && w) e = cudaMemcpy(dW, w, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dG, 0, (MLP_NPARAM + 1) * 4);
    if (e == cudaSuccess) {
        k_mlp_fwd_bwd<<<(n + MLP_TPB - 1) / MLP_TPB, MLP_TPB>>>(dP, dX, dY, dW, nullptr, n,
                                                               1.0f / (float)n, dG,
                                                               dG + MLP_NPARAM);
        note_launch(nullptr, 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(grad_out, dG, MLP_NPARAM * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(loss_out, dG + MLP_NPARAM, 4, cudaMemcpyDeviceToHost);
    cudaFree(dP);
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dW);
    cudaFree(dG);
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "mlp grad");
}

int rvsp_cuda_mlp_train(float* params, const float* X, const float* y, const float* w, int32_t n,
                        int32_t epochs, int32_t batch, float lr, uint64_t seed,
                        float* epoch_loss_out) {
    if (!params || !X || !y) return RVSP_ERROR_NULL_POINTER;
    if (n <= 0 || epochs <= 0 || batch <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
    float *dP = nullptr, *dX = nullptr, *dY = nullptr, *dW = nullptr, *dG = nullptr,
          *dM = nullptr, *dV = nullptr;
    int32_t* dI = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreate(&st);
    if (e == cudaSuccess) e = cudaMalloc(&dP, MLP_NPARAM * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * MLP_IN * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dY, (size_t)n * 4);
    if (e == cudaSuccess && w) e = cudaMalloc(&dW, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dG, (MLP_NPARAM + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dM, MLP_NPARAM * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dV, MLP_NPARAM * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dI, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMemcpy(dP, params, MLP_NPARAM * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dX, X, (size_t)n * MLP_IN * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dY, y, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && w) e = cudaMemcpy(dW, w, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dG, 0, (MLP_NPARAM + 1) * 4);
    if (e == cudaSuccess) e = cudaMemset(dM, 0, MLP_NPARAM * 4);
    if (e == cudaSuccess) e = cudaMemset(dV, 0, MLP_NPARAM * 4);
    std::vector<int32_t> perm(n);
    for (int32_t i = 0; i < n; ++i) perm[i] = i;
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int64_t step = 0;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        for (int32_t i = n - 1; i > 0; --i) {
            std::uniform_int_distribution<int32_t> d(0, i);
            std::swap(perm[i], perm[d(rng)]);
        }
        e = cudaMemcpyAsync(dI, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st);
        float* loss_slot = dG + MLP_NPARAM;
        if (e == cudaSuccess) e = cudaMemsetAsync(loss_slot, 0, 4, st);
        for (int32_t b0 = 0; b0 < n && e == cudaSuccess; b0 += batch) {
            const int32_t nb = std::min(batch, n - b0);
            k_mlp_fwd_bwd<<<(nb + MLP_TPB - 1) / MLP_TPB, MLP_TPB, 0, st>>>(
                dP, dX, dY, dW, dI + b0, nb, 1.0f / (float)nb, dG, loss_slot);
            ++step;
            const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
            k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(dP, dG, dM, dV, lr, b1, b2, eps, c1,
                                                            c2);
            note_launch(nullptr, 2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && epoch_loss_out) {
            float l = 0.0f;
            e = cudaMemcpyAsync(&l, loss_slot, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            // sum over batches of the mean batch loss -> mean per batch
            const int32_t nbatches = (n + batch - 1) / batch;
            epoch_loss_out[ep] = l / (float)nbatches;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpy(params, dP, MLP_NPARAM * 4, cudaMemcpyDeviceToHost);
    cudaFree(dP);
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dW);
    cudaFree(dG);
    cudaFree(dM);
    cudaFree(dV);
    cudaFree(dI);
    if (st) cudaStreamDestroy(st);
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "mlp train");
}

int rvsp_cuda_mlp_infer(const float* model, int32_t nfloats, const float* feat, const int32_t* ub,
                        int32_t n, float* mu_out, float* sigma_out, int32_t* cap_out) {
    if (!model || !feat || !ub || !cap_out) return RVSP_ERROR_NULL_POINTER;
    if (nfloats != kModelFloats || n <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
    MlpModel m;
    unpack(model, &m);
    float *dF = nullptr, *dMu = nullptr, *dSig = nullptr;
    int32_t *dU = nullptr, *dC = nullptr;
    cudaError_t e = cudaMalloc(&dF, (size_t)n * 16);
    if (e == cudaSuccess) e = cudaMalloc(&dU, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dC, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dMu, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dSig, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMemcpy(dF, feat, (size_t)n * 16, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dU, ub, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_mlp_infer<<<(n + 255) / 256, 256>>>(m, (const float4*)dF, dU, nullptr, n, dMu, dSig, dC);
        note_launch(nullptr, 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(cap_out, dC, (size_t)n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && mu_out) e = cudaMemcpy(mu_out, dMu, (size_t)n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && sigma_out)
        e = cudaMemcpy(sigma_out, dSig, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaFree(dF);
    cudaFree(dU);
    cudaFree(dC);
    cudaFree(dMu);
    cudaFree(dSig);
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "mlp infer");
}

}  // extern "C"
