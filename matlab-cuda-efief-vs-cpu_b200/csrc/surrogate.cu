// Surrogate MLP for adaptive frequency sweeps: (geometry, frequency) -> Zin.
//
// No counterpart in the reference.  The network maps normalised inputs
// (W, L, h, feed offset, f) through `n_layers` hidden layers of width
// `n_hidden` with SiLU to `n_out` outputs (Re, Im of the normalised Zin).
// Every linear layer computes with BF16 weights and FP32 accumulation; the
// optimizer keeps FP32 master weights and refreshes the BF16 copies after each
// Adam step.  Activations, gradients and moments are FP32.
//
// Parameter layout (FP32 master, also the host layout of get/set_params):
// for each linear layer l = 0..n_layers: W_l [out_l x in_l] row-major, then
// b_l [out_l].
//
// One training step (gather the minibatch, forward, MSE loss, backward,
// Adam) is a fixed sequence of kernels whose varying state -- the step count,
// hence the minibatch offset and Adam's bias correction -- lives in device
// memory, so the step is captured once into a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "efie_internal.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 16;

enum Epilogue { EPI_FWD_HIDDEN = 0, EPI_FWD_OUT = 1, EPI_BWD_DZ = 2, EPI_PARTIAL = 3 };
constexpr int KSPLIT = 512;   // K chunk of the weight-gradient products

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

template <typename T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// C[i][j] (M x N, row stride ldc) = sum_k A(i,k) B(k,j) with A(i,k) =
// A[i*sai + k*sak] (FP32) and B(k,j) = B[k*sbk + j*sbj]; 64x64 tiles, 4x4
// outputs per thread, FP32 accumulation.  blockIdx.z splits K in chunks of
// kchunk; EPI_PARTIAL stores chunk z's partial product at C + z M ldc, and
// k_sum_parts adds the chunks in order (bit-reproducible gradients).
template <typename TB, int EPI>
__global__ void __launch_bounds__(256) k_mlp_gemm(int M, int N, int K, const float *__restrict__ A, long sai,
                                                  long sak, const TB *__restrict__ B, long sbk, long sbj,
                                                  float *__restrict__ C, int ldc, const float *__restrict__ bias,
                                                  float *__restrict__ Aout, const float *__restrict__ Zprev,
                                                  int kchunk) {
    __shared__ float As[BK][BM + 4];
    __shared__ float Bs[BK][BN + 4];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int i0 = blockIdx.y * BM, j0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.f;
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        // A tile: BM x BK; B tile: BK x BN (4 elements per thread each)
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int e = tid + 256 * r;
            int ii, kk;
            if (sak == 1) { ii = e / BK; kk = e % BK; }   // contiguous along k
            else { ii = e % BM; kk = e / BM; }            // contiguous along i
            const int gi = i0 + ii, gk = k0 + kk;
            As[kk][ii] = (gi < M && gk < kend) ? A[(long)gi * sai + (long)gk * sak] : 0.f;
            int jj, kb;
            if (sbj == 1) { jj = e % BN; kb = e / BN; }
            else { jj = e / BK; kb = e % BK; }
            const int gj = j0 + jj, gkb = k0 + kb;
            Bs[kb][jj] = (gj < N && gkb < kend) ? to_f<TB>(B[(long)gkb * sbk + (long)gj * sbj]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            float x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                x[a] = As[kk][ty * 4 + a];
                y[a] = Bs[kk][tx * 4 + a];
            }
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) acc[a][b] = fmaf(x[a], y[b], acc[a][b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = i0 + ty * 4 + a, j = j0 + tx * 4 + b;
            if (i >= M || j >= N) continue;
            const long o = (long)i * ldc + j;
            if (EPI == EPI_FWD_HIDDEN) {
                const float z = acc[a][b] + bias[j];
                C[o] = z;
                Aout[o] = z * sigm(z);
            } else if (EPI == EPI_FWD_OUT) {
                C[o] = acc[a][b] + bias[j];
            } else if (EPI == EPI_BWD_DZ) {
                const float z = Zprev[o], s = sigm(z);
                C[o] = acc[a][b] * (s * (1.f + z * (1.f - s)));   // d silu / dz
            } else {
                C[(long)blockIdx.z * M * ldc + o] = acc[a][b];
            }
        }
}

// out[e] += sum_z part[z * count + e], z in order
__global__ void k_sum_parts(int nz, long count, const float *__restrict__ part, float *__restrict__ out) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    float t = out[e];
    for (int z = 0; z < nz; z++) t += part[(long)z * count + e];
    out[e] = t;
}

// db[j] += sum_i dZ[i][j]: one CTA per 32 columns, eight row lanes summed in
// a fixed order (bit-reproducible)
__global__ void __launch_bounds__(256) k_colsum(int M, int N, const float *__restrict__ dZ, float *__restrict__ db) {
    const int j = blockIdx.x * 32 + (threadIdx.x & 31);
    const int r = threadIdx.x >> 5;
    __shared__ float part[8][33];
    float s = 0.f;
    if (j < N)
        for (int i = r; i < M; i += 8) s += dZ[(long)i * N + j];
    part[r][threadIdx.x & 31] = s;
    __syncthreads();
    if (r == 0 && j < N) {
        float t = 0.f;
#pragma unroll
        for (int q = 0; q < 8; q++) t += part[q][threadIdx.x & 31];
        db[j] += t;
    }
}

// Rows perm[off + i] of X and T into the minibatch buffers; off from the
// run-local step count (off = (step mod nb) * bs).
__global__ void k_gather_batch(int bs, int nb, int n_in, int n_out, const int *__restrict__ perm,
                               const long long *__restrict__ step, const float *__restrict__ X,
                               const float *__restrict__ T, float *__restrict__ Xb, float *__restrict__ Tb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bs) return;
    const long long st = step[1];
    const int row = perm[(int)(st % nb) * bs + i];
    for (int c = 0; c < n_in; c++) Xb[(long)i * n_in + c] = X[(long)row * n_in + c];
    for (int c = 0; c < n_out; c++) Tb[(long)i * n_out + c] = T[(long)row * n_out + c];
}

// Mean squared error over the minibatch: dY = 2 (Y - T) / (bs n_out); the
// loss is added to hist[epoch] (epoch = run-local step / nb; the per-epoch
// mean over its minibatches) when hist is given, else to *loss.
__global__ void __launch_bounds__(256) k_mse(int bs, int n_out, const float *__restrict__ Y, const float *__restrict__ T,
                                             float *__restrict__ dY, const long long *__restrict__ step, int nb,
                                             double *__restrict__ hist, double *__restrict__ loss) {
    const int n = bs * n_out;
    const float scale = 1.0f / (float)n;
    float s = 0.f;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float d = Y[e] - T[e];
        dY[e] = 2.f * d * scale;
        s += d * d;
    }
    __shared__ float red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        double *dst = hist ? hist + (step[1] / nb) : loss;
        atomicAdd(dst, (double)t * (double)scale / (hist ? (double)nb : 1.0));
    }
}

// Adam with bias correction (t = global step + 1), FP32 master weights, BF16
// copies of the weight matrices (biases stay FP32).
__global__ void __launch_bounds__(256) k_adam(int n, float *__restrict__ w, const float *__restrict__ g,
                                              float *__restrict__ m, float *__restrict__ v,
                                              __nv_bfloat16 *__restrict__ wb, const long long *__restrict__ step,
                                              float lr, float b1, float b2, float eps, float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float t = (float)(step[0] + 1);
    const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_step_inc(long long *step) {
    step[0] += 1;   // Adam's step
    step[1] += 1;   // step of this training run
}

__global__ void k_to_bf16(int n, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace

struct efie_mlp {
    efie_ctx *ctx = nullptr;
    efie_mlp_config cfg{};
    int nl = 0;                                  // linear layers
    std::vector<int> fin, fout;                  // per layer
    std::vector<size_t> woff, boff;              // offsets into the parameter vector
    size_t np = 0;
    DevBuf w, wb, g, m, v;                       // params FP32, BF16 copy, grads, Adam moments
    DevBuf act;                                  // Z and A of every layer for `cap` rows
    DevBuf dz0, dz1;                             // backward ping-pong
    DevBuf gpart;                                // K-split partials of the weight gradients
    DevBuf Xd, Td, perm, Xb, Tb, dY, step, hist, loss;
    DevBuf Xin;                                  // inference input
    int cap = 0;                                 // rows the activation buffers hold
    int width = 0;                               // max(n_hidden, n_out): row stride of the buffers
    cudaGraphExec_t graph = nullptr;
    int graph_bs = 0, graph_nb = 0;
    efie_adam_opts graph_opts{};
    std::vector<void *> graph_ptrs;              // device buffers the captured step uses

    float *Z(int l) { return act.as<float>() + (size_t)cap * width * (2 * l); }
    float *A(int l) { return act.as<float>() + (size_t)cap * width * (2 * l + 1); }
    float *Y() { return Z(nl - 1); }
    std::vector<void *> step_ptrs() const {
        return {w.p,  wb.p, g.p,  m.p,  v.p,  act.p, dz0.p, dz1.p, gpart.p,
                Xd.p, Td.p, perm.p, Xb.p, Tb.p, dY.p, step.p, hist.p};
    }

    ~efie_mlp() {
        if (graph) cudaGraphExecDestroy(graph);
    }
};

namespace {

efie_status mlp_reserve(efie_mlp *p, int rows) {
    if (rows <= p->cap) return EFIE_OK;
    const int width = p->width;
    EFIE_TRY(p->act.reserve(sizeof(float) * (size_t)rows * width * 2 * p->nl));
    EFIE_TRY(p->dz0.reserve(sizeof(float) * (size_t)rows * width));
    EFIE_TRY(p->dz1.reserve(sizeof(float) * (size_t)rows * width));
    size_t wmax = 0;
    for (int l = 0; l < p->nl; l++) wmax = std::max(wmax, (size_t)p->fin[l] * p->fout[l]);
    EFIE_TRY(p->gpart.reserve(sizeof(float) * wmax * (size_t)cdiv(rows, KSPLIT)));
    p->cap = rows;
    if (p->graph) {  // the captured step addresses the old layout
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    return EFIE_OK;
}

// Forward of rows [0, n) of X (device, n x n_in) into the activation buffers.
efie_status mlp_forward(efie_mlp *p, const float *X, int n) {
    cudaStream_t s = p->ctx->stream;
    const float *in = X;
    for (int l = 0; l < p->nl; l++) {
        const int fi = p->fin[l], fo = p->fout[l];
        dim3 grid(cdiv(fo, BN), cdiv(n, BM), 1);
        const __nv_bfloat16 *W = p->wb.as<__nv_bfloat16>() + p->woff[l];
        const float *b = p->w.as<float>() + p->boff[l];
        // B(k, j) = W[j][k]
        if (l + 1 < p->nl)
            k_mlp_gemm<__nv_bfloat16, EPI_FWD_HIDDEN><<<grid, 256, 0, s>>>(n, fo, fi, in, fi, 1, W, 1, fi, p->Z(l), fo, b,
                                                                          p->A(l), nullptr, fi);
        else
            k_mlp_gemm<__nv_bfloat16, EPI_FWD_OUT><<<grid, 256, 0, s>>>(n, fo, fi, in, fi, 1, W, 1, fi, p->Z(l), fo, b,
                                                                       nullptr, nullptr, fi);
        EFIE_CUDA(cudaGetLastError());
        in = p->A(l);
    }
    return EFIE_OK;
}

// Backward from dY (device, n x n_out) with X the network input; gradients
// are added to p->g (the caller zeroes it).
efie_status mlp_backward(efie_mlp *p, const float *X, const float *dY, int n) {
    cudaStream_t s = p->ctx->stream;
    const int kchunk = KSPLIT;
    const float *dz = dY;
    float *bufs[2] = {p->dz0.as<float>(), p->dz1.as<float>()};
    int pb = 0;
    for (int l = p->nl - 1; l >= 0; l--) {
        const int fi = p->fin[l], fo = p->fout[l];
        const float *ain = l > 0 ? p->A(l - 1) : X;
        float *gW = p->g.as<float>() + p->woff[l], *gb = p->g.as<float>() + p->boff[l];
        // dW[o][i] += sum_m dz[m][o] ain[m][i]:  A(i=o, k=m) = dz[m*fo + o], B(k=m, j=i) = ain[m*fi + i]
        dim3 gw(cdiv(fi, BN), cdiv(fo, BM), cdiv(n, kchunk));
        k_mlp_gemm<float, EPI_PARTIAL><<<gw, 256, 0, s>>>(fo, fi, n, dz, 1, fo, ain, fi, 1, p->gpart.as<float>(), fi,
                                                         nullptr, nullptr, nullptr, kchunk);
        const long cnt = (long)fo * fi;
        k_sum_parts<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>((int)gw.z, cnt, p->gpart.as<float>(), gW);
        k_colsum<<<dim3(cdiv(fo, 32), 1), 256, 0, s>>>(n, fo, dz, gb);
        EFIE_CUDA(cudaGetLastError());
        if (l > 0) {
            // dZ_{l-1}[m][i] = (sum_o dz[m][o] W[o][i]) * silu'(Z_{l-1}[m][i])
            float *out = bufs[pb];
            pb ^= 1;
            const __nv_bfloat16 *W = p->wb.as<__nv_bfloat16>() + p->woff[l];
            dim3 gd(cdiv(fi, BN), cdiv(n, BM), 1);
            k_mlp_gemm<__nv_bfloat16, EPI_BWD_DZ><<<gd, 256, 0, s>>>(n, fi, fo, dz, fo, 1, W, fi, 1, out, fi, nullptr,
                                                                    nullptr, p->Z(l - 1), fo);
            EFIE_CUDA(cudaGetLastError());
            dz = out;
        }
    }
    return EFIE_OK;
}

efie_status mlp_upload_bf16(efie_mlp *p) {
    const int n = (int)p->np;
    k_to_bf16<<<cdiv(n, 256), 256, 0, p->ctx->stream>>>(n, p->w.as<float>(), p->wb.as<__nv_bfloat16>());
    EFIE_CUDA(cudaGetLastError());
    return EFIE_OK;
}

// One training step on the stream (captured into the graph).
efie_status mlp_train_step(efie_mlp *p, int bs, int nb, const efie_adam_opts &o) {
    cudaStream_t s = p->ctx->stream;
    const int ni = p->cfg.n_in, no = p->cfg.n_out;
    k_gather_batch<<<cdiv(bs, 128), 128, 0, s>>>(bs, nb, ni, no, p->perm.as<int>(), p->step.as<long long>(),
                                                 p->Xd.as<float>(), p->Td.as<float>(), p->Xb.as<float>(),
                                                 p->Tb.as<float>());
    EFIE_CUDA(cudaGetLastError());
    EFIE_TRY(mlp_forward(p, p->Xb.as<float>(), bs));
    k_mse<<<std::min(64, cdiv((long)bs * no, 256)), 256, 0, s>>>(bs, no, p->Y(), p->Tb.as<float>(), p->dY.as<float>(),
                                                                 p->step.as<long long>(), nb, p->hist.as<double>(),
                                                                 nullptr);
    EFIE_CUDA(cudaGetLastError());
    EFIE_CUDA(cudaMemsetAsync(p->g.p, 0, sizeof(float) * p->np, s));
    EFIE_TRY(mlp_backward(p, p->Xb.as<float>(), p->dY.as<float>(), bs));
    const int n = (int)p->np;
    k_adam<<<cdiv(n, 256), 256, 0, s>>>(n, p->w.as<float>(), p->g.as<float>(), p->m.as<float>(), p->v.as<float>(),
                                        p->wb.as<__nv_bfloat16>(), p->step.as<long long>(), o.lr, o.beta1, o.beta2,
                                        o.eps, o.weight_decay);
    k_step_inc<<<1, 1, 0, s>>>(p->step.as<long long>());
    EFIE_CUDA(cudaGetLastError());
    return EFIE_OK;
}

}  // namespace

extern "C" {

void efie_mlp_config_default(efie_mlp_config *c) {
    c->n_in = 5;
    c->n_hidden = 256;
    c->n_layers = 4;
    c->n_out = 2;
    c->seed = 1;
}

void efie_adam_opts_default(efie_adam_opts *o) {
    o->lr = 1e-3f;
    o->beta1 = 0.9f;
    o->beta2 = 0.999f;
    o->eps = 1e-8f;
    o->weight_decay = 0.f;
    o->batch = 1024;
    o->epochs = 100;
    o->seed = 1;
}

efie_status efie_mlp_create(efie_ctx *ctx, const efie_mlp_config *cfg, efie_mlp **out) {
    if (!ctx || !cfg || !out) return efie_fail(EFIE_ERR_ARGS, "null argument");
    *out = nullptr;
    if (cfg->n_in < 1 || cfg->n_in > 64 || cfg->n_out < 1 || cfg->n_out > 64 || cfg->n_hidden < 1 ||
        cfg->n_hidden > 4096 || cfg->n_layers < 1 || cfg->n_layers > EFIE_MLP_MAX_LAYERS)
        return efie_fail(EFIE_ERR_ARGS, "MLP shape out of range");
    DeviceGuard dg(ctx->device);
    efie_mlp *p = new (std::nothrow) efie_mlp();
    if (!p) return efie_fail(EFIE_ERR_NOMEM, "out of host memory");
    p->ctx = ctx;
    p->cfg = *cfg;
    p->nl = cfg->n_layers + 1;
    p->width = std::max(cfg->n_hidden, cfg->n_out);
    for (int l = 0; l < p->nl; l++) {
        p->fin.push_back(l == 0 ? cfg->n_in : cfg->n_hidden);
        p->fout.push_back(l + 1 == p->nl ? cfg->n_out : cfg->n_hidden);
        p->woff.push_back(p->np);
        p->np += (size_t)p->fin[l] * p->fout[l];
        p->boff.push_back(p->np);
        p->np += p->fout[l];
    }
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases
    std::vector<float> h(p->np);
    std::mt19937_64 rng(cfg->seed);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    for (int l = 0; l < p->nl; l++) {
        const float a = 1.f / std::sqrt((float)p->fin[l]);
        for (size_t e = 0; e < (size_t)p->fin[l] * p->fout[l]; e++) h[p->woff[l] + e] = a * u(rng);
        for (int e = 0; e < p->fout[l]; e++) h[p->boff[l] + e] = a * u(rng);
    }
    efie_status s = EFIE_OK;
    if (s == EFIE_OK) s = p->w.reserve(sizeof(float) * p->np);
    if (s == EFIE_OK) s = p->wb.reserve(sizeof(__nv_bfloat16) * p->np);
    if (s == EFIE_OK) s = p->g.reserve(sizeof(float) * p->np);
    if (s == EFIE_OK) s = p->m.reserve(sizeof(float) * p->np);
    if (s == EFIE_OK) s = p->v.reserve(sizeof(float) * p->np);
    if (s == EFIE_OK) s = p->step.reserve(2 * sizeof(long long));
    if (s == EFIE_OK) s = p->loss.reserve(sizeof(double));
    if (s == EFIE_OK) s = efie_cuda_check(cudaMemcpyAsync(p->w.p, h.data(), sizeof(float) * p->np,
                                                          cudaMemcpyHostToDevice, ctx->stream), "upload");
    if (s == EFIE_OK) s = efie_cuda_check(cudaMemsetAsync(p->m.p, 0, sizeof(float) * p->np, ctx->stream), "memset");
    if (s == EFIE_OK) s = efie_cuda_check(cudaMemsetAsync(p->v.p, 0, sizeof(float) * p->np, ctx->stream), "memset");
    if (s == EFIE_OK) s = efie_cuda_check(cudaMemsetAsync(p->step.p, 0, 2 * sizeof(long long), ctx->stream), "memset");
    if (s == EFIE_OK) s = mlp_upload_bf16(p);
    if (s == EFIE_OK) s = efie_cuda_check(cudaStreamSynchronize(ctx->stream), "sync");
    if (s != EFIE_OK) {
        delete p;
        return s;
    }
    *out = p;
    return EFIE_OK;
}

void efie_mlp_destroy(efie_mlp *p) {
    if (!p) return;
    DeviceGuard dg(p->ctx->device);
    delete p;
}

int64_t efie_mlp_num_params(const efie_mlp *p) { return p ? (int64_t)p->np : 0; }

efie_status efie_mlp_get_params(efie_mlp *p, float *params) {
    if (!p || !params) return efie_fail(EFIE_ERR_ARGS, "null argument");
    DeviceGuard dg(p->ctx->device);
    EFIE_CUDA(cudaMemcpyAsync(params, p->w.p, sizeof(float) * p->np, cudaMemcpyDeviceToHost, p->ctx->stream));
    EFIE_CUDA(cudaStreamSynchronize(p->ctx->stream));
    return EFIE_OK;
}

efie_status efie_mlp_set_params(efie_mlp *p, const float *params) {
    if (!p || !params) return efie_fail(EFIE_ERR_ARGS, "null argument");
    DeviceGuard dg(p->ctx->device);
    cudaStream_t s = p->ctx->stream;
    EFIE_CUDA(cudaMemcpyAsync(p->w.p, params, sizeof(float) * p->np, cudaMemcpyHostToDevice, s));
    EFIE_CUDA(cudaMemsetAsync(p->m.p, 0, sizeof(float) * p->np, s));
    EFIE_CUDA(cudaMemsetAsync(p->v.p, 0, sizeof(float) * p->np, s));
    EFIE_CUDA(cudaMemsetAsync(p->step.p, 0, 2 * sizeof(long long), s));
    EFIE_TRY(mlp_upload_bf16(p));
    EFIE_CUDA(cudaStreamSynchronize(s));
    return EFIE_OK;
}

efie_status efie_mlp_forward(efie_mlp *p, const float *X, int32_t n, float *Y) {
    if (!p || (!X && n > 0) || (!Y && n > 0) || n < 0) return efie_fail(EFIE_ERR_ARGS, "bad argument");
    if (n == 0) return EFIE_OK;
    DeviceGuard dg(p->ctx->device);
    cudaStream_t s = p->ctx->stream;
    const int chunk = std::max(p->cap, std::min(n, 1 << 14));
    EFIE_TRY(mlp_reserve(p, std::min(n, chunk)));
    EFIE_TRY(p->Xin.reserve(sizeof(float) * (size_t)std::min(n, chunk) * p->cfg.n_in));
    for (int r0 = 0; r0 < n; r0 += chunk) {
        const int m = std::min(chunk, n - r0);
        EFIE_CUDA(cudaMemcpyAsync(p->Xin.p, X + (size_t)r0 * p->cfg.n_in, sizeof(float) * m * p->cfg.n_in,
                                  cudaMemcpyHostToDevice, s));
        EFIE_TRY(mlp_forward(p, p->Xin.as<float>(), m));
        EFIE_CUDA(cudaMemcpyAsync(Y + (size_t)r0 * p->cfg.n_out, p->Y(), sizeof(float) * m * p->cfg.n_out,
                                  cudaMemcpyDeviceToHost, s));
    }
    EFIE_CUDA(cudaStreamSynchronize(s));
    return EFIE_OK;
}

efie_status efie_mlp_loss_grad(efie_mlp *p, const float *X, const float *T, int32_t n, double *loss, float *grad) {
    if (!p || !X || !T || n < 1) return efie_fail(EFIE_ERR_ARGS, "bad argument");
    DeviceGuard dg(p->ctx->device);
    cudaStream_t s = p->ctx->stream;
    const int ni = p->cfg.n_in, no = p->cfg.n_out;
    EFIE_TRY(mlp_reserve(p, n));
    EFIE_TRY(p->Xb.reserve(sizeof(float) * (size_t)n * ni));
    EFIE_TRY(p->Tb.reserve(sizeof(float) * (size_t)n * no));
    EFIE_TRY(p->dY.reserve(sizeof(float) * (size_t)n * no));
    EFIE_CUDA(cudaMemcpyAsync(p->Xb.p, X, sizeof(float) * n * ni, cudaMemcpyHostToDevice, s));
    EFIE_CUDA(cudaMemcpyAsync(p->Tb.p, T, sizeof(float) * n * no, cudaMemcpyHostToDevice, s));
    EFIE_TRY(mlp_forward(p, p->Xb.as<float>(), n));
    EFIE_CUDA(cudaMemsetAsync(p->loss.p, 0, sizeof(double), s));
    k_mse<<<std::min(64, cdiv((long)n * no, 256)), 256, 0, s>>>(n, no, p->Y(), p->Tb.as<float>(), p->dY.as<float>(),
                                                                p->step.as<long long>(), 1, nullptr,
                                                                p->loss.as<double>());
    EFIE_CUDA(cudaGetLastError());
    EFIE_CUDA(cudaMemsetAsync(p->g.p, 0, sizeof(float) * p->np, s));
    EFIE_TRY(mlp_backward(p, p->Xb.as<float>(), p->dY.as<float>(), n));
    if (loss) EFIE_CUDA(cudaMemcpyAsync(loss, p->loss.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (grad) EFIE_CUDA(cudaMemcpyAsync(grad, p->g.p, sizeof(float) * p->np, cudaMemcpyDeviceToHost, s));
    EFIE_CUDA(cudaStreamSynchronize(s));
    return EFIE_OK;
}

efie_status efie_mlp_train(efie_mlp *p, const float *X, const float *T, int32_t n, const efie_adam_opts *opts,
                           double *loss_history) {
    if (!p || !X || !T || n < 1) return efie_fail(EFIE_ERR_ARGS, "bad argument");
    efie_adam_opts o;
    if (opts) o = *opts;
    else efie_adam_opts_default(&o);
    if (o.epochs < 0 || o.batch < 1) return efie_fail(EFIE_ERR_ARGS, "bad training options");
    DeviceGuard dg(p->ctx->device);
    cudaStream_t s = p->ctx->stream;
    const int ni = p->cfg.n_in, no = p->cfg.n_out;
    const int bs = std::min<int>(o.batch, n);
    const int nb = n / bs;  // full minibatches per epoch (the permutation changes every epoch)
    EFIE_TRY(mlp_reserve(p, bs));
    EFIE_TRY(p->Xd.reserve(sizeof(float) * (size_t)n * ni));
    EFIE_TRY(p->Td.reserve(sizeof(float) * (size_t)n * no));
    EFIE_TRY(p->perm.reserve(sizeof(int) * (size_t)n));
    EFIE_TRY(p->Xb.reserve(sizeof(float) * (size_t)bs * ni));
    EFIE_TRY(p->Tb.reserve(sizeof(float) * (size_t)bs * no));
    EFIE_TRY(p->dY.reserve(sizeof(float) * (size_t)bs * no));
    EFIE_TRY(p->hist.reserve(sizeof(double) * (size_t)std::max(1, o.epochs)));
    EFIE_CUDA(cudaMemcpyAsync(p->Xd.p, X, sizeof(float) * (size_t)n * ni, cudaMemcpyHostToDevice, s));
    EFIE_CUDA(cudaMemcpyAsync(p->Td.p, T, sizeof(float) * (size_t)n * no, cudaMemcpyHostToDevice, s));
    EFIE_CUDA(cudaMemsetAsync(p->hist.p, 0, sizeof(double) * std::max(1, o.epochs), s));
    EFIE_CUDA(cudaMemsetAsync(p->step.as<long long>() + 1, 0, sizeof(long long), s));
    const bool rebuild = !p->graph || p->graph_bs != bs || p->graph_nb != nb || p->graph_ptrs != p->step_ptrs() ||
                         std::memcmp(&p->graph_opts, &o, sizeof(o)) != 0;
    if (rebuild) {
        if (p->graph) {
            cudaGraphExecDestroy(p->graph);
            p->graph = nullptr;
        }
        cudaStream_t cap;
        EFIE_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaStream_t saved = p->ctx->stream;
        p->ctx->stream = cap;
        cudaGraph_t g = nullptr;
        efie_status st = efie_cuda_check(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "capture");
        if (st == EFIE_OK) {
            st = mlp_train_step(p, bs, nb, o);
            cudaError_t e = cudaStreamEndCapture(cap, &g);
            if (st == EFIE_OK) st = efie_cuda_check(e, "end capture");
        }
        if (st == EFIE_OK) st = efie_cuda_check(cudaGraphInstantiate(&p->graph, g, 0), "instantiate");
        if (g) cudaGraphDestroy(g);
        p->ctx->stream = saved;
        cudaStreamDestroy(cap);
        if (st != EFIE_OK) return st;
        p->graph_bs = bs;
        p->graph_nb = nb;
        p->graph_opts = o;
        p->graph_ptrs = p->step_ptrs();
    }
    std::mt19937_64 rng(o.seed);
    std::vector<int> perm(n);
    for (int e = 0; e < o.epochs; e++) {
        for (int i = 0; i < n; i++) perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        EFIE_CUDA(cudaMemcpyAsync(p->perm.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        for (int b = 0; b < nb; b++) EFIE_CUDA(cudaGraphLaunch(p->graph, s));
        // perm is reused next epoch: wait until this epoch's gathers have read it
        EFIE_CUDA(cudaStreamSynchronize(s));
    }
    if (loss_history && o.epochs > 0)
        EFIE_CUDA(cudaMemcpyAsync(loss_history, p->hist.p, sizeof(double) * o.epochs, cudaMemcpyDeviceToHost, s));
    EFIE_CUDA(cudaStreamSynchronize(s));
    return EFIE_OK;
}

}  // extern "C"
