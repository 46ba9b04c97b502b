// The learned warm start: a small MLP (in -> 128 -> 128 -> out, tanh hidden
// layers) that maps a sweep point's parameters to a Newton start point. Its
// dense layers run on the tensor cores (k_gemm_tc: tcgen05.mma, BF16 operands,
// FP32 accumulation in tensor memory); training is this file's own forward,
// backward (MSE loss) and Adam kernels with FP32 master weights and BF16
// copies for the GEMMs. Inputs and targets are standardized per feature;
// predictions are de-standardized to FP64.
//
// No counterpart in the reference: ESPice warm-starts lanes from a nominal
// operating point (--warm-start); this module only changes where Newton
// starts, never the Newton that judges convergence.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/espice_learned.h"
#include "mlp_gemm.cuh"

using namespace espl::mlp;

namespace {

inline int up16(int v) { return (v + 15) & ~15; }

__global__ void k_to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16(src[i]);
}

// Standardized, zero-padded rows: dst[r, j] = (src[r, j] - mean[j]) / std[j]
// for j < cols, 0 for cols <= j < ld.
__global__ void k_standardize(const double* __restrict__ src, int rows, int cols, int ld, const float* __restrict__ mean,
                              const float* __restrict__ stdv, float* __restrict__ dst_f, __nv_bfloat16* __restrict__ dst_b) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)rows * ld) return;
    int r = (int)(i / ld), j = (int)(i % ld);
    float v = 0.0f;
    if (j < cols) v = (float)((src[(long long)r * cols + j] - (double)mean[j]) / (double)stdv[j]);
    if (dst_f) dst_f[i] = v;
    if (dst_b) dst_b[i] = __float2bfloat16(v);
}

// dY = 2 (Y - T) / (rows * cols) on the real columns (0 on the padding),
// its BF16 copy, and the loss sum.
__global__ void k_mse_grad(const float* __restrict__ y, const float* __restrict__ t, int rows, int cols, int ld,
                           float* __restrict__ dy, __nv_bfloat16* __restrict__ dyb, double* __restrict__ loss) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < (long long)rows * ld) {
        int j = (int)(i % ld);
        float g = 0.0f;
        if (j < cols) {
            float e = y[i] - t[i];
            l = e * e;
            g = 2.0f * e / ((float)rows * (float)cols);
        }
        dy[i] = g;
        dyb[i] = __float2bfloat16(g);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, (double)l);
}

// dZ = dH * (1 - H^2) (tanh), with its BF16 copy.
__global__ void k_tanh_back(const float* __restrict__ dh, const float* __restrict__ h, long long n,
                            float* __restrict__ dz, __nv_bfloat16* __restrict__ dzb) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = h[i];
    float g = dh[i] * (1.0f - v * v);
    dz[i] = g;
    dzb[i] = __float2bfloat16(g);
}

// out[j] += sum over rows of src[r, j] (bias gradients).
__global__ void k_colsum(const float* __restrict__ src, int rows, int ld, int cols, float* __restrict__ out) {
    int j = blockIdx.x;
    if (j >= cols) return;
    float s = 0.0f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += src[(long long)r * ld + j];
    __shared__ float part[256];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] += part[0];
}

// Adam with bias correction on the FP32 master parameters.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_destandardize(const float* __restrict__ y, int rows, int cols, int ld, const float* __restrict__ mean,
                                const float* __restrict__ stdv, double* __restrict__ out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)rows * cols) return;
    int r = (int)(i / cols), j = (int)(i % cols);
    out[i] = (double)y[(long long)r * ld + j] * (double)stdv[j] + (double)mean[j];
}

// Rows perm[0 .. rows) of the resident data set into the batch buffers.
__global__ void k_gather_rows(const __nv_bfloat16* __restrict__ xs, const float* __restrict__ ts,
                              const uint32_t* __restrict__ perm, int rows, int dp, int op,
                              __nv_bfloat16* __restrict__ xb, float* __restrict__ t) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nx = (long long)rows * dp, nt = (long long)rows * op;
    if (i < nx) {
        int r = (int)(i / dp), j = (int)(i % dp);
        xb[i] = xs[(long long)perm[r] * dp + j];
    }
    if (i < nt) {
        int r = (int)(i / op), j = (int)(i % op);
        t[i] = ts[(long long)perm[r] * op + j];
    }
}

inline unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// The BF16 weight image (weight_image_bytes): W1, W2, W3 from the FP32
// master weights as K-major core-matrix tiles, back to back.
__global__ void k_pack_image(const float* __restrict__ w1, const float* __restrict__ w2, const float* __restrict__ w3,
                             int dp, int op, unsigned char* __restrict__ image) {
    const long long n1 = 128LL * dp, n2 = 128LL * 128, n3 = (long long)op * 128;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n1) {
        const int r = (int)(i / dp), k = (int)(i % dp);
        *reinterpret_cast<__nv_bfloat16*>(image + tile_off_k(r, k, dp)) = __float2bfloat16(w1[i]);
        return;
    }
    i -= n1;
    unsigned char* t2 = image + n1 * 2;
    if (i < n2) {
        const int r = (int)(i / 128), k = (int)(i % 128);
        *reinterpret_cast<__nv_bfloat16*>(t2 + tile_off_k(r, k, 128)) = __float2bfloat16(w2[i]);
        return;
    }
    i -= n2;
    unsigned char* t3 = t2 + n2 * 2;
    if (i < n3) {
        const int r = (int)(i / 128), k = (int)(i % 128);
        *reinterpret_cast<__nv_bfloat16*>(t3 + tile_off_k(r, k, 128)) = __float2bfloat16(w3[i]);
    }
}

// Per column j of a rows x cols FP64 matrix (row-major): out[2 j] = the sum
// and out[2 j + 1] = the sum of squares over the rows. One block per column.
__global__ void k_col_stats(const double* __restrict__ a, long long rows, int cols, double* __restrict__ out) {
    const int j = blockIdx.x;
    double s = 0.0, s2 = 0.0;
    for (long long r = threadIdx.x; r < rows; r += blockDim.x) {
        const double v = a[r * cols + j];
        s += v;
        s2 += v * v;
    }
    __shared__ double ps[256], ps2[256];
    ps[threadIdx.x] = s;
    ps2[threadIdx.x] = s2;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            ps[threadIdx.x] += ps[threadIdx.x + w];
            ps2[threadIdx.x] += ps2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * j] = ps[0];
        out[2 * j + 1] = ps2[0];
    }
}

struct InferArgs {
    const double* x;          // rows x in_dim, raw parameters
    double* y;                // rows x out_dim, de-standardized predictions
    const float *w1, *b1, *w2, *b2, *w3, *b3;  // FP32 master weights (padded layouts)
    const float *in_mean, *in_std, *out_mean, *out_std;
    int rows, in_dim, dp, out_dim, op;
    int* err;
};

// The whole network for one 128-row tile in one CTA (mlp_layers): the
// standardized input tile and the three weight matrices in shared memory,
// the output layer de-standardized to FP64.
__global__ void __launch_bounds__(128) k_mlp_infer(InferArgs g) {
    extern __shared__ __align__(1024) unsigned char dsm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int H = 128, dp = g.dp, op = g.op;
    unsigned char* sx = dsm;                        // 128 x dp
    unsigned char* sw1 = sx + 128 * dp * 2;         // 128 x dp
    unsigned char* sw2 = sw1 + 128 * dp * 2;        // 128 x 128
    unsigned char* sw3 = sw2 + 128 * 128 * 2;       // op x 128
    unsigned char* sh = sw3 + (size_t)op * 128 * 2; // 128 x 128 activations
    const int warp = threadIdx.x >> 5;
    const int r0 = blockIdx.x * 128;
    if (threadIdx.x == 0) {
        mbar_init1(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(128u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // operands: standardized inputs and the BF16 weights
    for (int e = threadIdx.x; e < 128 * dp; e += blockDim.x) {
        int r = e / dp, k = e % dp;
        float v = 0.0f;
        if (r0 + r < g.rows && k < g.in_dim)
            v = (float)((g.x[(long long)(r0 + r) * g.in_dim + k] - (double)g.in_mean[k]) / (double)g.in_std[k]);
        *reinterpret_cast<__nv_bfloat16*>(sx + tile_off_k(r, k, dp)) = __float2bfloat16(v);
    }
    stage_weights(sw1, g.w1, H, dp);
    stage_weights(sw2, g.w2, H, H);
    stage_weights(sw3, g.w3, op, H);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    mlp_layers(sx, sw1, sw2, sw3, sh, g.b1, g.b2, g.b3, dp, op, g.out_dim, tmem, &bar, &failed,
               [&](int row, int o, float v) {
                   if (r0 + row < g.rows)
                       g.y[(long long)(r0 + row) * g.out_dim + o] =
                           (double)v * (double)g.out_std[o] + (double)g.out_mean[o];
               });
    if (failed && threadIdx.x == 0) atomicExch(g.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
}

}  // namespace

struct espl_mlp {
    int device = 0;
    int D = 0, Dp = 0, H = 128, O = 0, Op = 0, cap = 0;
    // parameters, packed: W1 [H x Dp], b1 [H], W2 [H x H], b2 [H], W3 [Op x H], b3 [Op]
    long long off_w1 = 0, off_b1 = 0, off_w2 = 0, off_b2 = 0, off_w3 = 0, off_b3 = 0, n_par = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *w1b = nullptr, *w2b = nullptr, *w3b = nullptr;
    float *in_mean = nullptr, *in_std = nullptr, *out_mean = nullptr, *out_std = nullptr;
    float* out_gain = nullptr;  // out_std, 0 for an output constant over the training set
    bool scaled = false;
    // the BF16 weight image of the step predictor, rebuilt when the weights
    // have changed (weights_version) since it was packed (image_version)
    unsigned char* image = nullptr;
    uint64_t weights_version = 1, image_version = 0;
    // batch buffers (cap rows)
    double *x_raw = nullptr, *y_raw = nullptr;
    __nv_bfloat16 *xb = nullptr, *h1b = nullptr, *h2b = nullptr, *dyb = nullptr, *dzb = nullptr;
    float *t = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr, *dy = nullptr, *dh = nullptr, *dz = nullptr;
    double* loss = nullptr;
    int* err = nullptr;
    long long adam_t = 0;
    double last_train_ms = 0.0;  // device time of the last training (events on the stream)
    double last_predict_ms = 0.0;  // device time of the last espl_mlp_predict (copies and kernel)
    // espl_mlp_predict's device buffers, grown on demand and kept until destroy
    double *pred_x = nullptr, *pred_y = nullptr;
    size_t pred_rows = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;
    std::string msg;
};

namespace {

#define MCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            if (h) h->msg = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            return e_ == cudaErrorMemoryAllocation ? (espl_status)ESPL_OUT_OF_MEMORY                \
                                                   : (espl_status)ESPL_DRIVER;                      \
        }                                                                                           \
    } while (0)

template <typename T>
espl_status alloc(espl_mlp* h, T** out, size_t count) {
    void* q = nullptr;
    MCK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    MCK(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), h->stream));
    h->owned.push_back(q);
    *out = static_cast<T*>(q);
    return ESPL_OK;
}

// One GEMM C = A B^T through the tensor cores (see mlp_gemm.cuh).
template <int EPI>
espl_status gemm(espl_mlp* h, const __nv_bfloat16* a, long long sam, long long sak, const __nv_bfloat16* b,
                 long long sbn, long long sbk, float* c, int ldc, int M, int N, int K, const float* bias = nullptr,
                 __nv_bfloat16* cb = nullptr, int splits = 1) {
    GemmArgs g{a, b, sam, sak, sbn, sbk, c, cb, bias, M, N, K, ldc, 0, h->err};
    int kps = (K + splits - 1) / splits;
    kps = (kps + kBK - 1) / kBK * kBK;
    g.k_per_split = std::max(kps, kBK);
    int gz = (K + g.k_per_split - 1) / g.k_per_split;
    if (N <= 16) {
        dim3 grid((M + kBM - 1) / kBM, (N + 15) / 16, gz);
        k_gemm_tc<16, EPI><<<grid, kGemmThreads, 0, h->stream>>>(g);
    } else if (N <= 32) {
        dim3 grid((M + kBM - 1) / kBM, (N + 31) / 32, gz);
        k_gemm_tc<32, EPI><<<grid, kGemmThreads, 0, h->stream>>>(g);
    } else {
        dim3 grid((M + kBM - 1) / kBM, (N + 127) / 128, gz);
        k_gemm_tc<128, EPI><<<grid, kGemmThreads, 0, h->stream>>>(g);
    }
    MCK(cudaGetLastError());
    return ESPL_OK;
}

espl_status refresh_bf16(espl_mlp* h) {
    k_to_bf16<<<blocks((long long)h->H * h->Dp), 256, 0, h->stream>>>(h->p + h->off_w1, h->w1b, (long long)h->H * h->Dp);
    k_to_bf16<<<blocks((long long)h->H * h->H), 256, 0, h->stream>>>(h->p + h->off_w2, h->w2b, (long long)h->H * h->H);
    k_to_bf16<<<blocks((long long)h->Op * h->H), 256, 0, h->stream>>>(h->p + h->off_w3, h->w3b, (long long)h->Op * h->H);
    MCK(cudaGetLastError());
    h->weights_version++;
    return ESPL_OK;
}

// Forward of `rows` standardized rows already in xb: h1, h2 (FP32 + BF16), y.
espl_status forward(espl_mlp* h, int rows) {
    espl_status s;
    const int H = h->H;
    if ((s = gemm<kEpiBiasTanh>(h, h->xb, h->Dp, 1, h->w1b, h->Dp, 1, h->h1, H, rows, H, h->Dp, h->p + h->off_b1,
                                h->h1b)))
        return s;
    if ((s = gemm<kEpiBiasTanh>(h, h->h1b, H, 1, h->w2b, H, 1, h->h2, H, rows, H, H, h->p + h->off_b2, h->h2b)))
        return s;
    return gemm<kEpiBias>(h, h->h2b, H, 1, h->w3b, H, 1, h->y, h->Op, rows, h->Op, H, h->p + h->off_b3);
}

// Gradients (into h->g) of `rows` rows with targets in h->t; the summed
// squared error is added to *loss.
espl_status backward(espl_mlp* h, int rows, double* loss) {
    espl_status s;
    const int H = h->H, Op = h->Op, Dp = h->Dp;
    MCK(cudaMemsetAsync(h->g, 0, sizeof(float) * h->n_par, h->stream));
    k_mse_grad<<<blocks((long long)rows * Op), 256, 0, h->stream>>>(h->y, h->t, rows, h->O, Op, h->dy, h->dyb,
                                                                    loss);
    const int splits = std::max(1, std::min(64, rows / 256));
    // layer 3: dW3 = dY^T H2, db3 = colsum dY, dH2 = dY W3
    if ((s = gemm<kEpiAtomic>(h, h->dyb, 1, Op, h->h2b, 1, H, h->g + h->off_w3, H, Op, H, rows, nullptr, nullptr,
                              splits)))
        return s;
    k_colsum<<<Op, 256, 0, h->stream>>>(h->dy, rows, Op, Op, h->g + h->off_b3);
    if ((s = gemm<kEpiStore>(h, h->dyb, Op, 1, h->w3b, 1, H, h->dh, H, rows, H, Op))) return s;
    k_tanh_back<<<blocks((long long)rows * H), 256, 0, h->stream>>>(h->dh, h->h2, (long long)rows * H, h->dz, h->dzb);
    // layer 2
    if ((s = gemm<kEpiAtomic>(h, h->dzb, 1, H, h->h1b, 1, H, h->g + h->off_w2, H, H, H, rows, nullptr, nullptr,
                              splits)))
        return s;
    k_colsum<<<H, 256, 0, h->stream>>>(h->dz, rows, H, H, h->g + h->off_b2);
    if ((s = gemm<kEpiStore>(h, h->dzb, H, 1, h->w2b, 1, H, h->dh, H, rows, H, H))) return s;
    k_tanh_back<<<blocks((long long)rows * H), 256, 0, h->stream>>>(h->dh, h->h1, (long long)rows * H, h->dz, h->dzb);
    // layer 1
    if ((s = gemm<kEpiAtomic>(h, h->dzb, 1, H, h->xb, 1, Dp, h->g + h->off_w1, Dp, H, Dp, rows, nullptr, nullptr,
                              splits)))
        return s;
    k_colsum<<<H, 256, 0, h->stream>>>(h->dz, rows, H, H, h->g + h->off_b1);
    MCK(cudaGetLastError());
    return ESPL_OK;
}

espl_status check_err(espl_mlp* h) {
    int e = 0;
    MCK(cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    if (e) {
        h->msg = "a tensor-core GEMM wait ran out";
        return ESPL_TIMEOUT;
    }
    return ESPL_OK;
}

// Uploads rows [r0, r0 + rows) of x (and y) standardized into the batch buffers.
espl_status upload(espl_mlp* h, const double* x, const double* y, const std::vector<uint32_t>* order, long long r0,
                   int rows) {
    std::vector<double> xs, ys;
    const double* xp = x + r0 * h->D;
    const double* yp = y ? y + r0 * h->O : nullptr;
    if (order) {
        xs.resize((size_t)rows * h->D);
        if (y) ys.resize((size_t)rows * h->O);
        for (int r = 0; r < rows; r++) {
            uint32_t src = (*order)[r0 + r];
            std::memcpy(&xs[(size_t)r * h->D], x + (size_t)src * h->D, sizeof(double) * h->D);
            if (y) std::memcpy(&ys[(size_t)r * h->O], y + (size_t)src * h->O, sizeof(double) * h->O);
        }
        xp = xs.data();
        yp = y ? ys.data() : nullptr;
    }
    MCK(cudaMemcpyAsync(h->x_raw, xp, sizeof(double) * rows * h->D, cudaMemcpyHostToDevice, h->stream));
    k_standardize<<<blocks((long long)rows * h->Dp), 256, 0, h->stream>>>(h->x_raw, rows, h->D, h->Dp, h->in_mean,
                                                                          h->in_std, nullptr, h->xb);
    if (yp) {
        MCK(cudaMemcpyAsync(h->y_raw, yp, sizeof(double) * rows * h->O, cudaMemcpyHostToDevice, h->stream));
        k_standardize<<<blocks((long long)rows * h->Op), 256, 0, h->stream>>>(h->y_raw, rows, h->O, h->Op,
                                                                              h->out_mean, h->out_std, h->t, nullptr);
    }
    MCK(cudaGetLastError());
    // the raw buffers are reused by the next upload; keep the copies ordered
    MCK(cudaStreamSynchronize(h->stream));
    return ESPL_OK;
}

// Uploads per-column means and standard deviations (sums and sums of
// squares over n rows in; a column whose deviation is at most 1e-12 is
// scaled by 1 and, for an output, marked constant: out_gain 0).
espl_status upload_scaling(espl_mlp* h, const std::vector<double>& xs, const std::vector<double>& ys, uint32_t n) {
    auto finish = [&](const std::vector<double>& sums, int cols, int ld, std::vector<float>& mean,
                      std::vector<float>& sd, std::vector<float>* gain) {
        mean.assign(ld, 0.0f);
        sd.assign(ld, 1.0f);
        if (gain) gain->assign(ld, 0.0f);
        for (int j = 0; j < cols; j++) {
            const double mu = sums[2 * j] / n;
            const double var = std::max(0.0, sums[2 * j + 1] / n - mu * mu);
            const double sdv = std::sqrt(var);
            mean[j] = (float)mu;
            sd[j] = (float)(sdv > 1e-12 ? sdv : 1.0);
            if (gain) (*gain)[j] = sdv > 1e-12 ? (float)sdv : 0.0f;
        }
    };
    std::vector<float> im, is, om, os, og;
    finish(xs, h->D, h->Dp, im, is, nullptr);
    finish(ys, h->O, h->Op, om, os, &og);
    MCK(cudaMemcpyAsync(h->in_mean, im.data(), sizeof(float) * h->Dp, cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(h->in_std, is.data(), sizeof(float) * h->Dp, cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(h->out_mean, om.data(), sizeof(float) * h->Op, cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(h->out_std, os.data(), sizeof(float) * h->Op, cudaMemcpyHostToDevice, h->stream));
    MCK(cudaMemcpyAsync(h->out_gain, og.data(), sizeof(float) * h->Op, cudaMemcpyHostToDevice, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    h->scaled = true;
    return ESPL_OK;
}

espl_status set_scaling(espl_mlp* h, const double* x, const double* y, uint32_t n) {
    auto sums = [&](const double* a, int cols) {
        std::vector<double> out(2 * (size_t)cols, 0.0);
        for (int j = 0; j < cols; j++) {
            double s = 0, s2 = 0;
            for (uint32_t r = 0; r < n; r++) s += a[(size_t)r * cols + j];
            const double mu = s / std::max<uint32_t>(n, 1);
            for (uint32_t r = 0; r < n; r++) {
                const double e = a[(size_t)r * cols + j] - mu;
                s2 += e * e;
            }
            // the second pass's centred sum, returned as the raw form the
            // finisher expects: sum of squares = centred + n mu^2
            out[2 * j] = s;
            out[2 * j + 1] = s2 + (double)n * mu * mu;
        }
        return out;
    };
    return upload_scaling(h, sums(x, h->D), sums(y, h->O), n);
}

// The same from rows already on the device (FP64, row-major).
espl_status set_scaling_device(espl_mlp* h, const double* x, const double* y, uint32_t n) {
    double* d = nullptr;
    MCK(cudaMalloc(&d, sizeof(double) * 2 * (h->D + h->O)));
    k_col_stats<<<h->D, 256, 0, h->stream>>>(x, n, h->D, d);
    k_col_stats<<<h->O, 256, 0, h->stream>>>(y, n, h->O, d + 2 * h->D);
    std::vector<double> all(2 * (size_t)(h->D + h->O));
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(all.data(), d, sizeof(double) * all.size(), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) {
        h->msg = std::string("column statistics: ") + cudaGetErrorString(e);
        return ESPL_DRIVER;
    }
    std::vector<double> xs(all.begin(), all.begin() + 2 * h->D), ys(all.begin() + 2 * h->D, all.end());
    return upload_scaling(h, xs, ys, n);
}

espl_status train_resident(espl_mlp* h, const double* xr, const double* yr, uint32_t n, const espl_train_opts* o,
                           double* epoch_loss);

}  // namespace

extern "C" {

espl_status espl_mlp_create(uint32_t in_dim, uint32_t out_dim, uint32_t capacity, uint64_t seed, uint32_t device,
                            espl_mlp** out) {
    if (!out) return ESPL_INVALID_ARGUMENT;
    *out = nullptr;
    if (in_dim == 0 || in_dim > 128 || out_dim == 0 || out_dim > 128 || capacity == 0) return ESPL_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ESPL_NO_IMAGE;
    if ((int)device >= ndev) return ESPL_INVALID_ARGUMENT;
    espl_mlp* h = new espl_mlp();
    auto bail = [&](espl_status s) {
        espl_mlp_destroy(h);
        return s;
    };
    h->device = (int)device;
    if (cudaSetDevice(h->device) != cudaSuccess) return bail(ESPL_DRIVER);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_gemm_tc<128, kEpiStore>) != cudaSuccess) return bail(ESPL_NO_IMAGE);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(ESPL_DRIVER);
    h->D = (int)in_dim;
    h->Dp = up16(h->D);
    h->O = (int)out_dim;
    h->Op = up16(h->O);
    h->cap = (int)((capacity + 127) / 128 * 128);
    const int H = h->H;
    h->off_w1 = 0;
    h->off_b1 = h->off_w1 + (long long)H * h->Dp;
    h->off_w2 = h->off_b1 + H;
    h->off_b2 = h->off_w2 + (long long)H * H;
    h->off_w3 = h->off_b2 + H;
    h->off_b3 = h->off_w3 + (long long)h->Op * H;
    h->n_par = h->off_b3 + h->Op;
    espl_status s;
#define AL(ptr, count) if ((s = alloc(h, &h->ptr, count))) return bail(s)
    AL(p, h->n_par);
    AL(g, h->n_par);
    AL(m, h->n_par);
    AL(v, h->n_par);
    AL(w1b, (size_t)H * h->Dp);
    AL(w2b, (size_t)H * H);
    AL(w3b, (size_t)h->Op * H);
    AL(in_mean, h->Dp);
    AL(in_std, h->Dp);
    AL(out_mean, h->Op);
    AL(out_std, h->Op);
    AL(out_gain, h->Op);
    AL(image, weight_image_bytes(h->Dp, h->Op));
    const size_t c = (size_t)h->cap;
    AL(x_raw, c * h->D);
    AL(y_raw, c * h->O);
    AL(xb, c * h->Dp);
    AL(t, c * h->Op);
    AL(h1, c * H);
    AL(h1b, c * H);
    AL(h2, c * H);
    AL(h2b, c * H);
    AL(y, c * h->Op);
    AL(dy, c * h->Op);
    AL(dyb, c * h->Op);
    AL(dh, c * H);
    AL(dz, c * H);
    AL(dzb, c * H);
    AL(loss, 1);
    AL(err, 1);
#undef AL
    // Glorot-uniform weights from the seed, zero biases (host draw, FP32).
    std::vector<float> par((size_t)h->n_par, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](long long off, int rows, int cols, int ld) {
        float a = std::sqrt(6.0f / (float)(rows + cols));
        std::uniform_real_distribution<float> u(-a, a);
        for (int r = 0; r < rows; r++)
            for (int cc = 0; cc < cols; cc++) par[(size_t)(off + (long long)r * ld + cc)] = u(rng);
    };
    fill(h->off_w1, H, h->D, h->Dp);
    fill(h->off_w2, H, H, H);
    fill(h->off_w3, h->O, H, H);
    if (cudaMemcpyAsync(h->p, par.data(), sizeof(float) * par.size(), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return bail(ESPL_DRIVER);
    std::vector<float> ones(std::max(h->Dp, h->Op), 1.0f);
    cudaMemcpyAsync(h->in_std, ones.data(), sizeof(float) * h->Dp, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->out_std, ones.data(), sizeof(float) * h->Op, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->out_gain, ones.data(), sizeof(float) * h->Op, cudaMemcpyHostToDevice, h->stream);
    if ((s = refresh_bf16(h))) return bail(s);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(ESPL_DRIVER);
    *out = h;
    return ESPL_OK;
}

espl_status espl_mlp_destroy(espl_mlp* h) {
    if (!h) return ESPL_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* q : h->owned) cudaFree(q);
    cudaFree(h->pred_x);
    cudaFree(h->pred_y);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return ESPL_OK;
}

espl_status espl_mlp_param_count(const espl_mlp* h, uint32_t* count) {
    if (!h || !count) return ESPL_INVALID_ARGUMENT;
    *count = (uint32_t)((long long)h->H * h->D + h->H + (long long)h->H * h->H + h->H + (long long)h->O * h->H + h->O);
    return ESPL_OK;
}

// Parameters in the API order W1 [128 x in], b1, W2 [128 x 128], b2,
// W3 [out x 128], b3 (row-major), FP32.
espl_status espl_mlp_get_params(espl_mlp* h, float* out) {
    if (!h || !out) return ESPL_INVALID_ARGUMENT;
    std::vector<float> par((size_t)h->n_par);
    MCK(cudaMemcpyAsync(par.data(), h->p, sizeof(float) * par.size(), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    size_t k = 0;
    const int H = h->H;
    for (int r = 0; r < H; r++)
        for (int c = 0; c < h->D; c++) out[k++] = par[(size_t)(h->off_w1 + (long long)r * h->Dp + c)];
    for (int r = 0; r < H; r++) out[k++] = par[(size_t)(h->off_b1 + r)];
    for (long long i = 0; i < (long long)H * H; i++) out[k++] = par[(size_t)(h->off_w2 + i)];
    for (int r = 0; r < H; r++) out[k++] = par[(size_t)(h->off_b2 + r)];
    for (int r = 0; r < h->O; r++)
        for (int c = 0; c < H; c++) out[k++] = par[(size_t)(h->off_w3 + (long long)r * H + c)];
    for (int r = 0; r < h->O; r++) out[k++] = par[(size_t)(h->off_b3 + r)];
    return ESPL_OK;
}

espl_status espl_mlp_set_params(espl_mlp* h, const float* in) {
    if (!h || !in) return ESPL_INVALID_ARGUMENT;
    std::vector<float> par((size_t)h->n_par, 0.0f);
    size_t k = 0;
    const int H = h->H;
    for (int r = 0; r < H; r++)
        for (int c = 0; c < h->D; c++) par[(size_t)(h->off_w1 + (long long)r * h->Dp + c)] = in[k++];
    for (int r = 0; r < H; r++) par[(size_t)(h->off_b1 + r)] = in[k++];
    for (long long i = 0; i < (long long)H * H; i++) par[(size_t)(h->off_w2 + i)] = in[k++];
    for (int r = 0; r < H; r++) par[(size_t)(h->off_b2 + r)] = in[k++];
    for (int r = 0; r < h->O; r++)
        for (int c = 0; c < H; c++) par[(size_t)(h->off_w3 + (long long)r * H + c)] = in[k++];
    for (int r = 0; r < h->O; r++) par[(size_t)(h->off_b3 + r)] = in[k++];
    MCK(cudaMemcpyAsync(h->p, par.data(), sizeof(float) * par.size(), cudaMemcpyHostToDevice, h->stream));
    espl_status s = refresh_bf16(h);
    if (s) return s;
    MCK(cudaStreamSynchronize(h->stream));
    return ESPL_OK;
}

espl_status espl_mlp_set_scaling(espl_mlp* h, const double* x, const double* y, uint32_t n) {
    if (!h || !x || !y || n == 0) return ESPL_INVALID_ARGUMENT;
    return set_scaling(h, x, y, n);
}

espl_status espl_mlp_loss_grad(espl_mlp* h, const double* x, const double* y, uint32_t n, double* loss, float* grad) {
    if (!h || !x || !y || n == 0 || (int)n > h->cap) return ESPL_INVALID_ARGUMENT;
    espl_status s;
    if ((s = upload(h, x, y, nullptr, 0, (int)n))) return s;
    if ((s = forward(h, (int)n))) return s;
    MCK(cudaMemsetAsync(h->loss, 0, sizeof(double), h->stream));
    if ((s = backward(h, (int)n, h->loss))) return s;
    if ((s = check_err(h))) return s;
    double l = 0;
    MCK(cudaMemcpyAsync(&l, h->loss, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    if (loss) *loss = l / ((double)n * h->O);
    if (grad) {
        // the same API order as espl_mlp_get_params, read from the gradient buffer
        float* keep = h->p;
        h->p = h->g;
        s = espl_mlp_get_params(h, grad);
        h->p = keep;
        if (s) return s;
    }
    return ESPL_OK;
}

espl_status espl_mlp_train(espl_mlp* h, const double* x, const double* y, uint32_t n, const espl_train_opts* o,
                           double* epoch_loss) {
    if (!h || !x || !y || n == 0 || !o || o->batch == 0 || (int)o->batch > h->cap || o->epochs == 0 ||
        o->batch > n)
        return ESPL_INVALID_ARGUMENT;
    espl_status s = ESPL_OK;
    if (!h->scaled && (s = set_scaling(h, x, y, n))) return s;
    double *xr = nullptr, *yr = nullptr;
    if (cudaMalloc(&xr, sizeof(double) * n * h->D) != cudaSuccess) {
        h->msg = "out of device memory for the training set";
        return ESPL_OUT_OF_MEMORY;
    }
    if (cudaMalloc(&yr, sizeof(double) * n * h->O) != cudaSuccess) {
        cudaFree(xr);
        h->msg = "out of device memory for the training set";
        return ESPL_OUT_OF_MEMORY;
    }
    if (cudaMemcpyAsync(xr, x, sizeof(double) * n * h->D, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(yr, y, sizeof(double) * n * h->O, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        s = ESPL_DRIVER;
    if (!s) s = train_resident(h, xr, yr, n, o, epoch_loss);
    cudaStreamSynchronize(h->stream);
    cudaFree(xr);
    cudaFree(yr);
    return s;
}

espl_status espl_mlp_train_device(espl_mlp* h, const double* x, const double* y, uint32_t n,
                                  const espl_train_opts* o, double* epoch_loss) {
    if (!h || !x || !y || n == 0 || !o || o->batch == 0 || (int)o->batch > h->cap || o->epochs == 0 ||
        o->batch > n)
        return ESPL_INVALID_ARGUMENT;
    espl_status s = ESPL_OK;
    if (!h->scaled && (s = set_scaling_device(h, x, y, n))) return s;
    return train_resident(h, x, y, n, o, epoch_loss);
}

}  // extern "C"

namespace {

// The training loop over rows already on the device (x: n x D, y: n x O,
// FP64, row-major), standardized once into BF16 inputs and FP32 targets.
espl_status train_resident(espl_mlp* h, const double* xr, const double* yr, uint32_t n, const espl_train_opts* o,
                           double* epoch_loss) {
    espl_status s = ESPL_OK;
    const uint32_t chunk_ep = std::max(1u, std::min(o->epochs, (uint32_t)((64u << 20) / (sizeof(uint32_t) * n))));
    // The data set stays on the device, standardized; the epochs'
    // permutations go up in chunks of up to 64 MB and every Adam step
    // gathers its rows on the device.
    double* lsum = nullptr;
    __nv_bfloat16* xs = nullptr;
    float* ts = nullptr;
    uint32_t* perm = nullptr;
    std::vector<void*> tmp;
    auto dalloc = [&](void** q, size_t bytes) {
        cudaError_t e = cudaMalloc(q, bytes);
        if (e == cudaSuccess) tmp.push_back(*q);
        return e;
    };
    auto cleanup = [&]() {
        cudaStreamSynchronize(h->stream);
        for (void* q : tmp) cudaFree(q);
    };
    if (dalloc((void**)&xs, sizeof(__nv_bfloat16) * n * h->Dp) || dalloc((void**)&ts, sizeof(float) * n * h->Op) ||
        dalloc((void**)&perm, sizeof(uint32_t) * n * chunk_ep) || dalloc((void**)&lsum, sizeof(double) * o->epochs)) {
        cleanup();
        h->msg = "out of device memory for the training set";
        return ESPL_OUT_OF_MEMORY;
    }
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, h->stream);
    cudaMemsetAsync(lsum, 0, sizeof(double) * o->epochs, h->stream);
    k_standardize<<<blocks((long long)n * h->Dp), 256, 0, h->stream>>>(xr, (int)n, h->D, h->Dp, h->in_mean, h->in_std,
                                                                        nullptr, xs);
    k_standardize<<<blocks((long long)n * h->Op), 256, 0, h->stream>>>(yr, (int)n, h->O, h->Op, h->out_mean,
                                                                        h->out_std, ts, nullptr);
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    std::mt19937_64 rng(o->seed);
    const float b1 = o->beta1, b2 = o->beta2;
    const uint32_t per_epoch = n / o->batch;
    const int rows = (int)o->batch;
    std::vector<uint32_t> perms((size_t)n * chunk_ep);
    for (uint32_t ep = 0; ep < o->epochs && !s; ep++) {
        const uint32_t slot = ep % chunk_ep;
        if (slot == 0) {
            const uint32_t count = std::min(chunk_ep, o->epochs - ep);
            for (uint32_t e = 0; e < count; e++) {
                std::shuffle(order.begin(), order.end(), rng);
                std::copy(order.begin(), order.end(), perms.begin() + (size_t)e * n);
            }
            // the permutation buffer is rewritten per chunk: order the copy
            // after the previous chunk's gathers
            if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
                cudaMemcpyAsync(perm, perms.data(), sizeof(uint32_t) * n * count, cudaMemcpyHostToDevice,
                                h->stream) != cudaSuccess) {
                s = ESPL_DRIVER;
                break;
            }
        }
        const uint32_t* ep_perm = perm + (size_t)slot * n;
        float lr = o->lr;
        if (o->lr_final > 0.0f && o->epochs > 1)
            lr = o->lr * std::pow(o->lr_final / o->lr, (float)ep / (float)(o->epochs - 1));
        for (uint32_t b = 0; b < per_epoch && !s; b++) {
            long long nb = (long long)rows * std::max(h->Dp, h->Op);
            k_gather_rows<<<blocks(nb), 256, 0, h->stream>>>(xs, ts, ep_perm + (size_t)b * rows, rows, h->Dp, h->Op,
                                                             h->xb, h->t);
            if ((s = forward(h, rows))) break;
            if ((s = backward(h, rows, lsum + ep))) break;
            h->adam_t++;
            float c1 = 1.0f - std::pow(b1, (float)h->adam_t), c2 = 1.0f - std::pow(b2, (float)h->adam_t);
            k_adam<<<blocks(h->n_par), 256, 0, h->stream>>>(h->p, h->g, h->m, h->v, h->n_par, lr, b1, b2, o->eps, c1,
                                                              c2);
            s = refresh_bf16(h);
        }
    }
    cudaEventRecord(ev1, h->stream);
    if (!s) s = check_err(h);
    {
        float ms = 0.0f;
        if (!s && cudaEventSynchronize(ev1) == cudaSuccess && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess)
            h->last_train_ms = ms;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    if (!s && epoch_loss) {
        std::vector<double> l(o->epochs);
        if (cudaMemcpyAsync(l.data(), lsum, sizeof(double) * o->epochs, cudaMemcpyDeviceToHost, h->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess)
            s = ESPL_DRIVER;
        for (uint32_t ep = 0; ep < o->epochs && !s; ep++)
            epoch_loss[ep] = l[ep] / ((double)per_epoch * rows * h->O);
    }
    cleanup();
    return s;
}

}  // namespace

extern "C" {

espl_status espl_mlp_predict(espl_mlp* h, const double* x, uint32_t n, double* y) {
    if (!h || !x || !y) return ESPL_INVALID_ARGUMENT;
    if (n == 0) return ESPL_OK;
    // One fused launch (k_mlp_infer): each CTA runs the whole network on 128
    // rows with the weights and activations in shared memory. The rows'
    // device buffers are the handle's, grown when a call needs more.
    if (n > h->pred_rows) {
        MCK(cudaStreamSynchronize(h->stream));
        cudaFree(h->pred_x);
        cudaFree(h->pred_y);
        h->pred_x = h->pred_y = nullptr;
        h->pred_rows = 0;
        if (cudaMalloc(&h->pred_x, sizeof(double) * (size_t)n * h->D) != cudaSuccess ||
            cudaMalloc(&h->pred_y, sizeof(double) * (size_t)n * h->O) != cudaSuccess) {
            cudaFree(h->pred_x);
            h->pred_x = nullptr;
            h->msg = "out of device memory for the predictions";
            return ESPL_OUT_OF_MEMORY;
        }
        h->pred_rows = n;
    }
    double *dx = h->pred_x, *dy = h->pred_y;
    espl_status s = ESPL_OK;
    const size_t smem = infer_smem_bytes(h->Dp, h->Op);
    InferArgs g{dx, dy, h->p + h->off_w1, h->p + h->off_b1, h->p + h->off_w2, h->p + h->off_b2, h->p + h->off_w3,
                h->p + h->off_b3, h->in_mean, h->in_std, h->out_mean, h->out_std, (int)n, h->D, h->Dp, h->O, h->Op,
                h->err};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, h->stream);
    if (cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaMemcpyAsync(dx, x, sizeof(double) * (size_t)n * h->D, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) {
        s = ESPL_DRIVER;
    } else {
        k_mlp_infer<<<(n + 127) / 128, 128, smem, h->stream>>>(g);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(y, dy, sizeof(double) * (size_t)n * h->O, cudaMemcpyDeviceToHost, h->stream) !=
                cudaSuccess)
            s = ESPL_DRIVER;
    }
    cudaEventRecord(ev1, h->stream);
    cudaStreamSynchronize(h->stream);
    float ms = 0.0f;
    if (!s && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) h->last_predict_ms = ms;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (s) {
        h->msg = "predict launch failed";
        return s;
    }
    return check_err(h);
}

// The layer-by-layer predictions through the training GEMMs (one launch per
// layer on capacity-sized chunks): the fused kernel's cross-check.
espl_status espl_mlp_predict_layers(espl_mlp* h, const double* x, uint32_t n, double* y) {
    if (!h || !x || !y) return ESPL_INVALID_ARGUMENT;
    espl_status s;
    double* out = nullptr;
    for (uint32_t r0 = 0; r0 < n; r0 += (uint32_t)h->cap) {
        int rows = (int)std::min<uint32_t>((uint32_t)h->cap, n - r0);
        if ((s = upload(h, x, nullptr, nullptr, r0, rows))) return s;
        if ((s = forward(h, rows))) return s;
        out = h->y_raw;  // rows x O doubles fit (cap x O)
        k_destandardize<<<blocks((long long)rows * h->O), 256, 0, h->stream>>>(h->y, rows, h->O, h->Op, h->out_mean,
                                                                              h->out_std, out);
        MCK(cudaGetLastError());
        MCK(cudaMemcpyAsync(y + (size_t)r0 * h->O, out, sizeof(double) * rows * h->O, cudaMemcpyDeviceToHost,
                            h->stream));
        MCK(cudaStreamSynchronize(h->stream));
    }
    return check_err(h);
}

espl_status espl_mlp_train_ms(const espl_mlp* h, double* device_ms) {
    if (!h || !device_ms) return ESPL_INVALID_ARGUMENT;
    *device_ms = h->last_train_ms;
    return ESPL_OK;
}

espl_status espl_mlp_predict_ms(const espl_mlp* h, double* device_ms) {
    if (!h || !device_ms) return ESPL_INVALID_ARGUMENT;
    *device_ms = h->last_predict_ms;
    return ESPL_OK;
}

espl_status espl_mlp_error_message(espl_mlp* h, char* buf, size_t cap) {
    if (!h || !buf || cap == 0) return ESPL_INVALID_ARGUMENT;
    size_t k = std::min(cap - 1, h->msg.size());
    std::memcpy(buf, h->msg.data(), k);
    buf[k] = 0;
    return ESPL_OK;
}

}  // extern "C"

uint32_t espl_mlp_view(espl_mlp* h, espl::mlp::MlpView* v, void* stream) {
    if (!h || !v) return ESPL_INVALID_ARGUMENT;
    if (h->image_version != h->weights_version) {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // the weights are written on the network's stream
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) return ESPL_DRIVER;
        const long long total = 128LL * h->Dp + 128LL * 128 + (long long)h->Op * 128;
        k_pack_image<<<blocks(total), 256, 0, st>>>(h->p + h->off_w1, h->p + h->off_w2, h->p + h->off_w3, h->Dp, h->Op,
                                                    h->image);
        if (cudaGetLastError() != cudaSuccess) return ESPL_DRIVER;
        h->image_version = h->weights_version;
    }
    v->image = h->image;
    v->b1 = h->p + h->off_b1;
    v->b2 = h->p + h->off_b2;
    v->b3 = h->p + h->off_b3;
    v->in_mean = h->in_mean;
    v->in_std = h->in_std;
    v->out_mean = h->out_mean;
    v->out_gain = h->out_gain;
    v->in_dim = h->D;
    v->dp = h->Dp;
    v->out_dim = h->O;
    v->op = h->Op;
    v->err = h->err;
    return ESPL_OK;
}
