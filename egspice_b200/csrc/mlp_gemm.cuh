// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05):
// C[m, n] = sum_k A(m, k) B(n, k), with A and B read from global memory
// through arbitrary element strides (so transposed views need no copy),
// staged into shared memory as K-major core matrices (8 rows x 16 bytes,
// no swizzle), multiplied by tcgen05.mma issued from one thread with the
// accumulator in tensor memory, and read back with tcgen05.ld for the
// epilogue. One CTA of 128 threads owns a 128 x BN tile of C; grid.z splits
// K (the partial tiles are added with FP32 atomics).
//
// Every wait on the MMA completion mbarrier is bounded; past the bound the
// kernel raises the caller's error flag, waits (bounded) for its own MMAs,
// frees its tensor memory and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace espl {
namespace mlp {

constexpr int kBM = 128;       // rows of C per CTA (the MMA's M)
constexpr int kBK = 64;        // K per staged chunk (four MMAs of K = 16)
constexpr int kGemmThreads = 128;

enum Epilogue : int {
    kEpiStore = 0,      // C = acc
    kEpiBiasTanh = 1,   // C = tanh(acc + bias), also Cb = bf16(C)
    kEpiBias = 2,       // C = acc + bias
    kEpiAtomic = 3,     // C += acc (split K)
};

struct GemmArgs {
    const __nv_bfloat16* a;
    const __nv_bfloat16* b;
    long long sam, sak;   // A(m, k) = a[m * sam + k * sak]
    long long sbn, sbk;   // B(n, k) = b[n * sbn + k * sbk]
    float* c;             // C(m, n) = c[m * ldc + n]
    __nv_bfloat16* cb;    // kEpiBiasTanh: bf16 copy of C, same layout
    const float* bias;    // per column n
    int M, N, K, ldc;
    int k_per_split;      // K range of one grid.z slice (multiple of kBK)
    int* err;             // set to 1 when a bounded wait ran out
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in a staged R x kBK tile: core matrix
// (r / 8, k / 8) at ((r / 8) * (kBK / 8) + k / 8) * 128, row r % 8 at 16 bytes
// each, element k % 8 at 2 bytes each.
__device__ __forceinline__ uint32_t tile_off(uint32_t r, uint32_t k) {
    return ((r >> 3) * (kBK / 8) + (k >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address,
// leading byte offset 128 (the next 8-element K block), stride byte offset
// (kBK / 8) * 128 (the next 8 rows), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)(((kBK / 8) * 128u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major,
// N = bn, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t bn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((bn >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_wait_parity(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false when the bound ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t tries = 0; tries < (1u << 22); tries++) {
        if (mbar_wait_parity(bar, parity)) return true;
        if (tries > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Stages rows [r0, r0 + rows) x K [k0, k0 + kBK) of a strided operand into
// a K-major tile; out-of-range elements are zero. Consecutive threads walk
// the contiguous dimension of the source.
__device__ __forceinline__ void stage_operand(unsigned char* tile, const __nv_bfloat16* src, long long s_row,
                                              long long s_k, int r0, int rows_total, int rows, int k0, int k_total) {
    const int tid = threadIdx.x;
    const int n = rows * kBK;
    if (s_k == 1) {
        for (int e = tid; e < n; e += kGemmThreads) {
            int r = e / kBK, k = e % kBK;
            int gr = r0 + r, gk = k0 + k;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (gr < rows_total && gk < k_total) v = src[(long long)gr * s_row + gk];
            *reinterpret_cast<__nv_bfloat16*>(tile + tile_off(r, k)) = v;
        }
    } else {
        for (int e = tid; e < n; e += kGemmThreads) {
            int k = e / rows, r = e % rows;
            int gr = r0 + r, gk = k0 + k;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (gr < rows_total && gk < k_total) v = src[(long long)gr * s_row + (long long)gk * s_k];
            *reinterpret_cast<__nv_bfloat16*>(tile + tile_off(r, k)) = v;
        }
    }
}

// BN: columns of C per CTA (16..128, a multiple of 16).
template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_tc(GemmArgs g) {
    constexpr uint32_t kTmemCols = BN <= 32 ? 32 : BN <= 64 ? 64 : 128;
    __shared__ __align__(1024) unsigned char sa[kBM * kBK * 2];
    __shared__ __align__(1024) unsigned char sb[BN * kBK * 2];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_per_split;
    const int ke = min(g.K, kb + g.k_per_split);
    if (threadIdx.x == 0) {
        mbar_init1(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = instr_desc(BN);
    uint32_t phase = 0;
    bool issued = false;
    for (int k0 = kb; k0 < ke; k0 += kBK) {
        stage_operand(sa, g.a, g.sam, g.sak, m0, g.M, kBM, k0, ke);
        stage_operand(sb, g.b, g.sbn, g.sbk, n0, g.N, BN, k0, ke);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < kBK / 16; j++) {
                uint64_t da = smem_desc(smem_u32(sa) + j * 256u);
                uint64_t db = smem_desc(smem_u32(sb) + j * 256u);
                tc_mma(tmem, da, db, idesc, (issued || j > 0) ? 1u : 0u);
            }
            tc_commit(&bar);
        }
        issued = true;
        // the tile buffers are reused: wait until the MMAs have read them
        bool ok = mbar_wait_bounded(&bar, phase);
        if (!ok) failed = 1;
        __syncthreads();
        if (failed) break;
        phase ^= 1u;
    }
    if (failed) {
        // give the MMAs in flight a second bounded wait before the tensor
        // memory they write is freed
        mbar_wait_bounded(&bar, phase);
        if (threadIdx.x == 0) atomicExch(g.err, 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (failed) {
    } else if (issued) {
        const int m = m0 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (m < g.M) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int n = n0 + c0 + i;
                    if (n >= g.N) continue;
                    float x = v[i];
                    float* cp = g.c + (long long)m * g.ldc + n;
                    if (EPI == kEpiAtomic) {
                        atomicAdd(cp, x);
                    } else if (EPI == kEpiBiasTanh) {
                        x = tanhf(x + g.bias[n]);
                        *cp = x;
                        g.cb[(long long)m * g.ldc + n] = __float2bfloat16(x);
                    } else if (EPI == kEpiBias) {
                        *cp = x + g.bias[n];
                    } else {
                        *cp = x;
                    }
                }
            }
        }
    } else if (EPI != kEpiAtomic) {
        // an empty K range: C = epilogue(0)
        const int m = m0 + warp * 32 + lane;
        if (m < g.M)
            for (int n = n0; n < min(g.N, n0 + BN); n++) {
                float x = 0.0f;
                float* cp = g.c + (long long)m * g.ldc + n;
                if (EPI == kEpiBiasTanh) {
                    x = tanhf(g.bias[n]);
                    g.cb[(long long)m * g.ldc + n] = __float2bfloat16(x);
                } else if (EPI == kEpiBias) {
                    x = g.bias[n];
                }
                *cp = x;
            }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace mlp
}  // namespace espl

namespace espl {
namespace mlp {

// Shared-memory descriptor of a K-major no-swizzle tile whose rows hold
// `k_cols` elements: the next 8-element K block is 128 bytes on, the next
// 8 rows (k_cols / 8) * 128 bytes on.
__device__ __forceinline__ uint64_t smem_desc_k(uint32_t addr, uint32_t k_cols) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)(((k_cols / 8) * 128u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ uint32_t tile_off_k(uint32_t r, uint32_t k, uint32_t k_cols) {
    return ((r >> 3) * (k_cols / 8) + (k >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

struct InferArgs {
    const double* x;          // rows x in_dim, raw parameters
    double* y;                // rows x out_dim, de-standardized predictions
    const float *w1, *b1, *w2, *b2, *w3, *b3;  // FP32 master weights (padded layouts)
    const float *in_mean, *in_std, *out_mean, *out_std;
    int rows, in_dim, dp, out_dim, op;
    int* err;
};

// Loads a FP32 weight matrix [n_rows x k_cols] (row-major, ld = k_cols) into
// a K-major BF16 tile.
__device__ __forceinline__ void stage_weights(unsigned char* tile, const float* w, int n_rows, int k_cols) {
    for (int e = threadIdx.x; e < n_rows * k_cols; e += blockDim.x) {
        int r = e / k_cols, k = e % k_cols;
        *reinterpret_cast<__nv_bfloat16*>(tile + tile_off_k(r, k, k_cols)) = __float2bfloat16(w[e]);
    }
}

// The whole network for one 128-row tile in one CTA: the standardized input
// tile and the three weight matrices in shared memory, each layer one chain
// of tcgen05.mma into tensor memory, its epilogue (bias, tanh) written back
// to shared memory as the next layer's BF16 operand, the output layer
// de-standardized to FP64. Dynamic shared memory: infer_smem_bytes.
__host__ __device__ inline size_t infer_smem_bytes(int dp, int op) {
    return (size_t)128 * dp * 2 + 128 * dp * 2 + 128 * 128 * 2 + (size_t)op * 128 * 2 + 128 * 128 * 2;
}

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
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
    const int row = warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    uint32_t phase = 0;
    for (int layer = 0; layer < 3; layer++) {
        const unsigned char* a = layer == 0 ? sx : sh;
        const unsigned char* b = layer == 0 ? sw1 : layer == 1 ? sw2 : sw3;
        const int kc = layer == 0 ? dp : H;
        const int n = layer == 2 ? op : H;
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t idesc = instr_desc((uint32_t)n);
            for (int j = 0; j < kc / 16; j++) {
                uint64_t da = smem_desc_k(smem_u32(a) + j * 256u, (uint32_t)kc);
                uint64_t db = smem_desc_k(smem_u32(b) + j * 256u, (uint32_t)kc);
                tc_mma(tmem, da, db, idesc, j > 0 ? 1u : 0u);
            }
            tc_commit(&bar);
        }
        if (!mbar_wait_bounded(&bar, phase)) failed = 1;
        __syncthreads();
        if (failed) {
            mbar_wait_bounded(&bar, phase);
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (layer < 2) {
            const float* bias = layer == 0 ? g.b1 : g.b2;
            for (int c0 = 0; c0 < H; c0 += 16) {
                float v[16];
                tc_ld16(trow + (uint32_t)c0, v);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float hv = tanhf(v[i] + bias[c0 + i]);
                    *reinterpret_cast<__nv_bfloat16*>(sh + tile_off_k(row, c0 + i, H)) = __float2bfloat16(hv);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
        } else {
            for (int c0 = 0; c0 < op; c0 += 16) {
                float v[16];
                tc_ld16(trow + (uint32_t)c0, v);
                if (r0 + row < g.rows) {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        int o = c0 + i;
                        if (o < g.out_dim)
                            g.y[(long long)(r0 + row) * g.out_dim + o] =
                                (double)(v[i] + g.b3[o]) * (double)g.out_std[o] + (double)g.out_mean[o];
                    }
                }
            }
        }
    }
    if (failed && threadIdx.x == 0) atomicExch(g.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
}

}  // namespace mlp
}  // namespace espl
