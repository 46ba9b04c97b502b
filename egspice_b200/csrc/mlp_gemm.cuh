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

// How an operand is staged: kStageK when K is contiguous (s_k == 1) and rows
// start on 16 bytes, kStageRows when rows are contiguous (s_row == 1) and K
// steps are 16 bytes, kStageAny otherwise. The first two move 8 elements per
// 16-byte load.
enum StageMode : int { kStageK = 0, kStageRows = 1, kStageAny = 2 };

__device__ __forceinline__ int stage_mode(const __nv_bfloat16* src, long long s_row, long long s_k) {
    if (reinterpret_cast<uintptr_t>(src) & 15u) return kStageAny;
    if (s_k == 1 && (s_row & 7) == 0) return kStageK;
    if (s_row == 1 && (s_k & 7) == 0) return kStageRows;
    return kStageAny;
}

// 8 contiguous elements from p; those at positions >= valid read as zero and
// are not touched.
__device__ __forceinline__ uint4 load8(const __nv_bfloat16* p, int valid) {
    if (valid >= 8) return __ldg(reinterpret_cast<const uint4*>(p));
    const unsigned short* q = reinterpret_cast<const unsigned short*>(p);
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint32_t lo = 2 * j < valid ? q[2 * j] : 0u;
        const uint32_t hi = 2 * j + 1 < valid ? q[2 * j + 1] : 0u;
        w[j] = lo | hi << 16;
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// A ROWS x kBK operand tile in flight: ROWS * kBK / 8 chunks of 16 bytes,
// ROWS / 16 per thread, chunk e = threadIdx.x + i * kGemmThreads.
//   kStageK:    chunk e holds row (e >> 6) * 8 + (e & 7), K block (e >> 3) & 7,
//               which is exactly tile bytes [16 e, 16 e + 16).
//   kStageRows: chunk e holds rows (e >> 6) * 8 .. + 7 at K index e & 63.
template <int ROWS>
struct StageBuf {
    uint4 v[ROWS / 16];
};

// Issues every global load of one tile (rows [r0, r0 + ROWS), K [k0, k0 +
// kBK), out-of-range elements zero) before any of them is consumed.
template <int ROWS>
__device__ __forceinline__ void stage_load(StageBuf<ROWS>& b, int mode, const __nv_bfloat16* src, long long s_row,
                                           long long s_k, int r0, int rows_total, int k0, int k_total) {
#pragma unroll
    for (int i = 0; i < ROWS / 16; i++) {
        const int e = threadIdx.x + i * kGemmThreads;
        if (mode == kStageK) {
            const int gr = r0 + (e >> 6) * 8 + (e & 7), gk = k0 + ((e >> 3) & 7) * 8;
            const int valid = gr < rows_total ? max(0, min(8, k_total - gk)) : 0;
            b.v[i] = load8(src + (long long)gr * s_row + gk, valid);
        } else if (mode == kStageRows) {
            const int gr = r0 + (e >> 6) * 8, gk = k0 + (e & 63);
            const int valid = gk < k_total ? max(0, min(8, rows_total - gr)) : 0;
            b.v[i] = load8(src + gr + (long long)gk * s_k, valid);
        }
    }
}

template <int ROWS>
__device__ __forceinline__ void stage_store(unsigned char* tile, const StageBuf<ROWS>& b, int mode) {
#pragma unroll
    for (int i = 0; i < ROWS / 16; i++) {
        const int e = threadIdx.x + i * kGemmThreads;
        if (mode == kStageK) {
            *reinterpret_cast<uint4*>(tile + (uint32_t)e * 16u) = b.v[i];
        } else if (mode == kStageRows) {
            const uint32_t w[4] = {b.v[i].x, b.v[i].y, b.v[i].z, b.v[i].w};
            const int rb = e >> 6, k = e & 63;
#pragma unroll
            for (int j = 0; j < 8; j++)
                *reinterpret_cast<unsigned short*>(tile + tile_off((uint32_t)(rb * 8 + j), (uint32_t)k)) =
                    (unsigned short)(w[j >> 1] >> ((j & 1) * 16));
        }
    }
}

// Stages rows [r0, r0 + rows) x K [k0, k0 + kBK) of an operand with any
// strides into a K-major tile, one element at a time; out-of-range elements
// are zero. Consecutive threads walk the contiguous dimension of the source.
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

constexpr int kEpPitch = 20;  // floats between the epilogue's staged rows

// Epilogue of C(m, n .. n + 3), the columns at or past N left alone; `vec`
// when C (and Cb) rows allow 16-byte (8-byte) stores.
template <int EPI>
__device__ __forceinline__ void epilogue4(const GemmArgs& g, int m, int n, float4 x, bool vec) {
    float v[4] = {x.x, x.y, x.z, x.w};
    const long long o = (long long)m * g.ldc + n;
    if constexpr (EPI == kEpiAtomic) {
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (n + j < g.N) atomicAdd(g.c + o + j, v[j]);
        return;
    }
    if constexpr (EPI == kEpiBias || EPI == kEpiBiasTanh) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float b = n + j < g.N ? g.bias[n + j] : 0.0f;
            v[j] = EPI == kEpiBiasTanh ? tanhf(v[j] + b) : v[j] + b;
        }
    }
    if (vec && n + 4 <= g.N) {
        *reinterpret_cast<float4*>(g.c + o) = make_float4(v[0], v[1], v[2], v[3]);
        if (EPI == kEpiBiasTanh) {
            __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]), hi = __floats2bfloat162_rn(v[2], v[3]);
            uint2 u;
            u.x = *reinterpret_cast<uint32_t*>(&lo);
            u.y = *reinterpret_cast<uint32_t*>(&hi);
            *reinterpret_cast<uint2*>(g.cb + o) = u;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (n + j < g.N) {
                g.c[o + j] = v[j];
                if (EPI == kEpiBiasTanh) g.cb[o + j] = __float2bfloat16(v[j]);
            }
    }
}

// BN: columns of C per CTA (16..128, a multiple of 16).
template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_tc(GemmArgs g) {
    constexpr uint32_t kTmemCols = BN <= 32 ? 32 : BN <= 64 ? 64 : 128;
    static_assert(kBK == 64 && BN % 16 == 0, "the staging chunk maps assume 64-element K tiles");
    static_assert(kGemmThreads * kEpPitch * 4 <= kBM * kBK * 2, "the epilogue rows fit in the A tile");
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
    const int ma = stage_mode(g.a, g.sam, g.sak), mb = stage_mode(g.b, g.sbn, g.sbk);
    StageBuf<kBM> ba;
    StageBuf<BN> bb;
    uint32_t phase = 0;
    bool issued = false;
    if (kb < ke) {
        stage_load<kBM>(ba, ma, g.a, g.sam, g.sak, m0, g.M, kb, ke);
        stage_load<BN>(bb, mb, g.b, g.sbn, g.sbk, n0, g.N, kb, ke);
    }
    for (int k0 = kb; k0 < ke; k0 += kBK) {
        if (ma == kStageAny) stage_operand(sa, g.a, g.sam, g.sak, m0, g.M, kBM, k0, ke);
        else stage_store<kBM>(sa, ba, ma);
        if (mb == kStageAny) stage_operand(sb, g.b, g.sbn, g.sbk, n0, g.N, BN, k0, ke);
        else stage_store<BN>(sb, bb, mb);
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
        // the next chunk's loads overlap the MMAs
        if (k0 + kBK < ke) {
            stage_load<kBM>(ba, ma, g.a, g.sam, g.sak, m0, g.M, k0 + kBK, ke);
            stage_load<BN>(bb, mb, g.b, g.sbn, g.sbk, n0, g.N, k0 + kBK, ke);
        }
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
        // Each warp reads its 32 accumulator rows 16 columns at a time and
        // passes them through shared memory (the A tile, free once the last
        // MMA completed; rows kEpPitch floats apart, so the 16-byte writes
        // of 8 consecutive rows fall in distinct banks), then writes them out
        // as 4-column runs, 4 lanes per row.
        float* ep = reinterpret_cast<float*>(sa) + warp * 32 * kEpPitch;
        const bool vec = (g.ldc & 3) == 0 && (reinterpret_cast<uintptr_t>(g.c) & 15u) == 0 &&
                         (EPI != kEpiBiasTanh || (reinterpret_cast<uintptr_t>(g.cb) & 7u) == 0);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            float4* own = reinterpret_cast<float4*>(ep + lane * kEpPitch);
#pragma unroll
            for (int q = 0; q < 4; q++) own[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int idx = lane + 32 * i, r = idx >> 2, q = idx & 3;
                const int m = m0 + warp * 32 + r, n = n0 + c0 + q * 4;
                const float4 x = *reinterpret_cast<const float4*>(ep + r * kEpPitch + q * 4);
                if (m < g.M && n < g.N) epilogue4<EPI>(g, m, n, x, vec);
            }
            __syncwarp();
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

// Loads a FP32 weight matrix [n_rows x k_cols] (row-major, ld = k_cols) into
// a K-major BF16 tile.
__device__ __forceinline__ void stage_weights(unsigned char* tile, const float* w, int n_rows, int k_cols) {
    for (int e = threadIdx.x; e < n_rows * k_cols; e += blockDim.x) {
        int r = e / k_cols, k = e % k_cols;
        *reinterpret_cast<__nv_bfloat16*>(tile + tile_off_k(r, k, k_cols)) = __float2bfloat16(w[e]);
    }
}

// Dynamic shared memory of a whole-network tile: the input tile, the three
// weight tiles and the hidden activations.
__host__ __device__ inline size_t infer_smem_bytes(int dp, int op) {
    return (size_t)128 * dp * 2 + 128 * dp * 2 + 128 * 128 * 2 + (size_t)op * 128 * 2 + 128 * 128 * 2;
}

// The three BF16 weight tiles (W1 128 x dp, W2 128 x 128, W3 op x 128) laid
// out exactly as a whole-network tile stages them, back to back: a kernel
// copies this image into shared memory with one bulk copy.
__host__ __device__ inline size_t weight_image_bytes(int dp, int op) {
    return (size_t)128 * dp * 2 + 128 * 128 * 2 + (size_t)op * 128 * 2;
}

// The three layers of one 128-row tile on the tensor cores. sx holds the
// standardized BF16 inputs (dp columns) and sw1 / sw2 / sw3 the BF16 weights,
// all K-major core-matrix tiles in shared memory; sh (128 x 128 BF16) takes
// the hidden activations. Each layer is one chain of tcgen05.mma (K = 16 per
// MMA) into the tensor memory at `tmem` (128 columns), committed to `bar`;
// its epilogue (bias, tanh) goes back to sh as the next layer's operand. The
// output layer calls out(row, o, acc + b3[o]) for every o < out_dim, row
// being this thread's tile row (still standardized). Every thread of the
// 128-thread block takes part. Returns false when a bounded wait ran out,
// after a second bounded wait for the MMAs in flight; the caller frees the
// tensor memory either way.
template <typename Out>
__device__ bool mlp_layers(const unsigned char* sx, const unsigned char* sw1, const unsigned char* sw2,
                           const unsigned char* sw3, unsigned char* sh, const float* b1, const float* b2,
                           const float* b3, int dp, int op, int out_dim, uint32_t tmem, uint64_t* bar, int* failed,
                           Out out) {
    const int H = 128;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
            tc_commit(bar);
        }
        if (!mbar_wait_bounded(bar, phase)) *failed = 1;
        __syncthreads();
        if (*failed) {
            mbar_wait_bounded(bar, phase);
            return false;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (layer < 2) {
            const float* bias = layer == 0 ? b1 : b2;
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
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int o = c0 + i;
                    if (o < out_dim) out(row, o, v[i] + b3[o]);
                }
            }
        }
    }
    return true;
}

// What a kernel outside the network's own module reads of a trained network
// (the transient's step predictor): the weight image (weight_image_bytes),
// the biases, the input standardization and the output scaling. out_gain[o]
// is the output's standard deviation, 0 for an output that was constant over
// the training set (its prediction is then out_mean[o] exactly).
struct MlpView {
    const unsigned char* image;
    const float *b1, *b2, *b3;
    const float *in_mean, *in_std, *out_mean, *out_gain;
    int in_dim, dp, out_dim, op;
    int* err;
};

}  // namespace mlp
}  // namespace espl

struct espl_mlp;
// Fills `v` for network `h` (packing the weight image first when the
// weights changed since the last call). ESPL_OK or a driver error code.
uint32_t espl_mlp_view(espl_mlp* h, espl::mlp::MlpView* v, void* stream);
