// The LU chain of a template in shared memory. The tape's index words are
// staged once per launch by bulk copies (cp.async.bulk, the TMA's 1-D form)
// completing on an mbarrier; the gather phase writes the assembled matrix
// into the tile's shared copy (in the factor's precision) as well as to
// global memory (FP64); the replay and the triangular solves then touch
// only shared memory, one thread per lane, with the 32 lanes interleaved
// (element i of lane j at i * 32 + j: a warp reads one element of all lanes
// as 32 consecutive words, conflict-free). Right-hand sides, the Newton step
// and the FP64 refinement residual stay in global memory, read once per
// row.
//
// FP64 tiles run the same operations in the same order as refactor64 and
// solve64 (src/solver/kernels/lane.zig:56-157), so a lane's factor and step
// are bitwise the global path's; FP32 tiles those of refactor32/solve32 and
// refine_mixed. A mixed lane that falls back to FP64 takes the global path.
#pragma once

#include "lane_tile.cuh"

namespace espl {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Tape arrays staged per tile, in this order; each starts on a 16-byte
// boundary and is copied padded to a 16-byte multiple (the global buffers
// carry that padding). The row view (RTPTR/RTCOL/RTPOS: per row, the
// columns and slots of its entries by ascending column) feeds the FP32
// tiles' refinement residual.
enum TapeArr { T_Q, T_COLPTR, T_PROW, T_UP, T_UI, T_LP, T_LI, T_FLAGS, T_PINV, T_RTPTR, T_RTCOL, T_RTPOS, T_COUNT };

__host__ __device__ inline uint32_t pad4(uint32_t words) { return (words + 3u) & ~3u; }

struct SmemPlan {
    uint32_t off[T_COUNT];   // u32-word offsets of the tape arrays
    uint32_t len[T_COUNT];   // padded word counts
    uint32_t tape_words;     // total (multiple of 4)
    uint32_t a_off, w_off, y_off, lx_off, ux_off, ud_off;  // byte offsets
    uint32_t bytes;          // total dynamic shared memory of the tile
};

// Layout of the tile's dynamic shared memory for template sizes (n, nnz,
// nnz_l, nnz_u): the staged tape, then A, the work vectors w and y, and
// the factor, all in FP32 for `f32` tiles and FP64 otherwise.
__host__ __device__ inline SmemPlan smem_plan(uint32_t n, uint32_t nnz, uint32_t nl, uint32_t nu, bool f32) {
    const uint32_t es = f32 ? 4u : 8u;
    SmemPlan p;
    uint32_t words[T_COUNT] = {n, n + 1, nnz, n + 1, nu, n + 1, nl, n, n,
                               f32 ? n + 1 : 0u, f32 ? nnz : 0u, f32 ? nnz : 0u};
    uint32_t o = 4;  // the first 16 bytes hold the mbarrier
    for (int k = 0; k < T_COUNT; k++) {
        p.off[k] = o;
        p.len[k] = pad4(words[k]);
        o += p.len[k];
    }
    p.tape_words = o - 4;
    uint32_t b = o * 4;
    b = (b + 15u) & ~15u;
    p.a_off = b;
    b += nnz * 32u * es;
    p.w_off = b;
    b += n * 32u * es;
    p.y_off = b;
    b += n * 32u * es;
    p.lx_off = b;
    b += nl * 32u * es;
    p.ux_off = b;
    b += nu * 32u * es;
    p.ud_off = b;
    b += n * 32u * es;
    p.bytes = (b + 15u) & ~15u;
    return p;
}

struct SmemTile {
    const uint32_t *q, *col_ptr, *prow, *up, *ui, *lp, *li, *flags, *pinv, *rt_ptr, *rt_col, *rt_pos;
    void *a, *w, *y, *lx, *ux, *ud;
};

__device__ __forceinline__ SmemTile smem_tile(unsigned char* base, const SmemPlan& p) {
    const uint32_t* u = reinterpret_cast<const uint32_t*>(base);
    SmemTile t;
    t.q = u + p.off[T_Q];
    t.col_ptr = u + p.off[T_COLPTR];
    t.prow = u + p.off[T_PROW];
    t.up = u + p.off[T_UP];
    t.ui = u + p.off[T_UI];
    t.lp = u + p.off[T_LP];
    t.li = u + p.off[T_LI];
    t.flags = u + p.off[T_FLAGS];
    t.pinv = u + p.off[T_PINV];
    t.rt_ptr = u + p.off[T_RTPTR];
    t.rt_col = u + p.off[T_RTCOL];
    t.rt_pos = u + p.off[T_RTPOS];
    t.a = base + p.a_off;
    t.w = base + p.w_off;
    t.y = base + p.y_off;
    t.lx = base + p.lx_off;
    t.ux = base + p.ux_off;
    t.ud = base + p.ud_off;
    return t;
}

// Stages the tape by bulk copies; thread 0 issues them, every thread of
// warp 0 waits (bounded: a copy of in-bounds memory completes, and past the
// bound the flag tells the caller to stay on the global path). The work
// vectors start at zero.
__device__ bool stage_tape(const GroupDev& d, unsigned char* base, const SmemPlan& p) {
    uint64_t* bar = reinterpret_cast<uint64_t*>(base);
    const uint32_t* src[T_COUNT] = {d.q, d.col_ptr, d.prow, d.up, d.ui, d.lp, d.li, d.flags, d.pinv,
                                    d.rt_ptr, d.rt_col, d.rt_pos};
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(bar, p.tape_words * 4u);
        uint32_t* u = reinterpret_cast<uint32_t*>(base);
        for (int k = 0; k < T_COUNT; k++)
            if (p.len[k]) bulk_g2s(u + p.off[k], src[k], p.len[k] * 4u, bar);
    }
    // zero w and y (both precisions share the invariant: all-zero bits)
    uint32_t* wz = reinterpret_cast<uint32_t*>(base + p.w_off);
    uint32_t nz = (p.lx_off - p.w_off) / 4u;  // w and y
    for (uint32_t i = threadIdx.x; i < nz; i += blockDim.x) wz[i] = 0u;
    __syncthreads();
    bool ok = true;
    if (threadIdx.x < 32) {
        uint32_t tries = 0;
        while (!mbar_try_wait(bar, 0)) {
            if (++tries > (1u << 26)) {
                ok = false;
                break;
            }
        }
    }
    return __syncthreads_and(ok || threadIdx.x >= 32) != 0;
}

#define SL(arr, i) (arr)[(size_t)(i) * 32 + lane]

// The replay in shared memory; T = double or float. 0 holds, 1 pivot or
// store failure, 2 only a multiplier past 1 / pivot_tol.
template <typename T>
__device__ int refactor_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    T* __restrict__ w = static_cast<T*>(s.w);
    T* __restrict__ lx = static_cast<T*>(s.lx);
    T* __restrict__ ux = static_cast<T*>(s.ux);
    T* __restrict__ ud = static_cast<T*>(s.ud);
    const T* __restrict__ a = static_cast<const T*>(s.a);
    const uint32_t P = d.P;
    for (uint32_t v = 0; v < d.n_void; v++)
        if (LM(d.a, d.void_slots[v]) != 0.0) return 1;
    constexpr bool f64 = sizeof(T) == 8;
    bool bad = false, nonfinite = false;
    const T growth = (T)1e-12;
    const T inf = (T)INFINITY;
    for (uint32_t k = 0; k < d.n; k++) {
        uint32_t c = s.q[k];
        for (uint32_t p = s.col_ptr[c]; p < s.col_ptr[c + 1]; p++) SL(w, s.prow[p]) = SL(a, p);
        for (uint32_t p = s.up[k]; p < s.up[k + 1]; p++) {
            uint32_t i = s.ui[p];
            T uki = SL(w, i);
            SL(w, i) = (T)0;
            SL(ux, p) = uki;
            nonfinite |= !(uki - uki == (T)0);
            for (uint32_t pl = s.lp[i]; pl < s.lp[i + 1]; pl++) SL(w, s.li[pl]) -= SL(lx, pl) * uki;
        }
        uint32_t fl = s.flags[k];
        if (fl & 1u) {
            SL(ud, k) = (T)1;
            for (uint32_t p = s.lp[k]; p < s.lp[k + 1]; p++) { SL(lx, p) = (T)0; SL(w, s.li[p]) = (T)0; }
            SL(w, k) = (T)0;
            for (uint32_t p = s.up[k]; p < s.up[k + 1]; p++) {
                uint32_t i = s.ui[p];
                for (uint32_t pl = s.lp[i]; pl < s.lp[i + 1]; pl++) SL(w, s.li[pl]) = (T)0;
            }
            continue;
        }
        T dk = SL(w, k);
        SL(w, k) = (T)0;
        bool dead = dk == (T)0 || !(fabs(dk) < inf);
        bad |= dead;
        if (dead) dk = (T)1;
        SL(ud, k) = dk;
        if constexpr (f64) {
            if (!(fl & 2u)) {
                uint64_t cb = dbits(fabs((double)dk));
                for (uint32_t p = s.lp[k]; p < s.lp[k + 1]; p++) {
                    uint32_t r = s.li[p];
                    T v = SL(w, r);
                    SL(w, r) = (T)0;
                    uint64_t vb = dbits(fabs((double)v));
                    cb = cb > vb ? cb : vb;
                    SL(lx, p) = v / dk;
                }
                bad |= !(fabs((double)dk) >= 1e-12 * bitsd(cb));
            } else {
                for (uint32_t p = s.lp[k]; p < s.lp[k + 1]; p++) {
                    uint32_t r = s.li[p];
                    T lv = SL(w, r) / dk;
                    nonfinite |= !(lv - lv == (T)0);
                    SL(lx, p) = lv;
                    SL(w, r) = (T)0;
                }
            }
        } else {
            T cmax = fabs(dk);
            for (uint32_t p = s.lp[k]; p < s.lp[k + 1]; p++) {
                uint32_t r = s.li[p];
                T v = SL(w, r);
                SL(w, r) = (T)0;
                cmax = fmaxf(cmax, fabsf(v));
                T lv = v / dk;
                nonfinite |= !(lv - lv == (T)0);
                SL(lx, p) = lv;
            }
            if (!(fl & 2u)) bad |= !(fabsf(dk) >= growth * cmax) || !(cmax / fabsf(dk) <= (T)kWide);
        }
    }
    if (nonfinite || bad) return 1;
    if constexpr (f64) {
        uint64_t worst = 0;
        for (uint32_t k = 0; k < d.n; k++) {
            if (s.flags[k] & 2u) continue;
            for (uint32_t p = s.lp[k]; p < s.lp[k + 1]; p++) {
                uint64_t b = dbits(fabs((double)SL(lx, p)));
                worst = worst > b ? worst : b;
            }
        }
        return bitsd(worst) <= kWide ? 0 : 2;
    }
    return 0;
}

// Forward and back substitution of y in place through the shared factors
// (luSolve's two sweeps).
template <typename T>
__device__ __forceinline__ void subst_smem(const GroupDev& d, const SmemTile& s, uint32_t lane) {
    T* __restrict__ y = static_cast<T*>(s.y);
    const T* __restrict__ lx = static_cast<const T*>(s.lx);
    const T* __restrict__ ux = static_cast<const T*>(s.ux);
    const T* __restrict__ ud = static_cast<const T*>(s.ud);
    for (uint32_t k = 0; k < d.n; k++) {
        T yk = SL(y, k);
        if (yk != (T)0)
            for (uint32_t p = s.lp[k]; p < s.lp[k + 1]; p++) SL(y, s.li[p]) -= SL(lx, p) * yk;
    }
    for (uint32_t k = d.n; k-- > 0;) {
        T zk = SL(y, k) / SL(ud, k);
        SL(y, k) = zk;
        if (zk != (T)0)
            for (uint32_t p = s.up[k]; p < s.up[k + 1]; p++) SL(y, s.ui[p]) -= SL(ux, p) * zk;
    }
}

// dx = -A^-1 rhs through the shared factors (luSolve with neg); rhs and dx
// are the lane's global rows.
template <typename T>
__device__ void solve_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    const uint32_t P = d.P;
    T* __restrict__ y = static_cast<T*>(s.y);
    for (uint32_t r = 0; r < d.n; r++) SL(y, s.pinv[r]) = (T)(-LM(d.rhs, r));
    subst_smem<T>(d, s, lane);
    for (uint32_t j = 0; j < d.n; j++) LM(d.dx, s.q[j]) = (double)SL(y, j);
}

// One FP64-residual refinement sweep of an FP32 solve (refine_mixed):
// r = rhs + A dx row by row, the products added by ascending column as the
// column sweep adds them (columns with dx = 0 skipped), then
// dx += -A^-1 r through the FP32 factors.
__device__ void refine_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    const uint32_t P = d.P;
    float* __restrict__ y = static_cast<float*>(s.y);
    for (uint32_t i = 0; i < d.n; i++) {
        double r = LM(d.rhs, i);
        for (uint32_t e = s.rt_ptr[i]; e < s.rt_ptr[i + 1]; e++) {
            double xc = LM(d.dx, s.rt_col[e]);
            if (xc != 0.0) r += LM(d.a, s.rt_pos[e]) * xc;
        }
        SL(y, s.pinv[i]) = (float)(-r);
    }
    subst_smem<float>(d, s, lane);
    for (uint32_t j = 0; j < d.n; j++) LM(d.dx, s.q[j]) += (double)SL(y, j);
}

// Copies a shared factor out to the lane's global factor arrays, for the
// global fallbacks (replay probe, peel) after a failed shared replay.
template <typename T>
__device__ void spill_factor(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    const uint32_t P = d.P;
    const T* lx = static_cast<const T*>(s.lx);
    const T* ux = static_cast<const T*>(s.ux);
    const T* ud = static_cast<const T*>(s.ud);
    for (uint32_t p = 0; p < d.nnz_l; p++) LM(d.lx, p) = (double)SL(lx, p);
    for (uint32_t p = 0; p < d.nnz_u; p++) LM(d.ux, p) = (double)SL(ux, p);
    for (uint32_t k = 0; k < d.n; k++) LM(d.udiag, k) = (double)SL(ud, k);
}

#undef SL

}  // namespace espl
