// The LU chain of a small template entirely in shared memory. The tape's
// index words are staged once per launch by bulk copies (cp.async.bulk, the
// TMA's 1-D form) completing on an mbarrier; the gather phase writes the
// assembled matrix and right-hand side into the tile's shared copies as well
// as to global memory; the replay, the triangular solves and the FP32
// refinement then touch only shared memory, one thread per lane, with the
// 32 lanes interleaved (element i of lane j at i * 32 + j: a warp reads one
// element of all lanes as 32 consecutive words, conflict-free).
//
// Same operations in the same order as refactor64/refactor32 and
// solve64/solve32 (src/solver/kernels/lane.zig:56-157), so a lane's factor
// and step are bitwise the global path's.
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
// carry that padding).
enum TapeArr { T_Q, T_COLPTR, T_ROWIDX, T_PROW, T_UP, T_UI, T_LP, T_LI, T_FLAGS, T_PINV, T_COUNT };

__host__ __device__ inline uint32_t pad4(uint32_t words) { return (words + 3u) & ~3u; }

struct SmemPlan {
    uint32_t off[T_COUNT];   // u32-word offsets of the tape arrays
    uint32_t len[T_COUNT];   // padded word counts
    uint32_t tape_words;     // total (multiple of 4)
    uint32_t a_off, rhs_off, w_off, y_off, lx_off, ux_off, ud_off, r_off, c_off, dx_off;  // byte offsets
    uint32_t bytes;          // total dynamic shared memory of the tile
};

// Layout of the tile's dynamic shared memory for template sizes (n, nnz,
// nnz_l, nnz_u). The LU arrays hold doubles, so a mixed lane can fall back to
// FP64 in place; an FP32 view uses the first half of each. `mixed` adds the
// refinement vectors.
__host__ __device__ inline SmemPlan smem_plan(uint32_t n, uint32_t nnz, uint32_t nl, uint32_t nu, bool mixed) {
    const uint32_t es = 8;
    SmemPlan p;
    uint32_t words[T_COUNT] = {n, n + 1, nnz, nnz, n + 1, nu, n + 1, nl, n, n};
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
    b += nnz * 32u * 8u;
    p.rhs_off = b;
    b += n * 32u * 8u;
    p.dx_off = b;
    b += n * 32u * 8u;
    p.r_off = b;           // FP64 refinement residual
    if (mixed) b += n * 32u * 8u;
    p.c_off = b;           // FP64 refinement correction
    if (mixed) b += n * 32u * 8u;
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
    const uint32_t *q, *col_ptr, *row_idx, *prow, *up, *ui, *lp, *li, *flags, *pinv;
    double *a, *rhs, *dx, *r, *corr;
    void *w, *y, *lx, *ux, *ud;
};

__device__ __forceinline__ SmemTile smem_tile(unsigned char* base, const SmemPlan& p) {
    const uint32_t* u = reinterpret_cast<const uint32_t*>(base);
    SmemTile t;
    t.q = u + p.off[T_Q];
    t.col_ptr = u + p.off[T_COLPTR];
    t.row_idx = u + p.off[T_ROWIDX];
    t.prow = u + p.off[T_PROW];
    t.up = u + p.off[T_UP];
    t.ui = u + p.off[T_UI];
    t.lp = u + p.off[T_LP];
    t.li = u + p.off[T_LI];
    t.flags = u + p.off[T_FLAGS];
    t.pinv = u + p.off[T_PINV];
    t.a = reinterpret_cast<double*>(base + p.a_off);
    t.rhs = reinterpret_cast<double*>(base + p.rhs_off);
    t.dx = reinterpret_cast<double*>(base + p.dx_off);
    t.r = reinterpret_cast<double*>(base + p.r_off);
    t.corr = reinterpret_cast<double*>(base + p.c_off);
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
    const uint32_t* src[T_COUNT] = {d.q, d.col_ptr, d.row_idx, d.prow, d.up, d.ui, d.lp, d.li, d.flags, d.pinv};
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
    uint32_t nz = (p.lx_off - p.w_off) / 4u;
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
__device__ int refactor_smem(const GroupDev& d, const SmemTile& s, uint32_t lane) {
    T* __restrict__ w = static_cast<T*>(s.w);
    T* __restrict__ lx = static_cast<T*>(s.lx);
    T* __restrict__ ux = static_cast<T*>(s.ux);
    T* __restrict__ ud = static_cast<T*>(s.ud);
    const double* __restrict__ a = s.a;
    for (uint32_t v = 0; v < d.n_void; v++)
        if (SL(a, d.void_slots[v]) != 0.0) return 1;
    constexpr bool f64 = sizeof(T) == 8;
    bool bad = false, nonfinite = false;
    const T growth = (T)1e-12;
    const T inf = (T)INFINITY;
    for (uint32_t k = 0; k < d.n; k++) {
        uint32_t c = s.q[k];
        for (uint32_t p = s.col_ptr[c]; p < s.col_ptr[c + 1]; p++) SL(w, s.prow[p]) = (T)SL(a, p);
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

// out = -A^-1 b through the shared factors (luSolve with neg), b and out by
// original row/column in shared memory.
template <typename T>
__device__ void solve_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, const double* b, double* out) {
    T* __restrict__ y = static_cast<T*>(s.y);
    const T* __restrict__ lx = static_cast<const T*>(s.lx);
    const T* __restrict__ ux = static_cast<const T*>(s.ux);
    const T* __restrict__ ud = static_cast<const T*>(s.ud);
    for (uint32_t r = 0; r < d.n; r++) SL(y, s.pinv[r]) = (T)(-SL(b, r));
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
    for (uint32_t j = 0; j < d.n; j++) SL(out, s.q[j]) = (double)SL(y, j);
}

// One FP64-residual refinement sweep of an FP32 solve in shared memory:
// r = rhs + A dx, dx += -A^-1 r.
__device__ void refine_smem(const GroupDev& d, const SmemTile& s, uint32_t lane) {
    for (uint32_t i = 0; i < d.n; i++) SL(s.r, i) = SL(s.rhs, i);
    for (uint32_t c = 0; c < d.n; c++) {
        double xc = SL(s.dx, c);
        if (xc == 0.0) continue;
        for (uint32_t p = s.col_ptr[c]; p < s.col_ptr[c + 1]; p++) SL(s.r, s.row_idx[p]) += SL(s.a, p) * xc;
    }
    solve_smem<float>(d, s, lane, s.r, s.corr);
    for (uint32_t i = 0; i < d.n; i++) SL(s.dx, i) += SL(s.corr, i);
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
