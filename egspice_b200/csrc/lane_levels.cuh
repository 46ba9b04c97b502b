// The LU of large templates, run by the whole CTA.
//
// A template whose factor fits neither the tile's shared memory nor the
// banded streaming replay (a power-grid mesh of 40,000 unknowns: 2 million
// factor entries per lane) would leave one thread per lane walking its whole
// factor while the other warps wait. Here the template's tiles run as parts
// of a few lanes, one CTA each, and every thread of the CTA works on the
// LU of its part: thread (share, lane) handles lane `lane` of the share of
// the work chosen by `share` (TileCtx.warp), a factor entry being one
// contiguous load of the part's lanes.
//
// Refactor (lvl_refactor): the frozen tape's columns in order (the replay of
// src/solver/kernels/lane.zig:56-125): a column's scatter, its U entries in
// the tape's topological order -- each entry's axpy of an L column split
// over the warps, a CTA barrier between entries -- and the pivot with its L
// entries split over the warps. The same operations on the same values as
// the one-thread replay, so the factor is the same to the bit.
//
// Solves (lvl_solve): row-oriented ("pull") sweeps over the level schedule
// of tape.h LevelPlan. Rows of a level are independent: with at least as
// many rows as warps each warp takes whole rows; with fewer, each row's
// entries are split over a group of warps and the group's partial sums are
// added in a fixed order after a barrier. The sums run in another order than
// the column sweeps of solve64, so a solve agrees with them to rounding.
//
// A linear template's A changes only with the companion coefficient and
// gmin, so a lane refactors only when that key changes (the reference's
// bypass of identical values, src/solver/direct.zig:313).
#pragma once

#include "lane_engine.cuh"

namespace espl {

// Per-lane reductions of the refactor, in the tile's shared memory.
struct LevelShared {
    uint32_t bad[32];              // a dead pivot, growth failure or filled void slot
    uint32_t nonfinite[32];        // OR of (u - u) bits: a NaN somewhere
    unsigned long long cmax[32];   // the column's largest |L| numerator (by bits)
    unsigned long long worst[32];  // the largest |L| over non-scaled columns (by bits)
};

template <typename T>
__device__ __forceinline__ uint64_t mag_bits(T v) {
    return dbits((double)fabs(v));
}

// sum over entries e = e0, e0 + stride, ... < e1 of vals[slot_e] y[col_e]
// for one lane (entries are (col, slot) pairs), in batches of eight: a
// batch's index, value and y loads are all issued before any is used (past
// the row's end they are skipped and read as zero), so eight gathers are in
// flight instead of one; a batch's products are added in a fixed order.
template <typename T>
__device__ __forceinline__ T row_dot(const uint2* __restrict__ e2, uint32_t e0, uint32_t e1, uint32_t stride,
                                     const T* __restrict__ vals, const T* __restrict__ y, uint32_t P, uint32_t l) {
    T acc = (T)0;
    for (uint32_t e = e0; e < e1; e += 8 * stride) {
        uint2 ce[8];
#pragma unroll
        for (int k = 0; k < 8; k++) ce[k] = e + k * stride < e1 ? e2[e + k * stride] : make_uint2(0u, kNone);
        T v[8], yv[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const bool ok = ce[k].y != kNone;
            v[k] = ok ? LM(vals, ce[k].y) : (T)0;
            yv[k] = ok ? LM(y, ce[k].x) : (T)0;
        }
        T s = v[0] * yv[0];
#pragma unroll
        for (int k = 1; k < 8; k++) s += v[k] * yv[k];
        acc += s;
    }
    return acc;
}

// One lane's refactor status (0 holds, 1 fails, 2 only a multiplier past
// 1 / pivot_tol) for every thread of the lane. `act`: the lane refactors;
// lanes that do not leave their factor as it is. All threads of the CTA call
// it.
template <typename T>
__device__ int lvl_refactor(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                            T* __restrict__ w, T* __restrict__ lx, T* __restrict__ ux, T* __restrict__ ud,
                            LevelShared& ls) {
    const uint32_t P = d.P;
    const double* __restrict__ a = d.a;
    constexpr bool F32 = sizeof(T) == 4;
    if (warp == 0) {
        uint32_t bad = 0;
        if (act)
            for (uint32_t v = 0; v < d.n_void; v++)
                if (LM(a, d.void_slots[v]) != 0.0) bad = 1;
        ls.bad[lane] = bad;
        ls.nonfinite[lane] = 0;
        ls.cmax[lane] = 0;
        ls.worst[lane] = 0;
    }
    __syncthreads();
    for (uint32_t k = 0; k < d.n; k++) {
        const uint32_t c = d.q[k];
        if (act)
            for (uint32_t p = d.col_ptr[c] + warp; p < d.col_ptr[c + 1]; p += nw) LM(w, d.prow[p]) = (T)LM(a, p);
        __syncthreads();
        const uint32_t u0 = d.up[k], u1 = d.up[k + 1];
        for (uint32_t p = u0; p < u1; p++) {
            const uint32_t i = d.ui[p];
            const T u = act ? LM(w, i) : (T)0;
            if (act) {
                for (uint32_t pl = d.lp[i] + warp; pl < d.lp[i + 1]; pl += nw) LM(w, d.li[pl]) -= LM(lx, pl) * u;
                if (warp == 0) {
                    LM(ux, p) = u;
                    ls.nonfinite[lane] |= (uint32_t)(mag_bits(u - u) != 0);
                }
            }
            __syncthreads();
        }
        // the taken rows of the work vector (each U entry's row) go back to zero
        if (act)
            for (uint32_t p = u0 + warp; p < u1; p += nw) LM(w, d.ui[p]) = (T)0;
        const uint32_t fl = d.flags[k];
        if (fl & 1u) {
            // a void column: unit pivot, no L entries, and every row its
            // takes filled is cleared
            if (act) {
                for (uint32_t p = d.lp[k] + warp; p < d.lp[k + 1]; p += nw) {
                    LM(lx, p) = (T)0;
                    LM(w, d.li[p]) = (T)0;
                }
                for (uint32_t p = u0; p < u1; p++) {
                    const uint32_t i = d.ui[p];
                    for (uint32_t pl = d.lp[i] + warp; pl < d.lp[i + 1]; pl += nw) LM(w, d.li[pl]) = (T)0;
                }
                if (warp == 0) {
                    LM(ud, k) = (T)1;
                    LM(w, k) = (T)0;
                }
            }
            __syncthreads();
            continue;
        }
        __syncthreads();
        T dk = act ? LM(w, k) : (T)1;
        const bool dead = dk == (T)0 || !(fabs(dk) < (T)INFINITY);
        if (dead) dk = (T)1;
        uint64_t cb = mag_bits(dk);
        uint32_t nf = 0;
        if (act)
            for (uint32_t p = d.lp[k] + warp; p < d.lp[k + 1]; p += nw) {
                const uint32_t r = d.li[p];
                const T v = LM(w, r);
                LM(w, r) = (T)0;
                const uint64_t vb = mag_bits(v);
                cb = cb > vb ? cb : vb;
                const T lv = v / dk;
                if (F32 || (fl & 2u)) nf |= (uint32_t)(mag_bits(lv - lv) != 0);
                LM(lx, p) = lv;
                if (!(fl & 2u)) {
                    const uint64_t lb = mag_bits(lv);
                    if (lb > ls.worst[lane]) atomicMax(&ls.worst[lane], lb);
                }
            }
        if (act) {
            atomicMax(&ls.cmax[lane], cb);
            if (nf) atomicOr(&ls.nonfinite[lane], 1u);
        }
        __syncthreads();
        if (warp == 0 && act) {
            LM(ud, k) = dk;
            LM(w, k) = (T)0;
            uint32_t bad = dead ? 1u : 0u;
            const double cmax = bitsd(ls.cmax[lane]);
            if (!(fl & 2u)) {
                if (F32)
                    bad |= (!(fabs((double)dk) >= 1e-12 * cmax) || !(cmax / fabs((double)dk) <= kWide)) ? 1u : 0u;
                else
                    bad |= !(fabs((double)dk) >= 1e-12 * cmax) ? 1u : 0u;
            }
            ls.bad[lane] |= bad;
            ls.cmax[lane] = 0;
        }
        __syncthreads();
    }
    const int rc = (ls.bad[lane] || ls.nonfinite[lane]) ? 1 : (bitsd(ls.worst[lane]) <= kWide || F32) ? 0 : 2;
    __syncthreads();
    return rc;
}

// One sweep of a level-scheduled solve over y (lane-interleaved): forward
// (BACK false) y_i -= sum L_ij y_j by the L rows; backward y_j = (y_j -
// sum U_jk y_k) / U_jj by the U rows. `red` holds one partial sum per thread.
template <typename T, bool BACK>
__device__ void lvl_sweep(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                          const uint32_t* __restrict__ lptr, const uint32_t* __restrict__ rows, uint32_t nlev,
                          const uint32_t* __restrict__ rptr, const uint32_t* __restrict__ ent,
                          const T* __restrict__ vals, const T* __restrict__ ud, T* __restrict__ y, T* red) {
    const uint32_t P = d.P;
    const uint2* __restrict__ e2 = reinterpret_cast<const uint2*>(ent);
    for (uint32_t v = 0; v < nlev; v++) {
        const uint32_t r0 = lptr[v], m = lptr[v + 1] - r0;
        if (m >= nw) {
            if (act)
                for (uint32_t k = r0 + warp; k < r0 + m; k += nw) {
                    const uint32_t i = rows[k];
                    T acc = LM(y, i) - row_dot<T>(e2, rptr[i], rptr[i + 1], 1u, vals, y, P, l);
                    if (BACK) acc = acc / LM(ud, i);
                    LM(y, i) = acc;
                }
        } else {
            // m < nw rows: gs shares per row (a power of two, so a row's
            // shares are an aligned run of threads), each summing a strided
            // part of the row; the parts are added by a butterfly of warp
            // shuffles inside each hardware warp, then (a row over several
            // warps) the warps' sums in order through shared memory -- a
            // fixed order either way
            uint32_t gs = 1;
            while (gs * 2 * m <= nw) gs *= 2;
            const uint32_t row = warp / gs, sub = warp % gs;
            const uint32_t tw = blockDim.x / nw, spw = 32u / tw;  // shares per hardware warp
            T part = (T)0;
            uint32_t i = 0;
            if (row < m) {
                i = rows[r0 + row];
                if (act) part = row_dot<T>(e2, rptr[i] + sub, rptr[i + 1], gs, vals, y, P, l);
            }
            for (uint32_t o = 1; o < gs && o < spw; o *= 2) part += __shfl_xor_sync(0xffffffffu, part, o * tw);
            if (gs > spw) {
                if ((threadIdx.x & 31u) < tw) red[(threadIdx.x >> 5) * tw + lane] = part;
                __syncthreads();
                if (row < m && sub == 0 && act) {
                    const uint32_t w0 = (row * gs) / spw, nwarps = gs / spw;
                    T sum = (T)0;
                    for (uint32_t k = 0; k < nwarps; k++) sum += red[(w0 + k) * tw + lane];
                    part = sum;
                }
            }
            if (row < m && sub == 0 && act) {
                T acc = LM(y, i) - part;
                if (BACK) acc = acc / LM(ud, i);
                LM(y, i) = acc;
            }
        }
        __syncthreads();
    }
}

// out = -A^-1 rhs through the lane's factors (luSolve with neg, solve64's
// contract), every thread of the CTA taking part.
template <typename T>
__device__ void lvl_solve(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                          const double* __restrict__ rhs, double* __restrict__ out, T* __restrict__ y,
                          const T* __restrict__ lx, const T* __restrict__ ux, const T* __restrict__ ud, T* red) {
    const uint32_t P = d.P;
    if (act)
        for (uint32_t r = warp; r < d.n; r += nw) LM(y, d.pinv[r]) = (T)(-LM(rhs, r));
    __syncthreads();
    lvl_sweep<T, false>(d, l, lane, warp, nw, act, d.fl_ptr, d.fl_rows, d.n_fl, d.rl_ptr, d.rl_ent, lx, nullptr, y,
                        red);
    lvl_sweep<T, true>(d, l, lane, warp, nw, act, d.bl_ptr, d.bl_rows, d.n_bl, d.ru_ptr, d.ru_ent, ux, ud, y, red);
    if (act)
        for (uint32_t j = warp; j < d.n; j += nw) LM(out, d.q[j]) = (double)LM(y, j);
    __syncthreads();
}

// One FP64-residual refinement sweep of a mixed solve (refine_mixed's
// contract), rows split over the warps through the row view of A:
// r = rhs + A dx, dx += -A^-1 r by the FP32 factors.
__device__ void lvl_refine(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                           float* red) {
    const uint32_t P = d.P;
    if (act)
        for (uint32_t i = warp; i < d.n; i += nw) {
            double r = LM(d.rhs, i);
            for (uint32_t e = d.rt_ptr[i]; e < d.rt_ptr[i + 1]; e++) r += LM(d.a, d.rt_pos[e]) * LM(d.dx, d.rt_col[e]);
            LM(d.rr, i) = r;
        }
    __syncthreads();
    lvl_solve<float>(d, l, lane, warp, nw, act, d.rr, d.corr, d.y32, d.lx32, d.ux32, d.udiag32, red);
    if (act)
        for (uint32_t i = warp; i < d.n; i += nw) LM(d.dx, i) += LM(d.corr, i);
    __syncthreads();
}

}  // namespace espl
