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
#include "lane_smem.cuh"

namespace espl {

// Per-lane reductions of the refactor, in the tile's shared memory.
struct LevelShared {
    uint32_t bad[32];              // a dead pivot, growth failure or filled void slot
    uint32_t nonfinite[32];        // OR of (u - u) bits: a NaN somewhere
    unsigned long long worst[32];  // the largest |L| over non-scaled columns (by bits)
    unsigned long long cmax[kRefGroups][32];  // each group's column's largest |L| numerator (by bits)
};

// A barrier of the threads of one column group (ids 1 .. kRefGroups; 0 is
// __syncthreads's).
__device__ __forceinline__ void group_sync(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// The ring of a streaming sweep (StreamDev): kRingSlots chunks staged by
// bulk copies (cp.async.bulk, the TMA's 1-D form), each completing on the
// mbarrier of its slot, up to kRingSlots chunks ahead of the levels that
// read them. `seq` counts the chunks the CTA has staged (the slot of the
// q-th is q % kRingSlots, its phase parity (q / kRingSlots) & 1); `fail`
// is set for good when a chunk's wait runs out.
constexpr uint32_t kRingSlots = 3, kRingChunk = 2048, kRingRows = 256;
// a chunk's plan (tape.h StreamPlan meta): 8 header words (the last four:
// the copy of the chunk kRingSlots ahead, which reuses its slot), at most
// kRingRows segments of 3 words, kRingRows rows and kRingRows + 1 offsets,
// padded to four words
constexpr uint32_t kRingMetaWords = (8 + 5 * kRingRows + 1 + 3) & ~3u;
struct RingShared {
    unsigned long long bar[kRingSlots];
    uint32_t seq, fail;
};
// A slot: kRingChunk entries' values for tw lanes (room for FP64), their
// columns, and the chunk's plan.
__host__ __device__ constexpr uint32_t ring_cols_off(uint32_t tw) { return kRingChunk * tw * 8u; }
__host__ __device__ constexpr uint32_t ring_meta_off(uint32_t tw) { return kRingChunk * (tw * 8u + 4u); }
__host__ __device__ constexpr uint32_t ring_slot_bytes(uint32_t tw) {
    return ring_meta_off(tw) + kRingMetaWords * 4u;
}
// After the slots, the y values of the chunk being solved (room for FP64):
// the entries' y (kRingChunk), then its rows' results (kRingRows), the
// rows' own y before the sweep and (backward) their U diagonals.
__host__ __device__ constexpr uint32_t ring_stage_bytes(uint32_t tw) {
    return (kRingChunk + 3u * kRingRows) * tw * 8u;
}
__host__ __device__ constexpr uint32_t ring_bytes(uint32_t tw) {
    return kRingSlots * ring_slot_bytes(tw) + ring_stage_bytes(tw);
}

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
//
// The columns run by levels (GroupDev cl_*): a level's columns read only the
// L of earlier levels, so its G groups of the CTA's threads (G up to
// kRefGroups) each factor their own columns at once, group g in work vector
// g (w, then wk), with barriers of the group between a column's steps and a
// CTA barrier between levels. A column's steps are those of the one-thread
// replay (src/solver/kernels/lane.zig:56-125): its scatter, its U entries in
// the tape's topological order (each entry's axpy of an L column split over
// the group, a barrier between entries), the pivot with its L entries
// split over the group; each row's updates come in the same order, so the
// factor is the same to the bit whatever the grouping.
template <typename T>
__device__ int lvl_refactor(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                            T* __restrict__ w, T* __restrict__ wk, T* __restrict__ lx, T* __restrict__ ux,
                            T* __restrict__ ud, LevelShared& ls, T* win = nullptr, uint32_t win_rows = 0) {
    const uint32_t P = d.P, tw = blockDim.x / nw;
    const double* __restrict__ a = d.a;
    constexpr bool F32 = sizeof(T) == 4;
    // Group 0's work vector keeps its last win_rows rows (the trailing
    // pivots: the top separators' dense chain of columns, which reads and
    // updates them step after step) in shared memory. Like w, the window is
    // zero between columns; it starts zeroed here.
    const uint32_t t0 = win && win_rows < d.n ? d.n - win_rows : (win ? 0u : d.n);
    if (win)
        for (uint32_t r = t0 + warp; r < d.n; r += nw) win[(r - t0) * tw + lane] = (T)0;
    if (warp == 0) {
        uint32_t bad = 0;
        if (act)
            for (uint32_t v = 0; v < d.n_void; v++)
                if (LM(a, d.void_slots[v]) != 0.0) bad = 1;
        ls.bad[lane] = bad;
        ls.nonfinite[lane] = 0;
        ls.worst[lane] = 0;
        for (uint32_t g = 0; g < kRefGroups; g++) ls.cmax[g][lane] = 0;
    }
    __syncthreads();
    for (uint32_t lv = 0; lv < d.n_cl; lv++) {
        const uint32_t b = d.cl_ptr[lv], G = d.cl_ptr[lv + 1] - b - 1;
        const uint32_t gsize = nw / G, g = warp / gsize, gw = warp % gsize;
        const uint32_t bid = 1 + g, bthreads = blockDim.x / G;
        T* __restrict__ wg = g == 0 ? w : wk + (size_t)(g - 1) * (d.n + 1) * P;
        const uint32_t tg = g == 0 ? t0 : d.n;
        // row r of the group's work vector
        auto W = [&](uint32_t r) -> T& { return r >= tg ? win[(r - tg) * tw + lane] : LM(wg, r); };
        unsigned long long& cmax = ls.cmax[g][lane];
        const uint32_t c0 = d.cl_gp[b + g], c1 = d.cl_gp[b + g + 1];
        for (uint32_t cc = c0; cc < c1; cc++) {
            const uint32_t k = d.cl_cols[cc];
            const uint32_t c = d.q[k];
            if (act)
                for (uint32_t p = d.col_ptr[c] + gw; p < d.col_ptr[c + 1]; p += gsize) W(d.prow[p]) = (T)LM(a, p);
            group_sync(bid, bthreads);
            const uint32_t u0 = d.up[k], u1 = d.up[k + 1];
            // Two U entries' loads in flight: an entry's first kPre L entries
            // of this thread's share (values and rows) are loaded two
            // entries ahead, into the register set of its parity, and its
            // row and L bounds (the U entry stream, read in sequence) four
            // ahead. None of them depends on the work vector.
            constexpr uint32_t kPre = 2;
            struct Pre {
                T v[kPre];
                uint32_t r[kPre];
                uint4 t;
            };
            const uint4* __restrict__ us = d.cl_ustream;
            const uint4 zero4 = make_uint4(0, 0, 0, 0);
            auto fill = [&](Pre& x, const uint4& t) {
                x.t = t;
#pragma unroll
                for (uint32_t r = 0; r < kPre; r++) {
                    const uint32_t pl = t.y + gw + r * gsize;
                    const bool ok = act && pl < t.z;
                    x.v[r] = ok ? LM(lx, pl) : (T)0;
                    x.r[r] = ok ? d.li[pl] : 0u;
                }
            };
            Pre A, B;
            uint4 q2 = zero4, q3 = zero4;  // the stream's entries p + 2 and p + 3
            if (u0 < u1) fill(A, us[u0]);
            if (u0 + 1 < u1) fill(B, us[u0 + 1]);
            if (u0 + 2 < u1) q2 = us[u0 + 2];
            if (u0 + 3 < u1) q3 = us[u0 + 3];
            auto step = [&](uint32_t p, Pre& x) {
                const uint32_t i = x.t.x, e0 = x.t.y + gw, e1 = x.t.z;
                const T u = act ? W(i) : (T)0;
                if (act) {
#pragma unroll
                    for (uint32_t r = 0; r < kPre; r++)
                        if (e0 + r * gsize < e1) W(x.r[r]) -= x.v[r] * u;
                    for (uint32_t pl = e0 + kPre * gsize; pl < e1; pl += gsize) W(d.li[pl]) -= LM(lx, pl) * u;
                    if (gw == 0) {
                        LM(ux, p) = u;
                        if (mag_bits(u - u) != 0) atomicOr(&ls.nonfinite[lane], 1u);
                    }
                }
                // this set now takes entry p + 2
                if (p + 2 < u1) fill(x, q2);
                q2 = q3;
                q3 = p + 4 < u1 ? us[p + 4] : zero4;
                group_sync(bid, bthreads);
            };
            for (uint32_t p = u0; p < u1; p += 2) {
                step(p, A);
                if (p + 1 < u1) step(p + 1, B);
            }
            // the taken rows of the work vector (each U entry's row) go back to zero
            if (act)
                for (uint32_t p = u0 + gw; p < u1; p += gsize) W(d.ui[p]) = (T)0;
            const uint32_t fl = d.flags[k];
            if (fl & 1u) {
                // a void column: unit pivot, no L entries, and every row its
                // takes filled is cleared
                if (act) {
                    for (uint32_t p = d.lp[k] + gw; p < d.lp[k + 1]; p += gsize) {
                        LM(lx, p) = (T)0;
                        W(d.li[p]) = (T)0;
                    }
                    for (uint32_t p = u0; p < u1; p++) {
                        const uint32_t i = d.ui[p];
                        for (uint32_t pl = d.lp[i] + gw; pl < d.lp[i + 1]; pl += gsize) W(d.li[pl]) = (T)0;
                    }
                    if (gw == 0) {
                        LM(ud, k) = (T)1;
                        W(k) = (T)0;
                    }
                }
                group_sync(bid, bthreads);
                continue;
            }
            group_sync(bid, bthreads);
            T dk = act ? W(k) : (T)1;
            const bool dead = dk == (T)0 || !(fabs(dk) < (T)INFINITY);
            if (dead) dk = (T)1;
            uint64_t cb = mag_bits(dk);
            uint32_t nf = 0;
            if (act)
                for (uint32_t p = d.lp[k] + gw; p < d.lp[k + 1]; p += gsize) {
                    const uint32_t r = d.li[p];
                    const T v = W(r);
                    W(r) = (T)0;
                    const uint64_t vb = mag_bits(v);
                    cb = cb > vb ? cb : vb;
                    const T lv2 = v / dk;
                    if (F32 || (fl & 2u)) nf |= (uint32_t)(mag_bits(lv2 - lv2) != 0);
                    LM(lx, p) = lv2;
                    if (!(fl & 2u)) {
                        const uint64_t lb = mag_bits(lv2);
                        if (lb > ls.worst[lane]) atomicMax(&ls.worst[lane], lb);
                    }
                }
            if (act) {
                atomicMax(&cmax, cb);
                if (nf) atomicOr(&ls.nonfinite[lane], 1u);
            }
            group_sync(bid, bthreads);
            if (gw == 0 && act) {
                LM(ud, k) = dk;
                W(k) = (T)0;
                uint32_t bad = dead ? 1u : 0u;
                const double cm = bitsd(cmax);
                if (!(fl & 2u)) {
                    if (F32)
                        bad |= (!(fabs((double)dk) >= 1e-12 * cm) || !(cm / fabs((double)dk) <= kWide)) ? 1u : 0u;
                    else
                        bad |= !(fabs((double)dk) >= 1e-12 * cm) ? 1u : 0u;
                }
                if (bad) atomicOr(&ls.bad[lane], 1u);
                cmax = 0;
            }
            group_sync(bid, bthreads);
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

// The factor's values of one precision into streaming order (StreamDev),
// after a refactor; the bulk copies that read them run in the async proxy,
// so each writer fences its stores for it before the barrier.
template <typename T>
__device__ void lvl_stream_store(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                                 const T* __restrict__ lx, const T* __restrict__ ux, T* __restrict__ vf,
                                 T* __restrict__ vb) {
    const uint32_t P = d.P, tw = blockDim.x / nw, part = l / tw;
    const StreamDev& sd = *d.stream;
    if (act) {
        for (uint32_t e = warp; e < sd.fw.entries; e += nw) {
            const uint32_t sl = sd.fw.slot[e];
            vf[((size_t)part * sd.fw.entries + e) * tw + lane] = sl == kNone ? (T)0 : LM(lx, sl);
        }
        for (uint32_t e = warp; e < sd.bw.entries; e += nw) {
            const uint32_t sl = sd.bw.slot[e];
            vb[((size_t)part * sd.bw.entries + e) * tw + lane] = sl == kNone ? (T)0 : LM(ux, sl);
        }
    }
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
}

__device__ __forceinline__ void ring_init(RingShared& r) {
    if (threadIdx.x == 0) {
        for (uint32_t k = 0; k < kRingSlots; k++) mbar_init(reinterpret_cast<uint64_t*>(&r.bar[k]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        r.seq = 0;
        r.fail = 0;
    }
    __syncthreads();
}

__device__ __forceinline__ bool ring_wait(RingShared& r, uint32_t q) {
    uint64_t* bar = reinterpret_cast<uint64_t*>(&r.bar[q % kRingSlots]);
    const uint32_t parity = (q / kRingSlots) & 1u;
    for (uint32_t tries = 0; tries < (1u << 22); tries++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (tries > 64) __nanosleep(64);
    }
    return false;
}

// One sweep over the streaming order. Each chunk brings the values and
// columns of its entries and its plan (segments: runs of one level's rows,
// with their longest row; the rows; their entry offsets) into a ring slot. When a chunk starts, its
// rows of earlier chunks are final, so the CTA gathers, all at once, the y
// of every entry whose column an earlier chunk (or no row of the sweep)
// computes, and each row's own y and U diagonal; an entry whose column a
// row of the same chunk computes (kStreamLocal) reads that row's result,
// which the row leaves in shared memory besides y. The levels then touch
// global memory only to store their rows.
//
// Rows are split over the threads as in lvl_sweep (a segment of at least
// nw rows: a row per logical warp; else gs logical warps per row, no more
// than its longest row needs, whose parts a butterfly of warp shuffles
// adds, and where a row spans hardware warps the warps' sums go through
// `red` and a second butterfly inside one hardware warp). A barrier ends each level; there thread 0 refills the
// slots whose chunks are done, so a chunk needs a barrier of its own for
// its copies only when it is not yet staged.
//
// Thread 0 issues the copies; every thread waits for a chunk before reading
// it, and the CTA agrees on the outcome (a barrier) before any thread reads
// the chunk's plan. A wait that runs out ends the sweep: no more copies are
// issued, thread 0 waits once more, bounded, for the copies still in
// flight, and ring.fail is set, so that the sweep and every later one of
// the CTA return false (their results are not used).
template <typename T, bool BACK>
__device__ bool lvl_sweep_ring(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                               const StreamSweep& sw, const T* __restrict__ vso, const T* __restrict__ ud,
                               T* __restrict__ y, T* red, RingShared& ring, unsigned char* slots) {
    const uint32_t P = d.P, tw = blockDim.x / nw, spw = 32u / tw, part = l / tw;
    const uint32_t sb = ring_slot_bytes(tw), nc = sw.n_chunks, q0 = ring.seq;
    const uint32_t hw = threadIdx.x >> 5, hl = threadIdx.x & 31u;
    const bool t0 = threadIdx.x == 0;
    // the chunk's y: entries' (kRingChunk), then its rows' results, the
    // rows' own y and U diagonals (kRingRows each); tw values per item
    T* ys = reinterpret_cast<T*>(slots + kRingSlots * sb);
    T* yo = ys + (kRingChunk + kRingRows) * tw;
    T* yd = yo + kRingRows * tw;
    if (ring.fail) return false;
    uint32_t sent = 0, confirmed = 0;  // thread 0: chunks issued, and waited for
    auto stage = [&](uint32_t lim) {   // thread 0: copies of the chunks before lim
        for (; sent < lim; sent++) {
            const uint32_t q = q0 + sent, slot = q % kRingSlots;
            unsigned char* base = slots + slot * sb;
            // the first chunks' copies from the plan in global memory, the
            // later ones from the header of the chunk whose slot they take
            uint32_t e0, len, m0, mlen;
            if (sent < kRingSlots) {
                e0 = sw.ch[sent];
                len = sw.ch[sent + 1] - e0;
                m0 = sw.mo[sent];
                mlen = sw.mo[sent + 1] - m0;
            } else {
                const uint4 h = *reinterpret_cast<const uint4*>(base + ring_meta_off(tw) + 16);
                e0 = h.x;
                len = h.y;
                m0 = h.z;
                mlen = h.w;
            }
            const uint32_t vbytes = len * tw * (uint32_t)sizeof(T);
            uint64_t* bar = reinterpret_cast<uint64_t*>(&ring.bar[slot]);
            mbar_arrive_expect_tx(bar, vbytes + len * 4u + mlen * 4u);
            bulk_g2s_once(base, vso + ((size_t)part * sw.entries + e0) * tw, vbytes, bar);
            bulk_g2s(base + ring_cols_off(tw), sw.col + e0, len * 4u, bar);
            bulk_g2s(base + ring_meta_off(tw), sw.meta + m0, mlen * 4u, bar);
        }
    };
    // the chunks staged so far by the schedule every thread follows (thread 0
    // issues them)
    uint32_t sched = nc < kRingSlots ? nc : kRingSlots;
    if (t0) stage(sched);
    bool failed = false;
    for (uint32_t c = 0; c < nc; c++) {
        if (c >= sched) {
            __syncthreads();  // every thread is done with chunk c - kRingSlots
            sched = min(nc, c + kRingSlots);
            if (t0) stage(sched);
        }
        const uint32_t slot = (q0 + c) % kRingSlots;
        unsigned char* base = slots + slot * sb;
        // (the barrier also orders the rows of earlier chunks before the gather)
        if (__syncthreads_or(!ring_wait(ring, q0 + c))) {
            failed = true;
            break;
        }
        confirmed = c + 1;
        const T* sv = reinterpret_cast<const T*>(base);
        const uint32_t* sc = reinterpret_cast<const uint32_t*>(base + ring_cols_off(tw));
        const uint32_t* meta = reinterpret_cast<const uint32_t*>(base + ring_meta_off(tw));
        const uint32_t ns = meta[0], nr = meta[1], len = meta[2];
        const uint32_t* sg = meta + 8;
        const uint32_t* ri = sg + 3 * ns;
        const uint32_t* rp = ri + nr;
        if (act) {
            // eight entries and a row per thread and batch, every load of a
            // batch in flight before its stores
            for (uint32_t b = warp; b < len || b < nr; b += 8 * nw) {
                T ve[8], vo = (T)0, vd = (T)1;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const uint32_t j = b + k * nw;
                    const uint32_t code = j < len ? sc[j] : kStreamLocal;
                    ve[k] = (code & kStreamLocal) ? (T)0 : LM(y, code);
                }
                if (b < nr) {
                    const uint32_t i = ri[b];
                    vo = LM(y, i);
                    if (BACK) vd = LM(ud, i);
                }
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const uint32_t j = b + k * nw;
                    if (j < len) ys[j * tw + lane] = ve[k];
                }
                if (b < nr) {
                    yo[b * tw + lane] = vo;
                    if (BACK) yd[b * tw + lane] = vd;
                }
            }
        }
        __syncthreads();
        // a row's sum over entries e = e0, e0 + stride, ... < e1 of the chunk
        auto dot = [&](uint32_t e0, uint32_t e1, uint32_t stride) {
            T acc = (T)0;
            for (uint32_t e = e0; e < e1; e += 8 * stride) {
                T v[8], yv[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const uint32_t ek = e + k * stride;
                    const bool ok = ek < e1;
                    const uint32_t j = ok ? ek : 0u, code = sc[j];
                    const uint32_t at = (code & kStreamLocal) ? kRingChunk + (code & ~kStreamLocal) : j;
                    v[k] = ok ? sv[j * tw + lane] : (T)0;
                    yv[k] = ok ? ys[at * tw + lane] : (T)0;
                }
                T s = v[0] * yv[0];
#pragma unroll
                for (int k = 1; k < 8; k++) s += v[k] * yv[k];
                acc += s;
            }
            return acc;
        };
        // row r of the chunk's result: y and its shared copy
        auto finish = [&](uint32_t r, T part_sum) {
            T acc = yo[r * tw + lane] - part_sum;
            if (BACK) acc = acc / yd[r * tw + lane];
            ys[(kRingChunk + r) * tw + lane] = acc;
            LM(y, ri[r]) = acc;
        };
        for (uint32_t g = 0; g < ns; g++) {
            const uint32_t k0 = sg[3 * g], k1 = sg[3 * g + 1], last = sg[3 * g + 2] & 1u, m = k1 - k0;
            const uint32_t longest = sg[3 * g + 2] >> 1;
            bool reused = false;  // red was read: a barrier before its next use
            if (m >= nw) {
                if (act)
                    for (uint32_t k = k0 + warp; k < k1; k += nw) finish(k, dot(rp[k], rp[k + 1], 1u));
            } else {
                // shares per row: enough for one pass of the dot's eight
                // entries over the longest row, as far as the rows leave
                // logical warps (the others wait at the level's barrier)
                uint32_t gs = 1;
                while (gs * 2 * m <= nw && gs * 8 < longest) gs *= 2;
                const uint32_t row = warp / gs, sub = warp % gs;
                const bool across = gs > spw;  // a row spans hardware warps
                T ps = (T)0;
                if (row < m && act) ps = dot(rp[k0 + row] + sub, rp[k0 + row + 1], gs);
                for (uint32_t o = 1; o < gs && o < spw; o *= 2) ps += __shfl_xor_sync(0xffffffffu, ps, o * tw);
                if (across) {
                    // hardware warp w's sum of its row at red[w * tw + lane];
                    // hardware warp r adds row r's nh warps' sums
                    const uint32_t nh = gs / spw;
                    if (hl < tw) red[hw * tw + lane] = ps;
                    __syncthreads();
                    ps = (hw < m && hl < nh * tw) ? red[hw * nh * tw + hl] : (T)0;
                    for (uint32_t o = tw; o < nh * tw; o *= 2) ps += __shfl_xor_sync(0xffffffffu, ps, o);
                    if (hw < m && hl < tw && act) finish(k0 + hw, ps);
                    reused = true;
                } else if (row < m && sub == 0 && act) {
                    finish(k0 + row, ps);
                }
            }
            if (last || reused) __syncthreads();
            if (last) {
                // the chunks before c are done, and c itself after its last segment
                const uint32_t lim = min(nc, c + kRingSlots + (g + 1 == ns ? 1u : 0u));
                if (lim > sched) {
                    sched = lim;
                    if (t0) stage(sched);
                }
            }
        }
    }
    __syncthreads();
    if (t0) {
        if (failed) {
            // the copies still in flight, once more
            for (uint32_t c = confirmed; c < sent; c++) ring_wait(ring, q0 + c);
            ring.fail = 1;
        }
        ring.seq = q0 + nc;
    }
    __syncthreads();
    return !failed;
}

// out = -A^-1 rhs through the lane's factors (luSolve with neg, solve64's
// contract), every thread of the CTA taking part.
template <typename T>
__device__ void lvl_solve(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                          const double* __restrict__ rhs, double* __restrict__ out, T* __restrict__ y,
                          const T* __restrict__ lx, const T* __restrict__ ux, const T* __restrict__ ud, T* red,
                          RingShared* ring = nullptr, unsigned char* slots = nullptr, const T* vf = nullptr,
                          const T* vb = nullptr) {
    const uint32_t P = d.P;
    if (act)
        for (uint32_t r = warp; r < d.n; r += nw) LM(y, d.pinv[r]) = (T)(-LM(rhs, r));
    __syncthreads();
    if (ring && vf) {
        // (a failed sweep leaves ring->fail set; the caller reads it)
        if (lvl_sweep_ring<T, false>(d, l, lane, warp, nw, act, d.stream->fw, vf, nullptr, y, red, *ring, slots))
            lvl_sweep_ring<T, true>(d, l, lane, warp, nw, act, d.stream->bw, vb, ud, y, red, *ring, slots);
    } else {
        lvl_sweep<T, false>(d, l, lane, warp, nw, act, d.fl_ptr, d.fl_rows, d.n_fl, d.rl_ptr, d.rl_ent, lx, nullptr,
                            y, red);
        lvl_sweep<T, true>(d, l, lane, warp, nw, act, d.bl_ptr, d.bl_rows, d.n_bl, d.ru_ptr, d.ru_ent, ux, ud, y,
                           red);
    }
    if (act)
        for (uint32_t j = warp; j < d.n; j += nw) LM(out, d.q[j]) = (double)LM(y, j);
    __syncthreads();
}

// One FP64-residual refinement sweep of a mixed solve (refine_mixed's
// contract), rows split over the warps through the row view of A:
// r = rhs + A dx, dx += -A^-1 r by the FP32 factors.
__device__ void lvl_refine(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t warp, uint32_t nw, bool act,
                           float* red, RingShared* ring = nullptr, unsigned char* slots = nullptr) {
    const uint32_t P = d.P;
    if (act)
        for (uint32_t i = warp; i < d.n; i += nw) {
            double r = LM(d.rhs, i);
            for (uint32_t e = d.rt_ptr[i]; e < d.rt_ptr[i + 1]; e++) r += LM(d.a, d.rt_pos[e]) * LM(d.dx, d.rt_col[e]);
            LM(d.rr, i) = r;
        }
    __syncthreads();
    lvl_solve<float>(d, l, lane, warp, nw, act, d.rr, d.corr, d.y32, d.lx32, d.ux32, d.udiag32, red, ring, slots,
                     d.stream ? d.stream->vf32 : nullptr, d.stream ? d.stream->vb32 : nullptr);
    if (act)
        for (uint32_t i = warp; i < d.n; i += nw) LM(d.dx, i) += LM(d.corr, i);
    __syncthreads();
}

}  // namespace espl
