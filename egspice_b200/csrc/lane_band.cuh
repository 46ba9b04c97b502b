// The banded streaming replay for templates too large for the shared-memory
// LU chain whose elimination stays within a narrow band of the pivot order
// (an RC ladder's elimination walks its chain: every column k touches only
// rows k - band .. k + band). The work vector lives in a ring of band_w rows and
// the recently produced L entries (the only ones a later axpy reads) in a
// ring of band_l slots, both in shared memory, so the dependent chain of the
// replay touches only shared memory. The replay program and the scattered A
// values stream from global memory through double-buffered shared-memory
// chunks that warps 1-3 fill while warp 0 replays the previous chunk, one
// thread per lane. L, U and the pivots go to the lane's global factor
// arrays, which the triangular solves read.
//
// The same operations on the same values in the same order as refactor64
// (FP64) and refactor32 (FP32), so the factor is bitwise theirs.
#pragma once

#include "lane_smem.cuh"

namespace espl {

// Streams count values into dst with warps 1-3 (thread t of nt), eight per
// thread in flight: all eight sources are loaded before any is stored, so
// the loads' latencies overlap instead of adding up.
template <typename F>
__device__ __forceinline__ void stream8(uint32_t t, uint32_t nt, uint32_t count, double* __restrict__ dst, F src) {
    for (uint32_t b0 = t; b0 < count; b0 += 8u * nt) {
        double v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t i = b0 + (uint32_t)j * nt;
            v[j] = i < count ? src(i) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t i = b0 + (uint32_t)j * nt;
            if (i < count) dst[i] = v[j];
        }
    }
}

struct BandAcc {
    bool bad, nonfinite;
    uint64_t worst;
};

template <typename T>
__device__ __forceinline__ void band_chunk(const GroupDev& d, uint32_t lane, uint32_t l,
                                           const uint32_t* __restrict__ prog, uint32_t nw,
                                           const double* __restrict__ abuf, T* __restrict__ w,
                                           T* __restrict__ lr, T* __restrict__ lx, T* __restrict__ ux,
                                           T* __restrict__ ud, BandAcc& acc) {
    const uint32_t P = d.P;
    const uint32_t wm = d.band_w - 1, lm = d.band_l - 1;
    constexpr bool f64 = sizeof(T) == 8;
    const T inf = (T)INFINITY;
#define WR(r) w[(size_t)((r) & wm) * 32 + lane]
#define LR(p) lr[(size_t)((p) & lm) * 32 + lane]
    uint32_t ei = 0;
    for (uint32_t pc = 0; pc < nw;) {
        const uint32_t h = prog[pc];
        const uint32_t op = h & 15u;
        if (op == kOpScat) {
            const uint32_t cnt = h >> 4;
            for (uint32_t j = 0; j < cnt; j++, ei++) WR(prog[pc + 1 + j] >> 16) = (T)abuf[ei * 32 + lane];
            pc += 1 + cnt;
        } else if (op == kOpTake) {
            const uint32_t cnt = h >> 4;
            const uint32_t ip = prog[pc + 1];
            const uint32_t i = ip >> 16;
            const T uki = WR(i);
            WR(i) = (T)0;
            LM(ux, ip & 0xffffu) = uki;
            acc.nonfinite |= !(uki - uki == (T)0);
            for (uint32_t j = 0; j < cnt; j++) {
                const uint32_t e = prog[pc + 2 + j];
                WR(e >> 16) -= LR(e & 0xffffu) * uki;
            }
            pc += 2 + cnt;
        } else {  // kOpPiv (band templates have no void column)
            const uint32_t fl = (h >> 4) & 15u, cnt = h >> 8;
            const uint32_t k = prog[pc + 1];
            T dk = WR(k);
            WR(k) = (T)0;
            bool dead = dk == (T)0 || !(fabs(dk) < inf);
            acc.bad |= dead;
            if (dead) dk = (T)1;
            LM(ud, k) = dk;
            if constexpr (f64) {
                if (!(fl & 2u)) {
                    uint64_t cb = dbits(fabs((double)dk));
                    for (uint32_t j = 0; j < cnt; j++) {
                        const uint32_t e = prog[pc + 2 + j];
                        const uint32_t r = e >> 16;
                        const T v = WR(r);
                        WR(r) = (T)0;
                        const uint64_t vb = dbits(fabs((double)v));
                        cb = cb > vb ? cb : vb;
                        const T lv = v / dk;
                        LM(lx, e & 0xffffu) = lv;
                        LR(e & 0xffffu) = lv;
                        const uint64_t lb = dbits(fabs((double)lv));
                        acc.worst = acc.worst > lb ? acc.worst : lb;
                    }
                    acc.bad |= !(fabs((double)dk) >= 1e-12 * bitsd(cb));
                } else {
                    for (uint32_t j = 0; j < cnt; j++) {
                        const uint32_t e = prog[pc + 2 + j];
                        const uint32_t r = e >> 16;
                        const T lv = WR(r) / dk;
                        acc.nonfinite |= !(lv - lv == (T)0);
                        LM(lx, e & 0xffffu) = lv;
                        LR(e & 0xffffu) = lv;
                        WR(r) = (T)0;
                    }
                }
            } else {
                T cmax = fabs(dk);
                for (uint32_t j = 0; j < cnt; j++) {
                    const uint32_t e = prog[pc + 2 + j];
                    const uint32_t r = e >> 16;
                    const T v = WR(r);
                    WR(r) = (T)0;
                    cmax = fmaxf(cmax, fabsf(v));
                    const T lv = v / dk;
                    acc.nonfinite |= !(lv - lv == (T)0);
                    LM(lx, e & 0xffffu) = lv;
                    LR(e & 0xffffu) = lv;
                }
                if (!(fl & 2u)) acc.bad |= !(fabsf(dk) >= (T)1e-12 * cmax) || !(cmax / fabsf(dk) <= (T)kWide);
            }
            pc += 2 + cnt;
        }
    }
#undef WR
#undef LR
}

// The banded replay of the tile's lanes; every thread of the tile calls it
// (warps 1-3 stream the chunks, warp 0 replays). `compute` marks the warp-0
// lanes that replay here; T = float for FP32 lanes (the FP32 factor arrays),
// double otherwise. Returns, for those lanes, 0 when the replay holds, 1
// for a failed pivot or a non-finite entry, 2 for only a multiplier past
// 1 / pivot_tol (FP64).
template <typename T>
__device__ int band_refactor(const GroupDev& d, uint32_t warp, uint32_t lane, uint32_t l, bool compute) {
    const uint32_t P = d.P;
    unsigned char* base = g_dsm + d.band_off;
    uint32_t* progbuf = reinterpret_cast<uint32_t*>(base);
    double* abuf = reinterpret_cast<double*>(base + 2u * d.band_cw * 4u);
    T* w = reinterpret_cast<T*>(base + 2u * d.band_cw * 4u + 2u * d.band_ce * 32u * 8u);
    T* lr = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(w) + d.band_w * 32u * 8u);
    constexpr bool f64 = sizeof(T) == 8;
    T* lx;
    T* ux;
    T* ud;
    if constexpr (f64) {
        lx = d.lx;
        ux = d.ux;
        ud = d.udiag;
    } else {
        lx = d.lx32;
        ux = d.ux32;
        ud = d.udiag32;
    }
    const uint32_t lbase = l - lane;  // the tile's first lane
    auto load = [&](uint32_t c, uint32_t b) {
        const uint32_t pc0 = d.band_cpc[c], nw = d.band_cpc[c + 1] - pc0;
        const uint32_t e0 = d.band_cent[c], ne = d.band_cent[c + 1] - e0;
        uint32_t* pb = progbuf + b * d.band_cw;
        double* ab = abuf + (size_t)b * d.band_ce * 32u;
        const uint32_t t = threadIdx.x - 32u, nt = blockDim.x - 32u;
        for (uint32_t i = t; i < nw; i += nt) pb[i] = d.lu_prog[pc0 + i];
        stream8(t, nt, ne * 32u, ab,
                [&](uint32_t i) { return d.a[(size_t)d.band_slot[e0 + (i >> 5)] * P + lbase + (i & 31u)]; });
    };
    // the work ring starts at zero; every column leaves it at zero
    {
        uint32_t* wz = reinterpret_cast<uint32_t*>(w);
        for (uint32_t i = threadIdx.x; i < d.band_w * 32u * 2u; i += blockDim.x) wz[i] = 0u;
    }
    bool void_hit = false;
    if (compute)
        for (uint32_t v = 0; v < d.n_void; v++)
            if (LM(d.a, d.void_slots[v]) != 0.0) void_hit = true;
    if (warp != 0) load(0, 0);
    __syncthreads();
    BandAcc acc{false, false, 0};
    const uint32_t nch = d.band_chunks;
    for (uint32_t c = 0; c < nch; c++) {
        if (warp != 0 && c + 1 < nch) load(c + 1, (c + 1) & 1u);
        if (compute && !void_hit) {
            const uint32_t b = c & 1u;
            band_chunk<T>(d, lane, l, progbuf + b * d.band_cw, d.band_cpc[c + 1] - d.band_cpc[c],
                          abuf + (size_t)b * d.band_ce * 32u, w, lr, lx, ux, ud, acc);
        }
        __syncthreads();
    }
    if (!compute) return 0;
    if (void_hit || acc.nonfinite || acc.bad) return 1;
    if constexpr (f64) return bitsd(acc.worst) <= kWide ? 0 : 2;
    return 0;
}

// The forward and back substitutions of the banded lanes (luSolve with neg,
// the same operations and order as solve64 / solve32), streamed by column
// blocks: y lives in a ring of band_w rows; pivot position j enters the
// forward ring (as -rhs of its row) when column j - band starts, and the
// back ring (as its forward result, kept in the lane's global y) when
// column j + band starts; dx[q[k]] is written as column k finishes. Warps
// 1-3 stage the next block's indices and factor values while warp 0 runs
// the current one.
template <typename T>
__device__ void band_solve(const GroupDev& d, uint32_t warp, uint32_t lane, uint32_t l, bool compute) {
    const uint32_t P = d.P, n = d.n, B = d.band_b, wm = d.band_w - 1;
    constexpr uint32_t kC = kSolveCols, kE = kSolveEntries;
    unsigned char* base = g_dsm + d.band_off;
    T* yr = reinterpret_cast<T*>(base + 2u * kSolveBufBytes);
    constexpr bool f64 = sizeof(T) == 8;
    const T* lxg;
    const T* uxg;
    const T* udg;
    T* yg;
    if constexpr (f64) {
        lxg = d.lx;
        uxg = d.ux;
        udg = d.udiag;
        yg = d.y;
    } else {
        lxg = d.lx32;
        uxg = d.ux32;
        udg = d.udiag32;
        yg = d.y32;
    }
    const uint32_t lbase = l - lane;
    const uint32_t t = threadIdx.x - 32u, nt = blockDim.x - 32u;
    auto bidx = [&](uint32_t b) { return reinterpret_cast<uint32_t*>(base + b * kSolveBufBytes); };
    auto bval = [&](uint32_t b) { return reinterpret_cast<double*>(base + b * kSolveBufBytes + kSolveIdxWords * 4u); };
    auto bcol = [&](uint32_t b) {
        return reinterpret_cast<double*>(base + b * kSolveBufBytes + kSolveIdxWords * 4u + kE * 32u * 8u);
    };
#define YR(r) yr[(size_t)((r) & wm) * 32 + lane]
    const uint32_t nblk = d.band_nblk;
    // forward: block c covers columns scol[c] .. scol[c + 1)
    auto load_fwd = [&](uint32_t c, uint32_t b) {
        const uint32_t k0 = d.band_scol[c], k1 = d.band_scol[c + 1], cols = k1 - k0;
        const uint32_t e0 = d.lp[k0], ne = d.lp[k1] - e0;
        uint32_t* ix = bidx(b);
        double* vv = bval(b);
        double* cv = bcol(b);
        for (uint32_t i = t; i <= cols; i += nt) ix[i] = d.lp[k0 + i] - e0;
        for (uint32_t i = t; i < ne; i += nt) ix[kC + 1 + i] = d.li[e0 + i];
        stream8(t, nt, ne * 32u, vv,
                [&](uint32_t i) { return (double)lxg[(size_t)(e0 + (i >> 5)) * P + lbase + (i & 31u)]; });
        stream8(t, nt, cols * 32u, cv, [&](uint32_t i) {
            const uint32_t k = k0 + (i >> 5), j = k + B;
            return (k >= 1 && j < n) ? d.rhs[(size_t)d.band_rowof[j] * P + lbase + (i & 31u)] : 0.0;
        });
    };
    if (compute)
        for (uint32_t j = 0; j <= B && j < n; j++) YR(j) = (T)(-LM(d.rhs, d.band_rowof[j]));
    if (warp != 0) load_fwd(0, 0);
    __syncthreads();
    for (uint32_t c = 0; c < nblk; c++) {
        if (warp != 0 && c + 1 < nblk) load_fwd(c + 1, (c + 1) & 1u);
        if (compute) {
            const uint32_t b = c & 1u, k0 = d.band_scol[c], cols = d.band_scol[c + 1] - k0;
            const uint32_t* ix = bidx(b);
            const double* vv = bval(b);
            const double* cv = bcol(b);
            for (uint32_t kk = 0; kk < cols; kk++) {
                const uint32_t k = k0 + kk;
                if (k >= 1 && k + B < n) YR(k + B) = (T)(-cv[kk * 32 + lane]);
                const T yk = YR(k);
                LM(yg, k) = yk;
                if (yk != (T)0)
                    for (uint32_t j = ix[kk]; j < ix[kk + 1]; j++) YR(ix[kC + 1 + j]) -= (T)vv[j * 32 + lane] * yk;
            }
        }
        __syncthreads();
    }
    // back: blocks in reverse, columns descending
    auto load_bwd = [&](uint32_t c, uint32_t b) {
        const uint32_t k0 = d.band_scol[c], k1 = d.band_scol[c + 1], cols = k1 - k0;
        const uint32_t e0 = d.up[k0], ne = d.up[k1] - e0;
        uint32_t* ix = bidx(b);
        double* vv = bval(b);
        double* cv = bcol(b);
        for (uint32_t i = t; i <= cols; i += nt) ix[i] = d.up[k0 + i] - e0;
        for (uint32_t i = t; i < ne; i += nt) ix[kC + 1 + i] = d.ui[e0 + i];
        for (uint32_t i = t; i < cols; i += nt) ix[kC + 1 + kE + i] = d.q[k0 + i];
        stream8(t, nt, ne * 32u, vv,
                [&](uint32_t i) { return (double)uxg[(size_t)(e0 + (i >> 5)) * P + lbase + (i & 31u)]; });
        stream8(t, nt, cols * 32u, cv,
                [&](uint32_t i) { return (double)udg[(size_t)(k0 + (i >> 5)) * P + lbase + (i & 31u)]; });
        stream8(t, nt, cols * 32u, cv + kC * 32u, [&](uint32_t i) {
            const uint32_t k = k0 + (i >> 5);
            return (k + 2 <= n && k >= B) ? (double)yg[(size_t)(k - B) * P + lbase + (i & 31u)] : 0.0;
        });
    };
    if (compute)
        for (uint32_t j = (n - 1 >= B ? n - 1 - B : 0); j < n; j++) YR(j) = LM(yg, j);
    if (warp != 0) load_bwd(nblk - 1, (nblk - 1) & 1u);
    __syncthreads();
    for (uint32_t cc = nblk; cc-- > 0;) {
        if (warp != 0 && cc > 0) load_bwd(cc - 1, (cc - 1) & 1u);
        if (compute) {
            const uint32_t b = cc & 1u, k0 = d.band_scol[cc], cols = d.band_scol[cc + 1] - k0;
            const uint32_t* ix = bidx(b);
            const double* vv = bval(b);
            const double* cv = bcol(b);
            for (uint32_t kk = cols; kk-- > 0;) {
                const uint32_t k = k0 + kk;
                if (k + 2 <= n && k >= B) YR(k - B) = (T)cv[kC * 32u + kk * 32 + lane];
                const T zk = YR(k) / (T)cv[kk * 32 + lane];
                YR(k) = zk;
                LM(d.dx, ix[kC + 1 + kE + kk]) = (double)zk;
                if (zk != (T)0)
                    for (uint32_t j = ix[kk]; j < ix[kk + 1]; j++) YR(ix[kC + 1 + j]) -= (T)vv[j * 32 + lane] * zk;
            }
        }
        __syncthreads();
    }
#undef YR
}

}  // namespace espl
