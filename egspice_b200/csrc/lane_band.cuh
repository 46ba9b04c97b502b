// The banded streaming replay for templates too large for the shared-memory
// LU chain whose elimination stays within a narrow band of the pivot order
// (an RC ladder's walks its chain: every column k touches only rows
// k - band .. k + band). The work vector lives in a ring of band_w rows and
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

// Shared-memory bytes of the band buffers of a template.
__host__ __device__ inline uint32_t band_bytes(uint32_t words, uint32_t entries, uint32_t w_ring, uint32_t l_ring) {
    return 2u * words * 4u + 2u * entries * 32u * 8u + (w_ring + l_ring) * 32u * 8u;
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
        const uint32_t t = threadIdx.x - 32u;
        for (uint32_t i = t; i < nw; i += blockDim.x - 32u) pb[i] = d.lu_prog[pc0 + i];
        for (uint32_t i = t; i < ne * 32u; i += blockDim.x - 32u) {
            const uint32_t e = i >> 5, ln = i & 31u;
            ab[i] = d.a[(size_t)d.band_slot[e0 + e] * P + lbase + ln];
        }
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

}  // namespace espl
