// Shared-memory staging of a tile's template and the LU chain in shared
// memory.
//
// Every lane of a template reads the same index words each Newton iteration
// (instance terminals, the stamp gather lists, the pivot tape), so a tile
// stages them once per launch by bulk copies (cp.async.bulk, the TMA's 1-D
// form) completing on an mbarrier, and runs on a copy of its template
// descriptor in shared memory whose index pointers are redirected to the
// staged copies. When the factor fits as well, the gather phase writes the
// assembled matrix into the tile's shared copy (in the factor's precision)
// besides global memory (FP64), and the replay and triangular solves touch
// only shared memory, one thread per lane, with the 32 lanes interleaved
// (element i of lane j at i * 32 + j: a warp reads one element of all lanes
// as 32 consecutive words, conflict-free). Right-hand sides, the Newton step
// and the FP64 refinement residual stay in global memory, read once per row.
//
// FP64 tiles run the same operations in the same order as refactor64 and
// solve64 (src/solver/kernels/lane.zig:56-157), so a lane's factor and step
// are bitwise the global path's; FP32 tiles those of refactor32/solve32 and
// refine_mixed. A mixed lane that falls back to FP64 takes the global path.
#pragma once

#include "lane_tile.cuh"
#include "tape.h"

namespace espl {

// The tile's dynamic shared memory. The LU chain derives its pointers from
// this symbol (not from pointers handed around), so the compiler addresses
// them as shared memory.
extern __shared__ __align__(16) unsigned char g_dsm[];

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

// The same for data read once (a lane's factor values streamed through a
// ring): an L2 policy of evict_first keeps it from displacing data that is
// read again.
__device__ __forceinline__ void bulk_g2s_once(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
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

// Index arrays a tile stages: the template's, then the tape, then the row
// view (RTPTR/RTCOL/RTPOS: per row, the columns and slots of its entries by
// ascending column) that the FP32 refinement residual reads. Each starts on
// a 16-byte boundary and is copied padded to a 16-byte multiple (the global
// buffers carry that padding); u8 arrays are copied as words.
enum StageArr {
    S_DIAG, S_VOID, S_CURROW, S_SLOTDIAG, S_RES_T, S_CAP_T, S_VSRC_T, S_DIO_T, S_MOS_T,
    S_GIPTR, S_GIENT, S_SITE,
    S_Q, S_PINV, S_COLPTR, S_PROW, S_UP, S_UI, S_LP, S_LI, S_FLAGS,
    S_RTPTR, S_RTCOL, S_RTPOS, S_PROG, S_SREC, S_COUNT
};

// One streamed block of the banded solves (lane_band.cuh): index words
// (column pointers, row indices, output columns), the block's factor entries
// and its per-column values, for 32 lanes.
constexpr uint32_t kSolveIdxWords = 160;  // >= kSolveCols + 1 + kSolveEntries + kSolveCols
constexpr uint32_t kSolveBufBytes = kSolveIdxWords * 4u + 64u * 32u * 8u + 2u * 32u * 32u * 8u;

// Staging modes of a template: nothing, the index arrays, or the index
// arrays and the LU chain.
enum : uint32_t { kStageNone = 0, kStageIndex = 1, kStageLu = 2 };

__host__ __device__ inline uint32_t pad4(uint32_t words) { return (words + 3u) & ~3u; }

__host__ __device__ inline uint32_t stage_words(const GroupDev& d, int k, uint32_t mode) {
    const bool rows = d.refine_rows != 0;
    // a tile replaying from the staged program reads neither the tape's
    // column pointers, scatter rows nor flags
    const bool by_prog = mode == kStageLu && d.n_rec != 0;
    switch (k) {
    case S_DIAG: return d.n;
    case S_VOID: return d.n_void;
    case S_CURROW: return (d.n + 3u) / 4u;
    case S_SLOTDIAG: return (d.nnz + 3u) / 4u;
    case S_RES_T: return 2 * d.n_res;
    case S_CAP_T: return 2 * d.n_cap;
    case S_VSRC_T: return 3 * d.n_vsrc;
    case S_DIO_T: return 2 * d.n_dio;
    case S_MOS_T: return 4 * d.n_mos;
    case S_GIPTR: return d.n_items + 1;
    case S_GIENT: return d.n_gi;
    case S_SITE: return d.n_sites;
    case S_Q: return d.n;
    case S_PINV: return d.n;
    case S_COLPTR: return by_prog ? 0u : d.n + 1;
    case S_PROW: return by_prog ? 0u : d.nnz;
    case S_UP: return d.n + 1;
    case S_UI: return d.nnz_u;
    case S_LP: return d.n + 1;
    case S_LI: return d.nnz_l;
    case S_FLAGS: return by_prog ? 0u : d.n;
    case S_RTPTR: return rows ? d.n + 1 : 0u;
    case S_RTCOL: return rows ? d.nnz : 0u;
    case S_RTPOS: return rows ? d.nnz : 0u;
    case S_PROG: return (mode == kStageLu && d.rec_stage) ? d.n_rec : 0u;
    case S_SREC: return (mode == kStageLu && d.srec_stage) ? d.n_srec : 0u;
    default: return 0u;
    }
}

__host__ __device__ inline const void* stage_src(const GroupDev& d, int k) {
    switch (k) {
    case S_DIAG: return d.diag;
    case S_VOID: return d.void_slots;
    case S_CURROW: return d.cur_row;
    case S_SLOTDIAG: return d.slot_diag;
    case S_RES_T: return d.res_t;
    case S_CAP_T: return d.cap_t;
    case S_VSRC_T: return d.vsrc_t;
    case S_DIO_T: return d.dio_t;
    case S_MOS_T: return d.mos_t;
    case S_GIPTR: return d.gi_ptr;
    case S_GIENT: return d.gi_ent;
    case S_SITE: return d.site_cell;
    case S_Q: return d.q;
    case S_PINV: return d.pinv;
    case S_COLPTR: return d.col_ptr;
    case S_PROW: return d.prow;
    case S_UP: return d.up;
    case S_UI: return d.ui;
    case S_LP: return d.lp;
    case S_LI: return d.li;
    case S_FLAGS: return d.flags;
    case S_RTPTR: return d.rt_ptr;
    case S_RTCOL: return d.rt_col;
    case S_RTPOS: return d.rt_pos;
    case S_PROG: return d.lu_rec;
    case S_SREC: return d.sol_rec;
    default: return nullptr;
    }
}

__device__ inline void stage_redirect(GroupDev& d, int k, const void* p) {
    const uint32_t* u = static_cast<const uint32_t*>(p);
    switch (k) {
    case S_DIAG: d.diag = u; break;
    case S_VOID: d.void_slots = u; break;
    case S_CURROW: d.cur_row = static_cast<const uint8_t*>(p); break;
    case S_SLOTDIAG: d.slot_diag = static_cast<const uint8_t*>(p); break;
    case S_RES_T: d.res_t = u; break;
    case S_CAP_T: d.cap_t = u; break;
    case S_VSRC_T: d.vsrc_t = u; break;
    case S_DIO_T: d.dio_t = u; break;
    case S_MOS_T: d.mos_t = u; break;
    case S_GIPTR: d.gi_ptr = u; break;
    case S_GIENT: d.gi_ent = u; break;
    case S_SITE: d.site_cell = u; break;
    case S_Q: d.q = u; break;
    case S_PINV: d.pinv = u; break;
    case S_COLPTR: d.col_ptr = u; break;
    case S_PROW: d.prow = u; break;
    case S_UP: d.up = u; break;
    case S_UI: d.ui = u; break;
    case S_LP: d.lp = u; break;
    case S_LI: d.li = u; break;
    case S_FLAGS: d.flags = u; break;
    case S_RTPTR: d.rt_ptr = u; break;
    case S_RTCOL: d.rt_col = u; break;
    case S_RTPOS: d.rt_pos = u; break;
    case S_PROG: d.lu_rec = u; break;
    case S_SREC: d.sol_rec = u; break;
    default: break;
    }
}

struct SmemPlan {
    uint32_t off[S_COUNT];   // u32-word offsets of the staged arrays
    uint32_t len[S_COUNT];   // padded word counts
    uint32_t idx_words;      // total staged words (multiple of 4)
    uint32_t a_off, w_off, lx_off, ux_off, ud_off;  // byte offsets of the LU chain (kStageLu)
    uint32_t band_off;       // byte offset of the banded replay's buffers
    uint32_t bytes;          // total dynamic shared memory of the tile
};

// Layout of the tile's dynamic shared memory in staging mode `mode`: the
// mbarrier, the index arrays, then (kStageLu) A, the work vector w (the
// solves' y aliases it: w is all-zero between replays, and each solve
// zeroes y after use), and the factor, in FP32 for `f32` tiles and FP64
// otherwise.
__host__ __device__ inline SmemPlan smem_plan(const GroupDev& d, uint32_t mode, bool f32) {
    SmemPlan p{};
    const uint32_t es = f32 ? 4u : 8u;
    uint32_t b = 0;
    if (mode != kStageNone) {
        uint32_t o = 4;  // the first 16 bytes hold the mbarrier
        for (int k = 0; k < S_COUNT; k++) {
            p.off[k] = o;
            p.len[k] = pad4(stage_words(d, k, mode));
            o += p.len[k];
        }
        p.idx_words = o - 4;
        b = o * 4;
    }
    if (mode == kStageLu) {
        b = (b + 15u) & ~15u;
        p.a_off = b;
        b += d.nnz * 32u * es;
        p.w_off = b;
        b += d.n * 32u * es;
        p.lx_off = b;
        b += d.nnz_l * 32u * es;
        p.ux_off = b;
        b += d.nnz_u * 32u * es;
        p.ud_off = b;
        b += d.n * 32u * es;
    }
    // the banded replay's and solves' buffers (lane_band.cuh, shared in
    // time) after the staged arrays
    if (mode != kStageLu && d.band_ok) {
        b = (b + 15u) & ~15u;
        p.band_off = b;
        uint32_t refac = 2u * d.band_cw * 4u + 2u * d.band_ce * 32u * 8u + (d.band_w + d.band_l) * 32u * 8u;
        uint32_t solve = 2u * kSolveBufBytes + d.band_w * 32u * 8u;
        b += refac > solve ? refac : solve;
    }
    p.bytes = (b + 15u) & ~15u;
    return p;
}

struct SmemTile {
    void *a, *w, *lx, *ux, *ud;
    SmemPlan plan;
};

__device__ __forceinline__ SmemTile smem_tile(unsigned char* base, const SmemPlan& p) {
    SmemTile t;
    t.plan = p;
    t.a = base + p.a_off;
    t.w = base + p.w_off;
    t.lx = base + p.lx_off;
    t.ux = base + p.ux_off;
    t.ud = base + p.ud_off;
    return t;
}

// Copies the tile's template descriptor to shared memory and stages its
// index arrays by bulk copies: thread 0 issues them, every thread of warp 0
// waits (bounded: a copy of in-bounds memory completes; past the bound the
// descriptor keeps its global pointers and the tile runs unstaged). In
// kStageLu the work vector starts at zero. Returns the descriptor the tile
// runs on.
__device__ const GroupDev* stage_template(const GroupDev& g, GroupDev& sd, unsigned char* base, bool f32) {
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&g);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
        for (uint32_t i = threadIdx.x; i < sizeof(GroupDev) / 4; i += blockDim.x) dst[i] = src[i];
    }
    const uint32_t mode = g.stage_mode;
    if (mode == kStageNone) {
        __syncthreads();
        return &sd;
    }
    const SmemPlan p = smem_plan(g, mode, f32);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base);
    uint32_t* u = reinterpret_cast<uint32_t*>(base);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(bar, p.idx_words * 4u);
        for (int k = 0; k < S_COUNT; k++)
            if (p.len[k]) bulk_g2s(u + p.off[k], stage_src(g, k), p.len[k] * 4u, bar);
    }
    if (mode == kStageLu) {
        uint32_t* wz = reinterpret_cast<uint32_t*>(base + p.w_off);
        uint32_t nz = (p.lx_off - p.w_off) / 4u;
        for (uint32_t i = threadIdx.x; i < nz; i += blockDim.x) wz[i] = 0u;
    }
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
    ok = __syncthreads_and(ok || threadIdx.x >= 32) != 0;
    if (threadIdx.x == 0) {
        if (ok)
            for (int k = 0; k < S_COUNT; k++)
                if (p.len[k]) stage_redirect(sd, k, u + p.off[k]);
        if (!ok) sd.stage_mode = kStageNone;
    }
    __syncthreads();
    return &sd;
}

#define SL(arr, i) (arr)[(size_t)(i) * 32 + lane]

// The template's tape words, read into registers once per call (the
// descriptor may sit in shared memory next to the stores of the chain).
struct TapeView {
    const uint32_t *__restrict__ q, *__restrict__ col_ptr, *__restrict__ prow, *__restrict__ up,
        *__restrict__ ui, *__restrict__ lp, *__restrict__ li, *__restrict__ flags, *__restrict__ pinv;
    uint32_t n;
};

// The staged tape of a kStageLu tile, addressed from the shared-memory symbol.
__device__ __forceinline__ TapeView tape_view_smem(const GroupDev& d, const SmemPlan& p) {
    const uint32_t* u = reinterpret_cast<const uint32_t*>(g_dsm);
    return TapeView{u + p.off[S_Q],  u + p.off[S_COLPTR], u + p.off[S_PROW],  u + p.off[S_UP],  u + p.off[S_UI],
                    u + p.off[S_LP], u + p.off[S_LI],     u + p.off[S_FLAGS], u + p.off[S_PINV], d.n};
}

// The replay in shared memory; T = double or float. 0 holds, 1 pivot or
// store failure, 2 only a multiplier past 1 / pivot_tol.
template <typename T>
__device__ __forceinline__ int refactor_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    T* __restrict__ w = static_cast<T*>(s.w);
    T* __restrict__ lx = static_cast<T*>(s.lx);
    T* __restrict__ ux = static_cast<T*>(s.ux);
    T* __restrict__ ud = static_cast<T*>(s.ud);
    const T* __restrict__ a = static_cast<const T*>(s.a);
    const uint32_t P = d.P;
    const TapeView t = tape_view_smem(d, s.plan);
    for (uint32_t v = 0; v < d.n_void; v++)
        if (LM(d.a, d.void_slots[v]) != 0.0) return 1;
    constexpr bool f64 = sizeof(T) == 8;
    bool bad = false, nonfinite = false;
    const T growth = (T)1e-12;
    const T inf = (T)INFINITY;
    for (uint32_t k = 0; k < t.n; k++) {
        uint32_t c = t.q[k];
        for (uint32_t p = t.col_ptr[c]; p < t.col_ptr[c + 1]; p++) SL(w, t.prow[p]) = SL(a, p);
        for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) {
            uint32_t i = t.ui[p];
            T uki = SL(w, i);
            SL(w, i) = (T)0;
            SL(ux, p) = uki;
            nonfinite |= !(uki - uki == (T)0);
            for (uint32_t pl = t.lp[i]; pl < t.lp[i + 1]; pl++) SL(w, t.li[pl]) -= SL(lx, pl) * uki;
        }
        uint32_t fl = t.flags[k];
        if (fl & 1u) {
            SL(ud, k) = (T)1;
            for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) { SL(lx, p) = (T)0; SL(w, t.li[p]) = (T)0; }
            SL(w, k) = (T)0;
            for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) {
                uint32_t i = t.ui[p];
                for (uint32_t pl = t.lp[i]; pl < t.lp[i + 1]; pl++) SL(w, t.li[pl]) = (T)0;
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
                for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) {
                    uint32_t r = t.li[p];
                    T v = SL(w, r);
                    SL(w, r) = (T)0;
                    uint64_t vb = dbits(fabs((double)v));
                    cb = cb > vb ? cb : vb;
                    SL(lx, p) = v / dk;
                }
                bad |= !(fabs((double)dk) >= 1e-12 * bitsd(cb));
            } else {
                for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) {
                    uint32_t r = t.li[p];
                    T lv = SL(w, r) / dk;
                    nonfinite |= !(lv - lv == (T)0);
                    SL(lx, p) = lv;
                    SL(w, r) = (T)0;
                }
            }
        } else {
            T cmax = fabs(dk);
            for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) {
                uint32_t r = t.li[p];
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
        for (uint32_t k = 0; k < t.n; k++) {
            if (t.flags[k] & 2u) continue;
            for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) {
                uint64_t b = dbits(fabs((double)SL(lx, p)));
                worst = worst > b ? worst : b;
            }
        }
        return bitsd(worst) <= kWide ? 0 : 2;
    }
    return 0;
}

// The replay from the template's 16-byte records (tape.h lu_records): the
// same operations on the same locations in the same order as
// refactor_smem, except that an FP32 tile multiplies a pivot column by the
// pivot's reciprocal instead of dividing each entry (the FP64 residual and
// Newton take up the rounding). Each record's loads are issued together and
// the next record is read while the current one runs. `d` is the tile's
// staged descriptor: lu_rec points into shared memory when the records are
// staged there.
template <typename T>
__device__ __forceinline__ int refactor_rec(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    T* __restrict__ w = static_cast<T*>(s.w);
    T* __restrict__ lx = static_cast<T*>(s.lx);
    T* __restrict__ ux = static_cast<T*>(s.ux);
    T* __restrict__ ud = static_cast<T*>(s.ud);
    const T* __restrict__ a = static_cast<const T*>(s.a);
    // staged in shared memory, or read from global memory through L1
    const uint4* __restrict__ rec = reinterpret_cast<const uint4*>(d.lu_rec);
    const uint32_t P = d.P;
    for (uint32_t v = 0; v < d.n_void; v++)
        if (LM(d.a, d.void_slots[v]) != 0.0) return 1;
    constexpr bool f64 = sizeof(T) == 8;
    bool bad = false, nonfinite = false;
    uint64_t worst = 0, cb = 0;
    const T growth = (T)1e-12;
    const T inf = (T)INFINITY;
    T uki = (T)0, dk = (T)1, rk = (T)1, cmax = (T)0;
    uint32_t pfl = 0;
    uint4 cur = rec[0];
    for (uint32_t pc = 1;; pc++) {
        const uint4 nxt = rec[pc];
        const uint32_t op = cur.x & 15u, m = (cur.x >> 4) & 15u;
        if (op == kRecScat) {
            const T v0 = SL(a, cur.y & 0xffffu);
            const T v1 = m > 1 ? SL(a, cur.z & 0xffffu) : (T)0;
            const T v2 = m > 2 ? SL(a, cur.w & 0xffffu) : (T)0;
            SL(w, cur.y >> 16) = v0;
            if (m > 1) SL(w, cur.z >> 16) = v1;
            if (m > 2) SL(w, cur.w >> 16) = v2;
        } else if (op == kRecTake || op == kRecAxpy) {
            // TAKE: u_ki leaves the work vector for U; both: w -= L(:, i) u_ki
            const bool take = op == kRecTake;
            const uint32_t e0 = take ? cur.z : cur.y, e1 = take ? cur.w : cur.z, e2 = cur.w;
            const uint32_t i = cur.x >> 16;
            if (take) uki = SL(w, i);
            const T w0 = m > 0 ? SL(w, e0 >> 16) : (T)0, l0 = m > 0 ? SL(lx, e0 & 0xffffu) : (T)0;
            const T w1 = m > 1 ? SL(w, e1 >> 16) : (T)0, l1 = m > 1 ? SL(lx, e1 & 0xffffu) : (T)0;
            const T w2 = (!take && m > 2) ? SL(w, e2 >> 16) : (T)0, l2 = (!take && m > 2) ? SL(lx, e2 & 0xffffu) : (T)0;
            if (take) {
                SL(w, i) = (T)0;
                SL(ux, cur.y) = uki;
                nonfinite |= !(uki - uki == (T)0);
            }
            if (m > 0) SL(w, e0 >> 16) = w0 - l0 * uki;
            if (m > 1) SL(w, e1 >> 16) = w1 - l1 * uki;
            if (!take && m > 2) SL(w, e2 >> 16) = w2 - l2 * uki;
        } else if (op == kRecPiv || op == kRecDiv) {
            if (op == kRecPiv) {
                const uint32_t k = cur.x >> 16;
                pfl = (cur.x >> 8) & 15u;
                dk = SL(w, k);
                SL(w, k) = (T)0;
                const bool dead = dk == (T)0 || !(fabs(dk) < inf);
                bad |= dead;
                if (dead) dk = (T)1;
                SL(ud, k) = dk;
                if constexpr (f64) cb = dbits(fabs((double)dk));
                else {
                    cmax = fabsf(dk);
                    rk = (T)1 / dk;
                }
            }
            const uint32_t e[3] = {cur.y, cur.z, cur.w};
            T v[3];
#pragma unroll
            for (int j = 0; j < 3; j++) v[j] = (uint32_t)j < m ? SL(w, e[j] >> 16) : (T)0;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                if ((uint32_t)j >= m) break;
                SL(w, e[j] >> 16) = (T)0;
                T lv;
                if constexpr (f64) {
                    lv = v[j] / dk;
                    if (!(pfl & 2u)) {
                        const uint64_t vb = dbits(fabs((double)v[j])), lb = dbits(fabs((double)lv));
                        cb = cb > vb ? cb : vb;
                        worst = worst > lb ? worst : lb;
                    } else {
                        nonfinite |= !(lv - lv == (T)0);
                    }
                } else {
                    lv = v[j] * rk;
                    cmax = fmaxf(cmax, fabsf(v[j]));
                    nonfinite |= !(lv - lv == (T)0);
                }
                SL(lx, e[j] & 0xffffu) = lv;
            }
            if ((cur.x & (1u << 12)) && !(pfl & 2u)) {
                if constexpr (f64) bad |= !(fabs((double)dk) >= 1e-12 * bitsd(cb));
                else bad |= !(fabsf(dk) >= growth * cmax) || !(cmax / fabsf(dk) <= (T)kWide);
            }
        } else if (op == kRecVoid) {
            const uint32_t k = cur.x >> 16;
            const TapeView t = tape_view_smem(d, s.plan);
            SL(ud, k) = (T)1;
            for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) { SL(lx, p) = (T)0; SL(w, t.li[p]) = (T)0; }
            SL(w, k) = (T)0;
            for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) {
                uint32_t i = t.ui[p];
                for (uint32_t pl = t.lp[i]; pl < t.lp[i + 1]; pl++) SL(w, t.li[pl]) = (T)0;
            }
        } else {
            break;
        }
        cur = nxt;
    }
    if (nonfinite || bad) return 1;
    if constexpr (f64) return bitsd(worst) <= kWide ? 0 : 2;
    return 0;
}

// Forward and back substitution of y in place through the shared factors
// (luSolve's two sweeps).
template <typename T>
__device__ __forceinline__ void subst_smem(const TapeView& t, const SmemTile& s, T* __restrict__ y, uint32_t lane) {
    const T* __restrict__ lx = static_cast<const T*>(s.lx);
    const T* __restrict__ ux = static_cast<const T*>(s.ux);
    const T* __restrict__ ud = static_cast<const T*>(s.ud);
    // the entries of one column update distinct rows: two at a time
    for (uint32_t k = 0; k < t.n; k++) {
        const T yk = SL(y, k);
        if (yk != (T)0) {
            uint32_t p = t.lp[k];
            const uint32_t pe = t.lp[k + 1];
            for (; p + 1 < pe; p += 2) {
                const uint32_t r0 = t.li[p], r1 = t.li[p + 1];
                const T y0 = SL(y, r0), y1 = SL(y, r1);
                const T l0 = SL(lx, p), l1 = SL(lx, p + 1);
                SL(y, r0) = y0 - l0 * yk;
                SL(y, r1) = y1 - l1 * yk;
            }
            if (p < pe) SL(y, t.li[p]) -= SL(lx, p) * yk;
        }
    }
    for (uint32_t k = t.n; k-- > 0;) {
        const T zk = SL(y, k) / SL(ud, k);
        SL(y, k) = zk;
        if (zk != (T)0) {
            uint32_t p = t.up[k];
            const uint32_t pe = t.up[k + 1];
            for (; p + 1 < pe; p += 2) {
                const uint32_t r0 = t.ui[p], r1 = t.ui[p + 1];
                const T y0 = SL(y, r0), y1 = SL(y, r1);
                const T u0 = SL(ux, p), u1 = SL(ux, p + 1);
                SL(y, r0) = y0 - u0 * zk;
                SL(y, r1) = y1 - u1 * zk;
            }
            if (p < pe) SL(y, t.ui[p]) -= SL(ux, p) * zk;
        }
    }
}

// dx = -A^-1 rhs through the shared factors (luSolve with neg); rhs and dx
// are the lane's global rows. y is the work vector w, zero again on return.
template <typename T>
__device__ __forceinline__ void solve_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    const uint32_t P = d.P;
    const TapeView t = tape_view_smem(d, s.plan);
    const double* __restrict__ rhs = d.rhs;
    double* __restrict__ dx = d.dx;
    T* __restrict__ y = static_cast<T*>(s.w);
    // the right-hand side comes from global memory: eight loads in flight
    uint32_t r = 0;
    for (; r + 7 < t.n; r += 8) {
        double b[8];
#pragma unroll
        for (int j = 0; j < 8; j++) b[j] = LM(rhs, r + j);
#pragma unroll
        for (int j = 0; j < 8; j++) SL(y, t.pinv[r + j]) = (T)(-b[j]);
    }
    for (; r < t.n; r++) SL(y, t.pinv[r]) = (T)(-LM(rhs, r));
    subst_smem<T>(t, s, y, lane);
    for (uint32_t j = 0; j < t.n; j++) {
        LM(dx, t.q[j]) = (double)SL(y, j);
        SL(y, j) = (T)0;
    }
}

// solve_smem from the template's solve records (tape.h solve_records): the
// same sweeps on the same locations in the same order, a record's loads
// issued together and the next record read while the current one runs,
// without the skip of zero entries (y - L * 0 is y).
template <typename T>
__device__ __forceinline__ void solve_rec(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    const uint32_t P = d.P;
    const TapeView t = tape_view_smem(d, s.plan);
    const double* __restrict__ rhs = d.rhs;
    double* __restrict__ dx = d.dx;
    T* __restrict__ y = static_cast<T*>(s.w);
    const T* __restrict__ lx = static_cast<const T*>(s.lx);
    const T* __restrict__ ux = static_cast<const T*>(s.ux);
    const T* __restrict__ ud = static_cast<const T*>(s.ud);
    uint32_t r = 0;
    for (; r + 7 < t.n; r += 8) {
        double b[8];
#pragma unroll
        for (int j = 0; j < 8; j++) b[j] = LM(rhs, r + j);
#pragma unroll
        for (int j = 0; j < 8; j++) SL(y, t.pinv[r + j]) = (T)(-b[j]);
    }
    for (; r < t.n; r++) SL(y, t.pinv[r]) = (T)(-LM(rhs, r));
    const uint4* __restrict__ rec = reinterpret_cast<const uint4*>(d.sol_rec);
    T yk = (T)0;
    uint4 cur = rec[0];
    for (uint32_t pc = 1;; pc++) {
        const uint4 nxt = rec[pc];
        const uint32_t op = cur.x & 15u, m = (cur.x >> 4) & 15u;
        if (op == kSolEnd) break;
        const T* __restrict__ f = (op == kSolFwd || op == kSolFwdC) ? lx : ux;
        const T y0 = m > 0 ? SL(y, cur.y >> 16) : (T)0, f0 = m > 0 ? SL(f, cur.y & 0xffffu) : (T)0;
        const T y1 = m > 1 ? SL(y, cur.z >> 16) : (T)0, f1 = m > 1 ? SL(f, cur.z & 0xffffu) : (T)0;
        const T y2 = m > 2 ? SL(y, cur.w >> 16) : (T)0, f2 = m > 2 ? SL(f, cur.w & 0xffffu) : (T)0;
        if (op == kSolFwd) {
            yk = SL(y, cur.x >> 16);
        } else if (op == kSolBwd) {
            const uint32_t k = cur.x >> 16;
            yk = SL(y, k) / SL(ud, k);
            SL(y, k) = yk;
        }
        if (m > 0) SL(y, cur.y >> 16) = y0 - f0 * yk;
        if (m > 1) SL(y, cur.z >> 16) = y1 - f1 * yk;
        if (m > 2) SL(y, cur.w >> 16) = y2 - f2 * yk;
        cur = nxt;
    }
    for (uint32_t j = 0; j < t.n; j++) {
        LM(dx, t.q[j]) = (double)SL(y, j);
        SL(y, j) = (T)0;
    }
}

// One FP64-residual refinement sweep of an FP32 solve (refine_mixed):
// r = rhs + A dx row by row, the products added by ascending column as the
// column sweep adds them (columns with dx = 0 skipped), then
// dx += -A^-1 r through the FP32 factors.
__device__ __forceinline__ void refine_smem(const GroupDev& d, const SmemTile& s, uint32_t lane, uint32_t l) {
    const uint32_t P = d.P;
    const TapeView t = tape_view_smem(d, s.plan);
    const uint32_t* u = reinterpret_cast<const uint32_t*>(g_dsm);
    const uint32_t *__restrict__ rt_ptr = u + s.plan.off[S_RTPTR], *__restrict__ rt_col = u + s.plan.off[S_RTCOL],
                   *__restrict__ rt_pos = u + s.plan.off[S_RTPOS];
    const double* __restrict__ rhs = d.rhs;
    const double* __restrict__ a = d.a;
    double* __restrict__ dx = d.dx;
    float* __restrict__ y = static_cast<float*>(s.w);
    for (uint32_t i = 0; i < t.n; i++) {
        double r = LM(rhs, i);
        for (uint32_t e = rt_ptr[i]; e < rt_ptr[i + 1]; e++) {
            double xc = LM(dx, rt_col[e]);
            if (xc != 0.0) r += LM(a, rt_pos[e]) * xc;
        }
        SL(y, t.pinv[i]) = (float)(-r);
    }
    subst_smem<float>(t, s, y, lane);
    for (uint32_t j = 0; j < t.n; j++) {
        LM(dx, t.q[j]) += (double)SL(y, j);
        SL(y, j) = 0.0f;
    }
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
