// The learned next-step predictor of the transient lanes: the Newton start
// of a lane's next attempt from its last three accepted solutions and the
// step about to be taken, through the small MLP of mlp_gemm.cuh on the
// tensor cores, in place of the reference's linear predictor
// (src/solver/lane_device.zig:388, src/solver/kernels/lane.zig:473-482).
//
// k_step_predict runs the whole network for 128 lanes of one template per
// CTA: it stages the network's BF16 weight image into shared memory with one
// bulk copy (cp.async.bulk on an mbarrier) while its threads build the lanes'
// standardized features straight from the lane-interleaved histories (one
// thread per lane, so every history load is a coalesced run across lanes),
// runs the three layers as tcgen05.mma chains into tensor memory, and writes
// each lane's start x = cur + (dt / h0)(cur - prev) + y lane-interleaved into
// the template's xpred, where k_tran reads it.
#pragma once

#include "lane_kernels.cuh"
#include "mlp_gemm.cuh"

namespace espl {

// The predictor's dynamic shared memory: the network's tiles and each lane's
// linear predictor x_lin (n FP64 values per lane, read by the epilogue).
__host__ __device__ inline size_t step_predict_smem(int dp, int op, uint32_t n) {
    return mlp::infer_smem_bytes(dp, op) + (size_t)n * 128 * 8;
}

struct StepPredictArgs {
    const GroupDev* d;    // the template's descriptor (device copy)
    const LaneState* st;  // every lane's state; the template's from d->lane0
    mlp::MlpView w;
    double dt_max;
};

// Lanes of one template, 128 per CTA, 128 threads (one per lane). Dynamic
// shared memory: step_predict_smem(dp, op, n). A lane that is not stepping,
// or has fewer than three accepted steps, gets a NaN row (k_tran starts it
// from the linear predictor).
__global__ void __launch_bounds__(128) k_step_predict(StepPredictArgs a) {
    using namespace mlp;
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(8) uint64_t wbar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const GroupDev& d = *a.d;
    const int dp = a.w.dp, op = a.w.op;
    const uint32_t n = d.n, P = d.P;
    unsigned char* sx = g_dsm;                          // 128 x dp
    unsigned char* sw1 = sx + 128 * dp * 2;             // the weight image: W1 128 x dp,
    unsigned char* sw2 = sw1 + 128 * dp * 2;            // W2 128 x 128,
    unsigned char* sw3 = sw2 + 128 * 128 * 2;           // W3 op x 128
    unsigned char* shid = sw3 + (size_t)op * 128 * 2;   // 128 x 128 activations
    double* sxl = reinterpret_cast<double*>(shid + 128 * 128 * 2);  // n x 128: each lane's x_lin
    const int warp = threadIdx.x >> 5;
    const uint32_t row = threadIdx.x;
    const uint32_t l = blockIdx.x * 128u + row;
    const bool valid = l < d.lanes;
    double r0 = 0.0, r1 = 0.0, dtf = 0.0;
    bool live = false;
    if (valid) {
        const LaneState& s = a.st[d.lane0 + l];
        live = s.status == 0 && s.steps >= 3;
        r0 = s.dt / s.dt_old0;
        r1 = s.dt / s.dt_old1;
        dtf = s.dt / a.dt_max;
    }
    if (threadIdx.x == 0) {
        mbar_init1(&bar);
        mbar_init1(&wbar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(128u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    const uint32_t image_bytes = (uint32_t)weight_image_bytes(dp, op);
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&wbar, image_bytes);
        bulk_g2s(sw1, a.w.image, image_bytes, &wbar);
    }
    // the features of this thread's lane, standardized, into row `row`
    auto put = [&](uint32_t k, float v) {
        *reinterpret_cast<__nv_bfloat16*>(sx + tile_off_k(row, k, (uint32_t)dp)) = __float2bfloat16(v);
    };
    const float *im = a.w.in_mean, *is = a.w.in_std;
    // unknowns in fours: the histories' loads of four rows are in flight at once
#pragma unroll 4
    for (uint32_t i = 0; i < n; i++) {
        float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
        if (live) {
            const size_t e = (size_t)i * P + l;
            double f[3];
            step_features(d.cur[e], d.prev[e], d.prev2[e], r0, r1, f);
            sxl[i * 128 + row] = f[0] + f[1];
            v0 = (float)((f[0] - (double)im[i]) / (double)is[i]);
            v1 = (float)((f[1] - (double)im[n + i]) / (double)is[n + i]);
            v2 = (float)((f[2] - (double)im[2 * n + i]) / (double)is[2 * n + i]);
        }
        put(i, v0);
        put(n + i, v1);
        put(2 * n + i, v2);
    }
    put(3 * n, live ? (float)((dtf - (double)im[3 * n]) / (double)is[3 * n]) : 0.0f);
    for (uint32_t k = 3 * n + 1; k < (uint32_t)dp; k++) put(k, 0.0f);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (!mbar_wait_bounded(&wbar, 0)) failed = 1;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (!failed) {
        const float *om = a.w.out_mean, *og = a.w.out_gain;
        mlp_layers(sx, sw1, sw2, sw3, shid, a.w.b1, a.w.b2, a.w.b3, dp, op, (int)n, tmem, &bar, &failed,
                   [&](int, int o, float v) {
                       if (!valid) return;
                       const size_t e = (size_t)o * P + l;
                       if (!live) {
                           d.xpred[e] = __longlong_as_double(0x7FF8000000000000LL);
                           return;
                       }
                       const double y = og[o] != 0.0f ? (double)v * (double)og[o] + (double)om[o] : (double)om[o];
                       d.xpred[e] = sxl[o * 128 + row] + y;
                   });
    } else {
        // the weights never arrived: give the bulk copy a second bounded wait
        // before the CTA's shared memory is released
        mbar_wait_bounded(&wbar, 0);
    }
    if (failed && threadIdx.x == 0) atomicExch(a.w.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
}

// Adds to *count the lanes of the tiles of a launch class that are still
// stepping (status 0), one thread per lane.
__global__ void __launch_bounds__(kTileThreads) k_count_stepping(TileMap m, const LaneState* st, uint32_t* count) {
    TileCtx c = tile_ctx(m);
    if (c.warp != 0) return;
    const bool run = c.valid && st[c.d->lane0 + c.l].status == 0;
    const unsigned b = __ballot_sync(c.tw == 32 ? 0xffffffffu : (1u << c.tw) - 1u, run);
    if (c.lane == 0 && b) atomicAdd(count, (uint32_t)__popc(b));
}

}  // namespace espl
