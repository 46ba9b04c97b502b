// Test harness only: the device's streaming .meas passes
// (egspice_b200/csrc/lane_meas.cuh, all __host__ __device__) compiled for
// the host, so the CPU tests run the kernels' own measure code over sample
// tables and compare it with the oracle. States are lane-interleaved with a
// stride of kLanes and the table is fed on lane 1, as a kernel lane would.
#define __host__
#define __device__

#include "../egspice_b200/csrc/lane_meas.cuh"

#include <vector>

namespace {
constexpr size_t kLanes = 3;
constexpr size_t kLane = 1;
}  // namespace

extern "C" int dev_meas_table(const espl_meas* passes, uint32_t n_passes, const double* x, const double* cols,
                              uint32_t n_cols, uint32_t n, double* value, double* at) {
    using namespace espl;
    std::vector<double> st((size_t)n_passes * kMeasWords * kLanes, -7.0);
    auto state = [&](uint32_t p) { return st.data() + (size_t)p * kMeasWords * kLanes + kLane; };
    for (uint32_t p = 0; p < n_passes; p++) meas_init(passes[p], state(p), kLanes);
    for (uint32_t k = 0; k < n; k++)
        for (uint32_t p = 0; p < n_passes; p++) {
            const espl_meas& c = passes[p];
            const double* row = cols + (size_t)k * n_cols;
            meas_feed(c, state(p), kLanes, p ? state(p - 1) : nullptr, x[k], row[c.row],
                      c.level_row ? row[c.level_row - 1] : 0.0);
        }
    for (uint32_t p = 0; p < n_passes; p++) meas_result(passes[p], state(p), kLanes, value[p], at[p]);
    return 0;
}
