// internal.hpp - the solver handle behind the C ABI (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../include/mcg.h"
#include "kernels.cuh"

namespace mcg {
// The radial-statistics state an output writes (a copy, so that outputs
// written on a worker thread see the state of the step they belong to).
struct StatsSnapshot {
    bool started = false;
    uint32_t start_step = 0;
    uint32_t samples = 0;
};
struct AsyncOutput;  // output_async.cpp
}  // namespace mcg

struct mcg_handle {
    mcg_params p{};
    mcg::DeviceState s{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int cur = 0;            // pops[cur] holds f(t) in pull layout
    int64_t step = 0;       // completed collisions
    uint64_t launches = 0;  // kernels launched through this handle
    mcg::FusedTiling tiling{};
    bool mom_stale = false;  // moment planes lag the last fused step

    // radial statistics (meanF/memoryMeanFields.cuh:39-45)
    int stats_mode = -1;  // -1 automatic from NSTATS_START_STEP, 0 off, 1 on
    int adjoint_tape = 20;  // moment records the periodic adjoint's innermost segments tape (mcg_set_adjoint_tape)
    int jet_adjoint_tapes = 0;  // segment tapes of the jet adjoint (0: as many as device memory allows)
    bool stats_started = false;
    uint32_t stats_start_step = 0;
    uint32_t stats_samples = 0;
    std::vector<uint64_t> ncols;  // interior (x,z) columns per radial bin

    // total kinetic energy state (meanF/memoryMeanFields.cuh:24-37)
    bool first_tke = true;
    float tke_total = 0.f, tke_avg = 0.f, tke_avg_prev = 0.f, tke_delta = 0.f, tke_abs_delta = 0.f;
    uint32_t uy_avg_samples = 0;

    float *d_inlet_profile = nullptr;   // [NZ][NX] inlet velocity multipliers (mcg_set_inlet_bessel)
    std::vector<float> inlet_coeffs;    // the Bessel coefficients it was made from
    double *d_scalar = nullptr;  // 8 doubles of device scratch for reductions
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // host state transfer (mcg_set/get_populations): a copy stream beside
    // `stream`, and per z-chunk events of the copies and of the kernels
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t xfer_start = nullptr;
    cudaEvent_t xfer_copy[16] = {}, xfer_kern[16] = {};
    std::vector<cudaEvent_t> prof_events;  // mcg_step_profiled

    mcg::AsyncOutput *async_out = nullptr;  // mcg_output_step_async pipeline (created on first use)
    char *d_vti_text = nullptr, *h_vti_text = nullptr;  // VTI text of mcg_output_step (first use)

    // output files (meanF/meanFieldsRT.cuh:23-33)
    std::string case_dir, mean_dir, vti_dir;
    FILE *f_tke_total = nullptr, *f_tke_avg = nullptr, *f_tke_diff = nullptr;
};

namespace mcg {

// Records the error text for mcg_last_error_string() and returns s.
mcg_status fail(mcg_status s, const std::string &msg);

// Entry points run their body through guarded(): an exception thrown inside
// (a host allocation failing) becomes an error status with its message
// instead of crossing the C ABI.
template <class F>
mcg_status guarded(F &&body) noexcept {
    try {
        return body();
    } catch (const std::bad_alloc &) {
        return fail(MCG_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(MCG_ERR_STATE, e.what());
    } catch (...) {
        return fail(MCG_ERR_STATE, "unexpected exception");
    }
}
mcg_status cuda_fail(cudaError_t e, const char *what);

// Radial count materialisation: samples * ncols[rb] on interior y rows.
void radial_counts(const mcg_handle *h, uint64_t *count);
void radial_counts_for(const mcg_handle *h, uint32_t samples, uint64_t *count);
StatsSnapshot stats_snapshot(const mcg_handle *h);
// kernels.cu:154-166 running average of the total kinetic energy, from the
// float64 device sum of this output step
void tke_update(mcg_handle *h, int32_t step, double total);

// io.cpp
mcg_status io_open(mcg_handle *h, const char *root);
mcg_status io_close(mcg_handle *h);
mcg_status io_write_case_metadata(mcg_handle *h);
mcg_status io_write_radial(mcg_handle *h);
mcg_status io_write_vti(mcg_handle *h, const std::string &path);
mcg_status io_write_tke_sample(mcg_handle *h, int32_t step);
// The same writers on host copies: radial sums [5][NY*NR_BINS], fields
// [5][Ncells] (rhor, rhob, ux, uy, uz), the statistics state of the output step.
mcg_status io_write_radial_host(mcg_handle *h, const StatsSnapshot &st, const double *sums);
// text: the four base64 arrays laid out by vti_text_layout (launch_vti_encode).
mcg_status io_write_vti_text(mcg_handle *h, const std::string &path, const char *text);
mcg_status io_write_tke_sample_snap(mcg_handle *h, int32_t step, const StatsSnapshot &st);
// Time-averaged jet profiles (profile.cpp), from the radial sums of uy
// (sum_uy [NY*NR_BINS], `samples` steps): the centreline velocity uc[y] (bin 0)
// and the half-width rh[y] (NaN where undefined), as the reference's
// post/plot_profiles.py:53-91 forms them.
void profile_metrics(const mcg_handle *h, const double *sum_uy, uint32_t samples, float *uc, float *rh);
// J = 1/2 sum_{y_lo<=y<=y_hi} ((uc - uc*)/U)^2 + ((rh - rh*)/D)^2 over the y
// where every value is defined, and src[y*NR_BINS + r] = dJ/duy of one node
// of bin r at one window step (dJ/d(mean) / (samples * columns of the bin)).
double profile_objective(const mcg_handle *h, const double *sum_uy, uint32_t samples, int y_lo, int y_hi,
                         const float *uc_target, const float *rh_target, float *src);
// Asynchronous outputs (output_async.cpp): wait for pending writes; release.
mcg_status async_flush(mcg_handle *h);
mcg_status async_enqueue(mcg_handle *h, int32_t step);
void async_release(mcg_handle *h);
mcg_status io_write_uy_average(mcg_handle *h);

}  // namespace mcg
