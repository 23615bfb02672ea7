// api.cu - C ABI of the solver (include/mcg.h).
//
// Owns device memory behind an opaque handle (the reference's LbmDevice and
// MeanFieldsDevice, memory.cuh:58-97 and meanF/memoryMeanFields.cuh:57-80),
// queues work on one stream, returns status codes instead of exiting.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.hpp"
#include "lattice.cuh"

namespace mcg {

namespace {
thread_local std::string g_last_error;
}

mcg_status fail(mcg_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

mcg_status cuda_fail(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? MCG_ERR_OOM : MCG_ERR_CUDA;
}

void radial_counts_for(const mcg_handle *h, uint32_t samples, uint64_t *count) {
    const int NY = h->p.NY, NRB = h->p.NX / 2;
    for (int y = 0; y < NY; ++y)
        for (int r = 0; r < NRB; ++r) {
            const bool interior = y >= 1 && y <= NY - 2;
            count[size_t(y) * NRB + r] = interior ? uint64_t(samples) * h->ncols[r] : 0;
        }
}

void radial_counts(const mcg_handle *h, uint64_t *count) { radial_counts_for(h, h->stats_samples, count); }

StatsSnapshot stats_snapshot(const mcg_handle *h) {
    StatsSnapshot s;
    s.started = h->stats_started;
    s.start_step = h->stats_start_step;
    s.samples = h->stats_samples;
    return s;
}

void tke_update(mcg_handle *h, int32_t step, double total) {
    h->tke_total = float(total);
    const unsigned sample_count = unsigned(step) / unsigned(h->p.NOUTPUT);
    const float count = float(sample_count);
    h->tke_avg = (h->tke_avg * count + h->tke_total) / (count + 1.0f);
}

}  // namespace mcg

using mcg::cuda_fail;
using mcg::fail;

#define MCG_CUDA(call, what)                                   \
    do {                                                       \
        cudaError_t e__ = (call);                              \
        if (e__ != cudaSuccess) return cuda_fail(e__, what);   \
    } while (0)

#define MCG_LAUNCH(h, call, what)                              \
    do {                                                       \
        cudaError_t e__ = (call);                              \
        if (e__ != cudaSuccess) return cuda_fail(e__, what);   \
        ++(h)->launches;                                       \
    } while (0)

#define MCG_REQUIRE(cond, msg)                                          \
    do {                                                                \
        if (!(cond)) return fail(MCG_ERR_INVALID_ARG, msg);             \
    } while (0)

namespace {

// Shared memory of one fused-step CTA: three CTAs per SM (228 KB per SM).
constexpr int kFusedSmemPerBlock = 75 * 1024;

float derive_omega(const mcg_params &p) {
    // omega_sponge (mathUtilities.cuh:60-90) with K = 0: 1/(0.5 + nu/cs^2)
    return 1.0f / std::fma(p.nu, mcg::kInvCs2, 0.5f);
}

mcg_status validate(const mcg_params *p) {
    MCG_REQUIRE(p != nullptr, "params is null");
    MCG_REQUIRE(p->NX >= 4 && p->NY >= 4 && p->NZ >= 4, "NX, NY, NZ must be >= 4 (ghost shell included)");
    const double n = double(p->NX) * p->NY * p->NZ;
    MCG_REQUIRE(n < 2147483647.0, "NX*NY*NZ must be < 2^31");
    MCG_REQUIRE(p->NX <= 256, "NX must be <= 256 (one CTA row of the fused step spans the x extent)");
    MCG_REQUIRE(p->boundary >= 0 && p->boundary <= 2, "unknown boundary mode");
    MCG_REQUIRE(p->storage == MCG_STORAGE_F32 || p->storage == MCG_STORAGE_F16, "unknown storage");
    MCG_REQUIRE(std::isfinite(p->taub) && p->taub > 0.5f, "taub must be > 0.5");
    MCG_REQUIRE(std::isfinite(p->taur) && p->taur > 0.5f, "taur must be > 0.5");
    MCG_REQUIRE(std::isfinite(p->nu) && p->nu > 0.0f, "nu must be > 0");
    MCG_REQUIRE(std::isfinite(p->sigma) && p->sigma >= 0.0f, "sigma must be finite and >= 0");
    MCG_REQUIRE(std::isfinite(p->beta_recolor) && p->beta_recolor >= 0.0f && p->beta_recolor <= 1.0f,
                "beta_recolor must be in [0,1]");
    MCG_REQUIRE(std::isfinite(p->rhor0) && p->rhor0 > 0.0f && std::isfinite(p->rhob0) && p->rhob0 > 0.0f,
                "rhor0, rhob0 must be > 0");
    MCG_REQUIRE(p->NOUTPUT > 0, "NOUTPUT must be > 0");
    MCG_REQUIRE(std::isfinite(p->jet_velocity) && std::isfinite(p->jet_radius), "jet parameters must be finite");
    MCG_REQUIRE(std::isfinite(p->sponge_K), "sponge_K must be finite");
    MCG_REQUIRE(p->sponge_K == 0.0f || p->sponge_cells >= 2, "sponge_cells must be >= 2 when sponge_K != 0");
    return MCG_OK;
}

void fill_physics(mcg_handle *h) {
    const mcg_params &p = h->p;
    mcg::Physics &ph = h->s.ph;
    ph.omega = derive_omega(p);
    ph.omega_b = 1.0f / p.taub;                                   // constants.cuh:67
    const float sigma_over_4cs4 = p.sigma / (4.0f * mcg::kCs4);  // constants.cuh:76
    const float A = sigma_over_4cs4 / p.taub;                     // forces.cuh:87-105
    ph.Ah = A / 2.0f;
    ph.beta = p.beta_recolor;
    ph.rhor0 = p.rhor0;
    ph.rhob0 = p.rhob0;
    ph.jet_x0 = p.jet_x0;
    ph.jet_z0 = p.jet_z0;
    ph.jet_r2 = p.jet_radius * p.jet_radius;
    ph.jet_velocity = p.jet_velocity;
    ph.inlet_noise = p.inlet_noise;
    ph.seed = p.seed;
    ph.sponge = p.sponge_K != 0.0f ? 1 : 0;
    ph.nu = p.nu;
    ph.sponge_K = p.sponge_K;
    const int y_end = p.NY - 2, y_start = y_end - p.sponge_cells + 1;
    ph.sponge_y_start = float(y_start);
    ph.sponge_inv_width = 1.0f / float(y_end - y_start);
    ph.NRB = p.NX / 2;
    ph.f16_rho0 = p.rhor0;
}

void compute_ncols(mcg_handle *h) {
    const mcg_params &p = h->p;
    const int NRB = p.NX / 2;
    h->ncols.assign(size_t(NRB), 0);
    for (int z = 1; z <= p.NZ - 2; ++z)
        for (int x = 1; x <= p.NX - 2; ++x) {
            const float dx = float(x) - p.jet_x0, dz = float(z) - p.jet_z0;
            const float r = std::sqrt(dx * dx + dz * dz);  // kernels.cu:207-210, float
            const unsigned rb = unsigned(r);
            if (rb < unsigned(NRB)) ++h->ncols[rb];
        }
}

size_t pop_buffer_bytes(const mcg_params &p) {
    const size_t N = size_t(p.NX) * p.NY * p.NZ;
    return p.storage == MCG_STORAGE_F16 ? size_t(mcg::kQ) * N * 4 : size_t(2 * mcg::kQ) * N * 4;
}

void release(mcg_handle *h) {
    mcg::async_release(h);
    mcg::io_close(h);
    void *ptrs[] = {h->s.pops[0], h->s.pops[1], h->s.mom,      h->s.psi[0], h->s.psi[1], h->s.radial,
                    h->s.uy_avg,  h->s.partials, h->s.flag, h->d_scalar, h->s.bmom,  h->d_inlet_profile, h->d_vti_text};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (h->h_vti_text) cudaFreeHost(h->h_vti_text);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->xfer_start) cudaEventDestroy(h->xfer_start);
    for (int k = 0; k < 16; ++k) {
        if (h->xfer_copy[k]) cudaEventDestroy(h->xfer_copy[k]);
        if (h->xfer_kern[k]) cudaEventDestroy(h->xfer_kern[k]);
    }
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

template <class T>
cudaError_t alloc_zero(T **ptr, size_t bytes) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(ptr), bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return e;
    }
    return cudaMemset(*ptr, 0, bytes);
}

mcg_status check_handle(const mcg_handle *h) {
    if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
    return MCG_OK;
}

// Automatic start of the radial statistics (meanF/meanFieldsRT.cuh:173-190).
bool stats_for_step(mcg_handle *h) {
    if (h->stats_mode == 0) return false;
    if (h->stats_mode == 1) {
        if (!h->stats_started) {
            h->stats_started = true;
            h->stats_start_step = uint32_t(h->step);
            h->stats_samples = 0;
        }
        return true;
    }
    if (!h->stats_started && h->step >= h->p.NSTATS_START_STEP) {
        h->stats_started = true;
        h->stats_start_step = uint32_t(h->step);
        h->stats_samples = 0;
    }
    return h->stats_started;
}

// One fused step (k_fused, then k_boundary for the jet).  The moment planes in
// HBM are not written by the fused kernel; they are refreshed on demand.
mcg_status one_fused_step(mcg_handle *h, bool *ran_boundary) {
    const bool jet = h->p.boundary == MCG_BOUNDARY_JET;
    const bool stats = stats_for_step(h);
    MCG_LAUNCH(h, mcg::launch_fused(h->s, h->tiling, h->cur, h->step, stats, h->stream), "fused step kernel");
    if (stats) ++h->stats_samples;
    if (jet && !h->tiling.boundary)
        MCG_LAUNCH(h, mcg::launch_boundary(h->s, h->cur ^ 1, h->step, -1, true, h->stream), "boundary kernel");
    if (ran_boundary) *ran_boundary = jet;
    h->cur ^= 1;
    ++h->step;
    h->mom_stale = true;
    return MCG_OK;
}

// After a synchronisation: whether a k_fused_bulk wait for a staged row ran
// out since the last check (the kernel sets flag[1] and finishes its march on
// stale rows, so the state is then invalid).  The flag is cleared.
mcg_status check_stage_waits(mcg_handle *h) {
    if (!h->tiling.bulk) return MCG_OK;
    int flag = 0;
    MCG_CUDA(cudaMemcpyAsync(&flag, h->s.flag + 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
             "download wait flag");
    MCG_CUDA(cudaStreamSynchronize(h->stream), "wait flag");
    if (!flag) return MCG_OK;
    MCG_CUDA(cudaMemsetAsync(h->s.flag + 1, 0, sizeof(int), h->stream), "clear wait flag");
    MCG_CUDA(cudaStreamSynchronize(h->stream), "wait flag");
    return fail(MCG_ERR_TIMEOUT, "fused step: a wait for a staged row ran out; the state is invalid");
}

mcg_status run_steps(mcg_handle *h, int32_t nsteps) {
    for (int32_t n = 0; n < nsteps; ++n)
        if (mcg_status s = one_fused_step(h, nullptr)) return s;
    return MCG_OK;
}

// Moment planes of the last completed step (what the reference's d.rhor ..
// d.Pixz hold after it): recomputed from that step's input buffer.
mcg_status ensure_moments(mcg_handle *h) {
    if (!h->mom_stale || h->step == 0) return MCG_OK;
    MCG_LAUNCH(h, mcg::launch_moments(h->s, h->cur ^ 1, h->step - 1, false, h->stream), "moments kernel");
    h->mom_stale = false;
    return MCG_OK;
}

}  // namespace

extern "C" {

int32_t mcg_abi_version(void) { return MCG_ABI_VERSION; }

int32_t mcg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char *mcg_last_error_string(void) { return mcg::g_last_error.c_str(); }

const char *mcg_status_string(mcg_status s) {
    switch (s) {
        case MCG_OK: return "ok";
        case MCG_ERR_INVALID_ARG: return "invalid argument";
        case MCG_ERR_OOM: return "out of memory";
        case MCG_ERR_CUDA: return "CUDA error";
        case MCG_ERR_NONFINITE: return "non-finite value";
        case MCG_ERR_IO: return "I/O error";
        case MCG_ERR_TIMEOUT: return "device wait timed out";
        case MCG_ERR_STATE: return "invalid state";
        case MCG_ERR_UNSUPPORTED: return "unsupported";
        case MCG_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

mcg_status mcg_params_default(mcg_params *p) {
    return mcg::guarded([&]() -> mcg_status {
        MCG_REQUIRE(p != nullptr, "params is null");
        std::memset(p, 0, sizeof(*p));
        // constants.cuh:8-76
        p->NX = 128; p->NY = 400; p->NZ = 128;
        p->NSTEP = 200000; p->NOUTPUT = 2000; p->NSTATS_START_STEP = 6000; p->write_vti_output = 1;
        p->sponge_cells = 34;
        p->jet_radius = 7.0f; p->jet_velocity = 0.05f;
        p->bubble_radius = 10.0f;
        p->rhor0 = 1.0f; p->rhob0 = 1.0f;
        p->Re = 5000.0f; p->We = 2000.0f;
        p->beta_recolor = 0.80f;
        p->sponge_K = 0.0f;
        p->boundary = MCG_BOUNDARY_JET;
        p->storage = MCG_STORAGE_F32;
        return mcg_params_derive(p);
    });
}

mcg_status mcg_params_derive(mcg_params *p) {
    return mcg::guarded([&]() -> mcg_status {
        MCG_REQUIRE(p != nullptr, "params is null");
        MCG_REQUIRE(p->Re > 0.0f && p->We > 0.0f, "Re and We must be > 0");
        const float cs2 = mcg::kCs2;
        p->jet_x0 = float(p->NX - 1) / 2.0f;  // constants.cuh:33-34
        p->jet_z0 = float(p->NZ - 1) / 2.0f;
        p->bubble_x0 = float(p->NX - 1) / 2.0f;  // constants.cuh:39-41
        p->bubble_y0 = float(p->NY - 1) / 2.0f;
        p->bubble_z0 = float(p->NZ - 1) / 2.0f;
        p->nu = (2.0f * p->jet_radius * p->jet_velocity) / p->Re;  // constants.cuh:60
        p->taur = 0.5f + p->nu / cs2;                              // constants.cuh:62-64
        p->taub = 0.5f + p->nu / cs2;
        p->sigma = (p->rhob0 * p->jet_velocity * p->jet_velocity * 2.0f * p->jet_radius) / p->We;  // constants.cuh:73
        return MCG_OK;
    });
}

mcg_status mcg_params_set_tau(mcg_params *p, float tau) {
    return mcg::guarded([&]() -> mcg_status {
        MCG_REQUIRE(p != nullptr, "params is null");
        MCG_REQUIRE(std::isfinite(tau) && tau > 0.5f, "tau must be > 0.5");
        p->nu = (tau - 0.5f) * mcg::kCs2;
        p->taur = tau;
        p->taub = tau;
        return MCG_OK;
    });
}

mcg_status mcg_create(const mcg_params *p, mcg_handle **out) {
    return mcg::guarded([&]() -> mcg_status {
        MCG_REQUIRE(out != nullptr, "out is null");
        *out = nullptr;
        mcg_status st = validate(p);
        if (st != MCG_OK) return st;
        if (mcg_device_count() <= 0) return fail(MCG_ERR_NO_DEVICE, "no CUDA device is visible");
        mcg_handle *h = new mcg_handle();
        h->p = *p;
        MCG_CUDA(cudaGetDevice(&h->device), "cudaGetDevice");
        mcg::Geometry &g = h->s.g;
        g.NX = p->NX; g.NY = p->NY; g.NZ = p->NZ;
        g.N = uint32_t(size_t(p->NX) * p->NY * p->NZ);
        g.sy = p->NX;
        g.sz = p->NX * p->NY;
        g.boundary = p->boundary;
        g.storage = p->storage;
        g.slots = mcg::kQ;  // one element (both colours) per direction: float2 or half2
        fill_physics(h);
        compute_ncols(h);
        const size_t N = g.N;
        const size_t M = size_t(p->NY) * (p->NX / 2);
        cudaError_t e = cudaSuccess;
        const size_t pb = pop_buffer_bytes(*p);
        if (e == cudaSuccess) e = alloc_zero(&h->s.pops[0], pb);
        if (e == cudaSuccess) e = alloc_zero(&h->s.pops[1], pb);
        if (e == cudaSuccess) e = alloc_zero(&h->s.mom, size_t(mcg::kMomCount) * N * 4);
        if (e == cudaSuccess) e = alloc_zero(&h->s.psi[0], N * 4);
        if (e == cudaSuccess) e = alloc_zero(&h->s.psi[1], N * 4);
        if (e == cudaSuccess) e = alloc_zero(&h->s.radial, 5 * M * 8);
        if (e == cudaSuccess) e = alloc_zero(&h->s.bmom, size_t(2) * p->NZ * mcg::kMomCount * p->NX * 4);
        h->tiling = mcg::fused_tiling(g, kFusedSmemPerBlock);
        if (e == cudaSuccess) e = mcg::fused_configure(h->tiling.smem_bytes);
        if (e == cudaSuccess) e = alloc_zero(&h->s.uy_avg, N * 4);
        h->s.partials_cap = mcg::conservation_blocks(g);
        if (e == cudaSuccess) e = alloc_zero(&h->s.partials, size_t(h->s.partials_cap) * 5 * 8);
        if (e == cudaSuccess) e = alloc_zero(&h->s.flag, sizeof(int) * 4);
        if (e == cudaSuccess) e = alloc_zero(&h->d_scalar, 8 * sizeof(double));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->xfer_start, cudaEventDisableTiming);
        for (int k = 0; k < 16 && e == cudaSuccess; ++k) {
            e = cudaEventCreateWithFlags(&h->xfer_copy[k], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->xfer_kern[k], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            const mcg_status s = cuda_fail(e, "mcg_create allocation");
            release(h);
            delete h;
            return s;
        }
        h->stream = h->own_stream;
        *out = h;
        return MCG_OK;
    });
}

mcg_status mcg_destroy(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (!h) return MCG_OK;
        cudaStreamSynchronize(h->stream);
        release(h);
        delete h;
        return MCG_OK;
    });
}

mcg_status mcg_set_stream(mcg_handle *h, void *stream) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
        return MCG_OK;
    });
}

mcg_status mcg_synchronize(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_CUDA(cudaStreamSynchronize(h->stream), "stream synchronize");
        return check_stage_waits(h);
    });
}

mcg_status mcg_set_stage_wait_limit(mcg_handle *h, int32_t tries) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(tries >= 0, "tries must be >= 0");
        h->tiling.wait_limit = tries;
        return MCG_OK;
    });
}

mcg_status mcg_get_params(const mcg_handle *h, mcg_params *out) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(out != nullptr, "out is null");
        *out = h->p;
        return MCG_OK;
    });
}

mcg_status mcg_device_bytes(const mcg_handle *h, uint64_t *out) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(out != nullptr, "out is null");
        const size_t N = h->s.g.N, M = size_t(h->p.NY) * (h->p.NX / 2);
        *out = 2 * pop_buffer_bytes(h->p) + size_t(mcg::kMomCount) * N * 4 + 2 * N * 4 + 5 * M * 8 + N * 4 +
               size_t(h->s.partials_cap) * 40 + 16 + 64;
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- initial conditions

static mcg_status reset_counters(mcg_handle *h) {
    h->cur = 0;
    h->step = 0;
    h->stats_started = false;
    h->stats_start_step = 0;
    h->stats_samples = 0;
    h->uy_avg_samples = 0;
    h->first_tke = true;
    h->tke_total = h->tke_avg = h->tke_avg_prev = h->tke_delta = h->tke_abs_delta = 0.f;
    const size_t M = size_t(h->p.NY) * (h->p.NX / 2);
    MCG_CUDA(cudaMemsetAsync(h->s.radial, 0, 5 * M * 8, h->stream), "clear radial sums");
    MCG_CUDA(cudaMemsetAsync(h->s.uy_avg, 0, size_t(h->s.g.N) * 4, h->stream), "clear uy average");
    return MCG_OK;
}

static mcg_status init_common(mcg_handle *h, int mode) {
    if (mcg_status s = reset_counters(h)) return s;
    const mcg_params &p = h->p;
    MCG_LAUNCH(h, mcg::launch_init_fields(h->s, mode, p.bubble_red_inside, p.bubble_radius * p.bubble_radius,
                                          p.bubble_x0, p.bubble_y0, p.bubble_z0, h->stream),
               "init fields");
    h->mom_stale = false;
    MCG_LAUNCH(h, mcg::launch_refresh_psi(h->s, h->stream), "init psi");
    MCG_LAUNCH(h, mcg::launch_init_pops(h->s, mode, p.init_noise, h->stream), "init populations");
    return MCG_OK;
}

mcg_status mcg_init_jet(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        return init_common(h, 0);
    });
}

mcg_status mcg_init_bubble(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        return init_common(h, 1);
    });
}

mcg_status mcg_init_equilibrium(mcg_handle *h, const float *rhor, const float *rhob, const float *ux,
                                const float *uy, const float *uz) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(rhor && rhob && ux && uy && uz, "field pointers must not be null");
        if (mcg_status s = reset_counters(h)) return s;
        if (mcg_status s = mcg_set_fields(h, rhor, rhob, ux, uy, uz)) return s;
        MCG_LAUNCH(h, mcg::launch_init_pops(h->s, 3, 0.0f, h->stream), "equilibrium populations");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "init equilibrium");
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- inlet profile

namespace {
// k-th positive zero of J0 (k >= 1): Newton's method on J0 (derivative -J1)
// from McMahon's asymptotic estimate (k - 1/4) pi.
double bessel_j0_zero(int k) {
    double x = (double(k) - 0.25) * M_PI;
    for (int it = 0; it < 60; ++it) {
        const double dx = std::cyl_bessel_j(0.0, x) / -std::cyl_bessel_j(1.0, x);
        x -= dx;
        if (std::fabs(dx) < 1e-15 * x) break;
    }
    return x;
}
}  // namespace

static_assert(mcg::kInletBesselMax == MCG_INLET_BESSEL_MAX, "inlet profile size");

mcg_status mcg_set_inlet_bessel(mcg_handle *h, const float *coeffs, int32_t n) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(n >= 0 && n <= MCG_INLET_BESSEL_MAX, "n must be in [0, MCG_INLET_BESSEL_MAX]");
        MCG_REQUIRE(n == 0 || coeffs != nullptr, "coeffs is null");
        for (int k = 0; k < n; ++k) MCG_REQUIRE(std::isfinite(coeffs[k]), "coefficients must be finite");
        const mcg_params &p = h->p;
        if (n == 0) {  // back to the top-hat
            h->s.inlet_profile = nullptr;
            h->inlet_coeffs.clear();
            return MCG_OK;
        }
        // multiplier m(r) = 1 + sum_k c_k J0(alpha_k r / R) of every column, with r
        // measured from the jet axis like the inlet mask (mathUtilities.cuh:14-21)
        const int NX = p.NX, NZ = p.NZ;
        std::vector<double> alpha(static_cast<size_t>(n));
        for (int k = 0; k < n; ++k) alpha[size_t(k)] = bessel_j0_zero(k + 1);
        std::vector<float> prof(size_t(NX) * NZ);
        const double R = p.jet_radius;
        for (int z = 0; z < NZ; ++z)
            for (int x = 0; x < NX; ++x) {
                const double dx = double(float(x) - p.jet_x0), dz = double(float(z) - p.jet_z0);
                const double r = std::sqrt(dx * dx + dz * dz);
                double m = 1.0;
                for (int k = 0; k < n; ++k) m += double(coeffs[k]) * std::cyl_bessel_j(0.0, alpha[size_t(k)] * r / R);
                prof[size_t(z) * NX + x] = float(m);
            }
        if (!h->d_inlet_profile)
            MCG_CUDA(cudaMalloc(&h->d_inlet_profile, prof.size() * sizeof(float)), "inlet profile allocation");
        MCG_CUDA(cudaMemcpyAsync(h->d_inlet_profile, prof.data(), prof.size() * sizeof(float), cudaMemcpyHostToDevice,
                                 h->stream),
                 "upload inlet profile");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "inlet profile");
        h->s.inlet_profile = h->d_inlet_profile;
        h->inlet_coeffs.assign(coeffs, coeffs + n);
        return MCG_OK;
    });
}

mcg_status mcg_get_tiling(const mcg_handle *h, int32_t *out) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(out != nullptr, "out is null");
        const mcg::FusedTiling &t = h->tiling;
        const int32_t march = t.bulk ? 2 : t.pipe;
        const int32_t v[MCG_TILING_FIELDS] = {t.ty, t.lz, t.tpr, t.ny_tiles, t.nz_chunks, t.smem_bytes, march, t.fixed_nx};
        for (int k = 0; k < MCG_TILING_FIELDS; ++k) out[k] = v[k];
        return MCG_OK;
    });
}

mcg_status mcg_get_inlet_profile(mcg_handle *h, float *profile) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(profile != nullptr, "profile is null");
        const size_t n = size_t(h->p.NX) * h->p.NZ;
        if (!h->s.inlet_profile) {
            for (size_t i = 0; i < n; ++i) profile[i] = 1.0f;
            return MCG_OK;
        }
        MCG_CUDA(cudaMemcpyAsync(profile, h->s.inlet_profile, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
                 "download inlet profile");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "inlet profile");
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- state transfer

namespace {
// Host state transfer in z-chunks of the reference layout, staged in the spare
// population buffer so that no device memory is allocated: the F32 spare
// buffer (2*27*N floats) holds every chunk at once, the F16 one (27*N words)
// half of them, reused in turn.  The host copies of chunk k+1 (copy stream)
// overlap the scatter or gather kernel of chunk k (solver stream).
struct XferPlan {
    int zc = 0, nchunks = 0, slots = 0;
    size_t pitch = 0;        // elements of one direction row of a chunk
    size_t slot_floats = 0;  // 2 colours x 27 rows
};

XferPlan xfer_plan(const mcg_handle *h) {
    const mcg::Geometry &g = h->s.g;
    XferPlan x;
    x.zc = std::max(1, (g.NZ + 7) / 8);
    x.nchunks = (g.NZ + x.zc - 1) / x.zc;
    x.pitch = size_t(x.zc) * size_t(g.sz);
    x.slot_floats = 2 * size_t(mcg::kQ) * x.pitch;
    const size_t cap = pop_buffer_bytes(h->p) / 4;
    x.slots = int(std::min<size_t>(size_t(x.nchunks), cap / x.slot_floats));
    return x;
}
}  // namespace

mcg_status mcg_set_populations(mcg_handle *h, const float *fr, const float *fb) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(fr && fb, "population pointers must not be null");
        if (mcg_status s = mcg::async_flush(h)) return s;
        const mcg::Geometry &g = h->s.g;
        const XferPlan x = xfer_plan(h);
        if (x.slots < 1 || x.nchunks > 16) return fail(MCG_ERR_STATE, "transfer plan does not fit the spare buffer");
        const size_t N = g.N;
        float *stage0 = static_cast<float *>(h->s.pops[1]);
        const float *src[2] = {fr, fb};
        // the spare buffer may still be read by queued work of the solver stream
        MCG_CUDA(cudaEventRecord(h->xfer_start, h->stream), "event record");
        MCG_CUDA(cudaStreamWaitEvent(h->copy_stream, h->xfer_start, 0), "stream wait");
        for (int k = 0; k < x.nchunks; ++k) {
            const int z0 = k * x.zc, nz = std::min(x.zc, g.NZ - z0);
            float *stage = stage0 + size_t(k % x.slots) * x.slot_floats;
            if (k >= x.slots) MCG_CUDA(cudaStreamWaitEvent(h->copy_stream, h->xfer_kern[k - x.slots], 0), "stream wait");
            for (int c = 0; c < 2; ++c)
                MCG_CUDA(cudaMemcpy2DAsync(stage + size_t(c) * mcg::kQ * x.pitch, x.pitch * 4, src[c] + size_t(z0) * g.sz,
                                           N * 4, size_t(nz) * g.sz * 4, mcg::kQ, cudaMemcpyHostToDevice,
                                           h->copy_stream),
                         "upload populations");
            MCG_CUDA(cudaEventRecord(h->xfer_copy[k], h->copy_stream), "event record");
            MCG_CUDA(cudaStreamWaitEvent(h->stream, h->xfer_copy[k], 0), "stream wait");
            MCG_LAUNCH(h, mcg::launch_scatter_chunk(h->s, 0, stage, x.pitch, z0, nz, h->stream), "scatter populations");
            MCG_CUDA(cudaEventRecord(h->xfer_kern[k], h->stream), "event record");
        }
        // both buffers carry the same ghost-plane slots (the ones no step rewrites)
        MCG_CUDA(cudaMemcpyAsync(h->s.pops[1], h->s.pops[0], pop_buffer_bytes(h->p), cudaMemcpyDeviceToDevice, h->stream),
                 "copy populations");
        h->cur = 0;
        MCG_CUDA(cudaStreamSynchronize(h->stream), "set populations");
        return MCG_OK;
    });
}

mcg_status mcg_get_populations(mcg_handle *h, float *fr, float *fb) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(fr && fb, "population pointers must not be null");
        if (mcg_status s = mcg::async_flush(h)) return s;
        // the spare buffer holds the last step's input state, from which the
        // moment planes the fields report are formed: form them before staging
        if (mcg_status s = ensure_moments(h)) return s;
        const mcg::Geometry &g = h->s.g;
        const XferPlan x = xfer_plan(h);
        if (x.slots < 1 || x.nchunks > 16) return fail(MCG_ERR_STATE, "transfer plan does not fit the spare buffer");
        const size_t N = g.N;
        const int rd = h->cur;
        float *stage0 = static_cast<float *>(h->s.pops[rd ^ 1]);
        float *dst[2] = {fr, fb};
        for (int k = 0; k < x.nchunks; ++k) {
            const int z0 = k * x.zc, nz = std::min(x.zc, g.NZ - z0);
            float *stage = stage0 + size_t(k % x.slots) * x.slot_floats;
            if (k >= x.slots) MCG_CUDA(cudaStreamWaitEvent(h->stream, h->xfer_copy[k - x.slots], 0), "stream wait");
            MCG_LAUNCH(h, mcg::launch_gather_chunk(h->s, rd, stage, x.pitch, z0, nz, h->stream), "gather populations");
            MCG_CUDA(cudaEventRecord(h->xfer_kern[k], h->stream), "event record");
            MCG_CUDA(cudaStreamWaitEvent(h->copy_stream, h->xfer_kern[k], 0), "stream wait");
            for (int c = 0; c < 2; ++c)
                MCG_CUDA(cudaMemcpy2DAsync(dst[c] + size_t(z0) * g.sz, N * 4, stage + size_t(c) * mcg::kQ * x.pitch,
                                           x.pitch * 4, size_t(nz) * g.sz * 4, mcg::kQ, cudaMemcpyDeviceToHost,
                                           h->copy_stream),
                         "download populations");
            MCG_CUDA(cudaEventRecord(h->xfer_copy[k], h->copy_stream), "event record");
        }
        // the spare buffer again holds the ghost-plane slots of the current one
        MCG_CUDA(cudaStreamWaitEvent(h->stream, h->xfer_copy[x.nchunks - 1], 0), "stream wait");
        MCG_CUDA(cudaMemcpyAsync(h->s.pops[rd ^ 1], h->s.pops[rd], pop_buffer_bytes(h->p), cudaMemcpyDeviceToDevice,
                                 h->stream),
                 "restore spare buffer");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "get populations");
        return MCG_OK;
    });
}

mcg_status mcg_set_fields(mcg_handle *h, const float *rhor, const float *rhob, const float *ux, const float *uy,
                          const float *uz) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        const size_t N = h->s.g.N;
        const float *src[5] = {rhor, rhob, ux, uy, uz};
        for (int k = 0; k < 5; ++k)
            if (src[k])
                MCG_CUDA(cudaMemcpyAsync(h->s.mom + size_t(k) * N, src[k], N * 4, cudaMemcpyHostToDevice, h->stream),
                         "upload field");
        MCG_LAUNCH(h, mcg::launch_refresh_psi(h->s, h->stream), "refresh psi");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "set fields");
        h->mom_stale = false;
        return MCG_OK;
    });
}

mcg_status mcg_get_fields(mcg_handle *h, float *rhor, float *rhob, float *ux, float *uy, float *uz) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = ensure_moments(h)) return s;
        const size_t N = h->s.g.N;
        float *dst[5] = {rhor, rhob, ux, uy, uz};
        for (int k = 0; k < 5; ++k)
            if (dst[k])
                MCG_CUDA(cudaMemcpyAsync(dst[k], h->s.mom + size_t(k) * N, N * 4, cudaMemcpyDeviceToHost, h->stream),
                         "download field");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "get fields");
        return MCG_OK;
    });
}

mcg_status mcg_get_stress(mcg_handle *h, float *pi6) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(pi6 != nullptr, "pi6 is null");
        if (mcg_status s = ensure_moments(h)) return s;
        const size_t N = h->s.g.N;
        MCG_CUDA(cudaMemcpyAsync(pi6, h->s.mom + size_t(mcg::kMomPXX) * N, 6 * N * 4, cudaMemcpyDeviceToHost, h->stream),
                 "download stress");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "get stress");
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- launch sequence

mcg_status mcg_macros(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_LAUNCH(h, mcg::launch_moments(h->s, h->cur, h->step, false, h->stream), "moments kernel");
        h->mom_stale = false;
        return MCG_OK;
    });
}

mcg_status mcg_accumulate_radial_moments(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (!h->stats_started) {
            h->stats_started = true;
            h->stats_start_step = uint32_t(h->step);
            h->stats_samples = 0;
        }
        MCG_LAUNCH(h, mcg::launch_accumulate_radial(h->s, h->stream), "radial statistics kernel");
        ++h->stats_samples;
        return MCG_OK;
    });
}

mcg_status mcg_collistream(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_LAUNCH(h, mcg::launch_collide(h->s, h->cur, h->step, h->stream), "collision kernel");
        h->cur ^= 1;
        ++h->step;
        return MCG_OK;
    });
}

mcg_status mcg_inlet_bc(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (h->step == 0) return fail(MCG_ERR_STATE, "mcg_inlet_bc needs a preceding mcg_collistream");
        MCG_LAUNCH(h, mcg::launch_boundary(h->s, h->cur, h->step - 1, 0, false, h->stream), "inlet kernel");
        return MCG_OK;
    });
}

mcg_status mcg_neumann_bc(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (h->step == 0) return fail(MCG_ERR_STATE, "mcg_neumann_bc needs a preceding mcg_collistream");
        MCG_LAUNCH(h, mcg::launch_boundary(h->s, h->cur, h->step - 1, 1, false, h->stream), "outlet kernel");
        return MCG_OK;
    });
}

mcg_status mcg_step(mcg_handle *h, int32_t nsteps) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(nsteps >= 0, "nsteps must be >= 0");
        return run_steps(h, nsteps);
    });
}

mcg_status mcg_step_timed(mcg_handle *h, int32_t nsteps, float *ms) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(nsteps >= 0 && ms != nullptr, "nsteps must be >= 0 and ms non-null");
        MCG_CUDA(cudaEventRecord(h->ev0, h->stream), "event record");
        if (mcg_status s = run_steps(h, nsteps)) return s;
        MCG_CUDA(cudaEventRecord(h->ev1, h->stream), "event record");
        MCG_CUDA(cudaEventSynchronize(h->ev1), "event synchronize");
        MCG_CUDA(cudaEventElapsedTime(ms, h->ev0, h->ev1), "event elapsed");
        return check_stage_waits(h);
    });
}

mcg_status mcg_step_profiled(mcg_handle *h, int32_t nsteps, float *ms_total, float *ms_kernels) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(nsteps >= 0 && ms_total != nullptr && ms_kernels != nullptr, "bad arguments");
        const bool jet = h->p.boundary == MCG_BOUNDARY_JET;
        const size_t need = size_t(nsteps) * 2 + 1;
        while (h->prof_events.size() < need) {
            cudaEvent_t e;
            MCG_CUDA(cudaEventCreate(&e), "event create");
            h->prof_events.push_back(e);
        }
        // kind of the launch that ends at event k+1: 0 fused step, 1 boundary
        std::vector<int> kind;
        kind.reserve(need);
        size_t ev = 0;
        MCG_CUDA(cudaEventRecord(h->prof_events[ev++], h->stream), "event record");
        for (int32_t n = 0; n < nsteps; ++n) {
            const bool stats = stats_for_step(h);
            MCG_LAUNCH(h, mcg::launch_fused(h->s, h->tiling, h->cur, h->step, stats, h->stream), "fused step kernel");
            if (stats) ++h->stats_samples;
            MCG_CUDA(cudaEventRecord(h->prof_events[ev++], h->stream), "event record");
            kind.push_back(0);
            if (jet && !h->tiling.boundary) {
                MCG_LAUNCH(h, mcg::launch_boundary(h->s, h->cur ^ 1, h->step, -1, true, h->stream), "boundary kernel");
                MCG_CUDA(cudaEventRecord(h->prof_events[ev++], h->stream), "event record");
                kind.push_back(1);
            }
            h->cur ^= 1;
            ++h->step;
            h->mom_stale = true;
        }
        MCG_CUDA(cudaEventSynchronize(h->prof_events[ev - 1]), "event synchronize");
        ms_kernels[0] = ms_kernels[1] = ms_kernels[2] = 0.0f;
        for (size_t k = 0; k + 1 < ev; ++k) {
            float ms = 0.0f;
            MCG_CUDA(cudaEventElapsedTime(&ms, h->prof_events[k], h->prof_events[k + 1]), "event elapsed");
            ms_kernels[kind[k]] += ms;
        }
        MCG_CUDA(cudaEventElapsedTime(ms_total, h->prof_events[0], h->prof_events[ev - 1]), "event elapsed");
        return check_stage_waits(h);
    });
}

mcg_status mcg_get_step(const mcg_handle *h, int64_t *step) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(step != nullptr, "step is null");
        *step = h->step;
        return MCG_OK;
    });
}

mcg_status mcg_launch_count(const mcg_handle *h, uint64_t *count) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(count != nullptr, "count is null");
        *count = h->launches;
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- statistics

mcg_status mcg_set_radial_statistics(mcg_handle *h, int32_t mode) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(mode >= -1 && mode <= 1, "mode must be -1, 0 or 1");
        h->stats_mode = mode;
        return MCG_OK;
    });
}

mcg_status mcg_get_radial(mcg_handle *h, double *sum_uy, double *sum_uy2, double *sum_ur, double *sum_ur2,
                          double *sum_uruy, uint64_t *count) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        const size_t M = size_t(h->p.NY) * (h->p.NX / 2);
        double *dst[5] = {sum_uy, sum_uy2, sum_ur, sum_ur2, sum_uruy};
        for (int k = 0; k < 5; ++k)
            if (dst[k])
                MCG_CUDA(cudaMemcpyAsync(dst[k], h->s.radial + size_t(k) * M, M * 8, cudaMemcpyDeviceToHost, h->stream),
                         "download radial sums");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "get radial");
        if (count) mcg::radial_counts(h, count);
        return MCG_OK;
    });
}

mcg_status mcg_get_radial_state(const mcg_handle *h, int32_t *started, uint32_t *start_step, uint32_t *samples) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (started) *started = h->stats_started ? 1 : 0;
        if (start_step) *start_step = h->stats_start_step;
        if (samples) *samples = h->stats_samples;
        return MCG_OK;
    });
}

mcg_status mcg_compute_tke(mcg_handle *h, int32_t step, float *tke_total, float *tke_avg) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = mcg::async_flush(h)) return s;  // the worker owns the tke state while outputs are pending
        if (mcg_status s = ensure_moments(h)) return s;
        MCG_LAUNCH(h, mcg::launch_tke(h->s, h->d_scalar, h->stream), "tke kernel");
        double tot = 0;
        MCG_CUDA(cudaMemcpyAsync(&tot, h->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "download tke");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "tke");
        mcg::tke_update(h, step, tot);  // kernels.cu:154-166: running average over output samples, float
        if (tke_total) *tke_total = h->tke_total;
        if (tke_avg) *tke_avg = h->tke_avg;
        return MCG_OK;
    });
}

mcg_status mcg_update_uy_average(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = ensure_moments(h)) return s;
        MCG_LAUNCH(h, mcg::launch_uy_average(h->s, h->uy_avg_samples, h->stream), "uy average kernel");
        ++h->uy_avg_samples;
        return MCG_OK;
    });
}

mcg_status mcg_get_uy_average(mcg_handle *h, float *uy_avg, uint32_t *samples) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (uy_avg)
            MCG_CUDA(cudaMemcpyAsync(uy_avg, h->s.uy_avg, size_t(h->s.g.N) * 4, cudaMemcpyDeviceToHost, h->stream),
                     "download uy average");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "get uy average");
        if (samples) *samples = h->uy_avg_samples;
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- diagnostics

mcg_status mcg_conservation_sums(mcg_handle *h, double out[5]) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(out != nullptr, "out is null");
        MCG_LAUNCH(h, mcg::launch_conservation(h->s, h->cur, h->s.partials, h->d_scalar, h->stream),
                   "conservation kernels");
        ++h->launches;  // two kernels
        MCG_CUDA(cudaMemcpyAsync(out, h->d_scalar, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                 "download sums");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "conservation sums");
        return MCG_OK;
    });
}

mcg_status mcg_check_finite(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = ensure_moments(h)) return s;
        MCG_LAUNCH(h, mcg::launch_check_finite(h->s, h->cur, h->s.flag, h->stream), "finite check kernel");
        int flag = 0;
        MCG_CUDA(cudaMemcpyAsync(&flag, h->s.flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "download flag");
        MCG_CUDA(cudaStreamSynchronize(h->stream), "finite check");
        if (flag) return fail(MCG_ERR_NONFINITE, "non-finite value in fields or populations");
        return MCG_OK;
    });
}

// ---------------------------------------------------------------- output

mcg_status mcg_output_open(mcg_handle *h, const char *root_dir) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(root_dir != nullptr, "root_dir is null");
        return mcg::io_open(h, root_dir);
    });
}

mcg_status mcg_output_close(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = mcg::async_flush(h)) return s;
        return mcg::io_close(h);
    });
}

mcg_status mcg_output_step(mcg_handle *h, int32_t step) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (h->case_dir.empty()) return fail(MCG_ERR_STATE, "mcg_output_open has not been called");
        if (mcg_status s = mcg::async_flush(h)) return s;
        // main.cu:73-103
        if (mcg_status s = mcg_compute_tke(h, step, nullptr, nullptr)) return s;
        if (mcg_status s = mcg::io_write_tke_sample(h, step)) return s;
        if (h->stats_started && h->stats_samples > 0)
            if (mcg_status s = mcg::io_write_radial(h)) return s;
        if (h->p.write_vti_output) {
            char name[64];
            std::snprintf(name, sizeof(name), "/lbm_%08d.vti", int(step));
            if (mcg_status s = mcg::io_write_vti(h, h->vti_dir + name)) return s;
        }
        return MCG_OK;
    });
}

mcg_status mcg_output_step_async(mcg_handle *h, int32_t step) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (h->case_dir.empty()) return fail(MCG_ERR_STATE, "mcg_output_open has not been called");
        if (mcg_status s = ensure_moments(h)) return s;
        return mcg::async_enqueue(h, step);
    });
}

mcg_status mcg_output_flush(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        return mcg::async_flush(h);
    });
}

mcg_status mcg_write_radial_outputs(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = mcg::async_flush(h)) return s;
        if (h->case_dir.empty()) return fail(MCG_ERR_STATE, "mcg_output_open has not been called");
        return mcg::io_write_radial(h);
    });
}

mcg_status mcg_write_vti(mcg_handle *h, const char *path) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = mcg::async_flush(h)) return s;
        MCG_REQUIRE(path != nullptr, "path is null");
        if (mcg_status s = ensure_moments(h)) return s;
        return mcg::io_write_vti(h, path);
    });
}

mcg_status mcg_write_uy_average(mcg_handle *h) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        if (mcg_status s = mcg::async_flush(h)) return s;
        if (h->case_dir.empty()) return fail(MCG_ERR_STATE, "mcg_output_open has not been called");
        return mcg::io_write_uy_average(h);
    });
}

mcg_status mcg_output_dirs(const mcg_handle *h, char *case_dir, char *mean_dir, char *vti_dir, size_t cap) {
    return mcg::guarded([&]() -> mcg_status {
        if (mcg_status s = check_handle(h)) return s;
        MCG_REQUIRE(cap > 0, "cap must be > 0");
        const std::string *src[3] = {&h->case_dir, &h->mean_dir, &h->vti_dir};
        char *dst[3] = {case_dir, mean_dir, vti_dir};
        for (int k = 0; k < 3; ++k) {
            if (!dst[k]) continue;
            if (src[k]->size() + 1 > cap) return fail(MCG_ERR_INVALID_ARG, "buffer too small for path");
            std::memcpy(dst[k], src[k]->c_str(), src[k]->size() + 1);
        }
        return MCG_OK;
    });
}

mcg_status mcg_write_constants_header(const mcg_params *p, const char *path) {
    return mcg::guarded([&]() -> mcg_status {
        MCG_REQUIRE(p != nullptr && path != nullptr, "null argument");
        FILE *f = std::fopen(path, "w");
        if (!f) return fail(MCG_ERR_IO, std::string("cannot open ") + path);
        // Same names and `name = static_cast<T>(value)` text form as constants.cuh:1-78,
        // values written so that float32 round-trips.
        std::fprintf(f, "#ifndef CONSTANTS_CUH\n#define CONSTANTS_CUH\n\n#include <array>\n#include \"utilities/types.cuh\"\n\n");
        std::fprintf(f, "// Steps\ninline constexpr int NSTEP = %d;\ninline constexpr int NOUTPUT = %d;\n", p->NSTEP, p->NOUTPUT);
        std::fprintf(f, "inline constexpr int NSTATS_START_STEP = %d;\n", p->NSTATS_START_STEP);
        std::fprintf(f, "inline constexpr bool write_vti_output = %s;\n\n", p->write_vti_output ? "true" : "false");
        std::fprintf(f, "// Grid\ninline constexpr label_t NX = static_cast<label_t>(%d);\n", p->NX);
        std::fprintf(f, "inline constexpr label_t NZ = static_cast<label_t>(%d);\n", p->NZ);
        std::fprintf(f, "inline constexpr label_t NY = static_cast<label_t>(%d);\n", p->NY);
        std::fprintf(f, "inline constexpr label_t sponge_cells = static_cast<label_t>(%d);\n\n", p->sponge_cells);
        std::fprintf(f, "inline constexpr label_t Ncells = NX * NY * NZ;\n");
        std::fprintf(f, "inline constexpr label_t NR_BINS = NX / static_cast<label_t>(2);\n");
        std::fprintf(f, "inline constexpr label_t NradialProfileCells = NY * NR_BINS;\n\n");
        std::fprintf(f, "inline constexpr label_t Q = 27;\n\n");
        std::fprintf(f, "inline constexpr std::size_t bytesCell = std::size_t(Ncells) * sizeof(real_t);\n");
        std::fprintf(f, "inline constexpr std::size_t fSize = std::size_t(Ncells) * (std::size_t)Q;\n");
        std::fprintf(f, "inline constexpr std::size_t bytesF = fSize * sizeof(pop_t);\n\n");
        std::fprintf(f, "// Jet parameters\n");
        std::fprintf(f, "inline constexpr real_t jet_radius = static_cast<real_t>(%.9g);\n", double(p->jet_radius));
        std::fprintf(f, "inline constexpr real_t jet_x0 = static_cast<real_t>(%.9g);\n", double(p->jet_x0));
        std::fprintf(f, "inline constexpr real_t jet_z0 = static_cast<real_t>(%.9g);\n", double(p->jet_z0));
        std::fprintf(f, "inline constexpr real_t jet_velocity = static_cast<real_t>(%.9g);\n\n", double(p->jet_velocity));
        std::fprintf(f, "// Bubble parameters\n");
        std::fprintf(f, "inline constexpr real_t bubble_radius = static_cast<real_t>(%.9g);\n", double(p->bubble_radius));
        std::fprintf(f, "inline constexpr real_t bubble_x0 = static_cast<real_t>(%.9g);\n", double(p->bubble_x0));
        std::fprintf(f, "inline constexpr real_t bubble_y0 = static_cast<real_t>(%.9g);\n", double(p->bubble_y0));
        std::fprintf(f, "inline constexpr real_t bubble_z0 = static_cast<real_t>(%.9g);\n", double(p->bubble_z0));
        std::fprintf(f, "inline constexpr real_t pi = static_cast<real_t>(3.141592653589793);\n\n");
        std::fprintf(f, "// Some useful constants\ninline constexpr real_t cs2 = static_cast<real_t>(1.0 / 3.0);\n");
        std::fprintf(f, "inline constexpr real_t cs4 = cs2 * cs2;\ninline constexpr real_t cs6 = cs4 * cs2;\n\n");
        std::fprintf(f, "inline constexpr real_t inv_cs2 = static_cast<real_t>(1) / cs2;\n");
        std::fprintf(f, "inline constexpr real_t inv_2cs2 = static_cast<real_t>(1) / (static_cast<real_t>(2) * cs2);\n");
        std::fprintf(f, "inline constexpr real_t inv_2cs4 = static_cast<real_t>(1) / (static_cast<real_t>(2) * cs4);\n");
        std::fprintf(f, "inline constexpr real_t inv_6cs6 = static_cast<real_t>(1.0) / (static_cast<real_t>(6.0) * cs6);\n");
        std::fprintf(f, "inline constexpr real_t inv_2cs6 = static_cast<real_t>(1.0) / (static_cast<real_t>(2.0) * cs6);\n\n");
        std::fprintf(f, "// FLuid parameters\n");
        std::fprintf(f, "inline constexpr real_t rhor0 = static_cast<real_t>(%.9g);\n", double(p->rhor0));
        std::fprintf(f, "inline constexpr real_t rhob0 = static_cast<real_t>(%.9g);\n\n", double(p->rhob0));
        std::fprintf(f, "inline constexpr real_t Re = static_cast<real_t>(%.9g);\n", double(p->Re));
        std::fprintf(f, "inline constexpr real_t nu = static_cast<real_t>(%.9g);\n\n", double(p->nu));
        std::fprintf(f, "inline constexpr real_t taur = static_cast<real_t>(%.9g);\n\n", double(p->taur));
        std::fprintf(f, "inline constexpr real_t taub = static_cast<real_t>(%.9g);\n\n", double(p->taub));
        std::fprintf(f, "inline constexpr real_t omegar = static_cast<real_t>(1) / taur;\n");
        std::fprintf(f, "inline constexpr real_t omegab = static_cast<real_t>(1) / taub;\n\n");
        std::fprintf(f, "// Weber number\ninline constexpr real_t We = static_cast<real_t>(%.9g);\n\n", double(p->We));
        std::fprintf(f, "inline constexpr real_t sigma = static_cast<real_t>(%.9g);\n", double(p->sigma));
        std::fprintf(f, "inline constexpr real_t beta_recolor = static_cast<real_t>(%.9g);\n\n", double(p->beta_recolor));
        std::fprintf(f, "inline constexpr real_t sigma_over_4cs4 = sigma / (static_cast<real_t>(4) * cs4);\n\n#endif\n");
        const bool ok = std::ferror(f) == 0;
        if (std::fclose(f) != 0 || !ok) return fail(MCG_ERR_IO, std::string("short write to ") + path);
        return MCG_OK;
    });
}

}  // extern "C"
