// mcg_jet.cpp - host driver: the reference's main.cu:17-120 on top of the C ABI.
//
// Runs the round jet with the constants.cuh defaults (or overrides given as
// `--NAME value`, names as in constants.cuh), writes the same files under
// ./JET_VTK/Re<Re>_We<We>/ (or --out DIR) and prints the same MLUPS and tke
// lines.  Unlike the reference it does not exit on the first CUDA error
// without a message: every failure prints mcg_last_error_string().
// `--async_output 1` writes the output steps through mcg_output_step_async:
// the same files, written by a worker thread while the steps continue.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/mcg.h"

namespace {

bool check(mcg_status s, const char *what) {
    if (s == MCG_OK) return true;
    std::fprintf(stderr, "%s failed: %s (%s)\n", what, mcg_status_string(s), mcg_last_error_string());
    return false;
}

bool set_param(mcg_params &p, const std::string &k, const char *v) {
    struct I { const char *n; int32_t *p; } ints[] = {
        {"NX", &p.NX}, {"NY", &p.NY}, {"NZ", &p.NZ}, {"NSTEP", &p.NSTEP}, {"NOUTPUT", &p.NOUTPUT},
        {"NSTATS_START_STEP", &p.NSTATS_START_STEP}, {"write_vti_output", &p.write_vti_output},
        {"sponge_cells", &p.sponge_cells}, {"storage", &p.storage}, {"boundary", &p.boundary}};
    struct F { const char *n; float *p; } flts[] = {
        {"jet_radius", &p.jet_radius}, {"jet_velocity", &p.jet_velocity}, {"bubble_radius", &p.bubble_radius},
        {"rhor0", &p.rhor0}, {"rhob0", &p.rhob0}, {"Re", &p.Re}, {"We", &p.We},
        {"beta_recolor", &p.beta_recolor}, {"inlet_noise", &p.inlet_noise}, {"init_noise", &p.init_noise}};
    for (auto &e : ints)
        if (k == e.n) { *e.p = std::atoi(v); return true; }
    for (auto &e : flts)
        if (k == e.n) { *e.p = float(std::atof(v)); return true; }
    if (k == "seed") { p.seed = std::strtoull(v, nullptr, 10); return true; }
    return false;
}

}  // namespace

int main(int argc, char **argv) {
    mcg_params p;
    mcg_params_default(&p);
    std::string out = ".";
    bool async_output = false;
    for (int a = 1; a + 1 < argc; a += 2) {
        const std::string k = argv[a];
        if (k.rfind("--", 0) != 0) { std::fprintf(stderr, "bad argument %s\n", argv[a]); return 2; }
        if (k == "--out") { out = argv[a + 1]; continue; }
        if (k == "--async_output") { async_output = std::atoi(argv[a + 1]) != 0; continue; }
        if (!set_param(p, k.substr(2), argv[a + 1])) { std::fprintf(stderr, "unknown parameter %s\n", argv[a]); return 2; }
    }
    if (!check(mcg_params_derive(&p), "params")) return 1;

    mcg_handle *h = nullptr;
    if (!check(mcg_create(&p, &h), "mcg_create")) return 1;
    if (!check(mcg_output_open(h, out.c_str()), "output")) return 1;
    if (p.NSTEP <= p.NSTATS_START_STEP)
        std::printf("Warning: NSTEP (%d) <= NSTATS_START_STEP (%d), so radial statistics will not start in this run.\n",
                    p.NSTEP, p.NSTATS_START_STEP);
    if (!check(mcg_init_jet(h), "init")) return 1;

    const double cells = double(p.NX) * p.NY * p.NZ;
    double total_ms = 0, window_ms = 0;
    int step = 0;
    while (step < p.NSTEP) {
        const int next_out = (step % p.NOUTPUT == 0) ? step : (step / p.NOUTPUT + 1) * p.NOUTPUT;
        const int next_win = (step / 100) * 100 + 99;
        int end = next_out < next_win ? next_out : next_win;
        if (end > p.NSTEP - 1) end = p.NSTEP - 1;
        float ms = 0;
        if (!check(mcg_step_timed(h, end - step + 1, &ms), "step")) return 1;
        window_ms += ms;
        step = end + 1;
        if (step % 100 == 0) {  // utilities/countmlups.cuh:20-64
            total_ms += window_ms;
            std::printf("step %d/%d | dt_window = %.3f ms | MLUPS = %.3f | MLUPS(avg) = %.3f\n", step, p.NSTEP,
                        window_ms, 100.0 * cells / (window_ms * 1e3), double(step) * cells / (total_ms * 1e3));
            window_ms = 0;
        }
        if (end % p.NOUTPUT == 0) {
            const mcg_status s = async_output ? mcg_output_step_async(h, end) : mcg_output_step(h, end);
            if (!check(s, "output")) return 1;
        }
    }
    if (!check(mcg_output_flush(h), "output")) return 1;
    if (!check(mcg_write_radial_outputs(h), "radial output")) return 1;
    mcg_destroy(h);
    return 0;
}
