// ref_dump.cu - TEST INFRASTRUCTURE ONLY.
//
// Driver for the reference's own CUDA build.  It calls the reference's public
// launch API exactly as main.cu:52-104 does (launch_Macros, then
// launch_accumulate_radial_moments when statistics run, launch_collistream,
// launch_inlet_bc, launch_neumann_bc), on the reference's LbmDevice memory
// (memory.cuh:58-97), compiled from the unmodified sources with a case header
// pre-included (oracle/ref_constants.py, oracle/build_ref.sh).
//
//   ref_dump run  <jet|bubble> <steps> <stats_from> <out_dir> [<state_dir>]
//       runs <steps> steps (radial statistics for step >= stats_from) from the
//       reference's initial condition, or from fr.bin/fb.bin/fields.bin in
//       <state_dir>, and writes fr.bin fb.bin fields.bin pi.bin radial.bin
//       count.bin tke.txt into <out_dir>.
//   ref_dump time <jet|bubble> <warmup> <steps> <stats 0|1>
//       times <steps> steps with CUDA events on the default stream and prints
//       one JSON line {"mlups":..,"ms_per_step":..}.
//   ref_dump outputs <out_dir>
//       the jet main loop of main.cu:17-120 for the compiled case (NSTEP,
//       NOUTPUT, NSTATS_START_STEP of the case header), in <out_dir> as the
//       working directory: the reference's own writers make the JET_VTK tree
//       (meanF/meanFieldsRT.cuh:93-381, io/save_data.cuh:137-215).
//   ref_dump vti <fields.bin> <out.vti>
//       write_vti (io/save_data.cuh:137-200) of the five float32 fields in
//       <fields.bin> (rhor, rhob, ux, uy, uz, Ncells each); host only.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <unistd.h>

#include "memory.cuh"
#include "launch.cuh"
#include "meanF/memoryMeanFields.cuh"
#include "meanF/meanFieldsRT.cuh"
#include "io/save_data.cuh"
#include "utilities/cudaConfig.cuh"

namespace {

bool read_file(const std::string &path, void *dst, size_t bytes) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t n = std::fread(dst, 1, bytes, f);
    std::fclose(f);
    return n == bytes;
}

bool write_file(const std::string &path, const void *src, size_t bytes) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t n = std::fwrite(src, 1, bytes, f);
    std::fclose(f);
    return n == bytes;
}

void one_step(const CudaConfig &cfg, const LbmDevice &d, MeanFieldsDevice &mf, bool jet, bool stats) {
    launch_Macros(cfg, d);
    if (stats) launch_accumulate_radial_moments(cfg, d, mf);
    launch_collistream(cfg, d);
    if (jet) {
        launch_inlet_bc(cfg, d);
        launch_neumann_bc(cfg, d);
    }
}

void init_case(const CudaConfig &cfg, const LbmDevice &d, bool jet) {
    if (jet) {
        launch_jetDensity(cfg, d);
        launch_Injet(cfg, d);
    } else {
        launch_bubble(cfg, d);
    }
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_dump run|time ...\n");
        return 2;
    }
    const std::string cmd = argv[1];
    if (cmd == "vti") {
        // host only: the reference's VTI writer on given fields
        if (argc < 4) return 2;
        const size_t n = size_t(Ncells);
        std::vector<float> fields(5 * n);
        if (!read_file(argv[2], fields.data(), fields.size() * 4)) {
            std::fprintf(stderr, "cannot read %s\n", argv[2]);
            return 3;
        }
        const float *f = fields.data();
        write_vti(argv[3], f, f + n, f + 2 * n, f + 3 * n, f + 4 * n, true);
        return 0;
    }
    if (cmd == "outputs") {
        // main.cu:17-120 with the jet initial condition, in <out_dir>
        if (argc < 3) return 2;
        if (chdir(argv[2]) != 0) {
            std::fprintf(stderr, "cannot enter %s\n", argv[2]);
            return 3;
        }
        MeanFieldsRuntime mf{};
        if (!initialize_mean_fields_runtime(0, mf)) return 4;
        const CudaConfig cfg = make_cudaConfig();
        LbmDevice d = allocate_device_memory();
        LbmHost h = allocate_host_memory();
        launch_jetDensity(cfg, d);
        launch_Injet(cfg, d);
        CUDA_CHECK(cudaDeviceSynchronize());
        for (int step = 0; step < NSTEP; ++step) {
            launch_Macros(cfg, d);
            update_radial_statistics_start(mf, step);
            if (mf.state.start_uy_average) {
                launch_accumulate_radial_moments(cfg, d, mf.device);
                ++mf.state.uy_avg_samples;
            }
            launch_collistream(cfg, d);
            launch_inlet_bc(cfg, d);
            launch_neumann_bc(cfg, d);
            if (step % NOUTPUT == 0) {
                CUDA_CHECK(cudaMemset(mf.device.tke_total, 0, sizeof(real_t)));
                launch_compute_total_tke(cfg, d, mf.device.tke_total);
                launch_update_tke_average(mf.device.tke_avg, mf.device.tke_total, step, 0);
                CUDA_CHECK(cudaDeviceSynchronize());
                CUDA_CHECK(cudaMemcpy(&mf.host.tke_total, mf.device.tke_total, sizeof(real_t), cudaMemcpyDeviceToHost));
                CUDA_CHECK(cudaMemcpy(&mf.host.tke_avg, mf.device.tke_avg, sizeof(real_t), cudaMemcpyDeviceToHost));
                process_tke_sample(mf, step);
                if (mf.state.start_uy_average && mf.state.uy_avg_samples > 0) write_radial_profile_outputs(mf);
                if constexpr (write_vti_output) write_vti_step_device(step, d, h);
            }
        }
        CUDA_CHECK(cudaDeviceSynchronize());
        write_radial_profile_outputs(mf);
        free_mean_fields_runtime(mf);
        free_device_memory(d);
        free_host_memory(h);
        return 0;
    }
    CUDA_CHECK(cudaSetDevice(0));
    const CudaConfig cfg = make_cudaConfig();
    LbmDevice d = allocate_device_memory();
    MeanFieldsDevice mf = allocate_mean_fields_device();
    const size_t N = size_t(Ncells);
    const size_t M = size_t(NradialProfileCells);

    if (cmd == "time") {
        if (argc < 6) return 2;
        const bool jet = std::string(argv[2]) == "jet";
        const int warm = std::atoi(argv[3]), steps = std::atoi(argv[4]);
        const bool stats = std::atoi(argv[5]) != 0;
        init_case(cfg, d, jet);
        for (int s = 0; s < warm; ++s) one_step(cfg, d, mf, jet, stats);
        cudaEvent_t a, b;
        CUDA_CHECK(cudaEventCreate(&a));
        CUDA_CHECK(cudaEventCreate(&b));
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaEventRecord(a));
        for (int s = 0; s < steps; ++s) one_step(cfg, d, mf, jet, stats);
        CUDA_CHECK(cudaEventRecord(b));
        CUDA_CHECK(cudaEventSynchronize(b));
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
        // countmlups.cuh:42-48: all cells, ghost shell included
        const double mlups = double(steps) * double(N) / (double(ms) * 1.0e3);
        std::printf("{\"mlups\": %.6f, \"ms_per_step\": %.6f, \"steps\": %d, \"cells\": %zu}\n", mlups,
                    double(ms) / steps, steps, N);
        free_mean_fields_device(mf);
        free_device_memory(d);
        return 0;
    }

    if (cmd != "run" || argc < 6) {
        std::fprintf(stderr, "usage: ref_dump run <jet|bubble> <steps> <stats_from> <out_dir> [<state_dir>]\n");
        return 2;
    }
    const bool jet = std::string(argv[2]) == "jet";
    const int steps = std::atoi(argv[3]);
    const int stats_from = std::atoi(argv[4]);
    const std::string out = argv[5];

    std::vector<float> fr(size_t(Q) * N), fb(size_t(Q) * N), fields(5 * N), pi(6 * N);
    if (argc >= 7) {
        const std::string in = argv[6];
        if (!read_file(in + "/fr.bin", fr.data(), fr.size() * 4) || !read_file(in + "/fb.bin", fb.data(), fb.size() * 4) ||
            !read_file(in + "/fields.bin", fields.data(), fields.size() * 4)) {
            std::fprintf(stderr, "cannot read state from %s\n", in.c_str());
            return 3;
        }
        CUDA_CHECK(cudaMemcpy(d.fir, fr.data(), bytesF, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(d.fib, fb.data(), bytesF, cudaMemcpyHostToDevice));
        float *dst[5] = {d.rhor, d.rhob, d.ux, d.uy, d.uz};
        for (int k = 0; k < 5; ++k)
            CUDA_CHECK(cudaMemcpy(dst[k], fields.data() + k * N, bytesCell, cudaMemcpyHostToDevice));
    } else {
        init_case(cfg, d, jet);
    }
    for (int s = 0; s < steps; ++s) one_step(cfg, d, mf, jet, s >= stats_from);

    CUDA_CHECK(cudaMemset(mf.tke_total, 0, sizeof(real_t)));
    launch_compute_total_tke(cfg, d, mf.tke_total);
    CUDA_CHECK(cudaDeviceSynchronize());

    CUDA_CHECK(cudaMemcpy(fr.data(), d.fir, bytesF, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(fb.data(), d.fib, bytesF, cudaMemcpyDeviceToHost));
    const float *src[5] = {d.rhor, d.rhob, d.ux, d.uy, d.uz};
    for (int k = 0; k < 5; ++k) CUDA_CHECK(cudaMemcpy(fields.data() + k * N, src[k], bytesCell, cudaMemcpyDeviceToHost));
    const float *psrc[6] = {d.Pixx, d.Pixy, d.Piyy, d.Piyz, d.Pizz, d.Pixz};
    for (int k = 0; k < 6; ++k) CUDA_CHECK(cudaMemcpy(pi.data() + k * N, psrc[k], bytesCell, cudaMemcpyDeviceToHost));
    std::vector<double> radial(5 * M);
    std::vector<unsigned long long> count(M);
    const double *rsrc[5] = {mf.radial_sum_uy, mf.radial_sum_uy2, mf.radial_sum_ur, mf.radial_sum_ur2,
                             mf.radial_sum_uruy};
    for (int k = 0; k < 5; ++k)
        CUDA_CHECK(cudaMemcpy(radial.data() + k * M, rsrc[k], M * sizeof(double), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(count.data(), mf.radial_count, M * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    float tke = 0;
    CUDA_CHECK(cudaMemcpy(&tke, mf.tke_total, sizeof(float), cudaMemcpyDeviceToHost));

    bool ok = write_file(out + "/fr.bin", fr.data(), fr.size() * 4) && write_file(out + "/fb.bin", fb.data(), fb.size() * 4) &&
              write_file(out + "/fields.bin", fields.data(), fields.size() * 4) &&
              write_file(out + "/pi.bin", pi.data(), pi.size() * 4) &&
              write_file(out + "/radial.bin", radial.data(), radial.size() * 8) &&
              write_file(out + "/count.bin", count.data(), count.size() * 8);
    FILE *t = std::fopen((out + "/tke.txt").c_str(), "w");
    if (t) {
        std::fprintf(t, "%.9g\n", double(tke));
        std::fclose(t);
    }
    free_mean_fields_device(mf);
    free_device_memory(d);
    if (!ok) {
        std::fprintf(stderr, "write failed in %s\n", out.c_str());
        return 4;
    }
    return 0;
}
