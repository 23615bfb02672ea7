// io.cpp - output files with the layouts the reference writes and its post/
// scripts read:
//   JET_VTK/Re<Re>_We<We>/case_info.txt                 meanF/meanFieldsRT.cuh:93-118
//   .../mean_profiles/tke_{total,avg,diff}.bin          meanF/meanFieldsRT.cuh:73-91,366-381
//   .../mean_profiles/radial_sum_{uy,uy2,ur,ur2,uruy}.bin, radial_count.bin,
//       radial_profile_metadata.txt                     meanF/meanFieldsRT.cuh:229-336
//   .../mean_profiles/uy_avg.bin                        post/binConversionVti.py:22-28
//   .../vti_data/lbm_%08d.vti                           io/save_data.cuh:137-215
#include <cmath>
#include <cstring>
#include <filesystem>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "internal.hpp"

namespace mcg {

namespace {

bool write_binary(const std::string &path, const void *data, size_t elem, size_t count) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t n = std::fwrite(data, elem, count, f);
    const bool closed = std::fclose(f) == 0;
    return n == count && closed;
}

int round_int(float v) { return static_cast<int>(std::lround(double(v))); }

}  // namespace

mcg_status io_open(mcg_handle *h, const char *root) {
    io_close(h);
    std::ostringstream name;
    name << "Re" << round_int(h->p.Re) << "_We" << round_int(h->p.We);
    const std::filesystem::path base = std::filesystem::path(root) / "JET_VTK" / name.str();
    h->case_dir = base.string();
    h->mean_dir = (base / "mean_profiles").string();
    h->vti_dir = (base / "vti_data").string();
    std::error_code ec;
    std::filesystem::create_directories(h->mean_dir, ec);
    if (ec) return fail(MCG_ERR_IO, "cannot create " + h->mean_dir);
    std::filesystem::create_directories(h->vti_dir, ec);
    if (ec) return fail(MCG_ERR_IO, "cannot create " + h->vti_dir);
    h->f_tke_total = std::fopen((h->mean_dir + "/tke_total.bin").c_str(), "wb");
    h->f_tke_avg = std::fopen((h->mean_dir + "/tke_avg.bin").c_str(), "wb");
    h->f_tke_diff = std::fopen((h->mean_dir + "/tke_diff.bin").c_str(), "wb");
    if (!h->f_tke_total || !h->f_tke_avg || !h->f_tke_diff) {
        io_close(h);
        return fail(MCG_ERR_IO, "cannot open tke files in " + h->mean_dir);
    }
    return io_write_case_metadata(h);
}

mcg_status io_close(mcg_handle *h) {
    FILE **fs[3] = {&h->f_tke_total, &h->f_tke_avg, &h->f_tke_diff};
    for (FILE **f : fs)
        if (*f) {
            std::fclose(*f);
            *f = nullptr;
        }
    return MCG_OK;
}

mcg_status io_write_case_metadata(mcg_handle *h) {
    const mcg_params &p = h->p;
    const std::string path = h->case_dir + "/case_info.txt";
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return fail(MCG_ERR_IO, "cannot write " + path);
    std::fprintf(f, "Re %d\n", round_int(p.Re));
    std::fprintf(f, "We %d\n", round_int(p.We));
    std::fprintf(f, "NX %u\n", unsigned(p.NX));
    std::fprintf(f, "NY %u\n", unsigned(p.NY));
    std::fprintf(f, "NZ %u\n", unsigned(p.NZ));
    std::fprintf(f, "NSTEP %d\n", p.NSTEP);
    std::fprintf(f, "NOUTPUT %d\n", p.NOUTPUT);
    std::fprintf(f, "NSTATS_START_STEP %d\n", p.NSTATS_START_STEP);
    std::fprintf(f, "NR_BINS %u\n", unsigned(p.NX / 2));
    std::fprintf(f, "write_vti_output %d\n", p.write_vti_output ? 1 : 0);
    std::fprintf(f, "jet_radius %.9g\n", double(p.jet_radius));
    std::fprintf(f, "jet_diameter %.9g\n", double(2.0f * p.jet_radius));
    std::fprintf(f, "jet_velocity %.9g\n", double(p.jet_velocity));
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) return fail(MCG_ERR_IO, "short write " + path);
    return MCG_OK;
}

static mcg_status write_radial_metadata(mcg_handle *h, const StatsSnapshot &st) {
    const mcg_params &p = h->p;
    const std::string path = h->mean_dir + "/radial_profile_metadata.txt";
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return fail(MCG_ERR_IO, "cannot write " + path);
    const unsigned NRB = unsigned(p.NX / 2);
    std::fprintf(f, "NX %u\n", unsigned(p.NX));
    std::fprintf(f, "NY %u\n", unsigned(p.NY));
    std::fprintf(f, "NZ %u\n", unsigned(p.NZ));
    std::fprintf(f, "NR_BINS %u\n", NRB);
    std::fprintf(f, "NradialProfileCells %u\n", unsigned(p.NY) * NRB);
    std::fprintf(f, "NOUTPUT %d\n", p.NOUTPUT);
    std::fprintf(f, "NPROFILE_OUTPUT %d\n", p.NOUTPUT);
    std::fprintf(f, "NSTATS_SAMPLE %d\n", 1);
    std::fprintf(f, "NSTATS_START_STEP %d\n", p.NSTATS_START_STEP);
    std::fprintf(f, "Re %d\n", round_int(p.Re));
    std::fprintf(f, "We %d\n", round_int(p.We));
    std::fprintf(f, "D %.9g\n", double(2.0f * p.jet_radius));
    std::fprintf(f, "U_jet %.9g\n", double(p.jet_velocity));
    std::fprintf(f, "jet_radius %.9g\n", double(p.jet_radius));
    std::fprintf(f, "jet_velocity %.9g\n", double(p.jet_velocity));
    std::fprintf(f, "uy_avg_started %d\n", st.started ? 1 : 0);
    std::fprintf(f, "start_step %u\n", st.start_step);
    std::fprintf(f, "uy_avg_start_step %u\n", st.start_step);
    std::fprintf(f, "uy_avg_samples %u\n", st.samples);
    std::fprintf(f, "radial_sample_count %u\n", st.samples);
    if (st.started && st.samples > 0) {
        std::fprintf(f, "uy_avg_first_sample_step %u\n", st.start_step);
        std::fprintf(f, "uy_avg_last_sample_step %u\n", st.start_step + st.samples - 1);
    }
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) return fail(MCG_ERR_IO, "short write " + path);
    return MCG_OK;
}

mcg_status io_write_radial(mcg_handle *h) {
    const StatsSnapshot st = stats_snapshot(h);
    if (!st.started || st.samples == 0) return write_radial_metadata(h, st);
    const size_t M = size_t(h->p.NY) * (h->p.NX / 2);
    std::vector<double> sums(5 * M);
    cudaError_t e = cudaMemcpyAsync(sums.data(), h->s.radial, 5 * M * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "download radial sums");
    return io_write_radial_host(h, st, sums.data());
}

mcg_status io_write_radial_host(mcg_handle *h, const StatsSnapshot &st, const double *sums) {
    if (!st.started || st.samples == 0) return write_radial_metadata(h, st);
    const size_t M = size_t(h->p.NY) * (h->p.NX / 2);
    std::vector<uint64_t> count(M);
    radial_counts_for(h, st.samples, count.data());
    static const char *names[5] = {"radial_sum_uy.bin", "radial_sum_uy2.bin", "radial_sum_ur.bin",
                                   "radial_sum_ur2.bin", "radial_sum_uruy.bin"};
    bool ok = true;
    for (int k = 0; k < 5; ++k) ok = write_binary(h->mean_dir + "/" + names[k], sums + k * M, 8, M) && ok;
    ok = write_binary(h->mean_dir + "/radial_count.bin", count.data(), 8, M) && ok;
    if (mcg_status s = write_radial_metadata(h, st)) return s;
    if (!ok) return fail(MCG_ERR_IO, "short write in " + h->mean_dir);
    return MCG_OK;
}

// The VTI text is encoded on the device from the moment planes
// (launch_vti_encode) and downloaded once; the host only writes it.
mcg_status io_write_vti(mcg_handle *h, const std::string &path) {
    const VtiText L = vti_text_layout(uint64_t(h->s.g.N));
    cudaError_t e = cudaSuccess;
    if (!h->d_vti_text) e = cudaMalloc(&h->d_vti_text, L.total);
    if (e == cudaSuccess && !h->h_vti_text) e = cudaMallocHost(&h->h_vti_text, L.total);
    if (e == cudaSuccess) {
        e = launch_vti_encode(h->s, h->d_vti_text, h->stream);
        if (e == cudaSuccess) ++h->launches;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_vti_text, h->d_vti_text, L.total, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "VTI text");
    return io_write_vti_text(h, path, h->h_vti_text);
}

mcg_status io_write_vti_text(mcg_handle *h, const std::string &path, const char *text) {
    const VtiText L = vti_text_layout(uint64_t(h->s.g.N));
    FILE *out = std::fopen(path.c_str(), "wb");
    if (!out) return fail(MCG_ERR_IO, "cannot open " + path);
    const int X = h->p.NX - 1, Y = h->p.NY - 1, Z = h->p.NZ - 1;
    std::fprintf(out, "<?xml version=\"1.0\"?>\n");
    std::fprintf(out, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
    std::fprintf(out, "  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n", X, Y, Z);
    std::fprintf(out, "    <Piece Extent=\"0 %d 0 %d 0 %d\">\n", X, Y, Z);
    std::fprintf(out, "      <PointData Scalars=\"rhor\" Vectors=\"u\">\n");
    static const char *names[4] = {"rhor", "rhob", "rho", "u"};
    for (int a = 0; a < 4; ++a) {
        std::fprintf(out, "        <DataArray type=\"Float32\" Name=\"%s\"%s format=\"binary\">\n", names[a],
                     a == 3 ? " NumberOfComponents=\"3\"" : "");
        std::fwrite(text + L.off[a], 1, L.len[a], out);
        std::fprintf(out, "\n        </DataArray>\n");
    }
    std::fprintf(out, "      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n");
    const bool ok = std::ferror(out) == 0;
    if (std::fclose(out) != 0 || !ok) return fail(MCG_ERR_IO, "short write " + path);
    return MCG_OK;
}

// update_tke_state + write_tke_outputs (meanF/meanFieldsRT.cuh:192-227, 366-381)
mcg_status io_write_tke_sample(mcg_handle *h, int32_t step) {
    return io_write_tke_sample_snap(h, step, stats_snapshot(h));
}

mcg_status io_write_tke_sample_snap(mcg_handle *h, int32_t step, const StatsSnapshot &st) {
    if (h->first_tke) {
        h->tke_delta = 0.f;
        h->tke_abs_delta = 0.f;
        h->first_tke = false;
    } else {
        h->tke_delta = h->tke_avg - h->tke_avg_prev;
        h->tke_abs_delta = std::fabs(h->tke_delta);
    }
    std::cout << std::scientific << "step " << step << " | tke_prev = " << h->tke_avg_prev
              << " | tke_avg = " << h->tke_avg << " | delta_tke_avg = " << h->tke_abs_delta;
    if (st.started)
        std::cout << " | uy_radial_avg = on | uy_avg_start_step = " << st.start_step
                  << " | uyavg_samples = " << st.samples << " | radial_count = on";
    else
        std::cout << " | uy_radial_avg = waiting | uyavg_samples = 0";
    std::cout << "\n";
    h->tke_avg_prev = h->tke_avg;
    if (!h->f_tke_total) return fail(MCG_ERR_STATE, "tke files are not open");
    bool ok = std::fwrite(&h->tke_total, 4, 1, h->f_tke_total) == 1;
    ok = std::fwrite(&h->tke_avg, 4, 1, h->f_tke_avg) == 1 && ok;
    ok = std::fwrite(&h->tke_abs_delta, 4, 1, h->f_tke_diff) == 1 && ok;
    std::fflush(h->f_tke_total);
    std::fflush(h->f_tke_avg);
    std::fflush(h->f_tke_diff);
    if (!ok) return fail(MCG_ERR_IO, "short write to tke files");
    return MCG_OK;
}

mcg_status io_write_uy_average(mcg_handle *h) {
    const size_t N = h->s.g.N;
    std::vector<float> buf(N);
    cudaError_t e = cudaMemcpyAsync(buf.data(), h->s.uy_avg, N * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "download uy average");
    const std::string path = h->mean_dir + "/uy_avg.bin";
    if (!write_binary(path, buf.data(), 4, N)) return fail(MCG_ERR_IO, "cannot write " + path);
    return MCG_OK;
}

}  // namespace mcg
