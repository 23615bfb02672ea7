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

mcg_status download_fields(mcg_handle *h, std::vector<float> &buf) {
    const size_t N = h->s.g.N;
    buf.resize(5 * N);
    cudaError_t e = cudaMemcpyAsync(buf.data(), h->s.mom, 5 * N * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "download fields");
    return MCG_OK;
}

}  // namespace

std::string base64_encode(const unsigned char *data, size_t len) {
    static const char tbl[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::string out((len + 2) / 3 * 4, '=');
    size_t o = 0, i = 0;
    for (; i + 2 < len; i += 3) {
        const uint32_t v = (uint32_t(data[i]) << 16) | (uint32_t(data[i + 1]) << 8) | uint32_t(data[i + 2]);
        out[o++] = tbl[(v >> 18) & 63];
        out[o++] = tbl[(v >> 12) & 63];
        out[o++] = tbl[(v >> 6) & 63];
        out[o++] = tbl[v & 63];
    }
    if (i < len) {
        const uint32_t b1 = (i + 1 < len) ? data[i + 1] : 0;
        const uint32_t v = (uint32_t(data[i]) << 16) | (b1 << 8);
        out[o++] = tbl[(v >> 18) & 63];
        out[o++] = tbl[(v >> 12) & 63];
        if (i + 1 < len) out[o++] = tbl[(v >> 6) & 63];
    }
    return out;
}

namespace {
// [UInt64 byte count][payload], base64 (VTK XML binary, header_type UInt64)
std::string vtk_block(const std::vector<unsigned char> &payload) {
    std::vector<unsigned char> buf(8 + payload.size());
    const uint64_t n = payload.size();
    std::memcpy(buf.data(), &n, 8);
    if (!payload.empty()) std::memcpy(buf.data() + 8, payload.data(), payload.size());
    return base64_encode(buf.data(), buf.size());
}
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

static mcg_status write_radial_metadata(mcg_handle *h) {
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
    std::fprintf(f, "uy_avg_started %d\n", h->stats_started ? 1 : 0);
    std::fprintf(f, "start_step %u\n", h->stats_start_step);
    std::fprintf(f, "uy_avg_start_step %u\n", h->stats_start_step);
    std::fprintf(f, "uy_avg_samples %u\n", h->stats_samples);
    std::fprintf(f, "radial_sample_count %u\n", h->stats_samples);
    if (h->stats_started && h->stats_samples > 0) {
        std::fprintf(f, "uy_avg_first_sample_step %u\n", h->stats_start_step);
        std::fprintf(f, "uy_avg_last_sample_step %u\n", h->stats_start_step + h->stats_samples - 1);
    }
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) return fail(MCG_ERR_IO, "short write " + path);
    return MCG_OK;
}

mcg_status io_write_radial(mcg_handle *h) {
    if (!h->stats_started || h->stats_samples == 0) return write_radial_metadata(h);
    const size_t M = size_t(h->p.NY) * (h->p.NX / 2);
    std::vector<double> sums(5 * M);
    std::vector<uint64_t> count(M);
    cudaError_t e = cudaMemcpyAsync(sums.data(), h->s.radial, 5 * M * 8, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "download radial sums");
    radial_counts(h, count.data());
    static const char *names[5] = {"radial_sum_uy.bin", "radial_sum_uy2.bin", "radial_sum_ur.bin",
                                   "radial_sum_ur2.bin", "radial_sum_uruy.bin"};
    bool ok = true;
    for (int k = 0; k < 5; ++k) ok = write_binary(h->mean_dir + "/" + names[k], sums.data() + k * M, 8, M) && ok;
    ok = write_binary(h->mean_dir + "/radial_count.bin", count.data(), 8, M) && ok;
    if (mcg_status s = write_radial_metadata(h)) return s;
    if (!ok) return fail(MCG_ERR_IO, "short write in " + h->mean_dir);
    return MCG_OK;
}

mcg_status io_write_vti(mcg_handle *h, const std::string &path) {
    std::vector<float> f;
    if (mcg_status s = download_fields(h, f)) return s;
    const size_t N = h->s.g.N;
    const float *rr = f.data(), *rb = rr + N, *ux = rb + N, *uy = ux + N, *uz = uy + N;
    std::vector<unsigned char> pl(N * 4);
    std::memcpy(pl.data(), rr, N * 4);
    const std::string e_rr = vtk_block(pl);
    std::memcpy(pl.data(), rb, N * 4);
    const std::string e_rb = vtk_block(pl);
    {
        float *q = reinterpret_cast<float *>(pl.data());
        for (size_t i = 0; i < N; ++i) q[i] = rr[i] + rb[i];
    }
    const std::string e_rho = vtk_block(pl);
    std::vector<unsigned char> pu(3 * N * 4);
    {
        float *q = reinterpret_cast<float *>(pu.data());
        for (size_t i = 0; i < N; ++i) {
            q[3 * i] = ux[i];
            q[3 * i + 1] = uy[i];
            q[3 * i + 2] = uz[i];
        }
    }
    const std::string e_u = vtk_block(pu);
    FILE *out = std::fopen(path.c_str(), "wb");
    if (!out) return fail(MCG_ERR_IO, "cannot open " + path);
    const int X = h->p.NX - 1, Y = h->p.NY - 1, Z = h->p.NZ - 1;
    std::fprintf(out, "<?xml version=\"1.0\"?>\n");
    std::fprintf(out, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
    std::fprintf(out, "  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n", X, Y, Z);
    std::fprintf(out, "    <Piece Extent=\"0 %d 0 %d 0 %d\">\n", X, Y, Z);
    std::fprintf(out, "      <PointData Scalars=\"rhor\" Vectors=\"u\">\n");
    const std::pair<const char *, const std::string *> arrays[3] = {{"rhor", &e_rr}, {"rhob", &e_rb}, {"rho", &e_rho}};
    for (const auto &a : arrays) {
        std::fprintf(out, "        <DataArray type=\"Float32\" Name=\"%s\" format=\"binary\">\n", a.first);
        std::fwrite(a.second->data(), 1, a.second->size(), out);
        std::fprintf(out, "\n        </DataArray>\n");
    }
    std::fprintf(out, "        <DataArray type=\"Float32\" Name=\"u\" NumberOfComponents=\"3\" format=\"binary\">\n");
    std::fwrite(e_u.data(), 1, e_u.size(), out);
    std::fprintf(out, "\n        </DataArray>\n");
    std::fprintf(out, "      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n");
    const bool ok = std::ferror(out) == 0;
    if (std::fclose(out) != 0 || !ok) return fail(MCG_ERR_IO, "short write " + path);
    return MCG_OK;
}

// update_tke_state + write_tke_outputs (meanF/meanFieldsRT.cuh:192-227, 366-381)
mcg_status io_write_tke_sample(mcg_handle *h, int32_t step) {
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
    if (h->stats_started)
        std::cout << " | uy_radial_avg = on | uy_avg_start_step = " << h->stats_start_step
                  << " | uyavg_samples = " << h->stats_samples << " | radial_count = on";
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
