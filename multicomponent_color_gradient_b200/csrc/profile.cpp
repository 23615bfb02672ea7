// profile.cpp - time-averaged profiles of the round jet from the radial
// statistics, and the profile-misfit objective of the jet adjoint with its
// gradient.
//
// Definitions follow the reference's post-processing (post/plot_profiles.py):
//   mean profile     U(y, r) = sum_uy(y, r) / count(y, r), count = samples x
//                    interior columns of bin r (post/mean_profile_io.py:182-212)
//   centreline       uc(y) = U(y, 0) (the first annulus, plot_profiles.py:129)
//   bin radius       the mean distance of the bin's interior columns from the
//                    jet axis, 0 for bin 0 (plot_profiles.py:73-91)
//   half-width       r_half(y): the first bin i > 0 with U(y, i)/uc(y) <= 1/2,
//                    linear interpolation of the ratio between bins i-1 and i
//                    (plot_profiles.py:53-70); undefined (NaN) when uc <= 0,
//                    no bin qualifies, or the two ratios are numerically equal
// The objective J = 1/2 sum_y ((uc - uc*)/U_jet)^2 + ((r_half - r_half*)/D)^2
// over y_lo <= y <= y_hi, each term where both of its values are defined.
// The bin of a crossing is piecewise constant in the data, so the gradient is
// that of the interpolation within the current bins.
#include <cmath>
#include <vector>

#include "internal.hpp"

namespace mcg {
namespace {

struct ProfileGrid {
    int NY, NRB;
    std::vector<double> ncols, radius;
};

ProfileGrid profile_grid(const mcg_handle *h) {
    ProfileGrid pg;
    pg.NY = h->p.NY;
    pg.NRB = h->p.NX / 2;
    pg.ncols.assign(size_t(pg.NRB), 0.0);
    pg.radius.assign(size_t(pg.NRB), 0.0);
    std::vector<double> rsum(size_t(pg.NRB), 0.0);
    for (int r = 0; r < pg.NRB; ++r) pg.ncols[size_t(r)] = double(h->ncols[size_t(r)]);
    for (int x = 1; x <= h->p.NX - 2; ++x)
        for (int z = 1; z <= h->p.NZ - 2; ++z) {
            const double dx = double(x) - double(h->p.jet_x0), dz = double(z) - double(h->p.jet_z0);
            const double r = std::sqrt(dx * dx + dz * dz);
            const int rb = int(r);
            if (rb < pg.NRB) rsum[size_t(rb)] += r;
        }
    for (int r = 0; r < pg.NRB; ++r)
        pg.radius[size_t(r)] = pg.ncols[size_t(r)] > 0 ? rsum[size_t(r)] / pg.ncols[size_t(r)] : double(r);
    pg.radius[0] = 0.0;
    return pg;
}

bool isclose(double a, double b) { return std::fabs(a - b) <= 1e-8 + 1e-5 * std::fabs(b); }

// Half-width of one profile row U[0..NRB) and, when g != null, its gradient
// with respect to U (g[0..NRB) is set).  NaN when undefined.
double half_width(const ProfileGrid &pg, const double *U, double *g) {
    if (g)
        for (int r = 0; r < pg.NRB; ++r) g[r] = 0.0;
    const double uc = U[0];
    if (!std::isfinite(uc) || uc <= 0.0) return NAN;
    int idx = -1;
    for (int r = 1; r < pg.NRB; ++r) {
        const double q = U[r] / uc;
        if (std::isfinite(q) && q <= 0.5) {
            idx = r;
            break;
        }
    }
    if (idx < 0) return NAN;
    const double r1 = pg.radius[size_t(idx - 1)], r2 = pg.radius[size_t(idx)];
    const double u1 = U[idx - 1] / uc, u2 = U[idx] / uc;
    if (!std::isfinite(u1) || !std::isfinite(u2) || isclose(u1, u2)) return NAN;
    const double dr = r2 - r1, du = u2 - u1;
    const double rh = r1 + (0.5 - u1) * dr / du;
    if (g) {
        const double d1 = dr * (0.5 - u2) / (du * du);   // d rh / d u1
        const double d2 = -dr * (0.5 - u1) / (du * du);  // d rh / d u2
        // u_k = U[k]/uc: dU[idx-1], dU[idx], and uc = U[0] through both ratios
        g[idx - 1] += d1 / uc;
        g[idx] += d2 / uc;
        g[0] += -(d1 * u1 + d2 * u2) / uc;
    }
    return rh;
}

void mean_profile(const ProfileGrid &pg, const double *sum_uy, uint32_t samples, int y, double *U) {
    const bool interior = y >= 1 && y <= pg.NY - 2;
    for (int r = 0; r < pg.NRB; ++r) {
        const double cnt = interior ? double(samples) * pg.ncols[size_t(r)] : 0.0;
        U[r] = cnt > 0 ? sum_uy[size_t(y) * pg.NRB + r] / cnt : NAN;
    }
}

}  // namespace

void profile_metrics(const mcg_handle *h, const double *sum_uy, uint32_t samples, float *uc, float *rh) {
    const ProfileGrid pg = profile_grid(h);
    std::vector<double> U(size_t(pg.NRB));
    for (int y = 0; y < pg.NY; ++y) {
        mean_profile(pg, sum_uy, samples, y, U.data());
        uc[y] = float(U[0]);
        rh[y] = float(half_width(pg, U.data(), nullptr));
    }
}

double profile_objective(const mcg_handle *h, const double *sum_uy, uint32_t samples, int y_lo, int y_hi,
                         const float *uc_target, const float *rh_target, float *src) {
    const ProfileGrid pg = profile_grid(h);
    const double U0 = double(h->p.jet_velocity), D = 2.0 * double(h->p.jet_radius);
    std::vector<double> U(size_t(pg.NRB)), g(size_t(pg.NRB)), dJdU(size_t(pg.NRB));
    for (size_t k = 0; k < size_t(pg.NY) * pg.NRB; ++k) src[k] = 0.0f;
    double J = 0.0;
    for (int y = y_lo; y <= y_hi; ++y) {
        mean_profile(pg, sum_uy, samples, y, U.data());
        for (int r = 0; r < pg.NRB; ++r) dJdU[size_t(r)] = 0.0;
        const double uc = U[0], uct = double(uc_target[y]);
        if (std::isfinite(uc) && std::isfinite(uct)) {
            const double e = (uc - uct) / U0;
            J += 0.5 * e * e;
            dJdU[0] += e / U0;
        }
        const double rh = half_width(pg, U.data(), g.data()), rht = double(rh_target[y]);
        if (std::isfinite(rh) && std::isfinite(rht)) {
            const double e = (rh - rht) / D;
            J += 0.5 * e * e;
            for (int r = 0; r < pg.NRB; ++r) dJdU[size_t(r)] += e / D * g[size_t(r)];
        }
        // U(y, r) = sum over the window's steps and the bin's columns / count
        for (int r = 0; r < pg.NRB; ++r) {
            const double cnt = double(samples) * pg.ncols[size_t(r)];
            if (cnt > 0) src[size_t(y) * pg.NRB + r] = float(dJdU[size_t(r)] / cnt);
        }
    }
    return J;
}

}  // namespace mcg
