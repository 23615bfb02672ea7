// mcg_oracle.cpp - TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's per-step update (Felipe-Aristi/
// Multicomponent_Color_Gradient), used as the checker for the CUDA path:
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
// it.  The product library never links or calls it.
//
// It follows the reference literally: push streaming into ONE in-place
// population buffer (memory.cuh:58-76), moments in separate arrays, the same
// expression order, the ghost-shell quirks (unwritten slots keep old values,
// lateral ghost densities are read unwrapped by the colour gradient, boundary
// writes are unwrapped).  It is templated on the arithmetic type: float gives
// the reference's own precision (compiled with -ffp-contract=off so no FMA
// contraction), double gives the FP64 oracle the FP16/FP32 error statements
// are made against.
//
// Parity pin: checked against fixtures produced by the reference's own CUDA
// build (oracle/ref_dump.cu, tests/golden/) and against lattice identities.
//
// Reference files restated (paths within the reference project):
//   stencil_ct.cuh:9-203        lattice tables, Hermite polynomials
//   lbm.cuh:16-78               feq, fneqr
//   lbm.cuh:82-165              Mfields_calculation
//   lbm.cuh:184-293             ColliStream_calculations
//   forces.cuh:13-105           force, cos2rule, A_calculation, preOmega2
//   collisionOperators.cuh:15-69  Omega2, cosphi, recolorDelta
//   utilities/mathUtilities.cuh:14-90  isJet, psi, clamp01, omega_sponge
//   utilities/bounds.cuh:6-60   interior, wrapx/wrapz
//   jet/jetIn.cuh:13-62, bubble/bubbleIn.cuh:10-39   initial conditions
//   jet/boundary_conditions.cuh:17-85,163-233         inlet, convective outlet
//   kernels.cu:136-233          tke, running averages, radial moments
//   main.cu:52-82               per-step sequence

#include "../include/mcg.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int Q = 27;
// Direction order of stencil_ct.cuh:9-16 (a table the interface fixes).
constexpr int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
constexpr int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
constexpr int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// Uniform in [0,1) with 24 random bits (exact in float).
inline float hash_uniform(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    uint64_t h = splitmix64(seed ^ splitmix64(a ^ splitmix64(b ^ splitmix64(c))));
    return static_cast<float>(h >> 40) * (1.0f / 16777216.0f);
}

// Lattice constants formed in T exactly as constants.cuh:45-53 and
// stencil_ct.cuh:42-189 form them in real_t.
template <class T>
struct Lattice {
    T cs2, cs4, cs6, inv_cs2, inv_2cs2, inv_2cs4, inv_6cs6, inv_2cs6;
    T w[Q], B[Q], invc[Q];
    T Hxx[Q], Hxy[Q], Hyy[Q], Hyz[Q], Hzz[Q], Hxz[Q];
    T Hxxy[Q], Hxxz[Q], Hxyy[Q], Hxzz[Q], Hyyz[Q], Hyzz[Q], Hxyz[Q];
    Lattice() {
        cs2 = static_cast<T>(1.0 / 3.0);
        cs4 = cs2 * cs2;
        cs6 = cs4 * cs2;
        inv_cs2 = static_cast<T>(1) / cs2;
        inv_2cs2 = static_cast<T>(1) / (static_cast<T>(2) * cs2);
        inv_2cs4 = static_cast<T>(1) / (static_cast<T>(2) * cs4);
        inv_6cs6 = static_cast<T>(1.0) / (static_cast<T>(6.0) * cs6);
        inv_2cs6 = static_cast<T>(1.0) / (static_cast<T>(2.0) * cs6);
        for (int i = 0; i < Q; ++i) {
            const int cx = CX[i], cy = CY[i], cz = CZ[i];
            const int s = cx * cx + cy * cy + cz * cz;
            w[i] = s == 0 ? T(8.0 / 27.0) : s == 1 ? T(2.0 / 27.0) : s == 2 ? T(1.0 / 54.0) : T(1.0 / 216.0);
            B[i] = i == 0 ? T(-10.0 / 27.0) : w[i];
            invc[i] = s == 0 ? T(0) : s == 1 ? T(1) : s == 2 ? T(0.7071067811865475) : T(0.5773502691896258);
            Hxx[i] = T(cx * cx) - cs2;
            Hxy[i] = T(cx * cy);
            Hyy[i] = T(cy * cy) - cs2;
            Hyz[i] = T(cy * cz);
            Hzz[i] = T(cz * cz) - cs2;
            Hxz[i] = T(cx * cz);
            Hxxy[i] = T(cx * cx * cy) - cs2 * T(cy);
            Hxxz[i] = T(cx * cx * cz) - cs2 * T(cz);
            Hxyy[i] = T(cx * cy * cy) - cs2 * T(cx);
            Hxzz[i] = T(cx * cz * cz) - cs2 * T(cx);
            Hyyz[i] = T(cy * cy * cz) - cs2 * T(cz);
            Hyzz[i] = T(cy * cz * cz) - cs2 * T(cy);
            Hxyz[i] = T(cx * cy * cz);
        }
    }
};

template <class T>
struct Oracle {
    mcg_params p{};
    int NX, NY, NZ, NRB;
    size_t N;
    Lattice<T> L;
    // physical constants in T
    T rhor0, rhob0, jet_x0, jet_z0, jet_radius, jet_velocity, nu, taub, omegab, beta, sigma_over_4cs4, sponge_K;
    int sponge_y_start, sponge_y_end;

    std::vector<T> fr, fb;  // populations, f[i*N + id] (memory.cuh:11-25)
    std::vector<T> rhor, rhob, ux, uy, uz, Pixx, Pixy, Piyy, Piyz, Pizz, Pixz;
    std::vector<double> s_uy, s_uy2, s_ur, s_ur2, s_uruy;
    std::vector<uint64_t> cnt;
    std::vector<T> uy_avg;
    std::vector<T> inlet_prof;  // per-column inlet velocity multipliers (empty: top-hat)
    uint32_t uy_avg_count = 0;
    T tke_total = 0, tke_avg = 0;
    int64_t step = 0;
    int stats_mode = -1;  // -1 automatic (NSTATS_START_STEP), 0 off, 1 on
    bool stats_started = false;
    uint32_t stats_start_step = 0, stats_samples = 0;

    explicit Oracle(const mcg_params &prm) : p(prm) {
        NX = p.NX; NY = p.NY; NZ = p.NZ;
        NRB = NX / 2;
        N = size_t(NX) * NY * NZ;
        fr.assign(size_t(Q) * N, T(0));
        fb.assign(size_t(Q) * N, T(0));
        for (auto *v : {&rhor, &rhob, &ux, &uy, &uz, &Pixx, &Pixy, &Piyy, &Piyz, &Pizz, &Pixz, &uy_avg})
            v->assign(N, T(0));
        for (auto *v : {&s_uy, &s_uy2, &s_ur, &s_ur2, &s_uruy}) v->assign(size_t(NY) * NRB, 0.0);
        cnt.assign(size_t(NY) * NRB, 0);
        rhor0 = T(p.rhor0); rhob0 = T(p.rhob0);
        jet_x0 = T(p.jet_x0); jet_z0 = T(p.jet_z0);
        jet_radius = T(p.jet_radius); jet_velocity = T(p.jet_velocity);
        nu = T(p.nu); taub = T(p.taub);
        omegab = T(1) / taub;                                   // constants.cuh:67
        beta = T(p.beta_recolor);
        sigma_over_4cs4 = T(p.sigma) / (T(4) * L.cs4);          // constants.cuh:76
        sponge_K = T(p.sponge_K);
        sponge_y_end = NY - 2;                                  // mathUtilities.cuh:52-53
        sponge_y_start = sponge_y_end - p.sponge_cells + 1;
    }

    size_t idx(int x, int y, int z) const { return size_t(x) + size_t(NX) * (size_t(y) + size_t(NY) * size_t(z)); }
    size_t fidx(size_t id, int i) const { return size_t(i) * N + id; }
    bool is_interior(int x, int y, int z) const {
        return x >= 1 && x <= NX - 2 && y >= 1 && y <= NY - 2 && z >= 1 && z <= NZ - 2;
    }
    int wrapx(int x) const { return x == 0 ? NX - 2 : (x == NX - 1 ? 1 : x); }  // bounds.cuh:23-34
    int wrapy(int y) const { return y == 0 ? NY - 2 : (y == NY - 1 ? 1 : y); }
    int wrapz(int z) const { return z == 0 ? NZ - 2 : (z == NZ - 1 ? 1 : z); }
    bool periodic() const { return p.boundary == MCG_BOUNDARY_PERIODIC; }

    // mathUtilities.cuh:14-21
    bool isJet(int x, int z) const {
        const T dx = T(x) - jet_x0, dz = T(z) - jet_z0;
        return dx * dx + dz * dz <= jet_radius * jet_radius;
    }
    static T psi(T a, T b) { return (a - b) / (a + b); }       // mathUtilities.cuh:24-28
    static T clamp01(T x) { return std::fmin(std::fmax(x, T(0)), T(1)); }
    // mathUtilities.cuh:56-90
    T omega_sponge(int y) const {
        const T inv_width = T(1.0) / T(sponge_y_end - sponge_y_start);
        const T s = clamp01((T(y) - T(sponge_y_start)) * inv_width);
        const T nus = nu * (T(1.0) + sponge_K * (s * s * s));
        const T tau = T(0.5) + nus * L.inv_cs2;
        return T(1.0) / tau;
    }

    // lbm.cuh:16-35
    T feq(int i, T rho, T vx, T vy, T vz) const {
        const T cu = vx * T(CX[i]) + vy * T(CY[i]) + vz * T(CZ[i]);
        const T usq = vx * vx + vy * vy + vz * vz;
        const T cu2 = cu * cu;
        const T A2eq = (cu * cu) * L.inv_2cs4 - usq * L.inv_2cs2 + cu * L.inv_cs2;
        const T A3eq = cu * (cu2 * L.inv_6cs6 - usq * L.inv_2cs4);
        return L.w[i] * rho * (T(1.0) + A2eq + A3eq);
    }
    // lbm.cuh:38-78
    T fneqr(int i, T pxx, T pxy, T pyy, T pyz, T pzz, T pxz, T vx, T vy, T vz) const {
        const T A2 = (pxx * L.Hxx[i] + T(2.0) * pxy * L.Hxy[i] + pyy * L.Hyy[i] + T(2.0) * pyz * L.Hyz[i] +
                      pzz * L.Hzz[i] + T(2.0) * pxz * L.Hxz[i]) * L.inv_2cs4;
        const T a3xxy = pxx * vy + T(2.0) * pxy * vx;
        const T a3xxz = pxx * vz + T(2.0) * pxz * vx;
        const T a3xyy = pyy * vx + T(2.0) * pxy * vy;
        const T a3xzz = pzz * vx + T(2.0) * pxz * vz;
        const T a3yyz = pyy * vz + T(2.0) * pyz * vy;
        const T a3yzz = pzz * vy + T(2.0) * pyz * vz;
        const T a3xyz = pxy * vz + pxz * vy + pyz * vx;
        const T A3 = (a3xxy * L.Hxxy[i] + a3xxz * L.Hxxz[i] + a3xyy * L.Hxyy[i] + a3xzz * L.Hxzz[i] +
                      a3yyz * L.Hyyz[i] + a3yzz * L.Hyzz[i] + T(2.0) * a3xyz * L.Hxyz[i]) * L.inv_2cs6;
        return L.w[i] * (A2 + A3);
    }

    // Initial populations with optional seeded noise f*(1+eps), eps uniform in [-a, a].
    T noisy(T f, size_t id, int i) const {
        if (p.init_noise == 0.0f) return f;
        const float u = hash_uniform(p.seed, 0x1D17ull, id, uint64_t(i));
        const float eps = (2.0f * u - 1.0f) * p.init_noise;
        return f * (T(1.0) + T(eps));
    }

    // jet/jetIn.cuh:13-35 (all cells) then jet/jetIn.cuh:37-62 (y=0 interior x,z)
    void init_jet() {
        for (int z = 0; z < NZ; ++z)
            for (int y = 0; y < NY; ++y)
                for (int x = 0; x < NX; ++x) {
                    const size_t id = idx(x, y, z);
                    rhor[id] = rhor0;
                    rhob[id] = T(0.0);
                    for (int i = 0; i < Q; ++i) {
                        fr[fidx(id, i)] = noisy(feq(i, rhor[id], 0, 0, 0), id, i);
                        fb[fidx(id, i)] = feq(i, rhob[id], 0, 0, 0);
                    }
                }
        for (int z = 1; z <= NZ - 2; ++z)
            for (int x = 1; x <= NX - 2; ++x) {
                const size_t id = idx(x, 0, z);
                const T j = isJet(x, z) ? T(1) : T(0);
                rhor[id] = (T(1.0) - j) * rhor0;
                rhob[id] = j * rhob0;
                for (int i = 0; i < Q; ++i) {
                    fr[fidx(id, i)] = feq(i, rhor[id], 0, 0, 0);
                    fb[fidx(id, i)] = feq(i, rhob[id], 0, 0, 0);
                }
            }
        step = 0;
    }

    // bubble/bubbleIn.cuh:10-39 (blue inside unless bubble_red_inside)
    void init_bubble() {
        const T R2 = T(p.bubble_radius) * T(p.bubble_radius);
        for (int z = 0; z < NZ; ++z)
            for (int y = 0; y < NY; ++y)
                for (int x = 0; x < NX; ++x) {
                    const size_t id = idx(x, y, z);
                    const T dx = T(x) - T(p.bubble_x0), dy = T(y) - T(p.bubble_y0), dz = T(z) - T(p.bubble_z0);
                    const T inside = (dx * dx + dy * dy + dz * dz) <= R2 ? T(1) : T(0);
                    if (p.bubble_red_inside) {
                        rhor[id] = inside * rhor0;
                        rhob[id] = (T(1.0) - inside) * rhob0;
                    } else {
                        rhor[id] = (T(1.0) - inside) * rhor0;
                        rhob[id] = inside * rhob0;
                    }
                    for (int i = 0; i < Q; ++i) {
                        fr[fidx(id, i)] = noisy(L.w[i] * rhor[id], id, i);
                        fb[fidx(id, i)] = noisy(L.w[i] * rhob[id], id, i);
                    }
                }
        if (periodic()) refresh_periodic_ghost_density();
        step = 0;
    }

    // lbm.cuh:82-165 over interior nodes (kernels.cu:60-76)
    void macros() {
#pragma omp parallel for schedule(static)
        for (int z = 1; z <= NZ - 2; ++z)
            for (int y = 1; y <= NY - 2; ++y)
                for (int x = 1; x <= NX - 2; ++x) {
                    const size_t id = idx(x, y, z);
                    T sumr = 0, sumb = 0, jx = 0, jy = 0, jz = 0;
                    T Axx = 0, Axy = 0, Ayy = 0, Ayz = 0, Azz = 0, Axz = 0;
                    for (int i = 0; i < Q; ++i) {
                        const T a = fr[fidx(id, i)], b = fb[fidx(id, i)];
                        sumr += a;
                        sumb += b;
                        const T gi = a + b;
                        jx += gi * T(CX[i]);
                        jy += gi * T(CY[i]);
                        jz += gi * T(CZ[i]);
                        Axx += gi * L.Hxx[i];
                        Axy += gi * L.Hxy[i];
                        Ayy += gi * L.Hyy[i];
                        Ayz += gi * L.Hyz[i];
                        Azz += gi * L.Hzz[i];
                        Axz += gi * L.Hxz[i];
                    }
                    rhor[id] = sumr;
                    rhob[id] = sumb;
                    const T rho = sumr + sumb;
                    const T inv = T(1.0) / rho;
                    const T vx = jx * inv, vy = jy * inv, vz = jz * inv;
                    ux[id] = vx; uy[id] = vy; uz[id] = vz;
                    Pixx[id] = Axx - rho * vx * vx;
                    Pixy[id] = Axy - rho * vx * vy;
                    Piyy[id] = Ayy - rho * vy * vy;
                    Piyz[id] = Ayz - rho * vy * vz;
                    Pizz[id] = Azz - rho * vz * vz;
                    Pixz[id] = Axz - rho * vx * vz;
                }
        if (periodic()) refresh_periodic_ghost_density();
    }

    // Extension (periodic box): ghost densities mirror the opposite interior
    // node so the unwrapped colour-gradient stencil sees a periodic field.
    void refresh_periodic_ghost_density() {
        for (int z = 0; z < NZ; ++z)
            for (int y = 0; y < NY; ++y)
                for (int x = 0; x < NX; ++x) {
                    if (is_interior(x, y, z)) continue;
                    const size_t id = idx(x, y, z);
                    const size_t src = idx(wrapx(x), wrapy(y), wrapz(z));
                    rhor[id] = rhor[src];
                    rhob[id] = rhob[src];
                }
    }

    // forces.cuh:13-43, 87-105
    void colour_gradient(size_t id, T &Fx, T &Fy, T &Fz) const {
        T sx = 0, sy = 0, sz = 0;
        const long off_y = NX, off_z = long(NX) * NY;
        for (int i = 1; i < Q; ++i) {
            const size_t n = size_t(long(id) + CX[i] + off_y * CY[i] + off_z * CZ[i]);  // no wrap
            const T psn = psi(rhor[n], rhob[n]);
            sx += L.w[i] * psn * T(CX[i]);
            sy += L.w[i] * psn * T(CY[i]);
            sz += L.w[i] * psn * T(CZ[i]);
        }
        Fx = L.inv_cs2 * sx;
        Fy = L.inv_cs2 * sy;
        Fz = L.inv_cs2 * sz;
    }

    // lbm.cuh:184-293 over interior nodes (kernels.cu:78-94)
    void collistream() {
        const T A = sigma_over_4cs4 / taub;          // forces.cuh:87-105 (tau_eff = taub)
        const T Ahalf = A / T(2.0);
#pragma omp parallel for schedule(static)
        for (int z = 1; z <= NZ - 2; ++z)
            for (int y = 1; y <= NY - 2; ++y)
                for (int x = 1; x <= NX - 2; ++x) {
                    const size_t id = idx(x, y, z);
                    const T rr = rhor[id], rb = rhob[id];
                    const T rT = rr + rb;
                    const T invrT = T(1) / rT;
                    const T aR = rr * invrT, aB = rb * invrT;
                    const T vx = ux[id], vy = uy[id], vz = uz[id];
                    const T pxx = Pixx[id], pxy = Pixy[id], pyy = Piyy[id], pyz = Piyz[id], pzz = Pizz[id],
                            pxz = Pixz[id];
                    const T oms = T(1.0) - omega_sponge(y);
                    const T Iind = T(4.0) * rr * rb * invrT * invrT;
                    const bool bulk = Iind <= T(1e-4);
                    T Fx = 0, Fy = 0, Fz = 0, absF = 0;
                    if (!bulk) {
                        colour_gradient(id, Fx, Fy, Fz);
                        absF = std::sqrt(Fx * Fx + Fy * Fy + Fz * Fz);
                    }
                    for (int i = 0; i < Q; ++i) {
                        const T Om1 = feq(i, rT, vx, vy, vz) + oms * fneqr(i, pxx, pxy, pyy, pyz, pzz, pxz, vx, vy, vz);
                        int xn = x + CX[i], yn = y + CY[i], zn = z + CZ[i];
                        xn = wrapx(xn);
                        zn = wrapz(zn);
                        if (periodic()) yn = wrapy(yn);
                        const size_t t = fidx(idx(xn, yn, zn), i);
                        if (bulk) {
                            fr[t] = aR * Om1;
                            fb[t] = aB * Om1;
                        } else {
                            // collisionOperators.cuh:15-24, forces.cuh:50-75
                            T cos2 = 0;
                            if (i != 0 && !(absF <= T(1.0e-4))) {
                                const T Fc = Fx * T(CX[i]) + Fy * T(CY[i]) + Fz * T(CZ[i]);
                                cos2 = (Fc * Fc) / (absF * absF);
                            }
                            const T Om2 = Ahalf * absF * (L.w[i] * cos2 - L.B[i]);
                            const T gi = Om1 + Om2;
                            // collisionOperators.cuh:28-69
                            T Delta = 0;
                            if (i != 0) {
                                const T rho = rr + rb;
                                const T fieq0 = L.w[i] * rho;
                                T Cos = 0;
                                if (!(absF <= T(1.0e-4))) {
                                    const T invF = T(1.0) / absF;
                                    const T dot = Fx * T(CX[i]) + Fy * T(CY[i]) + Fz * T(CZ[i]);
                                    Cos = dot * invF * L.invc[i];
                                }
                                const T coeff = beta * ((rr * rb) / (rho * rho));
                                Delta = coeff * Cos * fieq0;
                            }
                            fr[t] = aR * gi + Delta;
                            fb[t] = aB * gi - Delta;
                        }
                    }
                }
    }

    // Inlet velocity of a jet column: the top-hat U, times the column's radial
    // profile multiplier when one is set, times the seeded perturbation
    // (extensions; U itself when neither is set).
    T inlet_uy(int x, int z) const {
        T U = jet_velocity;
        if (!inlet_prof.empty()) U = U * inlet_prof[size_t(z) * NX + x];
        if (p.inlet_noise == 0.0f) return U;
        const float u = hash_uniform(p.seed, 0x1A1E7ull ^ uint64_t(step), uint64_t(x), uint64_t(z));
        const float f = 1.0f + (2.0f * u - 1.0f) * p.inlet_noise;
        return U * T(f);
    }

    // jet/boundary_conditions.cuh:17-85 over interior x,z (kernels.cu:98-114)
    void inlet() {
        const long off_z = long(NX) * NY;
        for (int z = 1; z <= NZ - 2; ++z)
            for (int x = 1; x <= NX - 2; ++x) {
                const size_t idB = idx(x, 0, z), idF = idx(x, 1, z);
                const bool j = isJet(x, z);
                rhor[idB] = (T(1.0) - (j ? T(1) : T(0))) * rhor0;
                rhob[idB] = (j ? T(1) : T(0)) * rhob0;
                if (!j) continue;
                const T rT = rhor[idB] + rhob[idB];
                const T uyb = inlet_uy(x, z);
                const T aR = rhor[idB] * (T(1) / rT), aB = rhob[idB] * (T(1) / rT);
                const T oms = T(1.0) - omegab;
                for (int i = 0; i < Q; ++i) {
                    if (CY[i] != 1) continue;
                    const size_t node = size_t(long(idF) + CX[i] + off_z * CZ[i]);  // no wrap
                    const T g = feq(i, rT, T(0), uyb, T(0)) +
                                oms * fneqr(i, Pixx[idF], Pixy[idF], Piyy[idF], Piyz[idF], Pizz[idF], Pixz[idF],
                                            ux[idF], uy[idF], uz[idF]);
                    fr[fidx(node, i)] = aR * g;
                    fb[fidx(node, i)] = aB * g;
                }
            }
    }

    // jet/boundary_conditions.cuh:163-233 over interior x,z (kernels.cu:116-132)
    void neumann() {
        const long off_z = long(NX) * NY;
        const T oms = T(1.0) - omega_sponge(NY - 2);
        for (int z = 1; z <= NZ - 2; ++z)
            for (int x = 1; x <= NX - 2; ++x) {
                const size_t idB = idx(x, NY - 1, z), idF = idx(x, NY - 2, z);
                const T uc = clamp01(uy[idF]);
                auto conv = [&](T b, T f) { return b - uc * (b - f); };
                const T rrB = conv(rhor[idB], rhor[idF]);
                const T rbB = conv(rhob[idB], rhob[idF]);
                const T uxB = conv(ux[idB], ux[idF]);
                const T uyB = conv(uy[idB], uy[idF]);
                const T uzB = conv(uz[idB], uz[idF]);
                rhor[idB] = rrB; rhob[idB] = rbB; ux[idB] = uxB; uy[idB] = uyB; uz[idB] = uzB;
                const T rhoT = rrB + rbB;
                const T inv = T(1.0) / rhoT;
                const T aR = rrB * inv, aB = rbB * inv;
                for (int i = 0; i < Q; ++i) {
                    if (CY[i] != -1) continue;
                    const size_t node = size_t(long(idF) + CX[i] + off_z * CZ[i]);  // no wrap
                    const T g = feq(i, rhoT, uxB, uyB, uzB) +
                                oms * fneqr(i, Pixx[idF], Pixy[idF], Piyy[idF], Piyz[idF], Pizz[idF], Pixz[idF],
                                            ux[idF], uy[idF], uz[idF]);
                    fr[fidx(node, i)] = aR * g;
                    fb[fidx(node, i)] = aB * g;
                }
            }
    }

    // kernels.cu:188-233 (float geometry, double sums)
    void accumulate_radial() {
#pragma omp parallel for schedule(static)
        for (int y = 1; y <= NY - 2; ++y)
            for (int z = 1; z <= NZ - 2; ++z)
                for (int x = 1; x <= NX - 2; ++x) {
                    const float dx = float(x) - p.jet_x0, dz = float(z) - p.jet_z0;
                    const float r = std::sqrt(dx * dx + dz * dz);
                    const uint32_t rb = static_cast<uint32_t>(r);
                    if (rb >= uint32_t(NRB)) continue;
                    const size_t id = idx(x, y, z);
                    const size_t m = size_t(y) * NRB + rb;
                    const double vy = double(uy[id]);
                    double vr = 0.0;
                    if (r > 1.0e-12f) vr = double((ux[id] * T(dx) + uz[id] * T(dz)) / T(r));
                    s_uy[m] += vy;
                    s_uy2[m] += vy * vy;
                    s_ur[m] += vr;
                    s_ur2[m] += vr * vr;
                    s_uruy[m] += vr * vy;
                    cnt[m] += 1;
                }
    }

    // kernels.cu:136-152 (sum in double)
    double total_tke() const {
        double s = 0;
        for (int z = 1; z <= NZ - 2; ++z)
            for (int y = 1; y <= NY - 2; ++y)
                for (int x = 1; x <= NX - 2; ++x) {
                    const size_t id = idx(x, y, z);
                    s += double(T(0.5) * (ux[id] * ux[id] + uy[id] * uy[id] + uz[id] * uz[id]));
                }
        return s;
    }

    // kernels.cu:168-186
    void update_uy_average() {
        const T c = T(uy_avg_count);
        for (int z = 1; z <= NZ - 2; ++z)
            for (int y = 1; y <= NY - 2; ++y)
                for (int x = 1; x <= NX - 2; ++x) {
                    const size_t id = idx(x, y, z);
                    uy_avg[id] = (uy_avg[id] * c + uy[id]) / (c + T(1));
                }
        ++uy_avg_count;
    }

    // main.cu:52-82 without the output block
    void run(int nsteps) {
        for (int n = 0; n < nsteps; ++n) {
            macros();
            bool acc = false;
            if (stats_mode == 1) {
                if (!stats_started) { stats_started = true; stats_start_step = uint32_t(step); stats_samples = 0; }
                acc = true;
            } else if (stats_mode == -1) {
                if (!stats_started && step >= p.NSTATS_START_STEP) {
                    stats_started = true;
                    stats_start_step = uint32_t(step);
                    stats_samples = 0;
                }
                acc = stats_started;
            }
            if (acc) { accumulate_radial(); ++stats_samples; }
            collistream();
            if (p.boundary == MCG_BOUNDARY_JET) { inlet(); neumann(); }
            ++step;
        }
    }

    // ---------------------------------------------------------------- adjoint
    // Discrete adjoint of `nsteps` steps of the periodic box in this class's own
    // form (push into one buffer): for J = sum over interior nodes of
    // (psi_T - target)^2 with psi_T the colour field of f(T), returns J,
    // dJ/dsigma, dJ/dtau and dJ/du0 of an initial state f0 = feq(rho_c, u0).
    // Step t maps f_t -> f_{t+1} by f_{t+1,i}(x + c_i) = C_i(M_t(x), F_t(x)); the
    // reverse step takes lambda of the pushed values, the collision's Jacobian
    // at each node (M and F), the gradient stencil's transpose and the moments'
    // transpose.  The state is left at f(0).
    void adjoint_periodic(const double *target, int nsteps, double out[3], double *du0) {
        const size_t NQ = size_t(Q) * N;
        std::vector<std::vector<T>> hr(size_t(nsteps) + 1), hb(size_t(nsteps) + 1);
        hr[0] = fr;
        hb[0] = fb;
        const int64_t step0 = step;
        for (int t = 0; t < nsteps; ++t) {
            run(1);
            hr[size_t(t) + 1] = fr;
            hb[size_t(t) + 1] = fb;
        }
        std::vector<double> lr(NQ, 0.0), lb(NQ, 0.0), nr(NQ, 0.0), nb(NQ, 0.0);
        std::vector<double> lm(size_t(11) * N, 0.0), lF(size_t(3) * N, 0.0);
        double Jv = 0, a_omega = 0, a_Ah = 0;
        auto load = [&](int t) {
            fr = hr[size_t(t)];
            fb = hb[size_t(t)];
            macros();  // moments of f(t); ghost densities mirrored
        };
        // terminal: lambda of f(T) from J
        load(nsteps);
        for (int z = 1; z <= NZ - 2; ++z)
            for (int y = 1; y <= NY - 2; ++y)
                for (int x = 1; x <= NX - 2; ++x) {
                    const size_t id = idx(x, y, z);
                    const double rr = double(rhor[id]), rb = double(rhob[id]), rho = rr + rb;
                    const double d = (rr - rb) / rho - target[id];
                    Jv += d * d;
                    const double lrr = 2 * d * 2 * rb / (rho * rho), lrb = -2 * d * 2 * rr / (rho * rho);
                    for (int i = 0; i < Q; ++i) {
                        lr[fidx(id, i)] = lrr;
                        lb[fidx(id, i)] = lrb;
                    }
                }
        const double A = double(sigma_over_4cs4 / taub), Ah = A / 2;
        for (int t = nsteps - 1; t >= 0; --t) {
            load(t);
            std::fill(lF.begin(), lF.end(), 0.0);
            // collision adjoint at every interior node
            for (int z = 1; z <= NZ - 2; ++z)
                for (int y = 1; y <= NY - 2; ++y)
                    for (int x = 1; x <= NX - 2; ++x) {
                        const size_t id = idx(x, y, z);
                        const double rr = rhor[id], rb = rhob[id], rho = rr + rb;
                        const double vx = ux[id], vy = uy[id], vz = uz[id];
                        const double pxx = Pixx[id], pxy = Pixy[id], pyy = Piyy[id], pyz = Piyz[id],
                                     pzz = Pizz[id], pxz = Pixz[id];
                        const double usq = vx * vx + vy * vy + vz * vz;
                        const double aR = rr / rho, aB = rb / rho;
                        const double oms = 1.0 - double(omega_sponge(y));
                        const bool iface = !(4.0 * rr * rb / (rho * rho) <= 1e-4);
                        double Fx = 0, Fy = 0, Fz = 0, absF = 0;
                        if (iface) {
                            T fx, fy, fz;
                            colour_gradient(id, fx, fy, fz);
                            Fx = fx; Fy = fy; Fz = fz;
                            absF = std::sqrt(Fx * Fx + Fy * Fy + Fz * Fz);
                        }
                        const bool hd = iface && !(absF <= 1e-4);
                        const double K = beta * rr * rb / rho;
                        // third-order terms of fneq (lbm.cuh:67-73)
                        const double a3[7] = {pxx * vy + 2 * pxy * vx, pxx * vz + 2 * pxz * vx, pyy * vx + 2 * pxy * vy,
                                              pzz * vx + 2 * pxz * vz, pyy * vz + 2 * pyz * vy, pzz * vy + 2 * pyz * vz,
                                              pxy * vz + pxz * vy + pyz * vx};
                        double l_aR = 0, l_aB = 0, l_rhoeq = 0, luP[3] = {0, 0, 0}, luQ = 0, l_oms = 0;
                        double S2[6] = {0, 0, 0, 0, 0, 0}, S3[7] = {0, 0, 0, 0, 0, 0, 0};
                        double sA[3] = {0, 0, 0}, sB = 0, sD[3] = {0, 0, 0}, sE = 0, sBB = 0, l_Ah = 0;
                        for (int i = 0; i < Q; ++i) {
                            const double cx = CX[i], cy = CY[i], cz = CZ[i];
                            const size_t tgt = fidx(idx(wrapx(x + CX[i]), wrapy(y + CY[i]), wrapz(z + CZ[i])), i);
                            const double Lr = lr[tgt], Lb = lb[tgt];
                            const double w = L.w[i];
                            const double cu = cx * vx + cy * vy + cz * vz;
                            const double fe = w * rho *
                                              (1 + cu * cu / (2 * double(L.cs4)) - usq / (2 * double(L.cs2)) +
                                               cu / double(L.cs2) + cu * (cu * cu / (6 * double(L.cs6)) - usq / (2 * double(L.cs4))));
                            const double H2[6] = {L.Hxx[i], L.Hxy[i], L.Hyy[i], L.Hyz[i], L.Hzz[i], L.Hxz[i]};
                            const double H3[7] = {L.Hxxy[i], L.Hxxz[i], L.Hxyy[i], L.Hxzz[i], L.Hyyz[i], L.Hyzz[i], L.Hxyz[i]};
                            const double A2 = (pxx * H2[0] + 2 * pxy * H2[1] + pyy * H2[2] + 2 * pyz * H2[3] + pzz * H2[4] +
                                               2 * pxz * H2[5]) / (2 * double(L.cs4));
                            double A3 = 0;
                            for (int k = 0; k < 6; ++k) A3 += a3[k] * H3[k];
                            A3 += 2 * a3[6] * H3[6];
                            const double fn = w * (A2 + A3 / (2 * double(L.cs6)));
                            const double fc = Fx * cx + Fy * cy + Fz * cz;
                            double om2A = 0;  // Omega2 / (A/2)
                            if (iface) om2A = absF * (w * ((i != 0 && hd) ? fc * fc / (absF * absF) : 0.0) - double(L.B[i]));
                            const double gi = fe + oms * fn + Ah * om2A;
                            l_aR += Lr * gi;
                            l_aB += Lb * gi;
                            const double lg = aR * Lr + aB * Lb, ld = Lr - Lb;
                            l_rhoeq += lg * fe;
                            const double P = 1 / double(L.cs2) + cu / double(L.cs4) + cu * cu / (2 * double(L.cs6)) -
                                             usq / (2 * double(L.cs4));
                            const double Qd = 1 / double(L.cs2) + cu / double(L.cs4);
                            const double wl = lg * w * rho;
                            luP[0] += wl * P * cx;
                            luP[1] += wl * P * cy;
                            luP[2] += wl * P * cz;
                            luQ += wl * Qd;
                            l_oms += lg * fn;
                            const double mu = oms * lg * w;
                            for (int k = 0; k < 6; ++k) S2[k] += mu * H2[k];
                            for (int k = 0; k < 7; ++k) S3[k] += mu * H3[k];
                            if (iface) {
                                sBB += lg * double(L.B[i]);
                                l_Ah += lg * om2A;
                                if (i != 0 && hd) {
                                    const double a = lg * w * fc, dd = ld * w * double(L.invc[i]);
                                    sA[0] += a * cx; sA[1] += a * cy; sA[2] += a * cz;
                                    sD[0] += dd * cx; sD[1] += dd * cy; sD[2] += dd * cz;
                                    sB += a * fc;
                                    sE += dd * fc;
                                }
                            }
                        }
                        const double c2 = 1 / (2 * double(L.cs4)), c3 = 1 / (2 * double(L.cs6));
                        double lP[6] = {S2[0] * c2, 2 * S2[1] * c2, S2[2] * c2, 2 * S2[3] * c2, S2[4] * c2, 2 * S2[5] * c2};
                        const double la[7] = {S3[0] * c3, S3[1] * c3, S3[2] * c3, S3[3] * c3, S3[4] * c3, S3[5] * c3,
                                              2 * S3[6] * c3};
                        // a3: xxy, xxz, xyy, xzz, yyz, yzz, xyz
                        lP[0] += la[0] * vy + la[1] * vz;
                        lP[2] += la[2] * vx + la[4] * vz;
                        lP[4] += la[3] * vx + la[5] * vy;
                        lP[1] += 2 * la[0] * vx + 2 * la[2] * vy + la[6] * vz;
                        lP[5] += 2 * la[1] * vx + 2 * la[3] * vz + la[6] * vy;
                        lP[3] += 2 * la[4] * vy + 2 * la[5] * vz + la[6] * vx;
                        double lu[3];
                        lu[0] = 2 * la[0] * pxy + 2 * la[1] * pxz + la[2] * pyy + la[3] * pzz + la[6] * pyz + luP[0] - vx * luQ;
                        lu[1] = la[0] * pxx + 2 * la[2] * pxy + 2 * la[4] * pyz + la[5] * pzz + la[6] * pxz + luP[1] - vy * luQ;
                        lu[2] = la[1] * pxx + 2 * la[3] * pxz + la[4] * pyy + 2 * la[5] * pyz + la[6] * pxy + luP[2] - vz * luQ;
                        double lK = 0;
                        if (iface) {
                            if (hd) {
                                const double i1 = 1 / absF, i3 = i1 * i1 * i1;
                                const double FF[3] = {Fx, Fy, Fz};
                                for (int k = 0; k < 3; ++k)
                                    lF[k * N + id] = Ah * (2 * i1 * sA[k] - FF[k] * i3 * sB - FF[k] * i1 * sBB) +
                                                     K * (sD[k] * i1 - FF[k] * i3 * sE);
                                lK = sE * i1;
                            } else if (absF > 0) {
                                const double q = -Ah * sBB / absF;
                                lF[0 * N + id] = q * Fx; lF[1 * N + id] = q * Fy; lF[2 * N + id] = q * Fz;
                            }
                        }
                        const double inv2 = 1 / (rho * rho);
                        lm[0 * N + id] = l_rhoeq / rho + (l_aR - l_aB) * rb * inv2 + lK * beta * rb * rb * inv2;
                        lm[1 * N + id] = l_rhoeq / rho - (l_aR - l_aB) * rr * inv2 + lK * beta * rr * rr * inv2;
                        for (int k = 0; k < 3; ++k) lm[(2 + k) * N + id] = lu[k];
                        for (int k = 0; k < 6; ++k) lm[(5 + k) * N + id] = lP[k];
                        a_omega -= l_oms;
                        a_Ah += l_Ah;
                    }
            // moments adjoint: psi gathered from the neighbours' F adjoints, then f(t)
            for (int z = 1; z <= NZ - 2; ++z)
                for (int y = 1; y <= NY - 2; ++y)
                    for (int x = 1; x <= NX - 2; ++x) {
                        const size_t id = idx(x, y, z);
                        const double rr = rhor[id], rb = rhob[id], rho = rr + rb;
                        const double vx = ux[id], vy = uy[id], vz = uz[id];
                        double lpsi = 0;
                        for (int j = 1; j < Q; ++j) {
                            const size_t nid = idx(wrapx(x - CX[j]), wrapy(y - CY[j]), wrapz(z - CZ[j]));
                            lpsi += double(L.w[j]) *
                                    (CX[j] * lF[0 * N + nid] + CY[j] * lF[1 * N + nid] + CZ[j] * lF[2 * N + nid]);
                        }
                        lpsi /= double(L.cs2);
                        const double lrr = lm[0 * N + id] + lpsi * 2 * rb / (rho * rho);
                        const double lrb = lm[1 * N + id] - lpsi * 2 * rr / (rho * rho);
                        const double lP[6] = {lm[5 * N + id], lm[6 * N + id], lm[7 * N + id],
                                              lm[8 * N + id], lm[9 * N + id], lm[10 * N + id]};
                        const double lux = lm[2 * N + id] - rho * (2 * vx * lP[0] + vy * lP[1] + vz * lP[5]);
                        const double luy = lm[3 * N + id] - rho * (2 * vy * lP[2] + vx * lP[1] + vz * lP[3]);
                        const double luz = lm[4 * N + id] - rho * (2 * vz * lP[4] + vx * lP[5] + vy * lP[3]);
                        double lrho = -(lP[0] * vx * vx + lP[1] * vx * vy + lP[2] * vy * vy + lP[3] * vy * vz +
                                        lP[4] * vz * vz + lP[5] * vx * vz);
                        lrho -= (lux * vx + luy * vy + luz * vz) / rho;
                        for (int i = 0; i < Q; ++i) {
                            const double lgi = lP[0] * L.Hxx[i] + lP[1] * L.Hxy[i] + lP[2] * L.Hyy[i] + lP[3] * L.Hyz[i] +
                                               lP[4] * L.Hzz[i] + lP[5] * L.Hxz[i] +
                                               (CX[i] * lux + CY[i] * luy + CZ[i] * luz) / rho + lrho;
                            nr[fidx(id, i)] = lrr + lgi;
                            nb[fidx(id, i)] = lrb + lgi;
                        }
                    }
            std::swap(lr, nr);
            std::swap(lb, nb);
        }
        // dJ/du0 of f0 = feq(rho_c, u0); the moments of f(0) are loaded
        for (size_t k = 0; k < size_t(3) * N; ++k) du0[k] = 0;
        for (int z = 1; z <= NZ - 2; ++z)
            for (int y = 1; y <= NY - 2; ++y)
                for (int x = 1; x <= NX - 2; ++x) {
                    const size_t id = idx(x, y, z);
                    const double rr = rhor[id], rb = rhob[id];
                    const double vx = ux[id], vy = uy[id], vz = uz[id], usq = vx * vx + vy * vy + vz * vz;
                    double gx = 0, gy = 0, gz = 0, gq = 0;
                    for (int i = 0; i < Q; ++i) {
                        const double cu = CX[i] * vx + CY[i] * vy + CZ[i] * vz;
                        const double P = 1 / double(L.cs2) + cu / double(L.cs4) + cu * cu / (2 * double(L.cs6)) -
                                         usq / (2 * double(L.cs4));
                        const double Qd = 1 / double(L.cs2) + cu / double(L.cs4);
                        const double wl = double(L.w[i]) * (lr[fidx(id, i)] * rr + lb[fidx(id, i)] * rb);
                        gx += wl * P * CX[i];
                        gy += wl * P * CY[i];
                        gz += wl * P * CZ[i];
                        gq += wl * Qd;
                    }
                    du0[id] = gx - vx * gq;
                    du0[N + id] = gy - vy * gq;
                    du0[2 * N + id] = gz - vz * gq;
                }
        // omega = 1/tau (nu = (tau - 1/2) cs^2), A/2 = sigma / (8 cs^4 tau)
        const double omega = double(omega_sponge(1)), tau = double(taub);
        out[0] = Jv;
        out[1] = a_Ah / (8 * double(L.cs4) * tau);
        out[2] = a_omega * (-omega * omega) + a_Ah * (-Ah / tau);
        fr = hr[0];
        fb = hb[0];
        step = step0;
    }
};

struct Handle {
    int precision;
    void *o;
};

template <class T>
Oracle<T> &as(Handle *h) { return *static_cast<Oracle<T> *>(h->o); }

#define DISPATCH(h, ...)                         \
    do {                                         \
        if ((h)->precision == 32) {              \
            auto &O = as<float>(h);              \
            __VA_ARGS__;                         \
        } else {                                 \
            auto &O = as<double>(h);             \
            __VA_ARGS__;                         \
        }                                        \
    } while (0)

template <class V>
void copy_out(const V &v, double *dst) {
    if (dst) for (size_t k = 0; k < v.size(); ++k) dst[k] = double(v[k]);
}
template <class V>
void copy_in(V &v, const double *src) {
    using T = typename V::value_type;
    if (src) for (size_t k = 0; k < v.size(); ++k) v[k] = T(src[k]);
}

}  // namespace

extern "C" {

void *orc_create(const mcg_params *p, int precision) {
    if (!p || (precision != 32 && precision != 64) || p->NX < 3 || p->NY < 3 || p->NZ < 3) return nullptr;
    Handle *h = new Handle{precision, nullptr};
    if (precision == 32) h->o = new Oracle<float>(*p);
    else h->o = new Oracle<double>(*p);
    return h;
}

void orc_destroy(void *hv) {
    Handle *h = static_cast<Handle *>(hv);
    if (!h) return;
    if (h->precision == 32) delete &as<float>(h);
    else delete &as<double>(h);
    delete h;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void orc_init_jet(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.init_jet()); }
void orc_init_bubble(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.init_bubble()); }

void orc_set_pops(void *hv, const double *fr, const double *fb) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, (copy_in(O.fr, fr), copy_in(O.fb, fb)));
}
void orc_get_pops(void *hv, double *fr, double *fb) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, (copy_out(O.fr, fr), copy_out(O.fb, fb)));
}
void orc_set_fields(void *hv, const double *rr, const double *rb, const double *vx, const double *vy,
                    const double *vz) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, (copy_in(O.rhor, rr), copy_in(O.rhob, rb), copy_in(O.ux, vx), copy_in(O.uy, vy), copy_in(O.uz, vz)));
}
// Discrete adjoint of the periodic box (see Oracle::adjoint_periodic).
// out: J, dJ/dsigma, dJ/dtau; du0: 3*Ncells.  Returns 0, or -1 if the case is
// not the periodic box.
int orc_adjoint_periodic(void *hv, const double *target, int nsteps, double *out, double *du0) {
    Handle *h = static_cast<Handle *>(hv);
    int rc = 0;
    DISPATCH(h, (O.periodic() ? (O.adjoint_periodic(target, nsteps, out, du0), 0) : (rc = -1)));
    return rc;
}

// Per-column inlet velocity multipliers (NX*NZ, x fastest); NULL restores the top-hat.
void orc_set_inlet_profile(void *hv, const double *prof) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, (prof ? (O.inlet_prof.assign(prof, prof + size_t(O.NX) * O.NZ), 0) : (O.inlet_prof.clear(), 0)));
}
void orc_get_fields(void *hv, double *rr, double *rb, double *vx, double *vy, double *vz) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, (copy_out(O.rhor, rr), copy_out(O.rhob, rb), copy_out(O.ux, vx), copy_out(O.uy, vy),
                 copy_out(O.uz, vz)));
}
void orc_get_stress(void *hv, double *pi6) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, {
        const size_t n = O.N;
        copy_out(O.Pixx, pi6);
        copy_out(O.Pixy, pi6 + n);
        copy_out(O.Piyy, pi6 + 2 * n);
        copy_out(O.Piyz, pi6 + 3 * n);
        copy_out(O.Pizz, pi6 + 4 * n);
        copy_out(O.Pixz, pi6 + 5 * n);
    });
}

void orc_macros(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.macros()); }
void orc_collistream(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, (O.collistream(), ++O.step)); }
void orc_inlet(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.inlet()); }
void orc_neumann(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.neumann()); }
void orc_accumulate_radial(void *hv) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, (O.accumulate_radial(), ++O.stats_samples));
}
void orc_set_stats_mode(void *hv, int mode) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.stats_mode = mode); }
void orc_step(void *hv, int nsteps) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.run(nsteps)); }
long long orc_get_step(void *hv) {
    Handle *h = static_cast<Handle *>(hv);
    long long s = 0;
    DISPATCH(h, s = O.step);
    return s;
}
void orc_get_radial(void *hv, double *sums5, uint64_t *count) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, {
        const size_t m = O.s_uy.size();
        if (sums5) {
            std::memcpy(sums5, O.s_uy.data(), m * 8);
            std::memcpy(sums5 + m, O.s_uy2.data(), m * 8);
            std::memcpy(sums5 + 2 * m, O.s_ur.data(), m * 8);
            std::memcpy(sums5 + 3 * m, O.s_ur2.data(), m * 8);
            std::memcpy(sums5 + 4 * m, O.s_uruy.data(), m * 8);
        }
        if (count) std::memcpy(count, O.cnt.data(), m * 8);
    });
}
void orc_get_radial_state(void *hv, int *started, unsigned *start_step, unsigned *samples) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, {
        *started = O.stats_started ? 1 : 0;
        *start_step = O.stats_start_step;
        *samples = O.stats_samples;
    });
}
double orc_total_tke(void *hv) {
    Handle *h = static_cast<Handle *>(hv);
    double s = 0;
    DISPATCH(h, s = O.total_tke());
    return s;
}
void orc_update_uy_average(void *hv) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, O.update_uy_average()); }
void orc_get_uy_average(void *hv, double *out) { Handle *h = static_cast<Handle *>(hv); DISPATCH(h, copy_out(O.uy_avg, out)); }

// Float64 sums over interior nodes of the populations: mass red, mass blue, momentum.
void orc_conservation_sums(void *hv, double out[5]) {
    Handle *h = static_cast<Handle *>(hv);
    DISPATCH(h, {
        double s[5] = {0, 0, 0, 0, 0};
        for (int z = 1; z <= O.NZ - 2; ++z)
            for (int y = 1; y <= O.NY - 2; ++y)
                for (int x = 1; x <= O.NX - 2; ++x) {
                    const size_t id = O.idx(x, y, z);
                    for (int i = 0; i < Q; ++i) {
                        const double a = double(O.fr[O.fidx(id, i)]), b = double(O.fb[O.fidx(id, i)]);
                        s[0] += a;
                        s[1] += b;
                        s[2] += (a + b) * CX[i];
                        s[3] += (a + b) * CY[i];
                        s[4] += (a + b) * CZ[i];
                    }
                }
        for (int k = 0; k < 5; ++k) out[k] = s[k];
    });
}

// Seeded hash shared with the product's device code (same formula, restated).
float orc_hash_uniform(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) { return hash_uniform(seed, a, b, c); }

}  // extern "C"
