// kernels.cu - the D3Q27 colour-gradient step on B200 (sm_100a).
//
// One step is two HBM passes over the lattice plus a plane-sized launch:
//   k_moments  pulls f(t) from pops[cur] (27+27 coalesced loads per node),
//              forms rho_r, rho_b, u, Pi^neq (lbm.cuh:82-165) and psi, and in
//              the same pass accumulates the radial statistics
//              (kernels.cu:188-233) with warp segmented reductions instead of
//              six global atomics per node.
//   k_boundary the inlet (jet/boundary_conditions.cuh:17-85) and convective
//              outlet (jet/boundary_conditions.cuh:163-233) of the same step,
//              one thread per boundary column; the values land in the y ghost
//              planes of pops[cur^1].
//   k_collide  relaxes every node (lbm.cuh:184-293): Hermite-regularised BGK,
//              colour-gradient perturbation and recolouring, with the
//              gradient from the 26 neighbouring psi values, and stores the
//              54 post-collision values at the node itself in pops[cur^1]
//              (fully coalesced stores; the next k_moments pulls them).
// The reference's in-place push buffer becomes a ping-pong pull pair; the
// populations a reference step never rewrites (y=1 slots fed by non-jet
// inlet columns, y=NY-2 slots fed by ghost columns) are the ghost-plane
// values of both buffers that no kernel writes, so results are the same.
#include <cuda_fp16.h>

#include "kernels.cuh"
#include "lattice.cuh"

namespace mcg {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ storage codecs

struct CodecF32 {
    const float *__restrict__ rd;
    float *__restrict__ wr;
    uint32_t N;
    template <int I>
    __device__ __forceinline__ void load(uint32_t s, float &r, float &b) const {
        r = __ldg(rd + size_t(I) * N + s);
        b = __ldg(rd + size_t(kQ + I) * N + s);
    }
    template <int I>
    __device__ __forceinline__ void store(uint32_t id, float r, float b) const {
        wr[size_t(I) * N + id] = r;
        wr[size_t(kQ + I) * N + id] = b;
    }
    // Write into a buffer other than wr (initialisation).
    __device__ __forceinline__ static void store_to(void *buf, uint32_t N, int i, uint32_t id, float r, float b,
                                                    float) {
        float *p = static_cast<float *>(buf);
        p[size_t(i) * N + id] = r;
        p[size_t(kQ + i) * N + id] = b;
    }
    __device__ __forceinline__ static void load_from(const void *buf, uint32_t N, int i, uint32_t s, float &r,
                                                     float &b, float) {
        const float *p = static_cast<const float *>(buf);
        r = p[size_t(i) * N + s];
        b = p[size_t(kQ + i) * N + s];
    }
};

// F16 word per (direction, node): x = g/w_i - rho0 (total offset by the rest
// equilibrium and scaled by 1/w_i), y = q, the minority-colour fraction
// 2 min(fr,fb)/g carrying the sign of fr-fb.  Pure nodes store q = +-0
// exactly, so a single-colour region keeps exactly zero of the other colour.
__device__ __forceinline__ __half2 f16_encode(float r, float b, float inv_w, float rho0) {
    const float g = r + b;
    const float h0 = g * inv_w - rho0;
    const float mn = fminf(r, b);
    float q = (g > 0.0f) ? __fdividef(2.0f * mn, g) : 0.0f;
    q = copysignf(fmaxf(q, 0.0f), r - b);
    return __floats2half2_rn(h0, q);
}
__device__ __forceinline__ void f16_decode(__half2 h, float w, float rho0, float &r, float &b) {
    const float2 v = __half22float2(h);
    const float g = w * (rho0 + v.x);
    const float minor = 0.5f * g * fabsf(v.y);
    const bool red_major = !signbit(v.y);
    r = red_major ? g - minor : minor;
    b = red_major ? minor : g - minor;
}

struct CodecF16 {
    const __half2 *__restrict__ rd;
    __half2 *__restrict__ wr;
    uint32_t N;
    float rho0;
    template <int I>
    __device__ __forceinline__ void load(uint32_t s, float &r, float &b) const {
        const __half2 h = __ldg(rd + size_t(I) * N + s);
        f16_decode(h, Dir<I>::w, rho0, r, b);
    }
    template <int I>
    __device__ __forceinline__ void store(uint32_t id, float r, float b) const {
        wr[size_t(I) * N + id] = f16_encode(r, b, 1.0f / Dir<I>::w, rho0);
    }
    __device__ __forceinline__ static void store_to(void *buf, uint32_t N, int i, uint32_t id, float r, float b,
                                                    float rho0) {
        static_cast<__half2 *>(buf)[size_t(i) * N + id] = f16_encode(r, b, 1.0f / dir_w(i), rho0);
    }
    __device__ __forceinline__ static void load_from(const void *buf, uint32_t N, int i, uint32_t s, float &r,
                                                     float &b, float rho0) {
        f16_decode(static_cast<const __half2 *>(buf)[size_t(i) * N + s], dir_w(i), rho0, r, b);
    }
};

template <class C>
__host__ __device__ C make_codec(const DeviceState &s, int cur);
template <>
__host__ __device__ CodecF32 make_codec<CodecF32>(const DeviceState &s, int cur) {
    return CodecF32{static_cast<const float *>(s.pops[cur]), static_cast<float *>(s.pops[cur ^ 1]), s.g.N};
}
template <>
__host__ __device__ CodecF16 make_codec<CodecF16>(const DeviceState &s, int cur) {
    return CodecF16{static_cast<const __half2 *>(s.pops[cur]), static_cast<__half2 *>(s.pops[cur ^ 1]), s.g.N,
                    s.ph.f16_rho0};
}

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ float psi_of(float a, float b) { return (a - b) / (a + b); }  // mathUtilities.cuh:24-28

__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// Relaxation rate at height y (mathUtilities.cuh:56-90); constant when K == 0.
__device__ __forceinline__ float omega_at(const Physics &ph, int y) {
    if (!ph.sponge) return ph.omega;
    const float s = clamp01((float(y) - ph.sponge_y_start) * ph.sponge_inv_width);
    const float nus = ph.nu * (1.0f + ph.sponge_K * (s * s * s));
    return 1.0f / (0.5f + nus * kInvCs2);
}

__device__ __forceinline__ bool is_jet_column(const Physics &ph, int x, int z) {  // mathUtilities.cuh:14-21
    const float dx = float(x) - ph.jet_x0, dz = float(z) - ph.jet_z0;
    return dx * dx + dz * dz <= ph.jet_r2;
}

__device__ __forceinline__ float inlet_velocity(const Physics &ph, int64_t step, int x, int z) {
    if (ph.inlet_noise == 0.0f) return ph.jet_velocity;
    const float u = hash_uniform(ph.seed, 0x1A1E7ull ^ uint64_t(step), uint64_t(x), uint64_t(z));
    return ph.jet_velocity * (1.0f + (2.0f * u - 1.0f) * ph.inlet_noise);
}

// Pull source of direction I for interior node (x,y,z) with id.
//  x and z are periodic over the interior through the ghost shell (the push
//  side wraps with bounds.cuh:23-60); y sources on a ghost plane are the
//  boundary's slots and are not wrapped (boundary writes are unwrapped,
//  boundary_conditions.cuh:73,137); in the periodic box y wraps too.
struct PullMap {
    int wxp, wxm, wzp, wzm, wyp, wym;
    bool gy_p, gy_m;
    __device__ __forceinline__ PullMap(const Geometry &g, int x, int y, int z, bool periodic) {
        wxp = (x == 1) ? (g.NX - 2) : 0;
        wxm = (x == g.NX - 2) ? -(g.NX - 2) : 0;
        wzp = (z == 1) ? g.sz * (g.NZ - 2) : 0;
        wzm = (z == g.NZ - 2) ? -g.sz * (g.NZ - 2) : 0;
        wyp = (periodic && y == 1) ? g.sy * (g.NY - 2) : 0;
        wym = (periodic && y == g.NY - 2) ? -g.sy * (g.NY - 2) : 0;
        gy_p = !periodic && y == 1;
        gy_m = !periodic && y == g.NY - 2;
    }
    template <int I>
    __device__ __forceinline__ uint32_t src(const Geometry &g, uint32_t id) const {
        using D = Dir<I>;
        int s = int(id) - (D::cx + g.sy * D::cy + g.sz * D::cz);
        bool ghost = false;
        if constexpr (D::cy == 1) ghost = gy_p;
        if constexpr (D::cy == -1) ghost = gy_m;
        int corr = 0;
        if constexpr (D::cx == 1) corr += wxp;
        if constexpr (D::cx == -1) corr += wxm;
        if constexpr (D::cz == 1) corr += wzp;
        if constexpr (D::cz == -1) corr += wzm;
        if (ghost) corr = 0;
        if constexpr (D::cy == 1) corr += wyp;
        if constexpr (D::cy == -1) corr += wym;
        return uint32_t(s + corr);
    }
};

// Same map for a runtime direction (init/gather kernels).
__device__ __forceinline__ uint32_t pull_src_rt(const Geometry &g, int x, int y, int z, int i) {
    const bool periodic = g.boundary == kBoundaryPeriodic;
    int xs = x - dir_cx(i), ys = y - dir_cy(i), zs = z - dir_cz(i);
    const bool ghost_plane = !periodic && (ys == 0 || ys == g.NY - 1);
    if (!ghost_plane) {
        if (xs == 0) xs = g.NX - 2;
        else if (xs == g.NX - 1) xs = 1;
        if (zs == 0) zs = g.NZ - 2;
        else if (zs == g.NZ - 1) zs = 1;
    }
    if (periodic) {
        if (ys == 0) ys = g.NY - 2;
        else if (ys == g.NY - 1) ys = 1;
    }
    return uint32_t(xs) + uint32_t(g.sy) * uint32_t(ys) + uint32_t(g.sz) * uint32_t(zs);
}

// Runtime-direction tables in constant memory for the non-hot kernels.
__constant__ int c_cx[kQ] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
__constant__ int c_cy[kQ] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
__constant__ int c_cz[kQ] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

// ------------------------------------------------------------------ boundary pieces

// Inlet column (x,z): density mask at y=0 and, for disc columns, the nine
// cy=+1 populations entering y=1 (jet/boundary_conditions.cuh:17-85).  They
// are stored in the ghost plane y=0 of `dst` at (x,0,z), where the y=1 nodes
// (x+cx, 1, z+cz) pull them.  `m` are the moments of fluid node (x,1,z).
template <class C>
__device__ __forceinline__ void inlet_column(const DeviceState &s, const C &codec_dst_only, void *dst, float *psi_dst,
                                             int x, int z, int64_t step, const NodeMoments &m) {
    const Geometry &g = s.g;
    const Physics &ph = s.ph;
    const uint32_t idB = uint32_t(x) + uint32_t(g.sz) * uint32_t(z);
    const bool jet = is_jet_column(ph, x, z);
    const float rrB = (1.0f - (jet ? 1.0f : 0.0f)) * ph.rhor0;
    const float rbB = (jet ? 1.0f : 0.0f) * ph.rhob0;
    s.mom[size_t(kMomRR) * g.N + idB] = rrB;
    s.mom[size_t(kMomRB) * g.N + idB] = rbB;
    psi_dst[idB] = psi_of(rrB, rbB);
    if (!jet) return;
    const float rT = rrB + rbB;
    const float aR = rrB * (1.0f / rT), aB = rbB * (1.0f / rT);
    const float oms = 1.0f - ph.omega_b;
    const EqTerms e = make_eq(0.0f, inlet_velocity(ph, step, x, z), 0.0f);
    const NeqTerms n = make_neq(m.pxx, m.pxy, m.pyy, m.pyz, m.pzz, m.pxz, m.ux, m.uy, m.uz);
    (void)codec_dst_only;
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (Dir<i>::cy == 1) {
            const float gi = feq<i>(rT, e) + oms * fneq<i>(n);
            C::store_to(dst, g.N, i, idB, aR * gi, aB * gi, ph.f16_rho0);
        }
    });
}

// Outlet column (x,z): convective update of the y=NY-1 state from fluid node
// F=(x,NY-2,z) and the nine cy=-1 populations entering y=NY-2
// (jet/boundary_conditions.cuh:163-233), stored in ghost plane y=NY-1 of dst.
template <class C>
__device__ __forceinline__ void outlet_column(const DeviceState &s, void *dst, float *psi_dst, int x, int z,
                                              const NodeMoments &m) {
    const Geometry &g = s.g;
    const Physics &ph = s.ph;
    const uint32_t idB = uint32_t(x) + uint32_t(g.sy) * uint32_t(g.NY - 1) + uint32_t(g.sz) * uint32_t(z);
    float *mom = s.mom;
    const size_t N = g.N;
    const float uc = clamp01(m.uy);
    auto conv = [uc](float b, float f) { return b - uc * (b - f); };
    const float rrB = conv(mom[kMomRR * N + idB], m.rr);
    const float rbB = conv(mom[kMomRB * N + idB], m.rb);
    const float uxB = conv(mom[kMomUX * N + idB], m.ux);
    const float uyB = conv(mom[kMomUY * N + idB], m.uy);
    const float uzB = conv(mom[kMomUZ * N + idB], m.uz);
    mom[kMomRR * N + idB] = rrB;
    mom[kMomRB * N + idB] = rbB;
    mom[kMomUX * N + idB] = uxB;
    mom[kMomUY * N + idB] = uyB;
    mom[kMomUZ * N + idB] = uzB;
    psi_dst[idB] = psi_of(rrB, rbB);
    const float rhoT = rrB + rbB;
    const float inv = 1.0f / rhoT;
    const float aR = rrB * inv, aB = rbB * inv;
    const float oms = 1.0f - omega_at(ph, g.NY - 2);
    const EqTerms e = make_eq(uxB, uyB, uzB);
    const NeqTerms n = make_neq(m.pxx, m.pxy, m.pyy, m.pyz, m.pzz, m.pxz, m.ux, m.uy, m.uz);
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (Dir<i>::cy == -1) {
            const float gi = feq<i>(rhoT, e) + oms * fneq<i>(n);
            C::store_to(dst, g.N, i, idB, aR * gi, aB * gi, ph.f16_rho0);
        }
    });
}

// ------------------------------------------------------------------ radial statistics

// Warp-collective: one warp = 32 consecutive x at fixed (y,z).  Lanes with the
// same radial bin form contiguous runs once split by the side of the jet axis
// (the bin is monotone in |x - x0| on each side), so a segmented scan leaves
// each run's sums in its last lane, which issues one float64 atomic per sum.
// Counts are not accumulated per node: every sample adds the fixed number of
// interior columns of a bin, so they are materialised on read.
__device__ __forceinline__ void radial_accumulate_warp(const DeviceState &s, int x, int y, int z, bool active,
                                                       float ux, float uy, float uz) {
    const Physics &ph = s.ph;
    const int lane = threadIdx.x & 31;
    unsigned key = 0xffffffffu;
    double v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0;
    if (active) {
        const float dx = float(x) - ph.jet_x0, dz = float(z) - ph.jet_z0;
        const float r = sqrtf(dx * dx + dz * dz);
        const unsigned rb = unsigned(r);
        if (rb < unsigned(ph.NRB)) {
            key = (rb << 1) | (dx < 0.0f ? 1u : 0u);
            float ur = 0.0f;
            if (r > 1.0e-12f) ur = (ux * dx + uz * dz) / r;
            const double duy = double(uy), dur = double(ur);
            v0 = duy;
            v1 = duy * duy;
            v2 = dur;
            v3 = dur * dur;
            v4 = dur * duy;
        }
    }
    if (__all_sync(kFull, key == 0xffffffffu)) return;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned ok = __shfl_up_sync(kFull, key, d);
        const double o0 = __shfl_up_sync(kFull, v0, d);
        const double o1 = __shfl_up_sync(kFull, v1, d);
        const double o2 = __shfl_up_sync(kFull, v2, d);
        const double o3 = __shfl_up_sync(kFull, v3, d);
        const double o4 = __shfl_up_sync(kFull, v4, d);
        if (lane >= d && ok == key) {
            v0 += o0; v1 += o1; v2 += o2; v3 += o3; v4 += o4;
        }
    }
    const unsigned next = __shfl_down_sync(kFull, key, 1);
    const bool tail = (lane == 31) || (next != key);
    if (tail && key != 0xffffffffu) {
        const size_t M = size_t(s.g.NY) * ph.NRB;
        const size_t m = size_t(y) * ph.NRB + (key >> 1);
        atomicAdd(s.radial + m, v0);
        atomicAdd(s.radial + M + m, v1);
        atomicAdd(s.radial + 2 * M + m, v2);
        atomicAdd(s.radial + 3 * M + m, v3);
        atomicAdd(s.radial + 4 * M + m, v4);
    }
}

// ------------------------------------------------------------------ the two step kernels

constexpr int kBX = 32, kBY = 8;

template <class C, bool kStats, bool kPeriodic>
__global__ void __launch_bounds__(kBX * kBY) k_moments(const DeviceState s, const C codec, int64_t step) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    const bool active = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    NodeMoments m{};
    if (active) {
        const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
        const PullMap pm(g, x, y, z, kPeriodic);
        float sumr = 0.f, sumb = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
        float Axx = 0.f, Axy = 0.f, Ayy = 0.f, Ayz = 0.f, Azz = 0.f, Axz = 0.f;
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            using D = Dir<i>;
            float fr, fb;
            codec.template load<i>(pm.template src<i>(g, id), fr, fb);
            sumr += fr;
            sumb += fb;
            const float gi = fr + fb;
            if constexpr (D::cx == 1) jx += gi;
            if constexpr (D::cx == -1) jx -= gi;
            if constexpr (D::cy == 1) jy += gi;
            if constexpr (D::cy == -1) jy -= gi;
            if constexpr (D::cz == 1) jz += gi;
            if constexpr (D::cz == -1) jz -= gi;
            Axx += gi * D::Hxx;
            if constexpr (D::Hxy != 0.0f) Axy += gi * D::Hxy;
            Ayy += gi * D::Hyy;
            if constexpr (D::Hyz != 0.0f) Ayz += gi * D::Hyz;
            Azz += gi * D::Hzz;
            if constexpr (D::Hxz != 0.0f) Axz += gi * D::Hxz;
        });
        const float rho = sumr + sumb;
        const float inv = 1.0f / rho;
        m.rr = sumr;
        m.rb = sumb;
        m.ux = jx * inv;
        m.uy = jy * inv;
        m.uz = jz * inv;
        m.pxx = Axx - rho * m.ux * m.ux;
        m.pxy = Axy - rho * m.ux * m.uy;
        m.pyy = Ayy - rho * m.uy * m.uy;
        m.pyz = Ayz - rho * m.uy * m.uz;
        m.pzz = Azz - rho * m.uz * m.uz;
        m.pxz = Axz - rho * m.ux * m.uz;
        const size_t N = g.N;
        float *mom = s.mom;
        mom[kMomRR * N + id] = m.rr;
        mom[kMomRB * N + id] = m.rb;
        mom[kMomUX * N + id] = m.ux;
        mom[kMomUY * N + id] = m.uy;
        mom[kMomUZ * N + id] = m.uz;
        mom[kMomPXX * N + id] = m.pxx;
        mom[kMomPXY * N + id] = m.pxy;
        mom[kMomPYY * N + id] = m.pyy;
        mom[kMomPYZ * N + id] = m.pyz;
        mom[kMomPZZ * N + id] = m.pzz;
        mom[kMomPXZ * N + id] = m.pxz;
        const float ps = psi_of(sumr, sumb);
        float *psi = s.psi[step & 1];
        psi[id] = ps;
        if constexpr (kPeriodic) {
            // ghost mirrors so the unwrapped gradient stencil sees a periodic field
            const int xs[2] = {x, x == 1 ? g.NX - 1 : (x == g.NX - 2 ? 0 : -1)};
            const int ys[2] = {y, y == 1 ? g.NY - 1 : (y == g.NY - 2 ? 0 : -1)};
            const int zs[2] = {z, z == 1 ? g.NZ - 1 : (z == g.NZ - 2 ? 0 : -1)};
#pragma unroll
            for (int k = 1; k < 8; ++k) {
                const int xx = xs[k & 1], yy = ys[(k >> 1) & 1], zz = zs[(k >> 2) & 1];
                if (xx >= 0 && yy >= 0 && zz >= 0)
                    psi[uint32_t(xx) + uint32_t(g.sy) * uint32_t(yy) + uint32_t(g.sz) * uint32_t(zz)] = ps;
            }
        }
    }
    if constexpr (kStats) radial_accumulate_warp(s, x, y, z, active, m.ux, m.uy, m.uz);
}

template <class C>
__global__ void __launch_bounds__(kBX * kBY, 4) k_collide(const DeviceState s, const C codec, int64_t step) {
    const Geometry &g = s.g;
    const Physics &ph = s.ph;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const size_t N = g.N;
    const float *__restrict__ mom = s.mom;
    const float rr = __ldg(mom + kMomRR * N + id), rb = __ldg(mom + kMomRB * N + id);
    const float vx = __ldg(mom + kMomUX * N + id), vy = __ldg(mom + kMomUY * N + id), vz = __ldg(mom + kMomUZ * N + id);
    const NeqTerms n = make_neq(__ldg(mom + kMomPXX * N + id), __ldg(mom + kMomPXY * N + id),
                                __ldg(mom + kMomPYY * N + id), __ldg(mom + kMomPYZ * N + id),
                                __ldg(mom + kMomPZZ * N + id), __ldg(mom + kMomPXZ * N + id), vx, vy, vz);
    const EqTerms e = make_eq(vx, vy, vz);
    const float rT = rr + rb;
    const float invrT = 1.0f / rT;
    const float aR = rr * invrT, aB = rb * invrT;
    const float oms = 1.0f - omega_at(ph, y);
    const float Iind = 4.0f * rr * rb * invrT * invrT;
    if (Iind <= 1e-4f) {  // bulk (lbm.cuh:216-247)
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const float gi = feq<i>(rT, e) + oms * fneq<i>(n);
            codec.template store<i>(id, aR * gi, aB * gi);
        });
        return;
    }
    // interface (lbm.cuh:249-292): colour gradient over the 26 neighbours,
    // read unwrapped like forces.cuh:31 (ghost psi is what the reference sees)
    const float *__restrict__ psi = s.psi[step & 1];
    float sx = 0.f, sy = 0.f, sz = 0.f;
    static_for<kQ - 1>([&](auto I) {
        constexpr int i = decltype(I)::value + 1;
        using D = Dir<i>;
        const float p = __ldg(psi + (int(id) + D::cx + g.sy * D::cy + g.sz * D::cz));
        const float wp = D::w * p;
        if constexpr (D::cx == 1) sx += wp;
        if constexpr (D::cx == -1) sx -= wp;
        if constexpr (D::cy == 1) sy += wp;
        if constexpr (D::cy == -1) sy -= wp;
        if constexpr (D::cz == 1) sz += wp;
        if constexpr (D::cz == -1) sz -= wp;
    });
    InterfaceTerms t;
    t.Fx = kInvCs2 * sx;
    t.Fy = kInvCs2 * sy;
    t.Fz = kInvCs2 * sz;
    t.absF = sqrtf(t.Fx * t.Fx + t.Fy * t.Fy + t.Fz * t.Fz);
    t.has_dir = !(t.absF <= 1.0e-4f);
    t.inv_absF = 1.0f / t.absF;
    t.inv_absF2 = 1.0f / (t.absF * t.absF);
    t.Ah_absF = ph.Ah * t.absF;
    t.coeff_rho = ph.beta * ((rr * rb) / (rT * rT)) * rT;
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const float gi = feq<i>(rT, e) + oms * fneq<i>(n) + omega2<i>(t);
        const float d = recolour<i>(t);
        codec.template store<i>(id, aR * gi + d, aB * gi - d);
    });
}

__device__ __forceinline__ NodeMoments load_moments(const DeviceState &s, uint32_t id) {
    const size_t N = s.g.N;
    const float *m = s.mom;
    NodeMoments r;
    r.rr = m[kMomRR * N + id]; r.rb = m[kMomRB * N + id];
    r.ux = m[kMomUX * N + id]; r.uy = m[kMomUY * N + id]; r.uz = m[kMomUZ * N + id];
    r.pxx = m[kMomPXX * N + id]; r.pxy = m[kMomPXY * N + id]; r.pyy = m[kMomPYY * N + id];
    r.pyz = m[kMomPYZ * N + id]; r.pzz = m[kMomPZZ * N + id]; r.pxz = m[kMomPXZ * N + id];
    return r;
}

// Jet boundary of step `step` from its moments: blockIdx.z == 0 is the inlet
// (y=0 plane), 1 the outlet (y=NY-1 plane).  Values go to the ghost planes of
// buffer `wbuf` (the one the collision of this step writes) and to the psi
// buffer of the next step; they run in their own small launch so the rarely
// taken boundary code does not inflate the bulk kernels' register budget.
template <class C>
__global__ void __launch_bounds__(256) k_boundary(const DeviceState s, int wbuf, int64_t step, int which) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < 1 || x > g.NX - 2 || z < 1 || z > g.NZ - 2) return;
    const int side = which >= 0 ? which : int(blockIdx.z);
    float *psi_next = s.psi[(step + 1) & 1];
    if (side == 0) {
        const uint32_t idF = uint32_t(x) + uint32_t(g.sy) + uint32_t(g.sz) * uint32_t(z);
        inlet_column<C>(s, C{}, s.pops[wbuf], psi_next, x, z, step, load_moments(s, idF));
    } else {
        const uint32_t idF = uint32_t(x) + uint32_t(g.sy) * uint32_t(g.NY - 2) + uint32_t(g.sz) * uint32_t(z);
        outlet_column<C>(s, s.pops[wbuf], psi_next, x, z, load_moments(s, idF));
    }
}

__global__ void __launch_bounds__(kBX * kBY) k_accumulate_radial(const DeviceState s) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    const bool active = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    float ux = 0, uy = 0, uz = 0;
    if (active) {
        const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
        ux = s.mom[kMomUX * size_t(g.N) + id];
        uy = s.mom[kMomUY * size_t(g.N) + id];
        uz = s.mom[kMomUZ * size_t(g.N) + id];
    }
    radial_accumulate_warp(s, x, y, z, active, ux, uy, uz);
}

// ------------------------------------------------------------------ initial state

// Densities of every node (jet/jetIn.cuh:13-62 or bubble/bubbleIn.cuh:10-22).
__global__ void k_init_fields(const DeviceState s, int mode, int red_inside, float r2, float bx, float by, float bz) {
    const Geometry &g = s.g;
    const Physics &ph = s.ph;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.NX || y >= g.NY) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    float rr, rb;
    if (mode == 0) {
        rr = ph.rhor0;
        rb = 0.0f;
        if (y == 0 && x >= 1 && x <= g.NX - 2 && z >= 1 && z <= g.NZ - 2) {
            const float j = is_jet_column(ph, x, z) ? 1.0f : 0.0f;
            rr = (1.0f - j) * ph.rhor0;
            rb = j * ph.rhob0;
        }
    } else {
        int xx = x, yy = y, zz = z;
        if (g.boundary == kBoundaryPeriodic) {  // ghosts mirror the opposite interior node
            xx = x == 0 ? g.NX - 2 : (x == g.NX - 1 ? 1 : x);
            yy = y == 0 ? g.NY - 2 : (y == g.NY - 1 ? 1 : y);
            zz = z == 0 ? g.NZ - 2 : (z == g.NZ - 1 ? 1 : z);
        }
        const float dx = float(xx) - bx, dy = float(yy) - by, dz = float(zz) - bz;
        const float in = ((dx * dx) + (dy * dy) + (dz * dz)) <= r2 ? 1.0f : 0.0f;
        if (red_inside) {
            rr = in * ph.rhor0;
            rb = (1.0f - in) * ph.rhob0;
        } else {
            rr = (1.0f - in) * ph.rhor0;
            rb = in * ph.rhob0;
        }
    }
    const size_t N = g.N;
    s.mom[kMomRR * N + id] = rr;
    s.mom[kMomRB * N + id] = rb;
    for (int k = kMomUX; k < kMomCount; ++k) s.mom[size_t(k) * N + id] = 0.0f;
}

// Populations of every interior node, written at their pull sources in both
// buffers (so slots no kernel rewrites hold the initial value in both).
template <class C>
__global__ void k_init_pops(const DeviceState s, int mode, const float *fr_ref, const float *fb_ref, float noise) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const size_t N = g.N;
    const float rr = s.mom[kMomRR * N + id], rb = s.mom[kMomRB * N + id];
    for (int i = 0; i < kQ; ++i) {
        float fr, fb;
        if (mode == 2) {
            fr = fr_ref[size_t(i) * N + id];
            fb = fb_ref[size_t(i) * N + id];
        } else {
            // jetDensity: feq(rho, 0) = w rho; bubble: w rho (jetIn.cuh:26-34, bubbleIn.cuh:25-39)
            const float w = dir_w(i);
            fr = w * rr;
            fb = w * rb;
            if (noise != 0.0f) {
                const float u = hash_uniform(s.ph.seed, 0x1D17ull, id, uint64_t(i));
                const float f = 1.0f + (2.0f * u - 1.0f) * noise;
                fr = fr * f;
                fb = fb * f;
            }
        }
        const uint32_t src = pull_src_rt(g, x, y, z, i);
        C::store_to(s.pops[0], g.N, i, src, fr, fb, s.ph.f16_rho0);
        C::store_to(s.pops[1], g.N, i, src, fr, fb, s.ph.f16_rho0);
    }
}

__global__ void k_refresh_psi(const DeviceState s) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.NX || y >= g.NY) return;
    int xx = x, yy = y, zz = z;
    if (g.boundary == kBoundaryPeriodic) {
        xx = x == 0 ? g.NX - 2 : (x == g.NX - 1 ? 1 : x);
        yy = y == 0 ? g.NY - 2 : (y == g.NY - 1 ? 1 : y);
        zz = z == 0 ? g.NZ - 2 : (z == g.NZ - 1 ? 1 : z);
    }
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const uint32_t src = uint32_t(xx) + uint32_t(g.sy) * uint32_t(yy) + uint32_t(g.sz) * uint32_t(zz);
    const size_t N = g.N;
    const float p = psi_of(s.mom[kMomRR * N + src], s.mom[kMomRB * N + src]);
    s.psi[0][id] = p;
    s.psi[1][id] = p;
}

template <class C>
__global__ void k_gather_pops(const DeviceState s, int cur, float *fr_ref, float *fb_ref) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.NX || y >= g.NY) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const size_t N = g.N;
    const bool interior = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    for (int i = 0; i < kQ; ++i) {
        float fr = 0.0f, fb = 0.0f;
        if (interior) C::load_from(s.pops[cur], g.N, i, pull_src_rt(g, x, y, z, i), fr, fb, s.ph.f16_rho0);
        fr_ref[size_t(i) * N + id] = fr;
        fb_ref[size_t(i) * N + id] = fb;
    }
}

// ------------------------------------------------------------------ reductions

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < NT / 32; ++k) r += sh[k];
    return r;
}

constexpr int kRedThreads = 256;

// Sum of 0.5|u|^2 over interior nodes (kernels.cu:136-152), float64.
__global__ void __launch_bounds__(kRedThreads) k_tke(const DeviceState s, double *out) {
    __shared__ double sh[kRedThreads / 32];
    const Geometry &g = s.g;
    const size_t N = g.N;
    double acc = 0.0;
    for (size_t id = size_t(blockIdx.x) * blockDim.x + threadIdx.x; id < N; id += size_t(gridDim.x) * blockDim.x) {
        const int x = int(id % g.NX), y = int((id / g.NX) % g.NY), z = int(id / (size_t(g.NX) * g.NY));
        if (x < 1 || x > g.NX - 2 || y < 1 || y > g.NY - 2 || z < 1 || z > g.NZ - 2) continue;
        const float vx = s.mom[kMomUX * N + id], vy = s.mom[kMomUY * N + id], vz = s.mom[kMomUZ * N + id];
        acc += double(0.5f * (vx * vx + vy * vy + vz * vz));
    }
    const double r = block_sum<kRedThreads>(acc, sh);
    if (threadIdx.x == 0) atomicAdd(out, r);
}

// Running mean of uy per interior node (kernels.cu:168-186).
__global__ void k_uy_average(const DeviceState s, uint32_t samples) {
    const Geometry &g = s.g;
    const size_t N = g.N;
    const float c = float(samples);
    for (size_t id = size_t(blockIdx.x) * blockDim.x + threadIdx.x; id < N; id += size_t(gridDim.x) * blockDim.x) {
        const int x = int(id % g.NX), y = int((id / g.NX) % g.NY), z = int(id / (size_t(g.NX) * g.NY));
        if (x < 1 || x > g.NX - 2 || y < 1 || y > g.NY - 2 || z < 1 || z > g.NZ - 2) continue;
        s.uy_avg[id] = (s.uy_avg[id] * c + s.mom[kMomUY * N + id]) / (c + 1.0f);
    }
}

constexpr int kConsBlocksMax = 4 * 148;

// Pass 1: per-block float64 partial sums of f(t) over interior nodes.
template <class C>
__global__ void __launch_bounds__(kRedThreads) k_conservation_partials(const DeviceState s, int cur,
                                                                       double *partials) {
    __shared__ double sh[kRedThreads / 32];
    const Geometry &g = s.g;
    const size_t N = g.N;
    double acc[5] = {0, 0, 0, 0, 0};
    for (size_t id = size_t(blockIdx.x) * blockDim.x + threadIdx.x; id < N; id += size_t(gridDim.x) * blockDim.x) {
        const int x = int(id % g.NX), y = int((id / g.NX) % g.NY), z = int(id / (size_t(g.NX) * g.NY));
        if (x < 1 || x > g.NX - 2 || y < 1 || y > g.NY - 2 || z < 1 || z > g.NZ - 2) continue;
        for (int i = 0; i < kQ; ++i) {
            float fr, fb;
            C::load_from(s.pops[cur], g.N, i, pull_src_rt(g, x, y, z, i), fr, fb, s.ph.f16_rho0);
            const double a = fr, b = fb;
            acc[0] += a;
            acc[1] += b;
            acc[2] += (a + b) * c_cx[i];
            acc[3] += (a + b) * c_cy[i];
            acc[4] += (a + b) * c_cz[i];
        }
    }
    for (int k = 0; k < 5; ++k) {
        const double r = block_sum<kRedThreads>(acc[k], sh);
        if (threadIdx.x == 0) partials[size_t(k) * gridDim.x + blockIdx.x] = r;
    }
}

// Pass 2: one block folds the partials in a fixed order (deterministic).
__global__ void __launch_bounds__(kRedThreads) k_conservation_final(const double *partials, int nblocks, double *out) {
    __shared__ double sh[kRedThreads / 32];
    for (int k = 0; k < 5; ++k) {
        double acc = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc += partials[size_t(k) * nblocks + b];
        const double r = block_sum<kRedThreads>(acc, sh);
        if (threadIdx.x == 0) out[k] = r;
    }
}

template <class C>
__global__ void k_check_finite(const DeviceState s, int cur, int *flag) {
    const Geometry &g = s.g;
    const size_t N = g.N;
    for (size_t id = size_t(blockIdx.x) * blockDim.x + threadIdx.x; id < N; id += size_t(gridDim.x) * blockDim.x) {
        const int x = int(id % g.NX), y = int((id / g.NX) % g.NY), z = int(id / (size_t(g.NX) * g.NY));
        if (x < 1 || x > g.NX - 2 || y < 1 || y > g.NY - 2 || z < 1 || z > g.NZ - 2) continue;
        bool bad = false;
        for (int k = 0; k < kMomCount; ++k) bad |= !isfinite(s.mom[size_t(k) * N + id]);
        for (int i = 0; i < kQ; ++i) {
            float fr, fb;
            C::load_from(s.pops[cur], g.N, i, pull_src_rt(g, x, y, z, i), fr, fb, s.ph.f16_rho0);
            bad |= !isfinite(fr) || !isfinite(fb);
        }
        if (bad) atomicOr(flag, 1);
    }
}

dim3 grid3(const Geometry &g) { return dim3((g.NX + kBX - 1) / kBX, (g.NY + kBY - 1) / kBY, g.NZ); }
dim3 grid_plane(const Geometry &g) { return dim3((g.NX + 31) / 32, (g.NZ + 7) / 8, 1); }
unsigned grid1(const Geometry &g) {
    const size_t want = (size_t(g.N) + kRedThreads - 1) / kRedThreads;
    return unsigned(want < size_t(8 * 148) ? want : size_t(8 * 148));
}

template <class C, bool kStats>
cudaError_t moments_dispatch(const DeviceState &s, int cur, int64_t step, cudaStream_t st) {
    const C codec = make_codec<C>(s, cur);
    if (s.g.boundary == kBoundaryPeriodic)
        k_moments<C, kStats, true><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, codec, step);
    else
        k_moments<C, kStats, false><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, codec, step);
    return cudaGetLastError();
}

template <class C>
cudaError_t moments_stats(const DeviceState &s, int cur, int64_t step, bool stats, cudaStream_t st) {
    return stats ? moments_dispatch<C, true>(s, cur, step, st) : moments_dispatch<C, false>(s, cur, step, st);
}

template <class C>
cudaError_t boundary_dispatch(const DeviceState &s, int wbuf, int64_t step, int which, cudaStream_t st) {
    dim3 grid = grid_plane(s.g);
    grid.z = which >= 0 ? 1 : 2;
    k_boundary<C><<<grid, dim3(32, 8), 0, st>>>(s, wbuf, step, which);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_moments(const DeviceState &s, int cur, int64_t step, bool stats, cudaStream_t st) {
    if (s.g.storage == kStoreF16) return moments_stats<CodecF16>(s, cur, step, stats, st);
    return moments_stats<CodecF32>(s, cur, step, stats, st);
}

cudaError_t launch_collide(const DeviceState &s, int cur, int64_t step, cudaStream_t st) {
    if (s.g.storage == kStoreF16)
        k_collide<CodecF16><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, make_codec<CodecF16>(s, cur), step);
    else
        k_collide<CodecF32><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, make_codec<CodecF32>(s, cur), step);
    return cudaGetLastError();
}

cudaError_t launch_boundary(const DeviceState &s, int wbuf, int64_t step, int which, cudaStream_t st) {
    if (s.g.storage == kStoreF16) return boundary_dispatch<CodecF16>(s, wbuf, step, which, st);
    return boundary_dispatch<CodecF32>(s, wbuf, step, which, st);
}

cudaError_t launch_accumulate_radial(const DeviceState &s, cudaStream_t st) {
    k_accumulate_radial<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s);
    return cudaGetLastError();
}

cudaError_t launch_init_fields(const DeviceState &s, int mode, int red_inside, float r2, float bx, float by, float bz,
                               float, cudaStream_t st) {
    k_init_fields<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, mode, red_inside, r2, bx, by, bz);
    return cudaGetLastError();
}

cudaError_t launch_init_pops(const DeviceState &s, int mode, const float *fr_ref, const float *fb_ref, float noise,
                             cudaStream_t st) {
    if (s.g.storage == kStoreF16)
        k_init_pops<CodecF16><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, mode, fr_ref, fb_ref, noise);
    else
        k_init_pops<CodecF32><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, mode, fr_ref, fb_ref, noise);
    return cudaGetLastError();
}

cudaError_t launch_refresh_psi(const DeviceState &s, cudaStream_t st) {
    k_refresh_psi<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s);
    return cudaGetLastError();
}

cudaError_t launch_gather_pops(const DeviceState &s, int cur, float *fr_ref, float *fb_ref, cudaStream_t st) {
    if (s.g.storage == kStoreF16)
        k_gather_pops<CodecF16><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, cur, fr_ref, fb_ref);
    else
        k_gather_pops<CodecF32><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, cur, fr_ref, fb_ref);
    return cudaGetLastError();
}

cudaError_t launch_tke(const DeviceState &s, double *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
    k_tke<<<grid1(s.g), kRedThreads, 0, st>>>(s, out);
    return cudaGetLastError();
}

cudaError_t launch_uy_average(const DeviceState &s, uint32_t samples, cudaStream_t st) {
    k_uy_average<<<grid1(s.g), kRedThreads, 0, st>>>(s, samples);
    return cudaGetLastError();
}

uint32_t conservation_blocks(const Geometry &g) {
    const size_t want = (size_t(g.N) + kRedThreads - 1) / kRedThreads;
    return uint32_t(want < size_t(kConsBlocksMax) ? want : size_t(kConsBlocksMax));
}

cudaError_t launch_conservation(const DeviceState &s, int cur, double *partials, double *out5, cudaStream_t st) {
    const uint32_t nb = conservation_blocks(s.g);
    if (s.g.storage == kStoreF16) k_conservation_partials<CodecF16><<<nb, kRedThreads, 0, st>>>(s, cur, partials);
    else k_conservation_partials<CodecF32><<<nb, kRedThreads, 0, st>>>(s, cur, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_conservation_final<<<1, kRedThreads, 0, st>>>(partials, int(nb), out5);
    return cudaGetLastError();
}

cudaError_t launch_check_finite(const DeviceState &s, int cur, int *flag, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    if (s.g.storage == kStoreF16) k_check_finite<CodecF16><<<grid1(s.g), kRedThreads, 0, st>>>(s, cur, flag);
    else k_check_finite<CodecF32><<<grid1(s.g), kRedThreads, 0, st>>>(s, cur, flag);
    return cudaGetLastError();
}

}  // namespace mcg
