// kernels.cu - the D3Q27 colour-gradient step on B200 (sm_100a).
//
// The step is one HBM pass, one launch (k_fused, or its pipelined forms
// k_fused_pipe and k_fused_bulk):
//   k_fused    a CTA owns a tile of rows (y) and marches a chunk of z planes.
//              For each plane it pulls f(t) for its rows plus a one-row halo
//              from the population buffer (row-blocked layout, so a pulled row
//              is nine contiguous segments), forms rho_r, rho_b, u, Pi^neq
//              (lbm.cuh:82-165) and psi into shared memory, accumulates the
//              radial statistics (kernels.cu:188-233) with warp segmented
//              reductions, and then relaxes the previous plane
//              (lbm.cuh:184-293): Hermite-regularised BGK, colour-gradient
//              perturbation and recolouring, with the gradient taken from the
//              same step's psi in shared memory (the reference needs a kernel
//              boundary for this), storing the post-collision values at each
//              node (pull layout, coalesced rows).  Moments never go to HBM.
//              The CTAs whose tiles hold the fluid rows 1 and NY-2 then write
//              the jet's inlet (jet/boundary_conditions.cuh:17-85) and
//              convective outlet (:163-233) columns of their chunk into the y
//              ghost planes of the new buffer (fused_boundary).
//   k_boundary the same boundary as a launch of its own, one thread per
//              column, from the fluid-plane moments the step leaves in bmom
//              (the granular sequence, and MCG_FUSED_BOUNDARY=0).
// The granular launch sequence of the reference (k_moments, k_collide,
// k_boundary, k_accumulate_radial) is kept for callers that drive the
// launchers one by one; it writes the moment planes to HBM like the reference.
// The reference's in-place push buffer becomes a ping-pong pull pair; the
// populations a reference step never rewrites (y=1 slots fed by non-jet
// inlet columns, y=NY-2 slots fed by ghost columns) are ghost-plane values of
// both buffers that no kernel writes, so results are the same.
#include <type_traits>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "kernels.cuh"
#include "lattice.cuh"

namespace mcg {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ storage codecs

// Float32 element per (direction, node): the pair (fr, fb), so a pull or a
// store of both colours is one 8-byte access.
struct CodecF32 {
    using Elem = float2;
    static constexpr int kGroupSlots = 3;
    static constexpr bool kSumDiff = false;  // pulls form sum fr and sum fb (reference order)
    // store_bulk takes P_i itself (collision_poly without a shift)
    static constexpr bool kShiftPoly = false;
    __device__ __forceinline__ float poly_shift() const { return 0.0f; }
    const float2 *__restrict__ rd;
    float2 *__restrict__ wr;
    int NX;
    // store through `wrow` = the node's row in the written buffer, offset by x
    template <int I>
    __device__ __forceinline__ void store_row(float2 *wrow, float r, float b) const {
        wrow[slot_pair(I) * NX] = make_float2(r, b);
    }
    // bulk node: fr_i = aR w_i P_i, fb_i = aB w_i P_i (lbm.cuh:216-247)
    __device__ __forceinline__ void store_bulk(float2 *wrow, float aR, float aB, const float (&P)[kQ]) const {
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            // both colours in one packed multiply and one store
            wrow[slot_pair(i) * NX] = __fmul2_rn(make_float2(aR * Dir<i>::w, aB * Dir<i>::w), make_float2(P[i], P[i]));
        });
    }
    // pull in two halves: the raw pair at `p` = the source node's element of
    // direction I, then the pair the colour sums add and the total gi
    using Raw = float2;
    template <int I>
    __device__ __forceinline__ Raw load_raw(const float2 *p) const {
        return __ldg(p);
    }
    template <int I>
    __device__ __forceinline__ float2 decode(Raw v, float &gi) const {
        gi = v.x + v.y;
        return v;
    }
    template <int I>
    __device__ __forceinline__ void store(size_t row, int x, float r, float b) const {
        wr[row + size_t(slot_pair(I)) * NX + x] = make_float2(r, b);
    }
    __device__ __forceinline__ static void store_to(void *buf, const Geometry &g, int i, int x, int y, int z, float r,
                                                    float b, float) {
        static_cast<float2 *>(buf)[pop_index(g, slot_pair(i), x, y, z)] = make_float2(r, b);
    }
    __device__ __forceinline__ static void load_from(const void *buf, const Geometry &g, int i, int x, int y, int z,
                                                     float &r, float &b, float) {
        const float2 v = static_cast<const float2 *>(buf)[pop_index(g, slot_pair(i), x, y, z)];
        r = v.x;
        b = v.y;
    }
};

// F16 word per (direction, node): x = g/w_i - rho0 (total offset by the rest
// equilibrium and scaled by 1/w_i), y = q, the minority-colour fraction
// 2 min(fr,fb)/g carrying the sign of fr-fb.  Pure nodes store q = +-0
// exactly, so a single-colour region keeps exactly zero of the other colour.
__device__ __forceinline__ __half2 f16_encode(float r, float b, float inv_w, float rho0) {
    // rounded operation by operation, so that every kernel that inlines it
    // (the jet boundary is written from several) gives the same word
    const float g = __fadd_rn(r, b);
    const float h0 = __fsub_rn(__fmul_rn(g, inv_w), rho0);
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
    using Elem = __half2;
    static constexpr int kGroupSlots = 3;
    static constexpr bool kSumDiff = true;  // pulls form sum (fr+fb) and sum (fr-fb)
    // store_bulk takes P_i - rho0, formed by collision_poly's constant term
    static constexpr bool kShiftPoly = true;
    __device__ __forceinline__ float poly_shift() const { return rho0; }
    const __half2 *__restrict__ rd;
    __half2 *__restrict__ wr;
    int NX;
    float rho0;
    template <int I>
    __device__ __forceinline__ void store_row(__half2 *wrow, float r, float b) const {
        wrow[slot_pair(I) * NX] = f16_encode(r, b, 1.0f / Dir<I>::w, rho0);
    }
    // bulk node: every direction splits its total g_i = w_i P_i in the same
    // proportion aR : aB, so the word is (P_i - rho0, q) (Ps = P - rho0 from
    // collision_poly) with one signed
    // minority fraction q = 2 min(aR, aB) for the node - the value f16_encode
    // forms from fr_i, fb_i up to float rounding, and exactly +-0 at a pure
    // node (aB or aR is exactly 0 there).
    __device__ __forceinline__ void store_bulk(__half2 *wrow, float aR, float aB, const float (&Ps)[kQ]) const {
        const float q = copysignf(fmaxf(2.0f * fminf(aR, aB), 0.0f), aR - aB);
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            wrow[slot_pair(i) * NX] = __floats2half2_rn(Ps[i], q);
        });
    }
    // pull in two halves: the raw word, then the total g = fr + fb and the
    // difference d = fr - fb.  With q the signed minority fraction, fr - fb =
    // g (1 - q) when red is the majority and -g (1 + q) otherwise, i.e.
    // g (sign(q) - q).
    // The read-only load asks L2 to fetch 256-byte blocks on a miss: the words
    // of a pulled row segment are then in L2 for the neighbouring warps'
    // loads (measured +0.3 % on the 128x256x128 jet, +1.2 % on 256-column
    // rows; no change in float32).
    using Raw = __half2;
    template <int I>
    __device__ __forceinline__ Raw load_raw(const __half2 *p) const {
        uint32_t u;
        asm("ld.global.nc.L2::256B.b32 %0, [%1];" : "=r"(u) : "l"(p));
        __half2 h;
        memcpy(&h, &u, sizeof h);
        return h;
    }
    template <int I>
    __device__ __forceinline__ float2 decode(Raw h, float &gi) const {
        const float2 v = __half22float2(h);
        const float gs = fmaf(Dir<I>::w, v.x, Dir<I>::w * rho0);
        gi = gs;
        return make_float2(gs, fmaf(-gs, v.y, copysignf(gs, v.y)));
    }
    template <int I>
    __device__ __forceinline__ void store(size_t row, int x, float r, float b) const {
        wr[row + size_t(slot_pair(I)) * NX + x] = f16_encode(r, b, 1.0f / Dir<I>::w, rho0);
    }
    __device__ __forceinline__ static void store_to(void *buf, const Geometry &g, int i, int x, int y, int z, float r,
                                                    float b, float rho0) {
        static_cast<__half2 *>(buf)[pop_index(g, slot_pair(i), x, y, z)] = f16_encode(r, b, 1.0f / dir_w(i), rho0);
    }
    __device__ __forceinline__ static void load_from(const void *buf, const Geometry &g, int i, int x, int y, int z,
                                                     float &r, float &b, float rho0) {
        f16_decode(static_cast<const __half2 *>(buf)[pop_index(g, slot_pair(i), x, y, z)], dir_w(i), rho0, r, b);
    }
};

template <class C>
__host__ __device__ C make_codec(const DeviceState &s, int cur);
template <>
__host__ __device__ CodecF32 make_codec<CodecF32>(const DeviceState &s, int cur) {
    return CodecF32{static_cast<const float2 *>(s.pops[cur]), static_cast<float2 *>(s.pops[cur ^ 1]), s.g.NX};
}
template <>
__host__ __device__ CodecF16 make_codec<CodecF16>(const DeviceState &s, int cur) {
    return CodecF16{static_cast<const __half2 *>(s.pops[cur]), static_cast<__half2 *>(s.pops[cur ^ 1]), s.g.NX,
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
    return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)) <= ph.jet_r2;
}

// Inlet velocity of jet column (x, z): the top-hat U (boundary_conditions.cuh:62),
// times the column's profile multiplier when a radial profile is set, times
// the seeded perturbation when inlet_noise != 0.
__device__ __forceinline__ float inlet_velocity(const DeviceState &s, int64_t step, int x, int z) {
    const Physics &ph = s.ph;
    float U = ph.jet_velocity;
    if (s.inlet_profile) U *= s.inlet_profile[x + s.g.NX * z];
    if (ph.inlet_noise == 0.0f) return U;
    const float u = hash_uniform(ph.seed, 0x1A1E7ull ^ uint64_t(step), uint64_t(x), uint64_t(z));
    return __fmul_rn(U, __fadd_rn(1.0f, __fmul_rn(__fsub_rn(2.0f * u, 1.0f), ph.inlet_noise)));
}

__host__ __device__ __forceinline__ int wrap_interior(int v, int n) { return v == 0 ? n - 2 : (v == n - 1 ? 1 : v); }

// Pull sources of interior node (x,y,z).  x and z are periodic over the
// interior through the ghost shell (the push side wraps with
// bounds.cuh:23-60); y sources on a ghost plane are the boundary's slots and
// are not wrapped laterally (boundary writes are unwrapped,
// boundary_conditions.cuh:73,137); in the periodic box y wraps too.
template <class C>
struct PullMap {
    long long own_row;              // offset of row (y,z)
    long long step_y, step_z;       // row offsets of y+1, z+1
    long long wzp, wzm, wyp, wym;   // wrap corrections (row offsets)
    int wxp, wxm;                   // wrap corrections (x)
    int NX;
    bool gy_p, gy_m;
    __device__ __forceinline__ PullMap(const Geometry &g, int x, int y, int z, bool periodic) {
        NX = g.NX;
        own_row = (long long)pop_row(g, y, z);
        step_y = (long long)g.slots * g.NX;
        step_z = step_y * g.NY;
        wxp = (x == 1) ? (g.NX - 2) : 0;
        wxm = (x == g.NX - 2) ? -(g.NX - 2) : 0;
        wzp = (z == 1) ? step_z * (g.NZ - 2) : 0;
        wzm = (z == g.NZ - 2) ? -step_z * (g.NZ - 2) : 0;
        wyp = (periodic && y == 1) ? step_y * (g.NY - 2) : 0;
        wym = (periodic && y == g.NY - 2) ? -step_y * (g.NY - 2) : 0;
        gy_p = !periodic && y == 1;
        gy_m = !periodic && y == g.NY - 2;
    }
    // offset of the group segment of direction I's source row, and source x
    template <int I>
    __device__ __forceinline__ void src(int x, size_t &grow, int &xs) const {
        using D = Dir<I>;
        const long long o = own_row - D::cy * step_y - D::cz * step_z;
        bool ghost = false;
        if constexpr (D::cy == 1) ghost = gy_p;
        if constexpr (D::cy == -1) ghost = gy_m;
        int xc = 0;
        long long oc = 0;
        if constexpr (D::cx == 1) xc = wxp;
        if constexpr (D::cx == -1) xc = wxm;
        if constexpr (D::cz == 1) oc = wzp;
        if constexpr (D::cz == -1) oc = wzm;
        if (ghost) {
            xc = 0;
            oc = 0;
        }
        if constexpr (D::cy == 1) oc += wyp;
        if constexpr (D::cy == -1) oc += wym;
        grow = size_t(o + oc) + size_t(dir_group(I) * C::kGroupSlots) * size_t(NX);
        xs = x - D::cx + xc;
    }
    // the source's first slot of direction I (red for float32)
    template <int I>
    __device__ __forceinline__ const typename C::Elem *ptr(const C &codec, int x) const {
        size_t grow;
        int xs;
        src<I>(x, grow, xs);
        return codec.rd + grow + size_t(dir_cx(I) + 1) * size_t(NX) + xs;
    }
};

// Pull sources of a node in rows y = 2 .. NY-3: no source lies on a y ghost
// plane or wraps in y, so the only corrections are the z wrap, the same for
// all directions of one cz, and the x wrap of columns 1 and NX-2.  One base
// pointer per cz (z wrap applied, offset by x) then serves nine directions,
// each a load at a constant offset from it, plus the x wrap for cx = +-1.
// The addresses are those of PullMap.
template <class C>
struct FastPullMap {
    const typename C::Elem *base[3];  // cz = -1, 0, +1
    long long step_y;
    int xwp, xwm;  // x wrap of cx = +1 (column 1) and cx = -1 (column NX-2)
    int NX;
    __device__ __forceinline__ FastPullMap(const Geometry &g, const C &codec, int x, int y, int z) {
        NX = g.NX;
        step_y = (long long)g.slots * g.NX;
        const long long step_z = step_y * g.NY;
        const typename C::Elem *own = codec.rd + pop_row(g, y, z) + x;
        base[0] = own + step_z + ((z == g.NZ - 2) ? -step_z * (g.NZ - 2) : 0);  // cz = -1: source plane z+1
        base[1] = own;
        base[2] = own - step_z + ((z == 1) ? step_z * (g.NZ - 2) : 0);          // cz = +1: source plane z-1
        xwp = (x == 1) ? (g.NX - 2) : 0;
        xwm = (x == g.NX - 2) ? -(g.NX - 2) : 0;
    }
    template <int I>
    __device__ __forceinline__ const typename C::Elem *ptr(const C &, int) const {
        using D = Dir<I>;
        const typename C::Elem *b = base[D::cz + 1];
        if constexpr (D::cx == 1) b += xwp;
        if constexpr (D::cx == -1) b += xwm;
        return b + (-(long long)D::cy * step_y + (long long)(dir_group(I) * C::kGroupSlots + D::cx + 1) * NX - D::cx);
    }
};

// Runtime-direction pull source (init/gather/diagnostic kernels): source
// coordinates of direction i for interior node (x,y,z).
__device__ __forceinline__ void pull_src_rt(const Geometry &g, int x, int y, int z, int i, int &xs, int &ys, int &zs) {
    const bool periodic = g.boundary == kBoundaryPeriodic;
    xs = x - dir_cx(i);
    ys = y - dir_cy(i);
    zs = z - dir_cz(i);
    const bool ghost_plane = !periodic && (ys == 0 || ys == g.NY - 1);
    if (!ghost_plane) {
        xs = wrap_interior(xs, g.NX);
        zs = wrap_interior(zs, g.NZ);
    }
    if (periodic) ys = wrap_interior(ys, g.NY);
}

__constant__ int c_cx[kQ] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
__constant__ int c_cy[kQ] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
__constant__ int c_cz[kQ] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

// ------------------------------------------------------------------ per-node pieces

// First of the opposite pairs (i, i+1), i = 2p+1, whose direction has a
// nonzero c_a c_b (a == b: c_a != 0); the moment sums start there.
__host__ __device__ constexpr int dir_comp(int i, int a) { return a == 0 ? dir_cx(i) : (a == 1 ? dir_cy(i) : dir_cz(i)); }
__host__ __device__ constexpr int first_pair(int a, int b) {
    for (int p = 0; p < (kQ - 1) / 2; ++p)
        if (dir_comp(2 * p + 1, a) * dir_comp(2 * p + 1, b) != 0) return p;
    return (kQ - 1) / 2;
}
template <bool kFirst>
__device__ __forceinline__ void moment_add(float &acc, float v) {
    if constexpr (kFirst)
        acc = v;
    else
        acc += v;
}

// A node's pull in two halves: pull_issue loads the 27 raw elements (float2
// or half2) into registers; densities_from / moments_from decode and sum them.
// Between the two a warp can do other work while the loads are in flight.
template <class C>
struct RawPull {
    typename C::Raw v[kQ];
};

template <class C, class Map>
__device__ __forceinline__ void pull_issue_map(const Map &pm, const C &codec, int x, RawPull<C> &raw) {
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        raw.v[i] = codec.template load_raw<i>(pm.template ptr<i>(codec, x));
    });
}

// Colour densities only of interior node (x,y,z): the colour sums of
// pull_moments below in the same order (direction index), so psi formed from
// either is bit-identical.  Nodes whose psi is all that is needed (halo rows
// and planes of a tile) take this.
// The pulled pairs come from `src.get<I>(gi)`: decoded from words already in
// registers (RawSource) or loaded and decoded on the spot (DecodedPull).
template <class C>
struct RawSource {
    const C &codec;
    const RawPull<C> &raw;
    template <int I>
    __device__ __forceinline__ float2 get(float &gi) const {
        return codec.template decode<I>(raw.v[I], gi);
    }
};

template <class Src>
__device__ __forceinline__ void densities_from(const Src &src, float &rr, float &rb) {
    using C = std::remove_cv_t<std::remove_reference_t<decltype(src.codec)>>;
    float2 sum = make_float2(0.f, 0.f);  // (sum fr, sum fb); C::kSumDiff: (sum fr+fb, sum fr-fb)
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        float gi;
        sum = __fadd2_rn(sum, src.template get<i>(gi));  // both colours in one packed add
    });
    if constexpr (C::kSumDiff) {
        rr = 0.5f * (sum.x + sum.y);
        rb = 0.5f * (sum.x - sum.y);
    } else {
        rr = sum.x;
        rb = sum.y;
    }
}

// Pull the 54 populations of interior node (x,y,z) and form its moments
// (lbm.cuh:106-164: densities, velocity, second-order Hermite moments minus
// the equilibrium part).  The loads are issued in direction-index order
// (measured: issuing them group by group was 5-20 % slower) into registers;
// the moments are then formed from the sums and differences of opposite
// pairs, about 100 operations instead of one multiply-add per direction and
// moment.
template <class Src>
__device__ __forceinline__ NodeMoments moments_from(const Src &src) {
    using C = std::remove_cv_t<std::remove_reference_t<decltype(src.codec)>>;
    float2 sum = make_float2(0.f, 0.f);  // (sum fr, sum fb); C::kSumDiff: (sum fr+fb, sum fr-fb)
    float gv[kQ];                        // totals fr + fb per direction
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        sum = __fadd2_rn(sum, src.template get<i>(gv[i]));
    });
    // Moments over the 13 opposite pairs (i, i+1), i odd: d = g_i - g_opp
    // carries the first moments, s = g_i + g_opp the second.  Near equilibrium
    // the two members of a pair are within a factor of two, so d is exact and
    // the momentum sums add small numbers.  The diagonal stresses take s times
    // the Hermite constants H_aa = c_a^2 - cs^2 (multiply-adds, as lbm.cuh
    // forms them): the rounding of the two constants cancels at rest, whereas
    // sum c_a^2 g - rho * float(1/3) is biased by 1e-8 rho at every node and
    // step, which accumulated to 3x the float32 error of the reference's
    // arithmetic in the kinetic energy.  (Summing whole (cy, cz) groups
    // before differencing lost digits of the momentum.)
    float Jx, Jy, Jz, Qxy, Qxz, Qyz;
    float Axx = gv[0] * Dir<0>::Hxx, Ayy = gv[0] * Dir<0>::Hyy, Azz = gv[0] * Dir<0>::Hzz;
    static_for<(kQ - 1) / 2>([&](auto P) {
        constexpr int p = decltype(P)::value, i = 2 * p + 1;
        using D = Dir<i>;
        static_assert(Dir<i + 1>::cx == -D::cx && Dir<i + 1>::cy == -D::cy && Dir<i + 1>::cz == -D::cz,
                      "directions i, i+1 (i odd) are opposite");
        const float d = gv[i] - gv[i + 1], sp = gv[i] + gv[i + 1];
        if constexpr (D::cx != 0) moment_add<p == first_pair(0, 0)>(Jx, D::cx > 0 ? d : -d);
        if constexpr (D::cy != 0) moment_add<p == first_pair(1, 1)>(Jy, D::cy > 0 ? d : -d);
        if constexpr (D::cz != 0) moment_add<p == first_pair(2, 2)>(Jz, D::cz > 0 ? d : -d);
        Axx = fmaf(sp, D::Hxx, Axx);
        Ayy = fmaf(sp, D::Hyy, Ayy);
        Azz = fmaf(sp, D::Hzz, Azz);
        if constexpr (D::cx * D::cy != 0) moment_add<p == first_pair(0, 1)>(Qxy, D::cx * D::cy > 0 ? sp : -sp);
        if constexpr (D::cx * D::cz != 0) moment_add<p == first_pair(0, 2)>(Qxz, D::cx * D::cz > 0 ? sp : -sp);
        if constexpr (D::cy * D::cz != 0) moment_add<p == first_pair(1, 2)>(Qyz, D::cy * D::cz > 0 ? sp : -sp);
    });
    float sumr = sum.x, sumb = sum.y;
    if constexpr (C::kSumDiff) {
        sumr = 0.5f * (sum.x + sum.y);
        sumb = 0.5f * (sum.x - sum.y);
    }
    NodeMoments m;
    const float rho = sumr + sumb;
    const float inv = 1.0f / rho;
    m.rr = sumr;
    m.rb = sumb;
    m.ux = Jx * inv;
    m.uy = Jy * inv;
    m.uz = Jz * inv;
    m.pxx = Axx - rho * m.ux * m.ux;
    m.pxy = Qxy - rho * m.ux * m.uy;
    m.pyy = Ayy - rho * m.uy * m.uy;
    m.pyz = Qyz - rho * m.uy * m.uz;
    m.pzz = Azz - rho * m.uz * m.uz;
    m.pxz = Qxz - rho * m.ux * m.uz;
    return m;
}

// Rows 2 .. NY-3 take FastPullMap, the two edge rows PullMap (ghost planes,
// y wrap); y is uniform over a warp at every call site, so the branch is too.
template <class C, bool kPeriodic>
__device__ __forceinline__ void pull_issue(const Geometry &g, const C &codec, int x, int y, int z, RawPull<C> &raw) {
    if (y >= 2 && y <= g.NY - 3)
        pull_issue_map(FastPullMap<C>(g, codec, x, y, z), codec, x, raw);
    else
        pull_issue_map(PullMap<C>(g, x, y, z, kPeriodic), codec, x, raw);
}
// One-piece pulls: each load is decoded where it is issued, which lets the
// compiler consume the words as they arrive (measured 2 % faster at 80
// registers than issuing all of them first).  The arithmetic and its order
// are the same either way, so the results are bit-identical.
template <class C, class Map>
struct DecodedPull {
    const Map &pm;
    const C &codec;
    int x;
    template <int I>
    __device__ __forceinline__ float2 get(float &gi) const {
        return codec.template decode<I>(codec.template load_raw<I>(pm.template ptr<I>(codec, x)), gi);
    }
};
template <class C, class Map>
__device__ __forceinline__ void pull_densities_map(const Map &pm, const C &codec, int x, float &rr, float &rb) {
    densities_from(DecodedPull<C, Map>{pm, codec, x}, rr, rb);
}
template <class C, class Map>
__device__ __forceinline__ NodeMoments pull_moments_map(const Map &pm, const C &codec, int x) {
    return moments_from(DecodedPull<C, Map>{pm, codec, x});
}
template <class C, bool kPeriodic>
__device__ __forceinline__ void pull_densities(const Geometry &g, const C &codec, int x, int y, int z, float &rr,
                                               float &rb) {
    if (y >= 2 && y <= g.NY - 3)
        pull_densities_map(FastPullMap<C>(g, codec, x, y, z), codec, x, rr, rb);
    else
        pull_densities_map(PullMap<C>(g, x, y, z, kPeriodic), codec, x, rr, rb);
}
template <class C, bool kPeriodic>
__device__ __forceinline__ NodeMoments pull_moments(const Geometry &g, const C &codec, int x, int y, int z) {
    if (y >= 2 && y <= g.NY - 3) return pull_moments_map(FastPullMap<C>(g, codec, x, y, z), codec, x);
    return pull_moments_map(PullMap<C>(g, x, y, z, kPeriodic), codec, x);
}

// Relax one node and store its 54 post-collision values (lbm.cuh:184-293).
// The bulk part feq + (1-omega) fneq of all 27 directions comes from
// collision_poly (lattice.cuh).  At interface nodes the perturbation Omega2
// (even in c: one evaluation per opposite pair) and the recolouring Delta
// (odd) are added per direction.  psi_at(cx,cy,cz) returns the neighbour's
// psi, read unwrapped like forces.cuh:31 (ghost psi is what the reference
// sees there).
template <class C, class PsiAt>
__device__ __forceinline__ void collide_node(const Geometry &g, const Physics &ph, const C &codec, size_t row, int x,
                                             int y, int z, const NodeMoments &m, PsiAt &&psi_at) {
    const NeqTerms n = make_neq(m.pxx, m.pxy, m.pyy, m.pyz, m.pzz, m.pxz, m.ux, m.uy, m.uz);
    const float rr = m.rr, rb = m.rb;
    const float rT = rr + rb;
    const float invrT = 1.0f / rT;
    const float aR = rr * invrT, aB = rb * invrT;
    const float oms = 1.0f - omega_at(ph, y);
    const float Iind = 4.0f * rr * rb * invrT * invrT;
    float P[kQ];  // P_i - shift, shift = 0 (float32) or rho0 (float16)
    const float shift = codec.poly_shift();
    collision_poly(rT, m.ux, m.uy, m.uz, n, oms, P, shift);
    auto full = [&](float p) {  // P_i from P_i - shift
        if constexpr (C::kShiftPoly)
            return p + shift;
        else
            return p;
    };
    typename C::Elem *const wrow = codec.wr + row + x;
    if (Iind <= 1e-4f) {  // bulk (lbm.cuh:216-247)
        codec.store_bulk(wrow, aR, aB, P);
        return;
    }
    // interface (lbm.cuh:249-292): colour gradient over the 26 neighbours
    float sx = 0.f, sy = 0.f, sz = 0.f;
    static_for<kQ - 1>([&](auto I) {
        constexpr int i = decltype(I)::value + 1;
        using D = Dir<i>;
        const float wp = D::w * psi_at(D::cx, D::cy, D::cz);
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
    {
        const float g0 = Dir<0>::w * full(P[0]) + omega2<0>(t);
        codec.template store_row<0>(wrow, aR * g0, aB * g0);
    }
    static_for<(kQ - 1) / 2>([&](auto Q) {
        constexpr int i = 2 * decltype(Q)::value + 1;
        const float o2 = omega2<i>(t);  // even: the same for i and its opposite
        const float gi = Dir<i>::w * full(P[i]) + o2, go = Dir<i + 1>::w * full(P[i + 1]) + o2;
        const float d = recolour<i>(t);  // odd: -d for the opposite
        codec.template store_row<i>(wrow, aR * gi + d, aB * gi - d);
        codec.template store_row<i + 1>(wrow, aR * go - d, aB * go + d);
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
    float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f, v4 = 0.f;
    if (active) {
        const float dx = float(x) - ph.jet_x0, dz = float(z) - ph.jet_z0;
        const float r = sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)));
        const unsigned rb = unsigned(r);
        if (rb < unsigned(ph.NRB)) {
            key = (rb << 1) | (dx < 0.0f ? 1u : 0u);
            float ur = 0.0f;
            if (r > 1.0e-12f) ur = (ux * dx + uz * dz) / r;
            v0 = uy;
            v1 = uy * uy;
            v2 = ur;
            v3 = ur * ur;
            v4 = ur * uy;
        }
    }
    if (__all_sync(kFull, key == 0xffffffffu)) return;
    // run sums in float32 (a run is at most 32 nodes of one row); the run
    // totals go into the float64 accumulators
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned ok = __shfl_up_sync(kFull, key, d);
        const float o0 = __shfl_up_sync(kFull, v0, d);
        const float o1 = __shfl_up_sync(kFull, v1, d);
        const float o2 = __shfl_up_sync(kFull, v2, d);
        const float o3 = __shfl_up_sync(kFull, v3, d);
        const float o4 = __shfl_up_sync(kFull, v4, d);
        if (lane >= d && ok == key) {
            v0 += o0; v1 += o1; v2 += o2; v3 += o3; v4 += o4;
        }
    }
    const unsigned next = __shfl_down_sync(kFull, key, 1);
    const bool tail = (lane == 31) || (next != key);
    if (tail && key != 0xffffffffu) {
        const size_t M = size_t(s.g.NY) * ph.NRB;
        const size_t mi = size_t(y) * ph.NRB + (key >> 1);
        atomicAdd(s.radial + mi, double(v0));
        atomicAdd(s.radial + M + mi, double(v1));
        atomicAdd(s.radial + 2 * M + mi, double(v2));
        atomicAdd(s.radial + 3 * M + mi, double(v3));
        atomicAdd(s.radial + 4 * M + mi, double(v4));
    }
}

// ------------------------------------------------------------------ boundary arithmetic

// The jet boundary columns are written from every fused kernel (and from
// k_boundary).  Their arithmetic is rounded operation by operation (no
// contraction into fused multiply-adds, which the compiler chooses per
// kernel), so that every kernel writes the same bits.  Same formulas as
// make_eq, make_neq, feq and fneq (lbm.cuh:16-78).
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }

__device__ __forceinline__ EqTerms bnd_eq(float ux, float uy, float uz) {
    return EqTerms{ux, uy, uz, radd(radd(rmul(ux, ux), rmul(uy, uy)), rmul(uz, uz))};
}
__device__ __forceinline__ NeqTerms bnd_neq(const NodeMoments &m) {
    NeqTerms n;
    n.pxx = m.pxx; n.pxy = m.pxy; n.pyy = m.pyy; n.pyz = m.pyz; n.pzz = m.pzz; n.pxz = m.pxz;
    n.a3xxy = radd(rmul(m.pxx, m.uy), rmul(2.0f * m.pxy, m.ux));
    n.a3xxz = radd(rmul(m.pxx, m.uz), rmul(2.0f * m.pxz, m.ux));
    n.a3xyy = radd(rmul(m.pyy, m.ux), rmul(2.0f * m.pxy, m.uy));
    n.a3xzz = radd(rmul(m.pzz, m.ux), rmul(2.0f * m.pxz, m.uz));
    n.a3yyz = radd(rmul(m.pyy, m.uz), rmul(2.0f * m.pyz, m.uy));
    n.a3yzz = radd(rmul(m.pzz, m.uy), rmul(2.0f * m.pyz, m.uz));
    n.a3xyz = radd(radd(rmul(m.pxy, m.uz), rmul(m.pxz, m.uy)), rmul(m.pyz, m.ux));
    return n;
}
template <int I>
__device__ __forceinline__ float bnd_feq(float rho, const EqTerms &e) {
    using D = Dir<I>;
    float cu = 0.0f;
    if constexpr (D::cx != 0) cu = radd(cu, D::fx * e.ux);
    if constexpr (D::cy != 0) cu = radd(cu, D::fy * e.uy);
    if constexpr (D::cz != 0) cu = radd(cu, D::fz * e.uz);
    const float cu2 = rmul(cu, cu);
    const float A2 = radd(rsub(rmul(cu2, kInv2Cs4), rmul(e.usq, kInv2Cs2)), rmul(cu, kInvCs2));
    const float A3 = rmul(cu, rsub(rmul(cu2, kInv6Cs6), rmul(e.usq, kInv2Cs4)));
    return rmul(rmul(D::w, rho), radd(radd(1.0f, A2), A3));
}
template <int I>
__device__ __forceinline__ float bnd_fneq(const NeqTerms &n) {
    using D = Dir<I>;
    float A2 = 0.0f;
    if constexpr (D::Hxx != 0.0f) A2 = radd(A2, rmul(n.pxx, D::Hxx));
    if constexpr (D::Hxy != 0.0f) A2 = radd(A2, rmul(2.0f * n.pxy, D::Hxy));
    if constexpr (D::Hyy != 0.0f) A2 = radd(A2, rmul(n.pyy, D::Hyy));
    if constexpr (D::Hyz != 0.0f) A2 = radd(A2, rmul(2.0f * n.pyz, D::Hyz));
    if constexpr (D::Hzz != 0.0f) A2 = radd(A2, rmul(n.pzz, D::Hzz));
    if constexpr (D::Hxz != 0.0f) A2 = radd(A2, rmul(2.0f * n.pxz, D::Hxz));
    A2 = rmul(A2, kInv2Cs4);
    float A3 = 0.0f;
    if constexpr (D::Hxxy != 0.0f) A3 = radd(A3, rmul(n.a3xxy, D::Hxxy));
    if constexpr (D::Hxxz != 0.0f) A3 = radd(A3, rmul(n.a3xxz, D::Hxxz));
    if constexpr (D::Hxyy != 0.0f) A3 = radd(A3, rmul(n.a3xyy, D::Hxyy));
    if constexpr (D::Hxzz != 0.0f) A3 = radd(A3, rmul(n.a3xzz, D::Hxzz));
    if constexpr (D::Hyyz != 0.0f) A3 = radd(A3, rmul(n.a3yyz, D::Hyyz));
    if constexpr (D::Hyzz != 0.0f) A3 = radd(A3, rmul(n.a3yzz, D::Hyzz));
    if constexpr (D::Hxyz != 0.0f) A3 = radd(A3, rmul(2.0f * n.a3xyz, D::Hxyz));
    return rmul(D::w, radd(A2, rmul(A3, kInv2Cs6)));
}
// omega_at with the same rounding rule (the outlet's fluid plane)
__device__ __forceinline__ float bnd_omega_at(const Physics &ph, int y) {
    if (!ph.sponge) return ph.omega;
    const float s = clamp01(rmul(float(y) - ph.sponge_y_start, ph.sponge_inv_width));
    const float nus = rmul(ph.nu, radd(1.0f, rmul(ph.sponge_K, rmul(rmul(s, s), s))));
    return 1.0f / radd(0.5f, rmul(nus, kInvCs2));
}

__device__ __forceinline__ NodeMoments load_moments(const float *m, size_t stride, size_t id) {
    NodeMoments r;
    r.rr = m[kMomRR * stride + id]; r.rb = m[kMomRB * stride + id];
    r.ux = m[kMomUX * stride + id]; r.uy = m[kMomUY * stride + id]; r.uz = m[kMomUZ * stride + id];
    r.pxx = m[kMomPXX * stride + id]; r.pxy = m[kMomPXY * stride + id]; r.pyy = m[kMomPYY * stride + id];
    r.pyz = m[kMomPYZ * stride + id]; r.pzz = m[kMomPZZ * stride + id]; r.pxz = m[kMomPXZ * stride + id];
    return r;
}

// ------------------------------------------------------------------ boundary pieces

// Inlet column (x,z): density mask at y=0 and, for disc columns, the nine
// cy=+1 populations entering y=1 (jet/boundary_conditions.cuh:17-85).  They
// are stored in the ghost plane y=0 of `dst` at (x,0,z), where the y=1 nodes
// (x+cx, 1, z+cz) pull them.  `m` are the moments of fluid node (x,1,z).
template <class C>
__device__ __forceinline__ void inlet_column(const DeviceState &s, void *dst, float *psi_dst, int x, int z,
                                             int64_t step, const NodeMoments &m) {
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
    const float rT = radd(rrB, rbB);
    const float aR = rmul(rrB, 1.0f / rT), aB = rmul(rbB, 1.0f / rT);
    const float oms = rsub(1.0f, ph.omega_b);
    const EqTerms e = bnd_eq(0.0f, inlet_velocity(s, step, x, z), 0.0f);
    const NeqTerms n = bnd_neq(m);
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (Dir<i>::cy == 1) {
            const float gi = radd(bnd_feq<i>(rT, e), rmul(oms, bnd_fneq<i>(n)));
            C::store_to(dst, g, i, x, 0, z, rmul(aR, gi), rmul(aB, gi), ph.f16_rho0);
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
    auto conv = [uc](float b, float f) { return rsub(b, rmul(uc, rsub(b, f))); };
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
    const float rhoT = radd(rrB, rbB);
    const float inv = 1.0f / rhoT;
    const float aR = rmul(rrB, inv), aB = rmul(rbB, inv);
    const float oms = rsub(1.0f, bnd_omega_at(ph, g.NY - 2));
    const EqTerms e = bnd_eq(uxB, uyB, uzB);
    const NeqTerms n = bnd_neq(m);
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (Dir<i>::cy == -1) {
            const float gi = radd(bnd_feq<i>(rhoT, e), rmul(oms, bnd_fneq<i>(n)));
            C::store_to(dst, g, i, x, g.NY - 1, z, rmul(aR, gi), rmul(aB, gi), ph.f16_rho0);
        }
    });
}

// ------------------------------------------------------------------ the fused step

constexpr int kFusedThreads = 256;
// Row lengths the fused kernels are specialised for (the 128-column rows of
// the 128x256x128 jet, the 256-column rows of the 256x512x256 one); other
// row lengths take the runtime-geometry kernels.
constexpr int kFusedNX = 128;
constexpr int kFusedNX2 = 256;

#ifndef MCG_FUSED_MIN_BLOCKS
#define MCG_FUSED_MIN_BLOCKS 3  // CTAs per SM the register budget is sized for
#endif

// First row of this CTA's y-tile.  With the jet boundary in the step the
// tiles are numbered from the outlet end: the outlet tile's CTAs, which also
// write the outlet columns, then start first in each chunk instead of last.
// Neighbouring CTAs still hold neighbouring tiles.
__device__ __forceinline__ int tile_y0(const FusedTiling &T) {
    const int t = T.boundary ? T.ny_tiles - 1 - int(blockIdx.x) : int(blockIdx.x);
    return 1 + t * T.ty;
}

// Own-row results of a pulled node: the moments into the stage row, the
// fluid-plane moments for the boundary (fused_boundary or k_boundary), the
// adjoint's moment record.
template <class C>
__device__ __forceinline__ void tile_store_moments(const DeviceState &s, int x, int y, int zp, const NodeMoments &m,
                                                   float ps, float *msm_row, int tpr) {
    const Geometry &g = s.g;
    float *q = msm_row + x;
    q[kMomRR * tpr] = m.rr;
    q[kMomRB * tpr] = m.rb;
    q[kMomUX * tpr] = m.ux;
    q[kMomUY * tpr] = m.uy;
    q[kMomUZ * tpr] = m.uz;
    q[kMomPXX * tpr] = m.pxx;
    q[kMomPXY * tpr] = m.pxy;
    q[kMomPYY * tpr] = m.pyy;
    q[kMomPYZ * tpr] = m.pyz;
    q[kMomPZZ * tpr] = m.pzz;
    q[kMomPXZ * tpr] = m.pxz;
    if (g.boundary == kBoundaryJet && (y == 1 || y == g.NY - 2)) {
        // fluid-plane moments for the boundary launch
        float *b = s.bmom + ((size_t(y == 1 ? 0 : 1) * g.NZ + zp) * kMomCount) * g.NX + x;
        const float v[kMomCount] = {m.rr, m.rb, m.ux, m.uy, m.uz, m.pxx, m.pxy, m.pyy, m.pyz, m.pzz, m.pxz};
#pragma unroll
        for (int k = 0; k < kMomCount; ++k) b[size_t(k) * g.NX] = v[k];
    }
    if (s.tape) {
        // moment record of the pulled state (the adjoint sweep reads it)
        float *t = s.tape + (uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(zp));
        const size_t N = g.N;
        const float v[kTapePlanes] = {m.rr, m.rb, m.ux, m.uy, m.uz, m.pxx, m.pxy, m.pyy, m.pyz, m.pzz, m.pxz, ps};
#pragma unroll
        for (int k = 0; k < kTapePlanes; ++k) t[size_t(k) * N] = v[k];
    }
}

// One node of a tile row in plane zp, pulled in two halves.  tile_pull_issue
// loads the node's words (at a position that is not pulled, its psi);
// tile_pull_finish puts psi into `ring_row` (all columns, halo rows
// included), and for own rows the moments into `msm_row`, the fluid-plane
// moments for the boundary launch, the adjoint's moment record, and the
// radial statistics.  tile_pull_finish is warp-collective when kStats: all
// 32 lanes of a warp (one row) call it together.  TilePull holds the loads
// between the two.
template <class C>
struct TilePull {
    RawPull<C> raw;  // the node's pulled words, when `pull`
    float ps;        // psi of a position that is not pulled (ghost)
    bool pull;
};

template <class C, bool kPeriodic>
__device__ __forceinline__ void tile_pull_issue(const DeviceState &s, const C &codec, const float *__restrict__ psi_g,
                                                int x, int y, int zp, TilePull<C> &t) {
    const Geometry &g = s.g;
    t.pull = false;
    if (x >= g.NX) return;
    int xn = x, yn = y, zn = zp;
    if constexpr (kPeriodic) {
        xn = wrap_interior(x, g.NX);
        yn = wrap_interior(y, g.NY);
        zn = wrap_interior(zp, g.NZ);
        t.pull = true;
    } else {
        t.pull = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && zp >= 1 && zp <= g.NZ - 2;
    }
    if (t.pull)
        pull_issue<C, kPeriodic>(g, codec, xn, yn, zn, t.raw);
    else
        t.ps = psi_g[uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(zp)];
}

// A node's statistics sample held for a later radial_accumulate_warp call.
struct RadialSample {
    float ux, uy, uz;
    int y, z;
    bool active;
};

template <class C, bool kStats, bool kPeriodic>
__device__ __forceinline__ void tile_pull_finish(const DeviceState &s, const C &codec, int x, int y, int zp,
                                                 bool own_row, const TilePull<C> &t, float *ring_row, float *msm_row,
                                                 int tpr, RadialSample *defer = nullptr) {
    const Geometry &g = s.g;
    const bool xin = x >= 1 && x <= g.NX - 2;
    NodeMoments m{};
    bool have = false;
    if (x < g.NX) {
        float ps;
        if (t.pull && own_row) {  // own_row is uniform per warp: a warp covers part of one row
            m = moments_from(RawSource<C>{codec, t.raw});
            have = true;
            ps = psi_of(m.rr, m.rb);
        } else if (t.pull) {
            float rr, rb;
            densities_from(RawSource<C>{codec, t.raw}, rr, rb);
            ps = psi_of(rr, rb);
        } else {
            ps = t.ps;
        }
        ring_row[x] = ps;
        if (own_row && xin) tile_store_moments<C>(s, x, y, zp, m, ps, msm_row, tpr);
    }
    if constexpr (kStats) {
        if (defer) {
            *defer = RadialSample{m.ux, m.uy, m.uz, y, zp, have && xin};
        } else if (own_row) {
            radial_accumulate_warp(s, x, y, zp, have && xin, m.ux, m.uy, m.uz);
        }
    }
}

// tile_pull_issue + tile_pull_finish in one piece, for marches with nothing
// to overlap: the own-row / halo branch comes before the loads, so each
// branch consumes its loads as they arrive (issuing all of them before the
// branch keeps every word live at once and spills at 80 registers).
template <class C, bool kStats, bool kPeriodic>
__device__ __forceinline__ void tile_pull(const DeviceState &s, const C &codec, const float *__restrict__ psi_g, int x,
                                          int y, int zp, bool own_row, float *ring_row, float *msm_row, int tpr) {
    const Geometry &g = s.g;
    const bool xin = x >= 1 && x <= g.NX - 2;
    NodeMoments m{};
    bool have = false;
    if (x < g.NX) {
        int xn = x, yn = y, zn = zp;
        bool pull;
        if constexpr (kPeriodic) {
            xn = wrap_interior(x, g.NX);
            yn = wrap_interior(y, g.NY);
            zn = wrap_interior(zp, g.NZ);
            pull = true;
        } else {
            pull = xin && y >= 1 && y <= g.NY - 2 && zp >= 1 && zp <= g.NZ - 2;
        }
        float ps;
        if (pull && own_row) {  // uniform per warp: a warp covers part of one row
            m = pull_moments<C, kPeriodic>(g, codec, xn, yn, zn);
            have = true;
            ps = psi_of(m.rr, m.rb);
        } else if (pull) {
            float rr, rb;
            pull_densities<C, kPeriodic>(g, codec, xn, yn, zn, rr, rb);
            ps = psi_of(rr, rb);
        } else {
            ps = psi_g[uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(zp)];
        }
        ring_row[x] = ps;
        if (own_row && xin) tile_store_moments<C>(s, x, y, zp, m, ps, msm_row, tpr);
    }
    if constexpr (kStats) {
        if (own_row) radial_accumulate_warp(s, x, y, zp, have && xin, m.ux, m.uy, m.uz);
    }
}

// Relax interior node (x, y, zc) of a tile: moments from the stage row
// `msm_row`, psi of planes zc-1, zc, zc+1 from the ring planes pm, p0, pp at
// ring row r.
template <class C>
__device__ __forceinline__ void tile_collide(const DeviceState &s, const C &codec, int x, int y, int zc, int r,
                                             const float *msm_row, const float *pm, const float *p0, const float *pp,
                                             int tpr) {
    const Geometry &g = s.g;
    const float *q = msm_row + x;
    NodeMoments m;
    m.rr = q[kMomRR * tpr];
    m.rb = q[kMomRB * tpr];
    m.ux = q[kMomUX * tpr];
    m.uy = q[kMomUY * tpr];
    m.uz = q[kMomUZ * tpr];
    m.pxx = q[kMomPXX * tpr];
    m.pxy = q[kMomPXY * tpr];
    m.pyy = q[kMomPYY * tpr];
    m.pyz = q[kMomPYZ * tpr];
    m.pzz = q[kMomPZZ * tpr];
    m.pxz = q[kMomPXZ * tpr];
    const int base = r * tpr + x;
    auto psi_at = [&](int cx, int cy, int cz) {
        const float *pl = cz < 0 ? pm : (cz > 0 ? pp : p0);
        return pl[base + cy * tpr + cx];
    };
    collide_node(g, s.ph, codec, pop_row(g, y, zc), x, y, zc, m, psi_at);
}

// The jet boundary of a fused step, from the CTAs whose tile holds fluid row
// 1 (inlet) or NY-2 (outlet), once their march is over: every column of the
// chunk from the fluid-plane moments the march left in bmom (written by this
// CTA's threads, visible after the barrier), into the ghost planes of the
// buffer the step writes and the next step's psi.  A column touches only its
// own ghost nodes and the outlet state it carries, which no other CTA of the
// launch reads.  Kept out of the march, where it added its instructions to
// every row.  The condition is uniform over the CTA.
template <class C>
__device__ __forceinline__ void fused_boundary(const DeviceState &s, const FusedTiling &T, int y0, int ty, int z0,
                                               int lz) {
    const Geometry &g = s.g;
    const bool inlet = y0 == 1, outlet = y0 + ty - 1 == g.NY - 2;
    if (!T.boundary || !(inlet || outlet)) return;
    __syncthreads();
    const int nx = g.NX - 2;
    for (int side = 0; side < 2; ++side) {
        if (!(side == 0 ? inlet : outlet)) continue;
        for (int i = threadIdx.x; i < lz * nx; i += blockDim.x) {
            const int x = 1 + i % nx, z = z0 + i / nx;
            const NodeMoments m =
                load_moments(s.bmom + (size_t(side) * g.NZ + z) * kMomCount * g.NX, size_t(g.NX), size_t(x));
            if (side == 0)
                inlet_column<C>(s, T.bnd_dst, T.bnd_psi, x, z, int64_t(T.bnd_step), m);
            else
                outlet_column<C>(s, T.bnd_dst, T.bnd_psi, x, z, m);
        }
    }
}

// Geometry of a fused launch: with kNX > 0 (rows of exactly kNX columns, one
// thread per column) the row length and slot counts are compile-time
// constants, so population, slot and shared-memory offsets fold into the
// loads' immediate offsets.
template <class C, int kNX>
__device__ __forceinline__ DeviceState fused_state(const DeviceState &s) {
    DeviceState l = s;
    if constexpr (kNX > 0) {
        l.g.NX = kNX;
        l.g.sy = kNX;
        l.g.slots = 9 * C::kGroupSlots;
    }
    return l;
}
template <class C, int kNX>
__device__ __forceinline__ C fused_codec(const DeviceState &s, int cur) {
    C c = make_codec<C>(s, cur);
    if constexpr (kNX > 0) c.NX = kNX;
    return c;
}

template <class C, bool kStats, bool kPeriodic, int kNX>
__global__ void __launch_bounds__(kFusedThreads, MCG_FUSED_MIN_BLOCKS) k_fused(const DeviceState s_arg,
                                                                              const FusedTiling T, int cur,
                                                                              int64_t step) {
    extern __shared__ float sm[];
    const DeviceState s = fused_state<C, kNX>(s_arg);
    const Geometry &g = s.g;
    const int tpr = kNX > 0 ? kNX : T.tpr;
    const int rpt = kFusedThreads / tpr;
    // row group of this thread; groups beyond rpt (when tpr does not divide
    // the block) start past every row and only take part in the barriers
    const int lr0 = threadIdx.x / tpr;
    const int lr = lr0 < rpt ? lr0 : T.ty + 2;
    const int x = threadIdx.x - lr0 * tpr;
    const int y0 = tile_y0(T);
    const int ty = min(T.ty, g.NY - 1 - y0);
    const int z0 = 1 + int(blockIdx.y) * T.lz;
    const int lz = min(T.lz, g.NZ - 1 - z0);
    const int pstride = (T.ty + 2) * tpr;  // one psi plane of the ring
    float *ring = sm;                      // [3][ty+2][tpr]
    float *msm = sm + 3 * pstride;         // [2][ty][11][tpr]
    const int mplane = T.ty * kMomCount * tpr;
    const C codec = fused_codec<C, kNX>(s_arg, cur);
    const float *__restrict__ psi_g = s_arg.psi[step & 1];  // indexed on the parameter, not the local copy
    const bool xin = x >= 1 && x <= g.NX - 2;
    // Odd chunks march down: the plane two neighbouring chunks both pull (one
    // as its halo, one as its own) is then pulled by both at the same end of
    // their marches, close in time, and the second pull finds it in L2.
    const bool down = T.alternate && (blockIdx.y & 1);
    for (int k = 0; k <= lz + 1; ++k) {
        const int zp = down ? z0 + lz - k : z0 - 1 + k;
        float *ringp = ring + (zp % 3) * pstride;
        float *msmp = msm + (zp & 1) * mplane;
        const bool own_plane = zp >= z0 && zp < z0 + lz;
        // ---- pull plane zp: psi for rows y0-1 .. y0+ty, moments for own rows
        for (int r = lr; r < ty + 2; r += rpt) {
            tile_pull<C, kStats, kPeriodic>(s, codec, psi_g, x, y0 - 1 + r, zp, own_plane && r >= 1 && r <= ty,
                                            ringp + r * tpr, msmp + (r - 1) * kMomCount * tpr, tpr);
        }
        __syncthreads();
        // ---- relax the plane behind the march front, whose neighbours are all pulled
        const int zc = down ? zp + 1 : zp - 1;
        if (zc >= z0 && zc < z0 + lz) {
            const float *pm = ring + ((zc + 2) % 3) * pstride;  // plane zc-1
            const float *p0 = ring + (zc % 3) * pstride;        // plane zc
            const float *pp = ring + ((zc + 1) % 3) * pstride;  // plane zc+1
            const float *mc = msm + (zc & 1) * mplane;
            for (int r = 1 + lr; r <= ty; r += rpt) {
                if (!xin) continue;
                tile_collide(s, codec, x, y0 - 1 + r, zc, r, mc + (r - 1) * kMomCount * tpr, pm, p0, pp, tpr);
            }
        }
        __syncthreads();
    }
    fused_boundary<C>(s, T, y0, ty, z0, lz);
}

// ------------------------------------------------------------------ software-pipelined fused step

// The tile march of k_fused with the pull and the relaxation in the same
// phase: iteration k pulls march plane k and relaxes march plane k-2, whose
// psi neighbours (planes k-3 .. k-1) and moments were pulled in earlier
// iterations.  The pull writes ring slot k mod 4 and stage slot k mod 3; the
// relaxation reads ring slots k-3 .. k-1 and stage slot k-2 - all different -
// so one __syncthreads per iteration suffices.  Between barriers the warps of
// a CTA drift apart, and the memory-bound pull of one warp overlaps the
// ALU-bound relaxation of another.
constexpr int kPipeRing = 4, kPipeStage = 3;
// CTAs per SM the pipelined kernel's register budget is sized for: float32
// (3-row tiles, 3 CTAs, 80 registers) measured faster than 2 CTAs at 128
// registers; float16 keeps 2 (its words in flight across the relaxation need
// the registers).
template <class C>
struct PipeBlocks {
    static constexpr int value = std::is_same<C, CodecF16>::value ? 2 : 3;
};

template <class C, bool kStats, bool kPeriodic, int kNX>
__global__ void __launch_bounds__(kFusedThreads, PipeBlocks<C>::value) k_fused_pipe(const DeviceState s_arg,
                                                                                  const FusedTiling T, int cur,
                                                                                  int64_t step) {
    extern __shared__ float sm[];
    const DeviceState s = fused_state<C, kNX>(s_arg);
    const Geometry &g = s.g;
    const int tpr = kNX > 0 ? kNX : T.tpr;
    const int rpt = kFusedThreads / tpr;
    const int lr0 = threadIdx.x / tpr;
    const int lr = lr0 < rpt ? lr0 : T.ty + 2;  // idle groups (tpr not dividing the block) skip every row
    const int x = threadIdx.x - lr0 * tpr;
    const int pstride = (T.ty + 2) * tpr;
    const int mplane = T.ty * kMomCount * tpr;
    float *ring = sm;                        // [4][ty+2][tpr]
    float *msm = sm + kPipeRing * pstride;   // [3][ty][11][tpr]
    const C codec = fused_codec<C, kNX>(s_arg, cur);
    const float *__restrict__ psi_g = s_arg.psi[step & 1];  // indexed on the parameter, not the local copy
    const bool xin = x >= 1 && x <= g.NX - 2;
    // Float16 words (27 registers a node) stay in flight across the relaxation
    // of another row: measured +4 % on 128x256x128.  Float32 (27 float2, 54
    // registers) pulls then relaxes: its 3-CTA, 80-register default is faster
    // than the overlap, which spills there.
    constexpr bool kOverlap = std::is_same<C, CodecF16>::value;
    // One CTA per y-tile (blockIdx.x) and z chunk (blockIdx.y): CTAs of
    // neighbouring y-tiles run the same planes at about the same time, so the
    // halo rows one pulls are the own rows another pulled and hit L2.  Odd
    // chunks march down: two neighbouring chunks then pull their shared
    // boundary plane at the same end of their marches (L2 again).
    {
        const int y0 = tile_y0(T);
        const int z0 = 1 + int(blockIdx.y) * T.lz;
        const int lz = min(T.lz, g.NZ - 1 - z0);
        const bool down = T.alternate && (blockIdx.y & 1);
        const int ty = min(T.ty, g.NY - 1 - y0);
        auto plane = [&](int k) { return down ? z0 + lz - k : z0 - 1 + k; };
        RadialSample held{};   // statistics of this warp's last own row, taken
        bool pending = false;  // after the next row's loads are issued
        for (int k = 0; k <= lz + 2; ++k) {
            const bool do_pull = k <= lz + 1;
            const int c = k - 2;  // march index of the plane relaxed in this iteration
            const bool do_relax = c >= 1 && c <= lz;
            const int zp = plane(k);
            float *ringp = ring + (k % kPipeRing) * pstride;
            float *msmp = msm + (k % kPipeStage) * mplane;
            const bool own_plane = k >= 1 && k <= lz;
            const int zc = plane(c);
            const float *pm = ring + (((down ? c + 1 : c - 1) + kPipeRing) % kPipeRing) * pstride;  // plane zc-1
            const float *p0 = ring + ((c + kPipeRing) % kPipeRing) * pstride;                       // plane zc
            const float *pp = ring + (((down ? c - 1 : c + 1) + kPipeRing) % kPipeRing) * pstride;  // plane zc+1
            const float *mc = msm + ((c + kPipeStage) % kPipeStage) * mplane;
            // rows of this thread: pull rows lr, lr+rpt, ... (< ty+2) and relax rows
            // 1+lr, 1+lr+rpt, ... (<= ty), interleaved so that a warp has loads of
            // one row in flight while it relaxes another.  With one row group (rows
            // of 256 columns) the upper half of the row's threads takes the rows in
            // a rotated order, so that one half pulls while the other relaxes, as
            // two row groups do; the order of the rows within an iteration is free.
            // (split at a warp boundary: the statistics are warp-collective)
            const int rot = (rpt == 1 && x >= (tpr / 64) * 32) ? (ty + 2) / 2 : 0;
            for (int ri = lr; ri < ty + 2; ri += rpt) {
                const int r = rot ? (ri + rot) % (ty + 2) : ri;
                const bool own = own_plane && r >= 1 && r <= ty;
                const int rc = r + 1;
                if constexpr (kOverlap) {
                    // the loads of row r are in flight while this warp takes the
                    // statistics of its previous own row and relaxes row r+1
                    TilePull<C> tp;
                    if (do_pull) tile_pull_issue<C, kPeriodic>(s, codec, psi_g, x, y0 - 1 + r, zp, tp);
                    if constexpr (kStats) {
                        if (pending) {  // warp-uniform
                            radial_accumulate_warp(s, x, held.y, held.z, held.active, held.ux, held.uy, held.uz);
                            pending = false;
                        }
                    }
                    if (do_relax && rc <= ty && xin)
                        tile_collide(s, codec, x, y0 - 1 + rc, zc, rc, mc + (rc - 1) * kMomCount * tpr, pm, p0, pp,
                                     tpr);
                    if (do_pull) {
                        tile_pull_finish<C, kStats, kPeriodic>(s, codec, x, y0 - 1 + r, zp, own, tp, ringp + r * tpr,
                                                               msmp + (r - 1) * kMomCount * tpr, tpr,
                                                               kStats && own ? &held : nullptr);
                        if (kStats && own) pending = true;
                    }
                } else {
                    if (do_pull)
                        tile_pull<C, kStats, kPeriodic>(s, codec, psi_g, x, y0 - 1 + r, zp, own, ringp + r * tpr,
                                                        msmp + (r - 1) * kMomCount * tpr, tpr);
                    if (do_relax && rc <= ty && xin)
                        tile_collide(s, codec, x, y0 - 1 + rc, zc, rc, mc + (rc - 1) * kMomCount * tpr, pm, p0, pp,
                                     tpr);
                }
            }
            __syncthreads();
        }
        if constexpr (kStats) {
            if (pending) radial_accumulate_warp(s, x, held.y, held.z, held.active, held.ux, held.uy, held.uz);
        }
        fused_boundary<C>(s, T, y0, ty, z0, lz);
    }
}

// ------------------------------------------------------------------ bulk-staged pipelined fused step

// One-dimensional bulk copies (cp.async.bulk, no multicast) into shared
// memory, completed on an mbarrier; one GPU, the CTA's own shared memory.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Waits for the phase of parity `parity` of `bar` to complete: at most
// `limit` tries, each suspending the thread for about a microsecond at most.
// Returns false when the limit ran out (limit 0: at once).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
            : "memory");
        if (done) return true;
    }
    return false;
}
// Barrier of the `count` threads of one row group (named barrier `id` > 0);
// returns the OR of `pred` over them.
__device__ __forceinline__ bool group_barrier_or(int id, int count, bool pred) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"(uint32_t(pred)), "r"(id), "r"(count)
        : "memory");
    return out != 0;
}

// Row image of a staged pull: the 9 (cy, cz) source segments of row (y, z)
// (3 slots x NX elements each, group g = dir_group at g*3*NX), copied
// verbatim from the population buffer.  Direction I of node x reads slot
// (g, cx+1) at column x - cx, with the lateral wrap of PullMap: columns 1
// and NX-2 wrap for cx = +1 / -1, except in a segment that comes from a y
// ghost plane (the boundary's unwrapped slots).
template <class C, int kNX>
struct StagedRow {
    const typename C::Elem *img;
    int x;
    int wxp, wxm;
    bool gy_p, gy_m;
    __device__ __forceinline__ StagedRow(const typename C::Elem *img_, int x_, int y, const Geometry &g, bool periodic)
        : img(img_), x(x_) {
        wxp = (x == 1) ? (kNX - 2) : 0;
        wxm = (x == kNX - 2) ? -(kNX - 2) : 0;
        gy_p = !periodic && y == 1;
        gy_m = !periodic && y == g.NY - 2;
    }
    template <int I>
    __device__ __forceinline__ typename C::Raw load() const {
        using D = Dir<I>;
        int xc = 0;
        if constexpr (D::cx == 1) xc = wxp;
        if constexpr (D::cx == -1) xc = wxm;
        if constexpr (D::cy == 1) xc = gy_p ? 0 : xc;
        if constexpr (D::cy == -1) xc = gy_m ? 0 : xc;
        return img[(dir_group(I) * C::kGroupSlots + D::cx + 1) * kNX + x - D::cx + xc];
    }
};

// Issues the 9 segment copies of pulled row (y, z) (own coordinates, wrapped
// for the periodic box) into `img`, completing on `bar`.
template <class C, int kNX>
__device__ __forceinline__ void stage_row(const Geometry &g, const C &codec, bool periodic, int y, int z,
                                          typename C::Elem *img, uint64_t *bar) {
    constexpr uint32_t seg = uint32_t(C::kGroupSlots * kNX * sizeof(typename C::Elem));
    mbar_expect_tx(bar, 9 * seg);
    for (int grp = 0; grp < 9; ++grp) {
        const int cy = grp / 3 - 1, cz = grp % 3 - 1;
        int ys = y - cy, zs = z - cz;
        const bool ghost = !periodic && (ys == 0 || ys == g.NY - 1);
        if (!ghost) {
            zs = wrap_interior(zs, g.NZ);
            if (periodic) ys = wrap_interior(ys, g.NY);
        }
        const typename C::Elem *src =
            codec.rd + ((size_t(zs) * g.NY + ys) * kQ + size_t(grp) * C::kGroupSlots) * kNX;
        bulk_copy_g2s(img + grp * C::kGroupSlots * kNX, src, seg, bar);
    }
}

// The pipelined march of k_fused_pipe with each pulled row staged: the 9
// source segments of a row (3 KB each in float32 at 128 columns) arrive in
// shared memory by bulk copies while the row group (the 128 threads of one
// row, 4 warps) finishes its previous row and relaxes another.  Each row
// group owns one row image and one mbarrier; after its threads have read the
// image into registers (a barrier of the group), its first thread issues the
// copies of the group's next pulled row.  Pulls therefore hold no global
// loads in registers.  Ghost rows and planes are not pulled (psi from HBM).
// The pulled words, their order and the arithmetic are those of
// k_fused_pipe, so the results are bit-identical.
// Every wait has an iteration limit (T.wait_limit tries of about 1 us): when
// it runs out, the group sets flag[1], issues nothing more and finishes the
// march on whatever its image holds; before it exits, the group's first
// thread waits (again bounded) for the copies it has in flight.
constexpr int kBulkBarBytes = 128;  // mbarriers at the start of the shared memory
template <class C>
constexpr int bulk_image_bytes() { return kQ * kFusedNX * int(sizeof(typename C::Elem)); }

template <class C, bool kStats, bool kPeriodic>
__global__ void __launch_bounds__(kFusedThreads, 2) k_fused_bulk(const DeviceState s_arg, const FusedTiling T,
                                                                 int cur, int64_t step) {
    constexpr int kNX = kFusedNX;
    constexpr int tpr = kNX;
    constexpr int rpt = kFusedThreads / tpr;  // row groups
    using E = typename C::Elem;
    extern __shared__ __align__(128) unsigned char smb[];
    const DeviceState s = fused_state<C, kNX>(s_arg);
    const Geometry &g = s.g;
    const int grp = threadIdx.x / tpr;
    const int x = threadIdx.x - grp * tpr;
    const bool leader = x == 0;
    const int pstride = (T.ty + 2) * tpr;
    const int mplane = T.ty * kMomCount * tpr;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smb) + grp;
    E *img = reinterpret_cast<E *>(smb + kBulkBarBytes) + grp * (kQ * kNX);
    float *ring = reinterpret_cast<float *>(smb + kBulkBarBytes + rpt * bulk_image_bytes<C>());  // [4][ty+2][tpr]
    float *msm = ring + kPipeRing * pstride;                                                    // [3][ty][11][tpr]
    const C codec = fused_codec<C, kNX>(s_arg, cur);
    const float *__restrict__ psi_g = s_arg.psi[step & 1];
    const bool xin = x >= 1 && x <= kNX - 2;
    const int y0 = tile_y0(T);
    const int z0 = 1 + int(blockIdx.y) * T.lz;
    const int lz = min(T.lz, g.NZ - 1 - z0);
    const bool down = T.alternate && (blockIdx.y & 1);
    const int ty = min(T.ty, g.NY - 1 - y0);
    auto plane = [&](int k) { return down ? z0 + lz - k : z0 - 1 + k; };
    // a row of the march that is pulled (the periodic box pulls every row,
    // ghost rows as their wrapped interior rows)
    auto pulled = [&](int k, int r) {
        if constexpr (kPeriodic) return true;
        const int y = y0 - 1 + r, z = plane(k);
        return y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    };
    // the group's next pulled row after (k, r); k > lz+1 when there is none
    auto next_pull = [&](int &k, int &r) {
        do {
            r += rpt;
            if (r >= ty + 2) {
                r = grp;
                ++k;
            }
        } while (k <= lz + 1 && !pulled(k, r));
    };
    auto issue = [&](int k, int r) {
        int y = y0 - 1 + r, z = plane(k);
        if constexpr (kPeriodic) {
            y = wrap_interior(y, g.NY);
            z = wrap_interior(z, g.NZ);
        }
        stage_row<C, kNX>(g, codec, kPeriodic, y, z, img, bar);
    };
    if (threadIdx.x == 0) {
        for (int k = 0; k < rpt; ++k) mbar_init(reinterpret_cast<uint64_t *>(smb) + k, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const uint32_t limit = uint32_t(T.wait_limit);
    bool failed = false;    // uniform over the row group
    bool in_flight = false; // leader: copies issued and not yet waited for
    uint32_t parity = 0;     // of the next phase this thread waits for
    if (leader && grp < ty + 2) {
        int k = 0, r = grp;
        if (!pulled(k, r)) next_pull(k, r);
        if (k <= lz + 1) {
            issue(k, r);
            in_flight = true;
        }
    }
    for (int k = 0; k <= lz + 2; ++k) {
        const bool do_pull = k <= lz + 1;
        const int c = k - 2;
        const bool do_relax = c >= 1 && c <= lz;
        const int zp = plane(k);
        float *ringp = ring + (k % kPipeRing) * pstride;
        float *msmp = msm + (k % kPipeStage) * mplane;
        const bool own_plane = k >= 1 && k <= lz;
        const int zc = plane(c);
        const float *pm = ring + (((down ? c + 1 : c - 1) + kPipeRing) % kPipeRing) * pstride;
        const float *p0 = ring + ((c + kPipeRing) % kPipeRing) * pstride;
        const float *pp = ring + (((down ? c - 1 : c + 1) + kPipeRing) % kPipeRing) * pstride;
        const float *mc = msm + ((c + kPipeStage) % kPipeStage) * mplane;
        for (int r = grp; r < ty + 2; r += rpt) {
            const bool own = own_plane && r >= 1 && r <= ty;
            const int y = y0 - 1 + r;
            if (do_pull) {
                if (pulled(k, r)) {
                    bool late = false;
                    if (!failed) {
                        late = !mbar_wait(bar, parity, limit);
                        if (!late) {
                            parity ^= 1u;
                            if (leader) in_flight = false;  // the copies have landed
                        }
                    }
                    int xn = x, yn = y, zn = zp;
                    if constexpr (kPeriodic) {
                        xn = wrap_interior(x, kNX);
                        yn = wrap_interior(y, g.NY);
                        zn = wrap_interior(zp, g.NZ);
                    }
                    const bool pull = kPeriodic || xin;
                    RawPull<C> raw;
                    if (pull) {
                        const StagedRow<C, kNX> src(img, xn, yn, g, kPeriodic);
                        static_for<kQ>([&](auto I) {
                            constexpr int i = decltype(I)::value;
                            raw.v[i] = src.template load<i>();
                        });
                    }
                    // every thread of the group has read the image
                    const bool now_failed = group_barrier_or(1 + grp, tpr, late);
                    if (now_failed && !failed) {
                        failed = true;
                        if (leader) atomicExch(s.flag + 1, 1);
                    }
                    if (leader && !failed) {
                        int kn = k, rn = r;
                        next_pull(kn, rn);
                        if (kn <= lz + 1) {
                            issue(kn, rn);
                            in_flight = true;
                        }
                    }
                    NodeMoments m{};
                    float ps = 0.0f;
                    if (pull && own) {  // own is uniform per warp
                        m = moments_from(RawSource<C>{codec, raw});
                        ps = psi_of(m.rr, m.rb);
                    } else if (pull) {
                        float rr, rb;
                        densities_from(RawSource<C>{codec, raw}, rr, rb);
                        ps = psi_of(rr, rb);
                    } else {
                        ps = psi_g[uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(zp)];
                    }
                    ringp[r * tpr + x] = ps;
                    if (own && xin)
                        tile_store_moments<C>(s, x, y, zp, m, ps, msmp + (r - 1) * kMomCount * tpr, tpr);
                    if constexpr (kStats) {
                        if (own) radial_accumulate_warp(s, x, y, zp, pull && xin, m.ux, m.uy, m.uz);
                    }
                } else {
                    ringp[r * tpr + x] =
                        psi_g[uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(zp)];
                }
            }
            const int rc = r + 1;
            if (do_relax && rc <= ty && xin)
                tile_collide(s, codec, x, y0 - 1 + rc, zc, rc, mc + (rc - 1) * kMomCount * tpr, pm, p0, pp, tpr);
        }
        __syncthreads();
    }
    // copies still in flight after a wait ran out land before the CTA exits
    if (leader && in_flight) mbar_wait(bar, parity, limit > 0 ? limit : kBulkDrainLimit);
    fused_boundary<C>(s, T, y0, ty, z0, lz);
}

// Shared memory of k_fused_bulk with `ty`-row tiles: mbarriers, one row image
// per row group, the psi ring and the moment stage of k_fused_pipe.
template <class C>
constexpr int bulk_smem_for(int ty) {
    return kBulkBarBytes + (kFusedThreads / kFusedNX) * bulk_image_bytes<C>() +
           (kPipeRing * (ty + 2) + kPipeStage * kMomCount * ty) * kFusedNX * 4;
}
// rows per tile of k_fused_bulk: float32 2 (3 KB segments, 27 KB images),
// float16 4; both fit two CTAs per SM
template <class C>
constexpr int bulk_rows() { return std::is_same<C, CodecF16>::value ? 4 : 2; }
template <class C>
constexpr int bulk_smem_bytes() { return bulk_smem_for<C>(bulk_rows<C>()); }

// ------------------------------------------------------------------ granular sequence

constexpr int kBX = 32, kBY = 8;

// launch_Macros equivalent: moments and psi of every interior node to HBM.
template <class C, bool kPeriodic>
__global__ void __launch_bounds__(kBX * kBY) k_moments(const DeviceState s, const C codec, int64_t step) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const NodeMoments m = pull_moments<C, kPeriodic>(g, codec, x, y, z);
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
    const float ps = psi_of(m.rr, m.rb);
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

// launch_collistream equivalent: relax from the moment planes and psi in HBM.
template <class C>
__global__ void __launch_bounds__(kBX * kBY, 4) k_collide(const DeviceState s, const C codec, int64_t step) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const size_t N = g.N;
    const float *__restrict__ mom = s.mom;
    NodeMoments m;
    m.rr = __ldg(mom + kMomRR * N + id);
    m.rb = __ldg(mom + kMomRB * N + id);
    m.ux = __ldg(mom + kMomUX * N + id);
    m.uy = __ldg(mom + kMomUY * N + id);
    m.uz = __ldg(mom + kMomUZ * N + id);
    m.pxx = __ldg(mom + kMomPXX * N + id);
    m.pxy = __ldg(mom + kMomPXY * N + id);
    m.pyy = __ldg(mom + kMomPYY * N + id);
    m.pyz = __ldg(mom + kMomPYZ * N + id);
    m.pzz = __ldg(mom + kMomPZZ * N + id);
    m.pxz = __ldg(mom + kMomPXZ * N + id);
    const float *__restrict__ psi = s.psi[step & 1];
    auto psi_at = [&](int cx, int cy, int cz) { return __ldg(psi + (int(id) + cx + g.sy * cy + g.sz * cz)); };
    collide_node(g, s.ph, codec, pop_row(g, y, z), x, y, z, m, psi_at);
}


// Jet boundary of step `step`: blockIdx.z == 0 is the inlet (y=0 plane), 1 the
// outlet (y=NY-1 plane), unless `which` selects one.  Values go to the ghost
// planes of buffer `wbuf` (the one the collision of this step writes) and to
// the psi buffer of the next step.
template <class C>
__global__ void __launch_bounds__(256) k_boundary(const DeviceState s, int wbuf, int64_t step, int which,
                                                  int from_bmom) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < 1 || x > g.NX - 2 || z < 1 || z > g.NZ - 2) return;
    const int side = which >= 0 ? which : int(blockIdx.z);
    float *psi_next = s.psi[(step + 1) & 1];
    NodeMoments m;
    if (from_bmom) {
        m = load_moments(s.bmom + (size_t(side) * g.NZ + z) * kMomCount * g.NX, size_t(g.NX), size_t(x));
    } else {
        const int yF = side == 0 ? 1 : g.NY - 2;
        m = load_moments(s.mom, size_t(g.N), size_t(x) + size_t(g.sy) * size_t(yF) + size_t(g.sz) * size_t(z));
    }
    if (side == 0) inlet_column<C>(s, s.pops[wbuf], psi_next, x, z, step, m);
    else outlet_column<C>(s, s.pops[wbuf], psi_next, x, z, m);
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
            xx = wrap_interior(x, g.NX);
            yy = wrap_interior(y, g.NY);
            zz = wrap_interior(z, g.NZ);
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

// Populations of every interior node, written at their pull sources.  The
// current buffer takes every slot; the other one only the slots on a y ghost
// plane, which no step rewrites (they must hold the initial value in both
// buffers).  Every other slot of the other buffer is written by the first
// step before anything reads it.  Directions are unrolled, so the pull
// source and the equilibrium take compile-time lattice constants.
template <class C>
__global__ void k_init_pops(const DeviceState s, int mode, float noise) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const size_t N = g.N;
    const float rr = s.mom[kMomRR * N + id], rb = s.mom[kMomRB * N + id];
    const float ux = s.mom[kMomUX * N + id], uy = s.mom[kMomUY * N + id], uz = s.mom[kMomUZ * N + id];
    const float usq = ux * ux + uy * uy + uz * uz;
    const bool periodic = g.boundary == kBoundaryPeriodic;
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        using D = Dir<i>;
        float fr, fb;
        if (mode == 3) {
            // per colour, the third-order equilibrium at the node's velocity (lbm.cuh:16-35)
            const float cu = D::fx * ux + D::fy * uy + D::fz * uz;
            const float A2 = (cu * cu) * kInv2Cs4 - usq * kInv2Cs2 + cu * kInvCs2;
            const float A3 = cu * ((cu * cu) * kInv6Cs6 - usq * kInv2Cs4);
            const float e = D::w * (1.0f + A2 + A3);
            fr = e * rr;
            fb = e * rb;
        } else {
            // jetDensity: feq(rho, 0) = w rho; bubble: w rho (jetIn.cuh:26-34, bubbleIn.cuh:25-39)
            fr = D::w * rr;
            fb = D::w * rb;
            if (noise != 0.0f) {
                const float u = hash_uniform(s.ph.seed, 0x1D17ull, id, uint64_t(i));
                const float f = 1.0f + (2.0f * u - 1.0f) * noise;
                fr = fr * f;
                fb = fb * f;
            }
        }
        int xs, ys, zs;
        pull_src_rt(g, x, y, z, i, xs, ys, zs);
        C::store_to(s.pops[0], g, i, xs, ys, zs, fr, fb, s.ph.f16_rho0);
        if (!periodic && (ys == 0 || ys == g.NY - 1)) C::store_to(s.pops[1], g, i, xs, ys, zs, fr, fb, s.ph.f16_rho0);
    });
}

__global__ void k_refresh_psi(const DeviceState s) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.NX || y >= g.NY) return;
    int xx = x, yy = y, zz = z;
    if (g.boundary == kBoundaryPeriodic) {
        xx = wrap_interior(x, g.NX);
        yy = wrap_interior(y, g.NY);
        zz = wrap_interior(z, g.NZ);
    }
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const uint32_t src = uint32_t(xx) + uint32_t(g.sy) * uint32_t(yy) + uint32_t(g.sz) * uint32_t(zz);
    const size_t N = g.N;
    const float p = psi_of(s.mom[kMomRR * N + src], s.mom[kMomRB * N + src]);
    s.psi[0][id] = p;
    s.psi[1][id] = p;
}

// Host state transfer in z-chunks of the reference layout f[i*Ncells + id].
// A chunk holds planes [z0, z0 + nz) of both colours, staged as
// stage[colour][i][id - z0*NX*NY] with `pitch` elements per direction row, so
// that the host copy of each colour is one 2-D copy of 27 rows.
//
// Scatter: the populations of the chunk's interior nodes go to their pull
// sources in buffer `wbuf` (the sources of planes z0 and z0+nz-1 lie in the
// neighbouring chunks' planes; every source is written by exactly one node).
template <class C>
__global__ void k_scatter_chunk(const DeviceState s, int wbuf, const float *__restrict__ stage, size_t pitch, int z0) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = z0 + int(blockIdx.z);
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const size_t lid = size_t(x) + size_t(g.sy) * size_t(y) + size_t(g.sz) * size_t(blockIdx.z);
    const float *fr = stage, *fb = stage + size_t(kQ) * pitch;
    for (int i = 0; i < kQ; ++i) {
        int xs, ys, zs;
        pull_src_rt(g, x, y, z, i, xs, ys, zs);
        C::store_to(s.pops[wbuf], g, i, xs, ys, zs, fr[size_t(i) * pitch + lid], fb[size_t(i) * pitch + lid],
                    s.ph.f16_rho0);
    }
}

// Gather: f(t) = pops[cur] pulled at the chunk's nodes into the stage; ghost
// nodes give 0.
template <class C>
__global__ void k_gather_chunk(const DeviceState s, int cur, float *__restrict__ stage, size_t pitch, int z0) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = z0 + int(blockIdx.z);
    if (x >= g.NX || y >= g.NY) return;
    const size_t lid = size_t(x) + size_t(g.sy) * size_t(y) + size_t(g.sz) * size_t(blockIdx.z);
    const bool interior = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    float *fr = stage, *fb = stage + size_t(kQ) * pitch;
    for (int i = 0; i < kQ; ++i) {
        float r = 0.0f, b = 0.0f;
        if (interior) {
            int xs, ys, zs;
            pull_src_rt(g, x, y, z, i, xs, ys, zs);
            C::load_from(s.pops[cur], g, i, xs, ys, zs, r, b, s.ph.f16_rho0);
        }
        fr[size_t(i) * pitch + lid] = r;
        fb[size_t(i) * pitch + lid] = b;
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
            int xs, ys, zs;
            pull_src_rt(g, x, y, z, i, xs, ys, zs);
            float fr, fb;
            C::load_from(s.pops[cur], g, i, xs, ys, zs, fr, fb, s.ph.f16_rho0);
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
            int xs, ys, zs;
            pull_src_rt(g, x, y, z, i, xs, ys, zs);
            float fr, fb;
            C::load_from(s.pops[cur], g, i, xs, ys, zs, fr, fb, s.ph.f16_rho0);
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


template <class C, bool kStats, bool kPeriodic, int kNX>
cudaError_t fused_attr_nx(int smem) {
    cudaError_t e = cudaFuncSetAttribute(k_fused<C, kStats, kPeriodic, kNX>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_fused_pipe<C, kStats, kPeriodic, kNX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem);
}

template <class C, bool kStats, bool kPeriodic>
cudaError_t fused_attr(int smem) {
    cudaError_t e = fused_attr_nx<C, kStats, kPeriodic, 0>(smem);
    if (e != cudaSuccess) return e;
    e = fused_attr_nx<C, kStats, kPeriodic, kFusedNX>(smem);
    if (e != cudaSuccess) return e;
    e = fused_attr_nx<C, kStats, kPeriodic, kFusedNX2>(smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_fused_bulk<C, kStats, kPeriodic>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bulk_smem_bytes<C>());
}

template <class C, bool kStats, bool kPeriodic, int kNX>
cudaError_t fused_launch_nx(const DeviceState &s, const FusedTiling &t, int cur, int64_t step, cudaStream_t st) {
    if constexpr (kNX == kFusedNX) {
        if (t.bulk) {
            k_fused_bulk<C, kStats, kPeriodic>
                <<<dim3(t.ny_tiles, t.nz_chunks), dim3(kFusedThreads), size_t(t.smem_bytes), st>>>(s, t, cur, step);
            return cudaGetLastError();
        }
    }
    if (t.pipe) {
        k_fused_pipe<C, kStats, kPeriodic, kNX>
            <<<dim3(t.ny_tiles, t.nz_chunks), dim3(kFusedThreads), size_t(t.smem_bytes), st>>>(s, t, cur, step);
        return cudaGetLastError();
    }
    k_fused<C, kStats, kPeriodic, kNX>
        <<<dim3(t.ny_tiles, t.nz_chunks), dim3(kFusedThreads), size_t(t.smem_bytes), st>>>(s, t, cur, step);
    return cudaGetLastError();
}

template <class C, bool kStats, bool kPeriodic>
cudaError_t fused_launch(const DeviceState &s, const FusedTiling &t, int cur, int64_t step, cudaStream_t st) {
    if (t.fixed_nx == kFusedNX) return fused_launch_nx<C, kStats, kPeriodic, kFusedNX>(s, t, cur, step, st);
    if (t.fixed_nx == kFusedNX2) return fused_launch_nx<C, kStats, kPeriodic, kFusedNX2>(s, t, cur, step, st);
    return fused_launch_nx<C, kStats, kPeriodic, 0>(s, t, cur, step, st);
}

template <class C, bool kStats>
cudaError_t fused_dispatch(const DeviceState &s, const FusedTiling &t, int cur, int64_t step, cudaStream_t st) {
    if (s.g.boundary == kBoundaryPeriodic) return fused_launch<C, kStats, true>(s, t, cur, step, st);
    return fused_launch<C, kStats, false>(s, t, cur, step, st);
}

template <class C>
cudaError_t moments_dispatch(const DeviceState &s, int cur, int64_t step, cudaStream_t st) {
    const C codec = make_codec<C>(s, cur);
    if (s.g.boundary == kBoundaryPeriodic)
        k_moments<C, true><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, codec, step);
    else
        k_moments<C, false><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, codec, step);
    return cudaGetLastError();
}

template <class C>
cudaError_t boundary_dispatch(const DeviceState &s, int wbuf, int64_t step, int which, bool from_bmom,
                              cudaStream_t st) {
    dim3 grid = grid_plane(s.g);
    grid.z = which >= 0 ? 1 : 2;
    k_boundary<C><<<grid, dim3(32, 8), 0, st>>>(s, wbuf, step, which, from_bmom ? 1 : 0);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ discrete adjoint

// Adjoint of one step of the periodic box, float32 populations.  The forward
// step maps the stored post-collision values S_t to S_{t+1}:
//   f_i(x) = S_t,i(x - c_i); M(x) = moments(f(x)); psi(x) = psi(M(x));
//   F(x) = (1/cs2) sum_j w_j c_j psi(x + c_j);  S_{t+1},i(x) = C_i(M(x), F(x)).
// Given lambda_{t+1} = dJ/dS_{t+1} the adjoint forms lambda_t = dJ/dS_t in two
// node-parallel passes: k_adj_collide takes C's Jacobian (moments and F of the
// node), k_adj_moments gathers the F-adjoints of the neighbours into the
// node's psi-adjoint, goes back through the moments and scatters along the
// transposed streaming.  The bulk/interface switch (I <= 1e-4) and the
// |F| <= 1e-4 cut-off are taken as in the forward step (derivatives inside
// the branch the forward state selects).
//
// Every pass reads the state S_t only through its moment record M: the 11
// moment planes of the pulled populations and psi (plane kTapePsi), interior
// nodes; neighbours are addressed with the periodic wrap.

__device__ __forceinline__ double block_sum_any(double v, double *sh, int nthreads) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = t & 31, wid = t >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (t == 0)
        for (int k = 0; k < nthreads / 32; ++k) r += sh[k];
    __syncthreads();
    return r;
}

// block_sum_any of three values in one pass: two barriers instead of nine.
// Each value is summed in the same order as block_sum_any sums it.  sh holds
// 3 * (threads / 32) doubles; the sums are valid in thread 0.
__device__ __forceinline__ void block_sum3(double (&v)[3], double *sh, int nthreads) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) v[k] += __shfl_down_sync(kFull, v[k], o);
    }
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = t & 31, wid = t >> 5, nw = nthreads / 32;
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < 3; ++k) sh[k * nw + wid] = v[k];
    __syncthreads();
    if (t == 0) {
        for (int k = 0; k < 3; ++k) {
            double r = 0.0;
            for (int j = 0; j < nw; ++j) r += sh[k * nw + j];
            v[k] = r;
        }
    }
}

// J = sum over interior nodes of (psi_T - psi*)^2 and lambda_T = dJ/dS_T.
__global__ void __launch_bounds__(kBX * kBY) k_adj_terminal(const DeviceState s, const float *__restrict__ M,
                                                           const float *__restrict__ target, float *lam, double *J) {
    __shared__ double sh[kBX * kBY / 32];
    const Geometry &g = s.g;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    const bool in = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    double jloc = 0.0;
    if (in) {
        const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
        const size_t N = g.N;
        const float rr = M[kMomRR * N + id], rb = M[kMomRB * N + id];
        const float rho = rr + rb;
        const float d = M[kTapePsi * N + id] - target[id];
        jloc = double(d) * double(d);
        const float lpsi = 2.0f * d;
        const float inv2 = 1.0f / (rho * rho);
        const float lrr = lpsi * 2.0f * rb * inv2, lrb = -lpsi * 2.0f * rr * inv2;
        const PullMap<CodecF32> pm(g, x, y, z, true);
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            size_t grow;
            int xs;
            pm.template src<i>(x, grow, xs);
            reinterpret_cast<float2 *>(lam)[grow + size_t(dir_cx(i) + 1) * g.NX + xs] = make_float2(lrr, lrb);
        });
    }
    const double r = block_sum_any(jloc, sh, kBX * kBY);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomicAdd(J, r);
}

// Exponents (a, b, c) of the 17 monomials cx^a cy^b cz^c of the collision
// polynomial (collision_poly): per-axis degree <= 2, total degree <= 3.
__host__ __device__ constexpr int poly_exp(int k, int axis) {
    constexpr int e[17][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0},
                              {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {2, 1, 0}, {2, 0, 1},
                              {1, 2, 0}, {1, 0, 2}, {0, 2, 1}, {0, 1, 2}, {1, 1, 1}};
    return e[k][axis];
}
__host__ __device__ constexpr int ipow1(int c, int e) { return e == 0 ? 1 : (e == 1 ? c : c * c); }
enum PolyTerm { kT000, kT100, kT010, kT001, kT200, kT020, kT002, kT110, kT101, kT011,
                kT210, kT201, kT120, kT102, kT021, kT012, kT111 };

// Adjoint of the bulk value g_i = w_i P(c_i) over the collision polynomial's
// coefficients, from the moments T_k = sum_i v_i m_k(c_i) of per-direction
// weights v (v = w lambda_g): Phi = (feq polynomial)/rho dotted with T, its
// u-gradient, and Psi = (fneq polynomial) dotted with T, with the S2 / S3
// Hermite sums Psi is made of.
struct PolyAdjoint {
    float S2[6], S3[7];
    float Phi, dPhi[3], Psi;
};
__device__ __forceinline__ PolyAdjoint poly_adjoint(const float (&T)[17], float ux, float uy, float uz,
                                                    const NeqTerms &n) {
    PolyAdjoint r;
    r.S2[0] = T[kT200] - kCs2 * T[kT000];
    r.S2[1] = T[kT110];
    r.S2[2] = T[kT020] - kCs2 * T[kT000];
    r.S2[3] = T[kT011];
    r.S2[4] = T[kT002] - kCs2 * T[kT000];
    r.S2[5] = T[kT101];
    r.S3[0] = T[kT210] - kCs2 * T[kT010];
    r.S3[1] = T[kT201] - kCs2 * T[kT001];
    r.S3[2] = T[kT120] - kCs2 * T[kT100];
    r.S3[3] = T[kT102] - kCs2 * T[kT100];
    r.S3[4] = T[kT021] - kCs2 * T[kT001];
    r.S3[5] = T[kT012] - kCs2 * T[kT010];
    r.S3[6] = T[kT111];
    r.Psi = kInv2Cs4 * (n.pxx * r.S2[0] + 2.0f * n.pxy * r.S2[1] + n.pyy * r.S2[2] + 2.0f * n.pyz * r.S2[3] +
                        n.pzz * r.S2[4] + 2.0f * n.pxz * r.S2[5]) +
            kInv2Cs6 * (n.a3xxy * r.S3[0] + n.a3xxz * r.S3[1] + n.a3xyy * r.S3[2] + n.a3xzz * r.S3[3] +
                        n.a3yyz * r.S3[4] + n.a3yzz * r.S3[5] + 2.0f * n.a3xyz * r.S3[6]);
    // feq_i / (w_i rho) = 1 + q cu + (q^2/2) cu^2 - (q/2) |u|^2 + (q^3/6) cu^3 - (q^2/2) |u|^2 cu, q = 1/cs^2
    const float usq = ux * ux + uy * uy + uz * uz;
    const float uTc = ux * T[kT100] + uy * T[kT010] + uz * T[kT001];
    const float lin = kInvCs2 - kInv2Cs4 * usq;
    const float t2x = T[kT200] * ux + T[kT110] * uy + T[kT101] * uz;
    const float t2y = T[kT110] * ux + T[kT020] * uy + T[kT011] * uz;
    const float t2z = T[kT101] * ux + T[kT011] * uy + T[kT002] * uz;
    // (1/3) d(cu^3)/du_a summed against T (c^3 = c on the lattice)
    const float cx3 = ux * ux * T[kT100] + 2.0f * ux * uy * T[kT210] + 2.0f * ux * uz * T[kT201] + uy * uy * T[kT120] +
                      uz * uz * T[kT102] + 2.0f * uy * uz * T[kT111];
    const float cy3 = uy * uy * T[kT010] + 2.0f * uy * ux * T[kT120] + 2.0f * uy * uz * T[kT021] + ux * ux * T[kT210] +
                      uz * uz * T[kT012] + 2.0f * ux * uz * T[kT111];
    const float cz3 = uz * uz * T[kT001] + 2.0f * uz * ux * T[kT102] + 2.0f * uz * uy * T[kT012] + ux * ux * T[kT201] +
                      uy * uy * T[kT021] + 2.0f * ux * uy * T[kT111];
    r.Phi = T[kT000] * (1.0f - kInv2Cs2 * usq) + lin * uTc + kInv2Cs4 * (ux * t2x + uy * t2y + uz * t2z) +
            kInv6Cs6 * (ux * cx3 + uy * cy3 + uz * cz3);
    const float q2 = 2.0f * kInv2Cs4, q3h = 3.0f * kInv6Cs6;
    r.dPhi[0] = -kInvCs2 * ux * T[kT000] - q2 * ux * uTc + lin * T[kT100] + q2 * t2x + q3h * cx3;
    r.dPhi[1] = -kInvCs2 * uy * T[kT000] - q2 * uy * uTc + lin * T[kT010] + q2 * t2y + q3h * cy3;
    r.dPhi[2] = -kInvCs2 * uz * T[kT000] - q2 * uz * uTc + lin * T[kT001] + q2 * t2z + q3h * cz3;
    return r;
}

// Per node: lambda_post (54 values at the node) -> adjoints of the node's
// moments (11, to lmom) and colour gradient (3, to lf); float64 partials of
// dJ/domega (acc[0]) and dJ/d(A/2) (acc[1]).
//
// Per direction the stored pair is r_i = aR g_i + D_i, b_i = aB g_i - D_i, so
// with lg_i = aR lr_i + aB lb_i and ld_i = lr_i - lb_i the node's sums are
//   d/d(aR - aB)-part  sum ld_i g_i,   d/drho  sum lg_i feq_i / rho,
//   d/du     sum lg_i w rho (c P_i - u Q_i)  (dfeq/du),
//   d/dPi    oms sum lg_i w H2_i / 2cs4 and the third-order a3 chain,
//   d/domega -sum lg_i fneq_i,  d/dF from Omega2 and D,  d/dK from D.
// Opposite directions i, i+1 are taken together: feq and fneq split into even
// and odd parts, Omega2 is even and D odd, so every sum needs only
// lg_i + lg_o, lg_i - lg_o, ld_i + ld_o and ld_i - ld_o.
template <bool kPeriodic>
__global__ void __launch_bounds__(kBX * kBY, 2) k_adj_collide(const DeviceState s, const float *__restrict__ M,
                                                             const float *lam, float *lmom, float *lf, double *acc,
                                                             AdjObjective obj) {
    __shared__ double sh[3 * (kBX * kBY / 32)];  // block_sum3
    const Geometry &g = s.g;
    const Physics &ph = s.ph;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    const bool in = x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2;
    double a_omega = 0.0, a_Ah = 0.0, a_J = 0.0;
    if (in) {
        const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
        const size_t N = g.N;
        const float *mom = M;
        const float rr = mom[kMomRR * N + id], rb = mom[kMomRB * N + id];
        const float ux = mom[kMomUX * N + id], uy = mom[kMomUY * N + id], uz = mom[kMomUZ * N + id];
        const NeqTerms n = make_neq(mom[kMomPXX * N + id], mom[kMomPXY * N + id], mom[kMomPYY * N + id],
                                    mom[kMomPYZ * N + id], mom[kMomPZZ * N + id], mom[kMomPXZ * N + id], ux, uy, uz);
        const float rho = rr + rb;
        const float invr = 1.0f / rho;
        const float aR = rr * invr, aB = rb * invr;
        const float oms = 1.0f - omega_at(ph, y);
        const bool interface = !(4.0f * rr * rb * invr * invr <= 1e-4f);
        float Fx = 0.f, Fy = 0.f, Fz = 0.f, absF = 0.f, K = 0.f;
        bool has_dir = false;
        if (interface) {
            // periodic box: neighbours wrap over the interior; jet: the record's
            // psi plane holds the ghost values the forward step read unwrapped
            const float *psi = M + size_t(kTapePsi) * N;
            const int xn[3] = {kPeriodic ? wrap_interior(x - 1, g.NX) : x - 1, x,
                               kPeriodic ? wrap_interior(x + 1, g.NX) : x + 1};
            const int yn[3] = {g.sy * (kPeriodic ? wrap_interior(y - 1, g.NY) : y - 1), g.sy * y,
                               g.sy * (kPeriodic ? wrap_interior(y + 1, g.NY) : y + 1)};
            const int zn[3] = {g.sz * (kPeriodic ? wrap_interior(z - 1, g.NZ) : z - 1), g.sz * z,
                               g.sz * (kPeriodic ? wrap_interior(z + 1, g.NZ) : z + 1)};
            float sx = 0.f, sy = 0.f, sz = 0.f;
            static_for<kQ - 1>([&](auto I) {
                constexpr int i = decltype(I)::value + 1;
                using D = Dir<i>;
                const float wp = D::w * psi[xn[D::cx + 1] + yn[D::cy + 1] + zn[D::cz + 1]];
                if constexpr (D::cx != 0) sx += D::fx * wp;
                if constexpr (D::cy != 0) sy += D::fy * wp;
                if constexpr (D::cz != 0) sz += D::fz * wp;
            });
            Fx = kInvCs2 * sx;
            Fy = kInvCs2 * sy;
            Fz = kInvCs2 * sz;
            absF = sqrtf(Fx * Fx + Fy * Fy + Fz * Fz);
            has_dir = !(absF <= 1.0e-4f);
            K = ph.beta * ((rr * rb) / (rho * rho)) * rho;
        }
        const float invF = has_dir ? 1.0f / absF : 0.0f;
        const float invF2 = invF * invF;
        const float Ah = ph.Ah;
        const size_t row = pop_row(g, y, z);
        // (lambda_r, lambda_b) of a direction: one float2, as the populations
        auto lam_at = [&](int slot) {
            return reinterpret_cast<const float2 *>(lam)[row + size_t(slot) * size_t(g.NX) + size_t(x)];
        };
        // Bulk part: g_i = w_i P(c_i) with P the collision polynomial, so the
        // sums over directions are the polynomial's coefficients dotted with
        // the moments T_k = sum_i w_i lambda_g,i m_k(c_i) (and U_k with
        // lambda_r - lambda_b for the colour split).  The moments are formed
        // group by group: per (cy, cz) the three cx values reduce to
        // (sum, sum cx, sum cx^2), which add into the 17 moments with the
        // weights cy^b cz^c.
        float Tm[17], Um[17];
#pragma unroll
        for (int k = 0; k < 17; ++k) Tm[k] = Um[k] = 0.f;
        static_for<9>([&](auto G) {
            constexpr int cy = decltype(G)::value / 3 - 1, cz = decltype(G)::value % 3 - 1;
            float mv[3], nv[3];
            static_for<3>([&](auto X) {
                constexpr int cx = decltype(X)::value - 1;
                constexpr int i = dir_of(cx, cy, cz);
                const float2 l = lam_at(slot_pair(i));
                mv[cx + 1] = Dir<i>::w * (aR * l.x + aB * l.y);
                nv[cx + 1] = Dir<i>::w * (l.x - l.y);
            });
            const float m2 = mv[2] + mv[0], n2 = nv[2] + nv[0];
            const float ms[3] = {m2 + mv[1], mv[2] - mv[0], m2};
            const float ns[3] = {n2 + nv[1], nv[2] - nv[0], n2};
            static_for<17>([&](auto K) {
                constexpr int k = decltype(K)::value;
                constexpr int wgt = ipow1(cy, poly_exp(k, 1)) * ipow1(cz, poly_exp(k, 2));
                constexpr int a = poly_exp(k, 0);
                if constexpr (wgt == 1) {
                    Tm[k] += ms[a];
                    Um[k] += ns[a];
                } else if constexpr (wgt == -1) {
                    Tm[k] -= ms[a];
                    Um[k] -= ns[a];
                }
            });
        });
        const PolyAdjoint pT = poly_adjoint(Tm, ux, uy, uz, n);
        const PolyAdjoint pU = poly_adjoint(Um, ux, uy, uz, n);
        const float(&S2)[6] = pT.S2;
        const float(&S3)[7] = pT.S3;
        const float l_rhoeq = rho * pT.Phi;  // sum lambda_g feq (feq is proportional to rho)
        const float l_oms = pT.Psi;          // sum lambda_g fneq
        float l_d = rho * pU.Phi + oms * pU.Psi;  // sum (lambda_r - lambda_b) g
        // interface nodes: the perturbation and recolouring terms, direction by direction
        float sAx = 0.f, sAy = 0.f, sAz = 0.f, sB = 0.f, sDx = 0.f, sDy = 0.f, sDz = 0.f, sE = 0.f, sBB = 0.f,
              l_Ah = 0.f;
        if (interface) {
            {  // rest direction: even only
                const float2 l0 = lam_at(slot_pair(0));
                const float lg = aR * l0.x + aB * l0.y, ld = l0.x - l0.y;
                const float o2A = -absF * Dir<0>::B;  // Omega2 / (A/2)
                l_d += ld * (Ah * o2A);
                sBB += lg * Dir<0>::B;
                l_Ah += lg * o2A;
            }
            static_for<(kQ - 1) / 2>([&](auto P) {
                constexpr int i = 2 * decltype(P)::value + 1;
                using D = Dir<i>;
                const float2 li = lam_at(slot_pair(i)), lo = lam_at(slot_pair(i + 1));
                const float lgi = aR * li.x + aB * li.y, lgo = aR * lo.x + aB * lo.y;
                const float ldi = li.x - li.y, ldo = lo.x - lo.y;
                const float gs = lgi + lgo, ds = ldi + ldo, dd = ldi - ldo;
                float fc = 0.f;
                if constexpr (D::cx != 0) fc += D::fx * Fx;
                if constexpr (D::cy != 0) fc += D::fy * Fy;
                if constexpr (D::cz != 0) fc += D::fz * Fz;
                const float o2A = absF * (D::w * (fc * fc) * invF2 - D::B);  // Omega2 / (A/2), even
                l_d += ds * (Ah * o2A);
                sBB += gs * D::B;
                l_Ah += gs * o2A;
                const float a = gs * D::w * fc, d = dd * D::w * D::invc;
                if constexpr (D::cx != 0) { sAx += D::fx * a; sDx += D::fx * d; }
                if constexpr (D::cy != 0) { sAy += D::fy * a; sDy += D::fy * d; }
                if constexpr (D::cz != 0) { sAz += D::fz * a; sDz += D::fz * d; }
                sB += a * fc;
                sE += d * fc;
            });
        }
        // fneq: Pi enters directly (H2) and through the third-order terms a3
        const float c2 = oms * kInv2Cs4, c3 = oms * kInv2Cs6;
        float lPxx = S2[0] * c2, lPxy = 2.0f * S2[1] * c2, lPyy = S2[2] * c2;
        float lPyz = 2.0f * S2[3] * c2, lPzz = S2[4] * c2, lPxz = 2.0f * S2[5] * c2;
        const float la_xxy = S3[0] * c3, la_xxz = S3[1] * c3, la_xyy = S3[2] * c3, la_xzz = S3[3] * c3;
        const float la_yyz = S3[4] * c3, la_yzz = S3[5] * c3, la_xyz = 2.0f * S3[6] * c3;
        lPxx += la_xxy * uy + la_xxz * uz;
        lPyy += la_xyy * ux + la_yyz * uz;
        lPzz += la_xzz * ux + la_yzz * uy;
        lPxy += 2.0f * la_xxy * ux + 2.0f * la_xyy * uy + la_xyz * uz;
        lPxz += 2.0f * la_xxz * ux + 2.0f * la_xzz * uz + la_xyz * uy;
        lPyz += 2.0f * la_yyz * uy + 2.0f * la_yzz * uz + la_xyz * ux;
        float lux = 2.0f * la_xxy * n.pxy + 2.0f * la_xxz * n.pxz + la_xyy * n.pyy + la_xzz * n.pzz + la_xyz * n.pyz;
        float luy = la_xxy * n.pxx + 2.0f * la_xyy * n.pxy + 2.0f * la_yyz * n.pyz + la_yzz * n.pzz + la_xyz * n.pxz;
        float luz = la_xxz * n.pxx + 2.0f * la_xzz * n.pxz + la_yyz * n.pyy + 2.0f * la_yzz * n.pyz + la_xyz * n.pxy;
        // feq: rho times the u-gradient of the feq polynomial against T
        lux += rho * pT.dPhi[0];
        luy += rho * pT.dPhi[1];
        luz += rho * pT.dPhi[2];
        // colour gradient: perturbation and recolouring
        float lFx = 0.f, lFy = 0.f, lFz = 0.f, lK = 0.f;
        if (interface) {
            if (has_dir) {
                const float i3 = invF2 * invF;
                lFx = Ah * (2.0f * invF * sAx - Fx * i3 * sB - Fx * invF * sBB) + K * (sDx * invF - Fx * i3 * sE);
                lFy = Ah * (2.0f * invF * sAy - Fy * i3 * sB - Fy * invF * sBB) + K * (sDy * invF - Fy * i3 * sE);
                lFz = Ah * (2.0f * invF * sAz - Fz * i3 * sB - Fz * invF * sBB) + K * (sDz * invF - Fz * i3 * sE);
                lK = sE * invF;
            } else if (absF > 0.0f) {
                const float q = -Ah * sBB / absF;
                lFx = q * Fx;
                lFy = q * Fy;
                lFz = q * Fz;
            }
        }
        const float inv2 = invr * invr;
        const float l_rho = l_rhoeq * invr;  // feq is proportional to rho
        lmom[kMomRR * N + id] = l_rho + l_d * rb * inv2 + lK * ph.beta * rb * rb * inv2;
        lmom[kMomRB * N + id] = l_rho - l_d * rr * inv2 + lK * ph.beta * rr * rr * inv2;
        // the objective's source: J_t = (w/2) sum uy^2 over nodes with y >= y_obs,
        // or the profile objective's dJ/duy of the node's radial bin (the bin of
        // radial_accumulate_warp, same float arithmetic)
        float lobj = 0.f;
        if (obj.table) {
            const float dx = float(x) - ph.jet_x0, dz = float(z) - ph.jet_z0;
            const unsigned rbin = unsigned(sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz))));
            if (rbin < unsigned(ph.NRB)) lobj = obj.table[size_t(y) * ph.NRB + rbin];
        } else if (obj.weight != 0.0f && y >= obj.y_obs) {
            lobj = obj.weight * uy;
            a_J = 0.5 * double(obj.weight) * double(uy) * double(uy);
        }
        lmom[kMomUX * N + id] = lux;
        lmom[kMomUY * N + id] = luy + lobj;
        lmom[kMomUZ * N + id] = luz;
        lmom[kMomPXX * N + id] = lPxx;
        lmom[kMomPXY * N + id] = lPxy;
        lmom[kMomPYY * N + id] = lPyy;
        lmom[kMomPYZ * N + id] = lPyz;
        lmom[kMomPZZ * N + id] = lPzz;
        lmom[kMomPXZ * N + id] = lPxz;
        lf[0 * N + id] = lFx;
        lf[1 * N + id] = lFy;
        lf[2 * N + id] = lFz;
        a_omega = -double(l_oms);  // oms = 1 - omega
        a_Ah = double(l_Ah);
    }
    double r[3] = {a_omega, a_Ah, obj.J ? a_J : 0.0};
    block_sum3(r, sh, kBX * kBY);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicAdd(acc, r[0]);
        atomicAdd(acc + 1, r[1]);
        if (obj.J) atomicAdd(obj.J, r[2]);
    }
}

// Per node: the psi-adjoint gathered from the neighbours' F-adjoints, then back
// through the moments to the 54 pulled populations, stored at their pull
// sources (transposed streaming) in lam_out.
template <bool kPeriodic>
__global__ void __launch_bounds__(kBX * kBY) k_adj_moments(const DeviceState s, const float *__restrict__ M,
                                                          const float *lmom, const float *lf, float *lam_out) {
    // The block's F-adjoints with a one-node halo, [3][3 planes][kBY+2][kBX+2],
    // so the 26-neighbour gather reads shared memory.  A halo position holds
    // lf of the node whose psi it is: periodic neighbours wrap over the
    // interior; otherwise a position off the interior holds 0 (only interior
    // nodes relax, and read psi there).
    constexpr int TX = kBX + 2, TY = kBY + 2, TP = TX * TY * 3;
    __shared__ float tile[3 * TP];
    const Geometry &g = s.g;
    const size_t N = g.N;
    const int bx0 = int(blockIdx.x) * kBX - 1, by0 = int(blockIdx.y) * kBY - 1, bz0 = int(blockIdx.z) - 1;
    for (int t = threadIdx.y * kBX + threadIdx.x; t < TP; t += kBX * kBY) {
        const int xt = t % TX, yt = (t / TX) % TY, zt = t / (TX * TY);
        int xn = bx0 + xt, yn = by0 + yt, zn = bz0 + zt;
        bool ok;
        if constexpr (kPeriodic) {
            ok = xn >= 0 && xn <= g.NX - 1 && yn >= 0 && yn <= g.NY - 1 && zn >= 0 && zn <= g.NZ - 1;
            xn = wrap_interior(xn, g.NX);
            yn = wrap_interior(yn, g.NY);
            zn = wrap_interior(zn, g.NZ);
        } else {
            ok = xn >= 1 && xn <= g.NX - 2 && yn >= 1 && yn <= g.NY - 2 && zn >= 1 && zn <= g.NZ - 2;
        }
        float v0 = 0.f, v1 = 0.f, v2 = 0.f;
        if (ok) {
            const uint32_t nid = uint32_t(xn) + uint32_t(g.sy) * uint32_t(yn) + uint32_t(g.sz) * uint32_t(zn);
            v0 = lf[0 * N + nid];
            v1 = lf[1 * N + nid];
            v2 = lf[2 * N + nid];
        }
        tile[t] = v0;
        tile[TP + t] = v1;
        tile[2 * TP + t] = v2;
    }
    __syncthreads();
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const float *mom = M;
    const float rr = mom[kMomRR * N + id], rb = mom[kMomRB * N + id];
    const float ux = mom[kMomUX * N + id], uy = mom[kMomUY * N + id], uz = mom[kMomUZ * N + id];
    const float rho = rr + rb;
    // psi(y) enters F(y - c_j) with weight w_j c_j / cs2
    float lpsi = 0.f;
    const int tc = (1 * TY + int(threadIdx.y) + 1) * TX + int(threadIdx.x) + 1;  // the node in the tile
    static_for<kQ - 1>([&](auto I) {
        constexpr int i = decltype(I)::value + 1;
        using D = Dir<i>;
        const int tn = tc - (D::cz * TY + D::cy) * TX - D::cx;
        float dot = 0.f;
        if constexpr (D::cx != 0) dot += D::fx * tile[tn];
        if constexpr (D::cy != 0) dot += D::fy * tile[TP + tn];
        if constexpr (D::cz != 0) dot += D::fz * tile[2 * TP + tn];
        lpsi += D::w * dot;
    });
    lpsi *= kInvCs2;
    const float inv2 = 1.0f / (rho * rho);
    const float lrr = lmom[kMomRR * N + id] + lpsi * 2.0f * rb * inv2;
    const float lrb = lmom[kMomRB * N + id] - lpsi * 2.0f * rr * inv2;
    const float lPxx = lmom[kMomPXX * N + id], lPxy = lmom[kMomPXY * N + id], lPyy = lmom[kMomPYY * N + id];
    const float lPyz = lmom[kMomPYZ * N + id], lPzz = lmom[kMomPZZ * N + id], lPxz = lmom[kMomPXZ * N + id];
    // Pi = A - rho u u
    const float lux = lmom[kMomUX * N + id] - rho * (2.0f * ux * lPxx + uy * lPxy + uz * lPxz);
    const float luy = lmom[kMomUY * N + id] - rho * (2.0f * uy * lPyy + ux * lPxy + uz * lPyz);
    const float luz = lmom[kMomUZ * N + id] - rho * (2.0f * uz * lPzz + ux * lPxz + uy * lPyz);
    float lrho = -(lPxx * ux * ux + lPxy * ux * uy + lPyy * uy * uy + lPyz * uy * uz + lPzz * uz * uz + lPxz * ux * uz);
    // u = j / rho
    const float invr = 1.0f / rho;
    const float ljx = lux * invr, ljy = luy * invr, ljz = luz * invr;
    lrho -= (lux * ux + luy * uy + luz * uz) * invr;
    // lambda_g,i = lrho + lj.c_i + lP:H2(c_i) is a quadratic polynomial in c_i:
    // evaluated at the 27 directions by sum factorisation (per cz, then cy,
    // then cx) instead of a Hermite sum per direction
    const float k0 = lrho - kCs2 * (lPxx + lPyy + lPzz);
    const PullMap<CodecF32> pm(g, x, y, z, kPeriodic);
    static_for<3>([&](auto CZ) {
        constexpr int cz = decltype(CZ)::value - 1;
        const float az = cz == 0 ? k0 : (cz > 0 ? k0 + ljz + lPzz : k0 - ljz + lPzz);
        const float bxz = cz == 0 ? ljx : (cz > 0 ? ljx + lPxz : ljx - lPxz);  // coefficient of cx
        const float byz = cz == 0 ? ljy : (cz > 0 ? ljy + lPyz : ljy - lPyz);  // coefficient of cy
        static_for<3>([&](auto CY) {
            constexpr int cy = decltype(CY)::value - 1;
            const float c0 = cy == 0 ? az : (cy > 0 ? az + byz + lPyy : az - byz + lPyy);
            const float c1 = cy == 0 ? bxz : (cy > 0 ? bxz + lPxy : bxz - lPxy);
            const float c2 = c0 + lPxx;
            static_for<3>([&](auto CX) {
                constexpr int cx = decltype(CX)::value - 1;
                constexpr int i = dir_of(cx, cy, cz);
                const float lgi = cx == 0 ? c0 : (cx > 0 ? c2 + c1 : c2 - c1);
                size_t grow;
                int xs;
                pm.template src<i>(x, grow, xs);
                reinterpret_cast<float2 *>(lam_out)[grow + size_t(dir_cx(i) + 1) * g.NX + xs] =
                    make_float2(lrr + lgi, lrb + lgi);
            });
        });
    });
}

// Adjoint of the regularised non-equilibrium part over a set of directions:
// S2 = sum mu_i H2_i, S3 = sum mu_i H3_i with mu_i = (1-omega) lambda_i w_i give
// the adjoints of Pi (pxx, pxy, pyy, pyz, pzz, pxz) and the u added through
// the third-order terms a3 (lbm.cuh:38-78).
__device__ __forceinline__ void neq_adjoint(const float (&S2)[6], const float (&S3)[7], const NeqTerms &n, float ux,
                                            float uy, float uz, float (&lP)[6], float (&lu)[3]) {
    const float c2 = kInv2Cs4, c3 = kInv2Cs6;
    float lPxx = S2[0] * c2, lPxy = 2.0f * S2[1] * c2, lPyy = S2[2] * c2;
    float lPyz = 2.0f * S2[3] * c2, lPzz = S2[4] * c2, lPxz = 2.0f * S2[5] * c2;
    const float la_xxy = S3[0] * c3, la_xxz = S3[1] * c3, la_xyy = S3[2] * c3, la_xzz = S3[3] * c3;
    const float la_yyz = S3[4] * c3, la_yzz = S3[5] * c3, la_xyz = 2.0f * S3[6] * c3;
    lPxx += la_xxy * uy + la_xxz * uz;
    lPyy += la_xyy * ux + la_yyz * uz;
    lPzz += la_xzz * ux + la_yzz * uy;
    lPxy += 2.0f * la_xxy * ux + 2.0f * la_xyy * uy + la_xyz * uz;
    lPxz += 2.0f * la_xxz * ux + 2.0f * la_xzz * uz + la_xyz * uy;
    lPyz += 2.0f * la_yyz * uy + 2.0f * la_yzz * uz + la_xyz * ux;
    lu[0] += 2.0f * la_xxy * n.pxy + 2.0f * la_xxz * n.pxz + la_xyy * n.pyy + la_xzz * n.pzz + la_xyz * n.pyz;
    lu[1] += la_xxy * n.pxx + 2.0f * la_xyy * n.pxy + 2.0f * la_yyz * n.pyz + la_yzz * n.pzz + la_xyz * n.pxz;
    lu[2] += la_xxz * n.pxx + 2.0f * la_xzz * n.pxz + la_yyz * n.pyy + 2.0f * la_yzz * n.pyz + la_xyz * n.pxy;
    lP[0] = lPxx; lP[1] = lPxy; lP[2] = lPyy; lP[3] = lPyz; lP[4] = lPzz; lP[5] = lPxz;
}

template <int I>
__device__ __forceinline__ void neq_accumulate(float mu, float (&S2)[6], float (&S3)[7]) {
    using D = Dir<I>;
    S2[0] += mu * D::Hxx; S2[1] += mu * D::Hxy; S2[2] += mu * D::Hyy;
    S2[3] += mu * D::Hyz; S2[4] += mu * D::Hzz; S2[5] += mu * D::Hxz;
    if constexpr (D::Hxxy != 0.0f) S3[0] += mu * D::Hxxy;
    if constexpr (D::Hxxz != 0.0f) S3[1] += mu * D::Hxxz;
    if constexpr (D::Hxyy != 0.0f) S3[2] += mu * D::Hxyy;
    if constexpr (D::Hxzz != 0.0f) S3[3] += mu * D::Hxzz;
    if constexpr (D::Hyyz != 0.0f) S3[4] += mu * D::Hyyz;
    if constexpr (D::Hyzz != 0.0f) S3[5] += mu * D::Hyzz;
    if constexpr (D::Hxyz != 0.0f) S3[6] += mu * D::Hxyz;
}

__device__ __forceinline__ float inlet_noise_factor(const Physics &ph, int64_t step, int x, int z) {
    if (ph.inlet_noise == 0.0f) return 1.0f;
    const float u = hash_uniform(ph.seed, 0x1A1E7ull ^ uint64_t(step), uint64_t(x), uint64_t(z));
    return 1.0f + (2.0f * u - 1.0f) * ph.inlet_noise;
}

// One thread per interior column (x, z): the outlet at y = NY-1 and, in a jet
// column, the inlet at y = 0.  A ghost-plane slot enters only if an interior
// node pulls it (the boundary also writes slots nothing reads).
__global__ void __launch_bounds__(256) k_adj_boundary(const DeviceState s, int64_t step, const float *__restrict__ M,
                                                      const float *__restrict__ Bt, const float *__restrict__ lam,
                                                      const float *__restrict__ lf, float *lmom,
                                                      const float *__restrict__ LB_in, float *LB_out,
                                                      const float *__restrict__ bessel, int nb, double *dJdc) {
    const Geometry &g = s.g;
    const Physics &ph = s.ph;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    const bool col = x >= 1 && x <= g.NX - 2 && z >= 1 && z <= g.NZ - 2;
    const size_t N = g.N;
    const int NP = g.NX * g.NZ;
    const int ic = x + g.NX * z;
    float dc[kInletBesselMax];
#pragma unroll
    for (int k = 0; k < kInletBesselMax; ++k) dc[k] = 0.f;
    auto pulled = [&](int xp, int zp) { return xp >= 1 && xp <= g.NX - 2 && zp >= 1 && zp <= g.NZ - 2; };
    if (col) {
        // ---------------- outlet (boundary_conditions.cuh:163-233)
        const uint32_t idF = uint32_t(x) + uint32_t(g.sy) * uint32_t(g.NY - 2) + uint32_t(g.sz) * uint32_t(z);
        const float phi[5] = {M[kMomRR * N + idF], M[kMomRB * N + idF], M[kMomUX * N + idF], M[kMomUY * N + idF],
                              M[kMomUZ * N + idF]};
        const NeqTerms nF = make_neq(M[kMomPXX * N + idF], M[kMomPXY * N + idF], M[kMomPYY * N + idF],
                                     M[kMomPYZ * N + idF], M[kMomPZZ * N + idF], M[kMomPXZ * N + idF], phi[2], phi[3],
                                     phi[4]);
        float B[5], Bn[5];
        const float uc = clamp01(phi[3]);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            B[c] = Bt[c * NP + ic];
            Bn[c] = B[c] - uc * (B[c] - phi[c]);
        }
        const float rho = Bn[0] + Bn[1];
        const float inv = 1.0f / rho;
        const float aR = Bn[0] * inv, aB = Bn[1] * inv;
        const float oms = 1.0f - omega_at(ph, g.NY - 2);
        const EqTerms e = make_eq(Bn[2], Bn[3], Bn[4]);
        float lrho = 0.f, le[3] = {0.f, 0.f, 0.f}, laR = 0.f, laB = 0.f;
        float S2[6] = {0, 0, 0, 0, 0, 0}, S3[7] = {0, 0, 0, 0, 0, 0, 0};
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            using D = Dir<i>;
            if constexpr (D::cy == -1) {
                if (!pulled(x + D::cx, z + D::cz)) return;
                const float2 l = reinterpret_cast<const float2 *>(lam)[pop_index(g, slot_pair(i), x, g.NY - 1, z)];
                const float lr = l.x, lb = l.y;
                const float fe = feq<i>(rho, e), fn = fneq<i>(nF);
                const float gi = fe + oms * fn;
                const float lg = aR * lr + aB * lb;
                laR += lr * gi;
                laB += lb * gi;
                lrho += lg * fe * inv;
                float cu = 0.f;
                if constexpr (D::cx != 0) cu += D::fx * e.ux;
                cu += D::fy * e.uy;
                if constexpr (D::cz != 0) cu += D::fz * e.uz;
                const float P = kInvCs2 + cu * (2.0f * kInv2Cs4) + (cu * cu) * (3.0f * kInv6Cs6) - e.usq * kInv2Cs4;
                const float Q = kInvCs2 + cu * (2.0f * kInv2Cs4);
                const float wl = lg * D::w * rho;
                if constexpr (D::cx != 0) le[0] += wl * P * D::fx;
                le[1] += wl * P * D::fy;
                if constexpr (D::cz != 0) le[2] += wl * P * D::fz;
                const float q = wl * Q;
                le[0] -= q * e.ux;
                le[1] -= q * e.uy;
                le[2] -= q * e.uz;
                neq_accumulate<i>(oms * lg * D::w, S2, S3);
            }
        });
        const float inv2 = inv * inv;
        float lBn[5];
        lBn[0] = lrho + (laR - laB) * Bn[1] * inv2;
        lBn[1] = lrho - (laR - laB) * Bn[0] * inv2;
        lBn[2] = le[0];
        lBn[3] = le[1];
        lBn[4] = le[2];
        float luc = 0.f, lphi[5], lB[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            lBn[c] += LB_in[c * NP + ic];
            luc += lBn[c] * (phi[c] - B[c]);
            lphi[c] = uc * lBn[c];
            lB[c] = (1.0f - uc) * lBn[c];
        }
        if (phi[3] > 0.0f && phi[3] < 1.0f) lphi[3] += luc;  // d clamp01 / d uy
        float lP[6], lu[3] = {0.f, 0.f, 0.f};
        neq_adjoint(S2, S3, nF, phi[2], phi[3], phi[4], lP, lu);
        lmom[kMomRR * N + idF] += lphi[0];
        lmom[kMomRB * N + idF] += lphi[1];
        lmom[kMomUX * N + idF] += lphi[2] + lu[0];
        lmom[kMomUY * N + idF] += lphi[3] + lu[1];
        lmom[kMomUZ * N + idF] += lphi[4] + lu[2];
        lmom[kMomPXX * N + idF] += lP[0];
        lmom[kMomPXY * N + idF] += lP[1];
        lmom[kMomPYY * N + idF] += lP[2];
        lmom[kMomPYZ * N + idF] += lP[3];
        lmom[kMomPZZ * N + idF] += lP[4];
        lmom[kMomPXZ * N + idF] += lP[5];
        // psi(B) at (x, NY-1, z) entered the colour gradient of the step's
        // interior nodes (x, NY-2, z) - c over the cy = +1 directions
        float lpsi = 0.f;
        static_for<kQ>([&](auto I) {
            constexpr int i = decltype(I)::value;
            using D = Dir<i>;
            if constexpr (D::cy == 1) {
                const int xn = x - D::cx, zn = z - D::cz;
                if (!pulled(xn, zn)) return;
                const uint32_t nid = uint32_t(xn) + uint32_t(g.sy) * uint32_t(g.NY - 2) + uint32_t(g.sz) * uint32_t(zn);
                float dot = D::fy * lf[1 * N + nid];
                if constexpr (D::cx != 0) dot += D::fx * lf[0 * N + nid];
                if constexpr (D::cz != 0) dot += D::fz * lf[2 * N + nid];
                lpsi += D::w * dot;
            }
        });
        lpsi *= kInvCs2;
        const float rB = B[0] + B[1];
        const float i2 = 1.0f / (rB * rB);
        lB[0] += lpsi * 2.0f * B[1] * i2;
        lB[1] -= lpsi * 2.0f * B[0] * i2;
#pragma unroll
        for (int c = 0; c < 5; ++c) LB_out[c * NP + ic] = lB[c];
        // ---------------- inlet (boundary_conditions.cuh:17-85): jet columns only
        if (is_jet_column(ph, x, z)) {
            const uint32_t id1 = uint32_t(x) + uint32_t(g.sy) * 1u + uint32_t(g.sz) * uint32_t(z);
            const float u1x = M[kMomUX * N + id1], u1y = M[kMomUY * N + id1], u1z = M[kMomUZ * N + id1];
            const NeqTerms n1 = make_neq(M[kMomPXX * N + id1], M[kMomPXY * N + id1], M[kMomPYY * N + id1],
                                         M[kMomPYZ * N + id1], M[kMomPZZ * N + id1], M[kMomPXZ * N + id1], u1x, u1y,
                                         u1z);
            const float rT = ph.rhob0;  // the mask: red 0, blue rhob0 (aR = 0, aB = 1)
            const float U = inlet_velocity(s, step, x, z);
            const float omsb = 1.0f - ph.omega_b;
            float lU = 0.f;
            float T2[6] = {0, 0, 0, 0, 0, 0}, T3[7] = {0, 0, 0, 0, 0, 0, 0};
            static_for<kQ>([&](auto I) {
                constexpr int i = decltype(I)::value;
                using D = Dir<i>;
                if constexpr (D::cy == 1) {
                    if (!pulled(x + D::cx, z + D::cz)) return;
                    const float lg = reinterpret_cast<const float2 *>(lam)[pop_index(g, slot_pair(i), x, 0, z)].y;  // red = 0 * g
                    // d feq_i / d uy at u = (0, U, 0): w rho (c_y P - U Q), c.u = U
                    const float P = kInvCs2 + U * (2.0f * kInv2Cs4) + (U * U) * (3.0f * kInv6Cs6) - (U * U) * kInv2Cs4;
                    const float Q = kInvCs2 + U * (2.0f * kInv2Cs4);
                    lU += lg * D::w * rT * (P - U * Q);
                    neq_accumulate<i>(omsb * lg * D::w, T2, T3);
                }
            });
            float lP1[6], lu1[3] = {0.f, 0.f, 0.f};
            neq_adjoint(T2, T3, n1, u1x, u1y, u1z, lP1, lu1);
            lmom[kMomUX * N + id1] += lu1[0];
            lmom[kMomUY * N + id1] += lu1[1];
            lmom[kMomUZ * N + id1] += lu1[2];
            lmom[kMomPXX * N + id1] += lP1[0];
            lmom[kMomPXY * N + id1] += lP1[1];
            lmom[kMomPYY * N + id1] += lP1[2];
            lmom[kMomPYZ * N + id1] += lP1[3];
            lmom[kMomPZZ * N + id1] += lP1[4];
            lmom[kMomPXZ * N + id1] += lP1[5];
            // U = U0 (1 + sum_k c_k J0_k) (1 + noise): dU/dc_k = U0 (1 + noise) J0_k
            if (bessel) {
                const float dU = ph.jet_velocity * inlet_noise_factor(ph, step, x, z);
                for (int k = 0; k < nb; ++k) dc[k] = lU * dU * bessel[k * NP + ic];
            }
        }
    }
    if (bessel) {
        for (int k = 0; k < nb; ++k) {
            double v = dc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
            if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dJdc + k, v);
        }
    }
}

// The inverse: outlet state from src[5][NX*NZ] back to y = NY-1, with the psi
// the next step reads there (what the boundary launch writes).
__global__ void __launch_bounds__(256) k_restore_outlet_state(const DeviceState s, const float *src, float *psi) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.NX || z >= g.NZ) return;
    const uint32_t idB = uint32_t(x) + uint32_t(g.sy) * uint32_t(g.NY - 1) + uint32_t(g.sz) * uint32_t(z);
    const int NP = g.NX * g.NZ;
#pragma unroll
    for (int c = 0; c < 5; ++c) s.mom[size_t(c) * g.N + idB] = src[c * NP + x + g.NX * z];
    if (x >= 1 && x <= g.NX - 2 && z >= 1 && z <= g.NZ - 2)
        psi[idB] = psi_of(src[0 * NP + x + g.NX * z], src[1 * NP + x + g.NX * z]);
}

// Outlet state (rr, rb, ux, uy, uz at y = NY-1) of interior columns to dst[5][NX*NZ].
__global__ void __launch_bounds__(256) k_copy_outlet_state(const DeviceState s, float *dst) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.NX || z >= g.NZ) return;
    const uint32_t idB = uint32_t(x) + uint32_t(g.sy) * uint32_t(g.NY - 1) + uint32_t(g.sz) * uint32_t(z);
    const int NP = g.NX * g.NZ;
#pragma unroll
    for (int c = 0; c < 5; ++c) dst[c * NP + x + g.NX * z] = s.mom[size_t(c) * g.N + idB];
}

// dJ/du0 for an initial state f0_c,i = feq_i(rho_c, u0): pulls lambda_0 like
// the forward step pulls populations.
__global__ void __launch_bounds__(kBX * kBY) k_adj_initial(const DeviceState s, const float *__restrict__ M,
                                                          const float *lam0, float *du0) {
    const Geometry &g = s.g;
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.NX || y >= g.NY) return;
    const uint32_t id = uint32_t(x) + uint32_t(g.sy) * uint32_t(y) + uint32_t(g.sz) * uint32_t(z);
    const size_t N = g.N;
    if (!(x >= 1 && x <= g.NX - 2 && y >= 1 && y <= g.NY - 2 && z >= 1 && z <= g.NZ - 2)) {
        du0[id] = du0[N + id] = du0[2 * N + id] = 0.0f;
        return;
    }
    const float *mom = M;
    const float rr = mom[kMomRR * N + id], rb = mom[kMomRB * N + id];
    const float ux = mom[kMomUX * N + id], uy = mom[kMomUY * N + id], uz = mom[kMomUZ * N + id];
    const EqTerms e = make_eq(ux, uy, uz);
    const PullMap<CodecF32> pm(g, x, y, z, true);
    float gx = 0.f, gy = 0.f, gz = 0.f, gq = 0.f;
    static_for<kQ>([&](auto I) {
        constexpr int i = decltype(I)::value;
        using D = Dir<i>;
        size_t grow;
        int xs;
        pm.template src<i>(x, grow, xs);
        const float2 l = reinterpret_cast<const float2 *>(lam0)[grow + size_t(dir_cx(i) + 1) * g.NX + xs];
        const float lr = l.x, lb = l.y;
        float cu = 0.f;
        if constexpr (D::cx != 0) cu += D::fx * ux;
        if constexpr (D::cy != 0) cu += D::fy * uy;
        if constexpr (D::cz != 0) cu += D::fz * uz;
        const float P = kInvCs2 + cu * (2.0f * kInv2Cs4) + (cu * cu) * (3.0f * kInv6Cs6) - e.usq * kInv2Cs4;
        const float Q = kInvCs2 + cu * (2.0f * kInv2Cs4);
        const float wl = D::w * (lr * rr + lb * rb);
        if constexpr (D::cx != 0) gx += wl * P * D::fx;
        if constexpr (D::cy != 0) gy += wl * P * D::fy;
        if constexpr (D::cz != 0) gz += wl * P * D::fz;
        gq += wl * Q;
    });
    du0[id] = gx - ux * gq;
    du0[N + id] = gy - uy * gq;
    du0[2 * N + id] = gz - uz * gq;
}

}  // namespace

// ---------------------------------------------------------------------- host side

FusedTiling fused_tiling(const Geometry &g, int max_smem) {
    FusedTiling t{};
    t.tpr = ((g.NX + 31) / 32) * 32;
    const int per_row = t.tpr * 4;
    const int rpt = kFusedThreads / t.tpr;
    if (const char *v = std::getenv("MCG_FUSED_SMEM_KB")) max_smem = std::atoi(v) * 1024;  // tuning sweeps
    // software-pipelined march for rows of up to 128 columns (measured on
    // 128x256x128: +5 % float32, and +2 % float16 with its loads in flight
    // across the relaxation)
    t.pipe = t.tpr <= 128;
    // rows of 256 columns in float32 too, where one row group's upper half
    // takes the rows in a rotated order, on 1-row tiles at 3 CTAs per SM
    // (measured on 256x512x256: 11236 MLUPS at 24-plane chunks, against 10582
    // on 2-row tiles at 2 CTAs per SM and 10336 for the block-synchronous
    // march; float16 keeps the block-synchronous march on 2-row tiles, 16721
    // against 13171 pipelined)
    const bool pipe256 = t.tpr == 256 && g.storage == kStoreF32;
    if (pipe256) t.pipe = 1;
    if (const char *v = std::getenv("MCG_FUSED_PIPE")) t.pipe = std::atoi(v) != 0;  // tuning sweeps
    if (t.pipe) max_smem = std::max(max_smem, 112 * 1024);  // 4 ring + 3 stage planes: two CTAs per SM
    // rows per tile: at least one round of rows in parallel, 4 by default
    // (measured best on 128x256x128), fewer if shared memory
    // (3*(ty+2) + 2*11*ty) * tpr * 4 bytes does not fit
    int ty = std::max(4, rpt);
    // the float32 pipelined march runs 3 CTAs per SM (PipeBlocks) on one round
    // of rows (2 rows for 128 columns; measured +1.5 % over 4-row tiles at 2 CTAs)
    if (t.pipe && g.storage == kStoreF32) ty = std::max(2, rpt);
    if (t.pipe && pipe256) ty = 1;
    if (const char *v = std::getenv("MCG_FUSED_TY")) ty = std::max(1, std::atoi(v));  // tuning sweeps
    auto smem_of = [&](int h) {
        return (t.pipe ? kPipeRing * (h + 2) + kPipeStage * kMomCount * h : 3 * (h + 2) + 2 * kMomCount * h) * per_row;
    };
    while (ty > 1 && smem_of(ty) > max_smem) --ty;
    if (ty > rpt) ty -= ty % rpt;  // whole rounds of rows in parallel
    t.ty = ty;
    t.ny_tiles = (g.NY - 2 + ty - 1) / ty;
    // z chunks of the block-synchronous march: about thirteen CTAs per SM over
    // the launch (measured on the 256x512x256 jet: 32-plane chunks, 2040 CTAs;
    // float16 +2 %, float32 within 0.5 % of 51-plane ones)
    const int target = 13 * 148;
    int chunks = (target + t.ny_tiles - 1) / t.ny_tiles;
    if (chunks < 1) chunks = 1;
    int lz = (g.NZ - 2 + chunks - 1) / chunks;
    if (lz < 4) lz = 4;
    if (t.pipe) {
        // Chunks of the pipelined march, measured on 128x256x128 over 8..16
        // planes: float32 13 planes (10 chunks, 2.9 waves of 3 CTAs per SM;
        // +4.5 % over 16), float16 10 planes (13 chunks, 2.8 waves of 2 CTAs
        // per SM; +1 %).  The time follows the fill of the last wave more than
        // the halo planes.  Grids that give fewer than 1.5 waves of 16-plane
        // chunks keep the block-synchronous march, whose shorter chunks fill
        // the GPU.
        const int ctas16 = t.ny_tiles * ((g.NZ - 2 + 15) / 16);
        if (ctas16 >= 3 * 148 && !std::getenv("MCG_FUSED_LZ")) lz = pipe256 ? 24 : (g.storage == kStoreF16 ? 10 : 13);
        else if (!std::getenv("MCG_FUSED_PIPE")) t.pipe = 0;
    }
    if (const char *v = std::getenv("MCG_FUSED_LZ")) lz = std::max(1, std::atoi(v));  // tuning sweeps
    t.lz = lz;
    t.nz_chunks = (g.NZ - 2 + lz - 1) / lz;
    t.smem_bytes = t.pipe ? (kPipeRing * (ty + 2) + kPipeStage * kMomCount * ty) * per_row
                          : (3 * (ty + 2) + 2 * kMomCount * ty) * per_row;
    t.alternate = 1;
    if (const char *v = std::getenv("MCG_FUSED_ALTERNATE")) t.alternate = std::atoi(v) != 0;  // tuning sweeps
    // compile-time row length for rows of exactly 128 or 256 columns (measured
    // +5 % float32, +10 % float16 on 128x256x128); results are bit-identical
    t.fixed_nx = ((g.NX == kFusedNX || g.NX == kFusedNX2) && t.tpr == g.NX) ? g.NX : 0;
    if (const char *v = std::getenv("MCG_FUSED_FIXED_NX"))  // tuning sweeps and the equality test
        if (std::atoi(v) == 0) t.fixed_nx = 0;
    // rows staged by bulk copies (k_fused_bulk), on request only: the
    // pipelined march on rows of 128 columns (16-byte segments).  Measured on
    // 128x256x128 it is slower than the register-held pulls (float32 10868
    // vs 11387 MLUPS, float16 12950 vs 16197): a 27 KB row image per row
    // group leaves two CTAs per SM with one row in flight each.
    t.wait_limit = kBulkWaitLimit;
    // the jet's inlet and outlet columns from the fused step's own-row threads
    // of rows 1 and NY-2, instead of a k_boundary launch after it
    t.boundary = g.boundary == kBoundaryJet;
    if (const char *v = std::getenv("MCG_FUSED_BOUNDARY")) t.boundary = t.boundary && std::atoi(v) != 0;  // tests
    const bool f16 = g.storage == kStoreF16;
    const bool bulk_ok = t.pipe && t.fixed_nx == kFusedNX &&
                         t.ty <= (f16 ? bulk_rows<CodecF16>() : bulk_rows<CodecF32>());
    t.bulk = 0;
    if (const char *v = std::getenv("MCG_FUSED_BULK")) t.bulk = bulk_ok && std::atoi(v) != 0;
    if (t.bulk) t.smem_bytes = f16 ? bulk_smem_for<CodecF16>(t.ty) : bulk_smem_for<CodecF32>(t.ty);
    return t;
}

cudaError_t fused_configure(int smem) {
    cudaError_t e;
    if ((e = fused_attr<CodecF32, false, false>(smem)) != cudaSuccess) return e;
    if ((e = fused_attr<CodecF32, true, false>(smem)) != cudaSuccess) return e;
    if ((e = fused_attr<CodecF32, false, true>(smem)) != cudaSuccess) return e;
    if ((e = fused_attr<CodecF32, true, true>(smem)) != cudaSuccess) return e;
    if ((e = fused_attr<CodecF16, false, false>(smem)) != cudaSuccess) return e;
    if ((e = fused_attr<CodecF16, true, false>(smem)) != cudaSuccess) return e;
    if ((e = fused_attr<CodecF16, false, true>(smem)) != cudaSuccess) return e;
    return fused_attr<CodecF16, true, true>(smem);
}

cudaError_t launch_fused(const DeviceState &s, const FusedTiling &t_in, int cur, int64_t step, bool stats,
                         cudaStream_t st) {
    FusedTiling t = t_in;
    if (t.boundary) {
        t.bnd_dst = s.pops[cur ^ 1];
        t.bnd_psi = s.psi[(step + 1) & 1];
        t.bnd_step = step;
    }
    if (s.g.storage == kStoreF16)
        return stats ? fused_dispatch<CodecF16, true>(s, t, cur, step, st)
                     : fused_dispatch<CodecF16, false>(s, t, cur, step, st);
    return stats ? fused_dispatch<CodecF32, true>(s, t, cur, step, st)
                 : fused_dispatch<CodecF32, false>(s, t, cur, step, st);
}

cudaError_t launch_moments(const DeviceState &s, int cur, int64_t step, bool stats, cudaStream_t st) {
    cudaError_t e = s.g.storage == kStoreF16 ? moments_dispatch<CodecF16>(s, cur, step, st)
                                             : moments_dispatch<CodecF32>(s, cur, step, st);
    if (e != cudaSuccess || !stats) return e;
    return launch_accumulate_radial(s, st);
}

cudaError_t launch_collide(const DeviceState &s, int cur, int64_t step, cudaStream_t st) {
    if (s.g.storage == kStoreF16)
        k_collide<CodecF16><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, make_codec<CodecF16>(s, cur), step);
    else
        k_collide<CodecF32><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, make_codec<CodecF32>(s, cur), step);
    return cudaGetLastError();
}

cudaError_t launch_boundary(const DeviceState &s, int wbuf, int64_t step, int which, bool from_bmom,
                            cudaStream_t st) {
    if (s.g.storage == kStoreF16) return boundary_dispatch<CodecF16>(s, wbuf, step, which, from_bmom, st);
    return boundary_dispatch<CodecF32>(s, wbuf, step, which, from_bmom, st);
}

cudaError_t launch_accumulate_radial(const DeviceState &s, cudaStream_t st) {
    k_accumulate_radial<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s);
    return cudaGetLastError();
}

cudaError_t launch_init_fields(const DeviceState &s, int mode, int red_inside, float r2, float bx, float by, float bz,
                               cudaStream_t st) {
    k_init_fields<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, mode, red_inside, r2, bx, by, bz);
    return cudaGetLastError();
}

cudaError_t launch_init_pops(const DeviceState &s, int mode, float noise, cudaStream_t st) {
    if (s.g.storage == kStoreF16)
        k_init_pops<CodecF16><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, mode, noise);
    else
        k_init_pops<CodecF32><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, mode, noise);
    return cudaGetLastError();
}

cudaError_t launch_refresh_psi(const DeviceState &s, cudaStream_t st) {
    k_refresh_psi<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s);
    return cudaGetLastError();
}

cudaError_t launch_scatter_chunk(const DeviceState &s, int wbuf, const float *stage, size_t pitch, int z0, int nz,
                                 cudaStream_t st) {
    dim3 grid = grid3(s.g);
    grid.z = unsigned(nz);
    if (s.g.storage == kStoreF16)
        k_scatter_chunk<CodecF16><<<grid, dim3(kBX, kBY), 0, st>>>(s, wbuf, stage, pitch, z0);
    else
        k_scatter_chunk<CodecF32><<<grid, dim3(kBX, kBY), 0, st>>>(s, wbuf, stage, pitch, z0);
    return cudaGetLastError();
}

cudaError_t launch_gather_chunk(const DeviceState &s, int cur, float *stage, size_t pitch, int z0, int nz,
                                cudaStream_t st) {
    dim3 grid = grid3(s.g);
    grid.z = unsigned(nz);
    if (s.g.storage == kStoreF16)
        k_gather_chunk<CodecF16><<<grid, dim3(kBX, kBY), 0, st>>>(s, cur, stage, pitch, z0);
    else
        k_gather_chunk<CodecF32><<<grid, dim3(kBX, kBY), 0, st>>>(s, cur, stage, pitch, z0);
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

// ---- VTI text (base64, RFC 4648 alphabet, '=' padding) ----------------------

__device__ __forceinline__ uint32_t b64_char(uint32_t v) {
    return v < 26 ? 'A' + v : v < 52 ? 'a' + (v - 26) : v < 62 ? '0' + (v - 52) : v == 62 ? '+' : '/';
}

// Word e of array a's float32 payload.
__device__ __forceinline__ uint32_t vti_word(const float *__restrict__ m, uint64_t N, int a, uint64_t e) {
    if (a < 2) return __float_as_uint(m[a * N + e]);
    if (a == 2) return __float_as_uint(__fadd_rn(m[e], m[N + e]));
    const uint64_t node = e / 3;
    return __float_as_uint(m[(2 + (e - 3 * node)) * N + node]);
}

// One thread per 3-byte group of [count][payload] -> one 4-character word.
// blockIdx.y selects the array; stores are 4-byte words, coalesced per warp.
__global__ void __launch_bounds__(256) k_vti_encode(const float *__restrict__ m, uint64_t N, char *__restrict__ text,
                                                    VtiText L) {
    const int a = blockIdx.y;
    const uint64_t payload = (a == 3 ? 3 : 1) * N * 4, total = payload + 8, groups = (total + 2) / 3;
    uint32_t *out = reinterpret_cast<uint32_t *>(text + L.off[a]);
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < groups;
         g += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t v = 0, cw = 0;
        uint64_t ce = ~uint64_t(0);
        for (int k = 0; k < 3; ++k) {
            const uint64_t p = 3 * g + k;
            uint32_t b = 0;
            if (p < 8) {
                b = uint32_t(payload >> (8 * p)) & 0xffu;
            } else if (p < total) {
                const uint64_t q = p - 8, e = q >> 2;
                if (e != ce) {
                    ce = e;
                    cw = vti_word(m, N, a, e);
                }
                b = (cw >> (8 * (q & 3))) & 0xffu;
            }
            v = (v << 8) | b;
        }
        const uint64_t rest = total - 3 * g;
        const uint32_t valid = rest >= 3 ? 4u : uint32_t(rest) + 1u;  // characters that carry data
        uint32_t w = 0;
        for (uint32_t c = 0; c < 4; ++c) w |= (c < valid ? b64_char((v >> (18 - 6 * c)) & 63u) : uint32_t('=')) << (8 * c);
        out[g] = w;
    }
}

cudaError_t launch_vti_encode(const DeviceState &s, char *text, cudaStream_t st) {
    const uint64_t N = uint64_t(s.g.N);
    const VtiText L = vti_text_layout(N);
    const uint64_t groups = (8 + 3 * N * 4 + 2) / 3;
    const uint64_t want = (groups + 255) / 256;
    const unsigned bx = unsigned(want < uint64_t(8 * 148) ? want : uint64_t(8 * 148));
    k_vti_encode<<<dim3(bx, 4), 256, 0, st>>>(s.mom, N, text, L);
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

cudaError_t launch_adj_terminal(const DeviceState &s, const float *M, const float *target, float *lam, double *J,
                                cudaStream_t st) {
    k_adj_terminal<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, M, target, lam, J);
    return cudaGetLastError();
}

cudaError_t launch_adj_collide(const DeviceState &s, const float *M, const float *lam_in, float *lmom, float *lf,
                               double *acc, const AdjObjective &obj, cudaStream_t st) {
    if (s.g.boundary == kBoundaryPeriodic)
        k_adj_collide<true><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, M, lam_in, lmom, lf, acc, obj);
    else
        k_adj_collide<false><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, M, lam_in, lmom, lf, acc, obj);
    return cudaGetLastError();
}

cudaError_t launch_adj_moments(const DeviceState &s, const float *M, const float *lmom, const float *lf,
                               float *lam_out, cudaStream_t st) {
    if (s.g.boundary == kBoundaryPeriodic)
        k_adj_moments<true><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, M, lmom, lf, lam_out);
    else
        k_adj_moments<false><<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, M, lmom, lf, lam_out);
    return cudaGetLastError();
}

cudaError_t launch_adj_step(const DeviceState &s, const float *M, const float *lam_in, float *lmom, float *lf,
                            float *lam_out, double *acc, cudaStream_t st) {
    cudaError_t e = launch_adj_collide(s, M, lam_in, lmom, lf, acc, AdjObjective{0.0f, 0, nullptr}, st);
    if (e != cudaSuccess) return e;
    return launch_adj_moments(s, M, lmom, lf, lam_out, st);
}

cudaError_t launch_adj_boundary(const DeviceState &s, int64_t step, const float *M, const float *Bt,
                                const float *lam_next, const float *lf, float *lmom, const float *LB_in,
                                float *LB_out, const float *bessel, int nb, double *dJdc, cudaStream_t st) {
    const dim3 block(32, 8), grid((s.g.NX + 31) / 32, (s.g.NZ + 7) / 8);
    k_adj_boundary<<<grid, block, 0, st>>>(s, step, M, Bt, lam_next, lf, lmom, LB_in, LB_out, bessel, nb, dJdc);
    return cudaGetLastError();
}

cudaError_t launch_restore_outlet_state(const DeviceState &s, const float *src, float *psi, cudaStream_t st) {
    const dim3 block(32, 8), grid((s.g.NX + 31) / 32, (s.g.NZ + 7) / 8);
    k_restore_outlet_state<<<grid, block, 0, st>>>(s, src, psi);
    return cudaGetLastError();
}

cudaError_t launch_copy_outlet_state(const DeviceState &s, float *dst, cudaStream_t st) {
    const dim3 block(32, 8), grid((s.g.NX + 31) / 32, (s.g.NZ + 7) / 8);
    k_copy_outlet_state<<<grid, block, 0, st>>>(s, dst);
    return cudaGetLastError();
}

cudaError_t launch_adj_initial(const DeviceState &s, const float *M, const float *lam0, float *du0, cudaStream_t st) {
    k_adj_initial<<<grid3(s.g), dim3(kBX, kBY), 0, st>>>(s, M, lam0, du0);
    return cudaGetLastError();
}

}  // namespace mcg
