// lattice.cuh - D3Q27 lattice and the colour-gradient collision maths, float32.
//
// Direction order, weights, Hermite polynomials and the 1/|c| table are the
// ones the reference defines in stencil_ct.cuh:9-189 (the populations' memory
// layout depends on the order, and the Hermite constants are formed with the
// same float expressions so they fold to the same values).  The physics
// functions restate lbm.cuh:16-78 (equilibrium, regularised non-equilibrium),
// forces.cuh:50-105 (cos^2 rule, A) and collisionOperators.cuh:15-69
// (perturbation, recolouring).
#pragma once

#include <cstdint>
#include <utility>

namespace mcg {

constexpr int kQ = 27;

// constants.cuh:45-53 (float arithmetic, folded at compile time)
constexpr float kCs2 = static_cast<float>(1.0 / 3.0);
constexpr float kCs4 = kCs2 * kCs2;
constexpr float kCs6 = kCs4 * kCs2;
constexpr float kInvCs2 = 1.0f / kCs2;
constexpr float kInv2Cs2 = 1.0f / (2.0f * kCs2);
constexpr float kInv2Cs4 = 1.0f / (2.0f * kCs4);
constexpr float kInv6Cs6 = 1.0f / (6.0f * kCs6);
constexpr float kInv2Cs6 = 1.0f / (2.0f * kCs6);

__host__ __device__ constexpr int dir_cx(int i) {
    constexpr int t[kQ] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int dir_cy(int i) {
    constexpr int t[kQ] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int dir_cz(int i) {
    constexpr int t[kQ] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int dir_norm2(int i) {
    return dir_cx(i) * dir_cx(i) + dir_cy(i) * dir_cy(i) + dir_cz(i) * dir_cz(i);
}
__host__ __device__ constexpr float dir_w(int i) {
    return dir_norm2(i) == 0 ? float(8.0 / 27.0)
         : dir_norm2(i) == 1 ? float(2.0 / 27.0)
         : dir_norm2(i) == 2 ? float(1.0 / 54.0)
                             : float(1.0 / 216.0);
}
// Direction index of velocity (cx, cy, cz) (inverse of dir_cx/cy/cz).
__host__ __device__ constexpr int dir_of(int cx, int cy, int cz) {
    int r = -1;
    for (int i = 0; i < kQ; ++i)
        if (dir_cx(i) == cx && dir_cy(i) == cy && dir_cz(i) == cz) r = i;
    return r;
}
__host__ __device__ constexpr float dir_B(int i) { return i == 0 ? float(-10.0 / 27.0) : dir_w(i); }
__host__ __device__ constexpr float dir_invc(int i) {
    return dir_norm2(i) == 0 ? 0.0f
         : dir_norm2(i) == 1 ? 1.0f
         : dir_norm2(i) == 2 ? float(0.7071067811865475)
                             : float(0.5773502691896258);
}

// Compile-time view of one direction.
template <int I>
struct Dir {
    static constexpr int cx = dir_cx(I), cy = dir_cy(I), cz = dir_cz(I);
    static constexpr float fx = float(cx), fy = float(cy), fz = float(cz);
    static constexpr float w = dir_w(I);
    static constexpr float B = dir_B(I);
    static constexpr float invc = dir_invc(I);
    static constexpr float Hxx = float(cx * cx) - kCs2, Hxy = float(cx * cy), Hyy = float(cy * cy) - kCs2;
    static constexpr float Hyz = float(cy * cz), Hzz = float(cz * cz) - kCs2, Hxz = float(cx * cz);
    static constexpr float Hxxy = float(cx * cx * cy) - kCs2 * float(cy);
    static constexpr float Hxxz = float(cx * cx * cz) - kCs2 * float(cz);
    static constexpr float Hxyy = float(cx * cy * cy) - kCs2 * float(cx);
    static constexpr float Hxzz = float(cx * cz * cz) - kCs2 * float(cx);
    static constexpr float Hyyz = float(cy * cy * cz) - kCs2 * float(cz);
    static constexpr float Hyzz = float(cy * cz * cz) - kCs2 * float(cy);
    static constexpr float Hxyz = float(cx * cy * cz);
};

// Opposite direction of i in the reference order (pairs 2k-1, 2k).
__host__ __device__ constexpr int dir_opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

// Row-blocked population layout.  All populations of one lattice row (y,z)
// are contiguous; inside a row they are grouped by the row they are pulled
// from: group g = (cy+1)*3 + (cz+1), then cx.  One element holds both colours
// of a direction (a float2 (fr, fb), or a float16 pair; the adjoint's lambda
// pairs (lambda_r, lambda_b) the same way), so a pulled row is 9 contiguous
// segments of 3 x-rows.
__host__ __device__ constexpr int dir_group(int i) { return (dir_cy(i) + 1) * 3 + (dir_cz(i) + 1); }
__host__ __device__ constexpr int slot_pair(int i) { return dir_group(i) * 3 + (dir_cx(i) + 1); }

template <int... Is, class F>
__device__ __forceinline__ void static_for_impl(F &&f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
// f(std::integral_constant<int, i>) for i = 0..N-1, fully unrolled.
template <int N, class F>
__device__ __forceinline__ void static_for(F &&f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// Moments one collision needs: densities, velocity, non-equilibrium stress.
struct NodeMoments {
    float rr, rb;
    float ux, uy, uz;
    float pxx, pxy, pyy, pyz, pzz, pxz;
};

// Velocity-dependent terms shared by every direction of one node.
struct EqTerms {
    float ux, uy, uz, usq;
};
__device__ __forceinline__ EqTerms make_eq(float ux, float uy, float uz) {
    return EqTerms{ux, uy, uz, ux * ux + uy * uy + uz * uz};
}

// Third-order stress combinations of fneqr (lbm.cuh:67-73), per node.
struct NeqTerms {
    float pxx, pxy, pyy, pyz, pzz, pxz;
    float a3xxy, a3xxz, a3xyy, a3xzz, a3yyz, a3yzz, a3xyz;
};
__device__ __forceinline__ NeqTerms make_neq(float pxx, float pxy, float pyy, float pyz, float pzz, float pxz,
                                              float ux, float uy, float uz) {
    NeqTerms n;
    n.pxx = pxx; n.pxy = pxy; n.pyy = pyy; n.pyz = pyz; n.pzz = pzz; n.pxz = pxz;
    n.a3xxy = pxx * uy + 2.0f * pxy * ux;
    n.a3xxz = pxx * uz + 2.0f * pxz * ux;
    n.a3xyy = pyy * ux + 2.0f * pxy * uy;
    n.a3xzz = pzz * ux + 2.0f * pxz * uz;
    n.a3yyz = pyy * uz + 2.0f * pyz * uy;
    n.a3yzz = pzz * uy + 2.0f * pyz * uz;
    n.a3xyz = pxy * uz + pxz * uy + pyz * ux;
    return n;
}

// Third-order Hermite equilibrium (lbm.cuh:16-35).
template <int I>
__device__ __forceinline__ float feq(float rho, const EqTerms &e) {
    using D = Dir<I>;
    float cu = 0.0f;
    if constexpr (D::cx != 0) cu += D::fx * e.ux;
    if constexpr (D::cy != 0) cu += D::fy * e.uy;
    if constexpr (D::cz != 0) cu += D::fz * e.uz;
    const float A2 = (cu * cu) * kInv2Cs4 - e.usq * kInv2Cs2 + cu * kInvCs2;
    const float A3 = cu * ((cu * cu) * kInv6Cs6 - e.usq * kInv2Cs4);
    return D::w * rho * (1.0f + A2 + A3);
}

// Recursive-regularised non-equilibrium part (lbm.cuh:38-78).
template <int I>
__device__ __forceinline__ float fneq(const NeqTerms &n) {
    using D = Dir<I>;
    const float A2 = (n.pxx * D::Hxx + 2.0f * n.pxy * D::Hxy + n.pyy * D::Hyy + 2.0f * n.pyz * D::Hyz +
                      n.pzz * D::Hzz + 2.0f * n.pxz * D::Hxz) * kInv2Cs4;
    float A3 = 0.0f;
    if constexpr (D::Hxxy != 0.0f) A3 += n.a3xxy * D::Hxxy;
    if constexpr (D::Hxxz != 0.0f) A3 += n.a3xxz * D::Hxxz;
    if constexpr (D::Hxyy != 0.0f) A3 += n.a3xyy * D::Hxyy;
    if constexpr (D::Hxzz != 0.0f) A3 += n.a3xzz * D::Hxzz;
    if constexpr (D::Hyyz != 0.0f) A3 += n.a3yyz * D::Hyyz;
    if constexpr (D::Hyzz != 0.0f) A3 += n.a3yzz * D::Hyzz;
    if constexpr (D::Hxyz != 0.0f) A3 += 2.0f * n.a3xyz * D::Hxyz;
    return D::w * (A2 + A3 * kInv2Cs6);
}

// Directions 2k-1 and 2k are opposite (stencil_ct.cuh:9-16).  For such a pair
// the equilibrium and the regularised non-equilibrium split into a part even
// in c (same for both) and a part odd in c (sign flips), so one evaluation
// serves both directions.  feq_i = w rho (E + O), feq_ibar = w rho (E - O);
// fneq_i = w (A2 + A3), fneq_ibar = w (A2 - A3).
template <int I>
__device__ __forceinline__ void feq_pair(float rho, const EqTerms &e, float &fi, float &fo) {
    using D = Dir<I>;
    float cu = 0.0f;
    if constexpr (D::cx != 0) cu += D::fx * e.ux;
    if constexpr (D::cy != 0) cu += D::fy * e.uy;
    if constexpr (D::cz != 0) cu += D::fz * e.uz;
    const float even = 1.0f + ((cu * cu) * kInv2Cs4 - e.usq * kInv2Cs2);
    const float odd = cu * kInvCs2 + cu * ((cu * cu) * kInv6Cs6 - e.usq * kInv2Cs4);
    const float wr = D::w * rho;
    fi = wr * (even + odd);
    fo = wr * (even - odd);
}

template <int I>
__device__ __forceinline__ void fneq_pair(const NeqTerms &n, float &fi, float &fo) {
    using D = Dir<I>;
    const float A2 = (n.pxx * D::Hxx + 2.0f * n.pxy * D::Hxy + n.pyy * D::Hyy + 2.0f * n.pyz * D::Hyz +
                      n.pzz * D::Hzz + 2.0f * n.pxz * D::Hxz) * kInv2Cs4;
    float A3 = 0.0f;
    if constexpr (D::Hxxy != 0.0f) A3 += n.a3xxy * D::Hxxy;
    if constexpr (D::Hxxz != 0.0f) A3 += n.a3xxz * D::Hxxz;
    if constexpr (D::Hxyy != 0.0f) A3 += n.a3xyy * D::Hxyy;
    if constexpr (D::Hxzz != 0.0f) A3 += n.a3xzz * D::Hxzz;
    if constexpr (D::Hyyz != 0.0f) A3 += n.a3yyz * D::Hyyz;
    if constexpr (D::Hyzz != 0.0f) A3 += n.a3yzz * D::Hyzz;
    if constexpr (D::Hxyz != 0.0f) A3 += 2.0f * n.a3xyz * D::Hxyz;
    A3 *= kInv2Cs6;
    fi = D::w * (A2 + A3);
    fo = D::w * (A2 - A3);
}

// Bulk post-collision value over the weight, P[i] = (feq_i + oms fneq_i) / w_i
// (lbm.cuh:16-78), for all 27 directions at once.  As a function of c_i it is
// the polynomial
//   rho [1 + q u.c + (q^2/2)(u.c)^2 - (q/2)|u|^2 + (q^3/6)(u.c)^3 - (q^2/2)|u|^2 u.c]
//   + oms [(q^2/2) Pi:(cc - I/q) + (q^3/2) sum_k a3_k H3_k(c)],      q = 1/cs^2,
// which on the lattice (c_a^3 = c_a) has 17 coefficients of per-axis degree
// <= 2.  D3Q27 is the tensor product of three D1Q3 stencils, so the 27 values
// follow from the coefficients by three passes of 1-D evaluation at
// c = -1, 0, 1 (sum factorisation): about 70 adds instead of a Hermite
// evaluation per direction.  `shift` is taken off the constant coefficient,
// so P[i] comes out as P_i - shift (the float16 store keeps P_i - rho0).
__device__ __forceinline__ void collision_poly(float rho, float ux, float uy, float uz, const NeqTerms &n, float oms,
                                               float (&P)[kQ], float shift = 0.0f) {
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const float usq = ux2 + uy2 + uz2;
    const float lin = kInvCs2 - kInv2Cs4 * usq;
    // coefficients of 1, c_a, c_a^2, c_a c_b, c_a^2 c_b, c_x c_y c_z
    const float a0 = (rho - shift) - kInv2Cs2 * (rho * usq + oms * (n.pxx + n.pyy + n.pzz));
    const float Ax = rho * ux * (lin + kInv6Cs6 * ux2) - oms * kInv2Cs4 * (n.a3xyy + n.a3xzz);
    const float Ay = rho * uy * (lin + kInv6Cs6 * uy2) - oms * kInv2Cs4 * (n.a3xxy + n.a3yzz);
    const float Az = rho * uz * (lin + kInv6Cs6 * uz2) - oms * kInv2Cs4 * (n.a3xxz + n.a3yyz);
    const float rx2 = rho * ux2, ry2 = rho * uy2, rz2 = rho * uz2;
    const float Axx = kInv2Cs4 * (rx2 + oms * n.pxx);
    const float Ayy = kInv2Cs4 * (ry2 + oms * n.pyy);
    const float Azz = kInv2Cs4 * (rz2 + oms * n.pzz);
    const float Axy = (2.0f * kInv2Cs4) * (rho * ux * uy + oms * n.pxy);
    const float Axz = (2.0f * kInv2Cs4) * (rho * ux * uz + oms * n.pxz);
    const float Ayz = (2.0f * kInv2Cs4) * (rho * uy * uz + oms * n.pyz);
    const float Axxy = kInv2Cs6 * (rx2 * uy + oms * n.a3xxy);
    const float Axxz = kInv2Cs6 * (rx2 * uz + oms * n.a3xxz);
    const float Ayyx = kInv2Cs6 * (ry2 * ux + oms * n.a3xyy);
    const float Azzx = kInv2Cs6 * (rz2 * ux + oms * n.a3xzz);
    const float Ayyz = kInv2Cs6 * (ry2 * uz + oms * n.a3yyz);
    const float Azzy = kInv2Cs6 * (rz2 * uy + oms * n.a3yzz);
    const float Axyz = (2.0f * kInv2Cs6) * (rho * ux * uy * uz + oms * n.a3xyz);
    // P = B0(cx,cy) + cz B1(cx,cy) + cz^2 B2(cx,cy); B* = C*(cx) + cy C*'(cx) + cy^2 C*''(cx)
    float C0[3], C1[3], C2[3], D0[3], D1[3], E0[3];
    {
        const float s = a0 + Axx;
        C0[0] = s - Ax; C0[1] = a0; C0[2] = s + Ax;
    }
    {
        const float s = Ay + Axxy;
        C1[0] = s - Axy; C1[1] = Ay; C1[2] = s + Axy;
    }
    C2[0] = Ayy - Ayyx; C2[1] = Ayy; C2[2] = Ayy + Ayyx;
    {
        const float s = Az + Axxz;
        D0[0] = s - Axz; D0[1] = Az; D0[2] = s + Axz;
    }
    D1[0] = Ayz - Axyz; D1[1] = Ayz; D1[2] = Ayz + Axyz;
    E0[0] = Azz - Azzx; E0[1] = Azz; E0[2] = Azz + Azzx;
    static_for<3>([&](auto JX) {
        constexpr int jx = decltype(JX)::value;
        const float b0s = C0[jx] + C2[jx], b1s = D0[jx] + Ayyz;
        const float b0[3] = {b0s - C1[jx], C0[jx], b0s + C1[jx]};
        const float b1[3] = {b1s - D1[jx], D0[jx], b1s + D1[jx]};
        const float b2[3] = {E0[jx] - Azzy, E0[jx], E0[jx] + Azzy};
        static_for<3>([&](auto JY) {
            constexpr int jy = decltype(JY)::value;
            const float t = b0[jy] + b2[jy];
            P[dir_of(jx - 1, jy - 1, 0)] = b0[jy];
            P[dir_of(jx - 1, jy - 1, -1)] = t - b1[jy];
            P[dir_of(jx - 1, jy - 1, 1)] = t + b1[jy];
        });
    });
}

// Interface terms shared by all directions of one node.
struct InterfaceTerms {
    float Fx, Fy, Fz;     // colour gradient (forces.cuh:13-43)
    float absF;           // |F|
    bool has_dir;         // |F| > 1e-4: cos^2 and cos phi are non-zero (forces.cuh:61, collisionOperators.cuh:42)
    float inv_absF2;      // 1/|F|^2
    float inv_absF;       // 1/|F|
    float Ah_absF;        // (A/2)|F|
    float coeff_rho;      // beta * rr*rb/rho^2 * rho  (recolouring amplitude, collisionOperators.cuh:57-68)
};

// Perturbation operator (collisionOperators.cuh:15-24 with forces.cuh:50-75).
template <int I>
__device__ __forceinline__ float omega2(const InterfaceTerms &t) {
    using D = Dir<I>;
    float cos2 = 0.0f;
    if constexpr (I != 0) {
        if (t.has_dir) {
            float fc = 0.0f;
            if constexpr (D::cx != 0) fc += t.Fx * D::fx;
            if constexpr (D::cy != 0) fc += t.Fy * D::fy;
            if constexpr (D::cz != 0) fc += t.Fz * D::fz;
            cos2 = (fc * fc) * t.inv_absF2;
        }
    }
    return t.Ah_absF * (D::w * cos2 - D::B);
}

// Recolouring perturbation Delta_i (collisionOperators.cuh:28-69).
template <int I>
__device__ __forceinline__ float recolour(const InterfaceTerms &t) {
    using D = Dir<I>;
    if constexpr (I == 0) {
        return 0.0f;
    } else {
        if (!t.has_dir) return 0.0f;
        float fc = 0.0f;
        if constexpr (D::cx != 0) fc += t.Fx * D::fx;
        if constexpr (D::cy != 0) fc += t.Fy * D::fy;
        if constexpr (D::cz != 0) fc += t.Fz * D::fz;
        const float cosphi = fc * t.inv_absF * D::invc;
        return t.coeff_rho * cosphi * D::w;
    }
}

// Counter-based uniform hash in [0,1) with 24 random bits (exact in float).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ float hash_uniform(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    const uint64_t h = splitmix64(seed ^ splitmix64(a ^ splitmix64(b ^ splitmix64(c))));
    return static_cast<float>(h >> 40) * (1.0f / 16777216.0f);
}

}  // namespace mcg
