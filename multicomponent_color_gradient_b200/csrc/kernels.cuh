// kernels.cuh - device-side data layout and kernel entry points of the step.
//
// HBM layout (all structure-of-arrays, node index id = x + NX*(y + NY*z)):
//   pops[2]   two population buffers (ping-pong).  A buffer holds, at node s
//             and direction i, the value that streams OUT of s along c_i
//             (post-collision, pull layout): node x reads f_i(x) from
//             src(x,i) = x - c_i.  The y ghost planes hold what the boundary
//             delivers into the first/last fluid plane.
//               F32: float  [2 colours][27][N]
//               F16: __half2[27][N] = (total offset by w_i*rho0 over w_i,
//                                      colour fraction (fr-fb)/(fr+fb))
//   mom       11 float planes [11][N]: rr, rb, ux, uy, uz, Pixx, Pixy, Piyy,
//             Piyz, Pizz, Pixz - the reference's LbmDevice fields
//             (memory.cuh:11-25), ghost nodes included.
//   psi[2]    colour field psi = (rr-rb)/(rr+rb) per node, ping-pong by step
//             parity; ghost nodes carry what the reference's unwrapped
//             colour-gradient stencil reads there (forces.cuh:31-33).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mcg {

enum : int { kBoundaryJet = 0, kBoundaryClosed = 1, kBoundaryPeriodic = 2 };
enum : int { kStoreF32 = 0, kStoreF16 = 1 };
enum : int { kMomRR = 0, kMomRB, kMomUX, kMomUY, kMomUZ, kMomPXX, kMomPXY, kMomPYY, kMomPYZ, kMomPZZ, kMomPXZ, kMomCount };

struct Geometry {
    int NX, NY, NZ;
    uint32_t N;  // NX*NY*NZ (< 2^32)
    int sy, sz;  // strides of y and z: NX, NX*NY
    int boundary;
    int storage;
};

struct Physics {
    float omega;          // bulk relaxation rate omega_sponge(y) when sponge_K == 0 (mathUtilities.cuh:60-90)
    float omega_b;        // 1/taub, used by the inlet (boundary_conditions.cuh:62)
    float Ah;             // A/2 with A = sigma/(4 cs^4)/taub (forces.cuh:87-105)
    float beta;           // recolouring beta (constants.cuh:74)
    float rhor0, rhob0;
    float jet_x0, jet_z0, jet_r2, jet_velocity;
    float inlet_noise;
    uint64_t seed;
    // sponge (only when sponge_K != 0)
    int sponge;
    float nu, sponge_K, sponge_y_start, sponge_inv_width;
    // radial statistics
    int NRB;
    // F16 storage: populations are stored as (g/w - rho0) and (fr-fb)/g
    float f16_rho0;
};

struct DeviceState {
    Geometry g;
    Physics ph;
    void *pops[2];
    float *mom;       // [11][N]
    float *psi[2];    // [N] each
    double *radial;   // [5][NY*NRB]
    float *uy_avg;    // [N]
    double *partials; // reduction scratch
    uint32_t partials_cap;
    int *flag;        // device flag (non-finite detection)
};

// Launch helpers; all return cudaGetLastError() of the launch.
// step: the reference loop index of the step being computed.
cudaError_t launch_moments(const DeviceState &s, int cur, int64_t step, bool stats, cudaStream_t st);
cudaError_t launch_collide(const DeviceState &s, int cur, int64_t step, cudaStream_t st);
// Jet inlet (which=0), outlet (1) or both (-1) of step `step`, from the moments
// of that step, into the ghost planes of pops[wbuf] and psi[(step+1)&1].
cudaError_t launch_boundary(const DeviceState &s, int wbuf, int64_t step, int which, cudaStream_t st);
cudaError_t launch_accumulate_radial(const DeviceState &s, cudaStream_t st);

// Initial state.  mode 0: jet (jet/jetIn.cuh), 1: bubble (bubble/bubbleIn.cuh),
// 2: populations from reference-layout device arrays fr_ref/fb_ref.
cudaError_t launch_init_fields(const DeviceState &s, int mode, int red_inside, float bubble_r2, float bx, float by,
                               float bz, float noise, cudaStream_t st);
cudaError_t launch_init_pops(const DeviceState &s, int mode, const float *fr_ref, const float *fb_ref, float noise,
                             cudaStream_t st);
// psi of both buffers from the density planes, all nodes (periodic: ghosts mirrored).
cudaError_t launch_refresh_psi(const DeviceState &s, cudaStream_t st);
// Reference-layout gather of f(t) = pops[cur] pulled, interior nodes; ghosts 0.
cudaError_t launch_gather_pops(const DeviceState &s, int cur, float *fr_ref, float *fb_ref, cudaStream_t st);

// Diagnostics / mean fields.
cudaError_t launch_tke(const DeviceState &s, double *out, cudaStream_t st);
cudaError_t launch_uy_average(const DeviceState &s, uint32_t samples, cudaStream_t st);
// Float64 sums over interior nodes of f(t): mass r, mass b, momentum x,y,z.
// partials: scratch of at least conservation_blocks(g)*5 doubles.
uint32_t conservation_blocks(const Geometry &g);
cudaError_t launch_conservation(const DeviceState &s, int cur, double *partials, double *out5, cudaStream_t st);
cudaError_t launch_check_finite(const DeviceState &s, int cur, int *flag, cudaStream_t st);

}  // namespace mcg
