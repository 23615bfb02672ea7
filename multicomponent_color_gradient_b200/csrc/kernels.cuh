// kernels.cuh - device-side data layout and kernel entry points of the step.
//
// HBM layout (node index id = x + NX*(y + NY*z) for the per-node fields):
//   pops[2]   two population buffers (ping-pong), row-blocked: row (y,z) holds
//             `slots` = 27 x-rows of NX elements, grouped by pull source
//             (lattice.cuh slot_pair); element (slot, x, y, z) is at
//             ((z*NY + y)*27 + slot)*NX + x.  One element carries both colours
//             of a direction, so a pull or a store is one 8- or 4-byte access.
//             A buffer holds, at node s and direction i, the value that streams
//             OUT of s along c_i (post-collision, pull layout): node x reads
//             f_i(x) from x - c_i.  The y ghost planes hold what the boundary
//             delivers into the first/last fluid plane.
//               F32: float2 (fr, fb)
//               F16: __half2 ((total offset by w_i*rho0)/w_i, signed
//                              minority-colour fraction)
//             The adjoint's lambda arrays have the float32 layout: one
//             float2 (lambda_r, lambda_b) per direction and node.
//   mom       11 float planes [11][N]: rr, rb, ux, uy, uz, Pixx, Pixy, Piyy,
//             Piyz, Pizz, Pixz - the reference's LbmDevice fields
//             (memory.cuh:11-25), ghost nodes included.  The fused step does
//             not stream them; they are refreshed on demand (output steps,
//             granular launch sequence).
//   psi[2]    colour field psi = (rr-rb)/(rr+rb) per node, ping-pong by step
//             parity; the fused step reads only its ghost nodes, which carry
//             what the reference's unwrapped colour-gradient stencil reads
//             there (forces.cuh:31-33).
//   bmom      moments of the first and last fluid planes (y=1, y=NY-2),
//             [2][NZ][11][NX], for the boundary launch.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mcg {

enum : int { kBoundaryJet = 0, kBoundaryClosed = 1, kBoundaryPeriodic = 2 };
constexpr int kInletBesselMax = 8;  // coefficients of the radial inlet profile
enum : int { kStoreF32 = 0, kStoreF16 = 1 };
enum : int { kMomRR = 0, kMomRB, kMomUX, kMomUY, kMomUZ, kMomPXX, kMomPXY, kMomPYY, kMomPYZ, kMomPZZ, kMomPXZ, kMomCount };
// A moment record of one state: the kMomCount moment planes, then psi.
enum : int { kTapePsi = kMomCount, kTapePlanes = kMomCount + 1 };

struct Geometry {
    int NX, NY, NZ;
    uint32_t N;  // NX*NY*NZ (< 2^31)
    int sy, sz;  // strides of y and z in the per-node fields: NX, NX*NY
    int boundary;
    int storage;
    int slots;   // x-rows per lattice row in the population buffers: 27 (one element per direction)
};

__host__ __device__ __forceinline__ size_t pop_row(const Geometry &g, int y, int z) {
    return (size_t(z) * size_t(g.NY) + size_t(y)) * size_t(g.slots) * size_t(g.NX);
}
__host__ __device__ __forceinline__ size_t pop_index(const Geometry &g, int slot, int x, int y, int z) {
    return pop_row(g, y, z) + size_t(slot) * size_t(g.NX) + size_t(x);
}

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
    // F16 storage: populations are stored as (g/w - rho0) and the colour fraction
    float f16_rho0;
};

// Tiling of the fused step: a CTA owns rows [y0, y0+ty) of every plane of a
// z-chunk [z0, z0+lz) and marches z (up, or down for odd chunks when
// `alternate`); tpr threads per row (a multiple of 32,
// >= NX), blockDim.x / tpr rows in parallel.
struct FusedTiling {
    int ty, lz, tpr;
    int ny_tiles, nz_chunks;
    int smem_bytes;
    int alternate; // odd z-chunks march down, so neighbouring chunks pull their shared planes together
    int pipe;      // software-pipelined march (k_fused_pipe): one barrier per plane
    int fixed_nx;  // row length the kernel is compiled for (0: runtime geometry)
    int bulk;      // the pipelined march with rows staged by bulk copies (k_fused_bulk)
    int wait_limit;  // k_fused_bulk: tries (about 1 us each) of a wait for a staged row before it gives up
    int boundary;    // jet: the fused step writes the inlet and outlet columns itself (no k_boundary launch)
    // set by launch_fused for each launch when `boundary`: the buffer the step
    // writes, the next step's psi and the step (read only by the boundary rows)
    void *bnd_dst;
    float *bnd_psi;
    long long bnd_step;
};

// Tries of a k_fused_bulk wait by default (about a second), and of the wait
// for copies still in flight when a CTA gives up.
constexpr int kBulkWaitLimit = 1 << 20;
constexpr uint32_t kBulkDrainLimit = 1u << 20;

struct DeviceState {
    Geometry g;
    Physics ph;
    void *pops[2];
    float *mom;       // [11][N]
    float *psi[2];    // [N] each
    float *bmom;      // [2][NZ][11][NX]
    double *radial;   // [5][NY*NRB]
    float *uy_avg;    // [N]
    double *partials; // reduction scratch
    uint32_t partials_cap;
    int *flag;        // device flags: [0] non-finite value, [1] a k_fused_bulk wait ran out
    float *tape;      // null, or [kTapePlanes][N]: the fused step records the moments and psi it pulls there
    const float *inlet_profile;  // null (top-hat), or [NZ][NX] multipliers of the inlet velocity per column
};

// ---- the fused step (moments + colour gradient + collision in one pass) ----
FusedTiling fused_tiling(const Geometry &g, int max_smem_per_block);
cudaError_t fused_configure(int max_smem);
cudaError_t launch_fused(const DeviceState &s, const FusedTiling &t, int cur, int64_t step, bool stats,
                         cudaStream_t st);

// ---- granular launch sequence (launch.cuh order) ----
// step: the reference loop index of the step being computed.
cudaError_t launch_moments(const DeviceState &s, int cur, int64_t step, bool stats, cudaStream_t st);
cudaError_t launch_collide(const DeviceState &s, int cur, int64_t step, cudaStream_t st);
// Jet inlet (which=0), outlet (1) or both (-1) of step `step`, into the ghost
// planes of pops[wbuf] and psi[(step+1)&1].  from_bmom: moments of the fluid
// planes come from bmom (fused step) instead of mom (granular sequence).
cudaError_t launch_boundary(const DeviceState &s, int wbuf, int64_t step, int which, bool from_bmom,
                            cudaStream_t st);
cudaError_t launch_accumulate_radial(const DeviceState &s, cudaStream_t st);

// Initial state.  mode 0: jet (jet/jetIn.cuh), 1: bubble (bubble/bubbleIn.cuh),
// 3: per-colour equilibrium feq(rho_c, u) of the moment planes rr, rb, u.
cudaError_t launch_init_fields(const DeviceState &s, int mode, int red_inside, float bubble_r2, float bx, float by,
                               float bz, cudaStream_t st);
cudaError_t launch_init_pops(const DeviceState &s, int mode, float noise, cudaStream_t st);
// psi of both buffers from the density planes, all nodes (periodic: ghosts mirrored).
cudaError_t launch_refresh_psi(const DeviceState &s, cudaStream_t st);
// Host state transfer by z-chunks of the reference layout f[i*Ncells + id]:
// `stage` holds planes [z0, z0+nz) of both colours as
// stage[colour][i][id - z0*NX*NY], `pitch` elements per direction row.
// Scatter: the chunk's interior populations to their pull sources in
// pops[wbuf].  Gather: f(t) = pops[cur] pulled at the chunk's nodes (ghosts 0).
cudaError_t launch_scatter_chunk(const DeviceState &s, int wbuf, const float *stage, size_t pitch, int z0, int nz,
                                 cudaStream_t st);
cudaError_t launch_gather_chunk(const DeviceState &s, int cur, float *stage, size_t pitch, int z0, int nz,
                                cudaStream_t st);

// Diagnostics / mean fields.
cudaError_t launch_tke(const DeviceState &s, double *out, cudaStream_t st);
cudaError_t launch_uy_average(const DeviceState &s, uint32_t samples, cudaStream_t st);

// VTK XML image data, format="binary" (io/save_data.cuh:137-215): each array is
// the base64 text of [UInt64 byte count][little-endian float32 payload].  The
// four arrays are rhor, rhob, rho = rhor + rhob and u (ux, uy, uz interleaved
// per node); their texts lie back to back in one buffer.
struct VtiText {
    uint64_t len[4], off[4], total;
};
inline VtiText vti_text_layout(uint64_t N) {
    VtiText t{};
    uint64_t at = 0;
    for (int a = 0; a < 4; ++a) {
        const uint64_t bytes = 8 + (a == 3 ? 3 : 1) * N * 4;
        t.len[a] = (bytes + 2) / 3 * 4;
        t.off[a] = at;
        at += t.len[a];
    }
    t.total = at;
    return t;
}
// Encodes the first five moment planes of s.mom ([5][N]: rr, rb, ux, uy, uz)
// into text (vti_text_layout(N).total bytes, 4-byte aligned).
cudaError_t launch_vti_encode(const DeviceState &s, char *text, cudaStream_t st);
// Float64 sums over interior nodes of f(t): mass r, mass b, momentum x,y,z.
// partials: scratch of at least conservation_blocks(g)*5 doubles.
uint32_t conservation_blocks(const Geometry &g);
cudaError_t launch_conservation(const DeviceState &s, int cur, double *partials, double *out5, cudaStream_t st);
cudaError_t launch_check_finite(const DeviceState &s, int cur, int *flag, cudaStream_t st);

// Objective source of an adjoint step: J_t = (weight/2) sum of uy^2 over
// interior nodes with y >= y_obs (weight 0: none); J accumulates J_t (or null).
// With `table` ([NY][NRB]) the source instead is dJ/duy = table[y][rb] at the
// nodes of radial bin rb < NRB (the bins of the radial statistics), the
// adjoint of an objective of the time-averaged radial profiles of uy; J is
// then formed on the host.
struct AdjObjective {
    float weight;
    int y_obs;
    double *J;
    const float *table = nullptr;
};

// ---- discrete adjoint of the step (float32 populations) ----
// lambda buffers share the population layout; M is the moment record
// [kTapePlanes][N] of the state the pass belongs to (interior nodes).
// Terminal condition for J = sum (psi_T - target)^2, one adjoint step
// (lmom [11][N], lf [3][N] scratch; acc[0] += dJ/domega, acc[1] += dJ/d(A/2)),
// and dJ/du0 of a state f0 = feq(rho_c, u0) (du0 [3][N]).
cudaError_t launch_adj_terminal(const DeviceState &s, const float *M, const float *target, float *lam, double *J,
                                cudaStream_t st);
cudaError_t launch_adj_step(const DeviceState &s, const float *M, const float *lam_in, float *lmom, float *lf,
                            float *lam_out, double *acc, cudaStream_t st);
// The same step in two parts for the jet, with the boundary adjoint between
// them: the relaxation part (lam_in -> lmom, lf, objective source) and the
// moment part (lmom, lf -> lam_out).
cudaError_t launch_adj_collide(const DeviceState &s, const float *M, const float *lam_in, float *lmom, float *lf,
                               double *acc, const AdjObjective &obj, cudaStream_t st);
cudaError_t launch_adj_moments(const DeviceState &s, const float *M, const float *lmom, const float *lf,
                               float *lam_out, cudaStream_t st);
// Adjoint of the jet boundary of step `step` (inlet and convective outlet,
// jet/boundary_conditions.cuh:17-85,163-233) and of the outlet-plane psi the
// step read.  M: the step's moment record; Bt: [5][NX*NZ] outlet state
// (rr, rb, ux, uy, uz at y = NY-1) before the step's boundary; lam_next: the
// adjoint of the populations the step wrote; lf: the step's colour-gradient
// adjoint.  Adds into lmom at y = 1 and y = NY-2; LB_in: the adjoint of the
// outlet state after the boundary, LB_out: before it; bessel: [nb][NX*NZ] J0
// basis of the inlet profile (or null), dJdc[nb] += dJ/dc_k.
cudaError_t launch_adj_boundary(const DeviceState &s, int64_t step, const float *M, const float *Bt,
                                const float *lam_next, const float *lf, float *lmom, const float *LB_in,
                                float *LB_out, const float *bessel, int nb, double *dJdc, cudaStream_t st);
// The outlet state (5 planes at y = NY-1, interior columns) to dst[5][NX*NZ],
// and back (restoring also the outlet-plane psi in `psi`).
cudaError_t launch_copy_outlet_state(const DeviceState &s, float *dst, cudaStream_t st);
cudaError_t launch_restore_outlet_state(const DeviceState &s, const float *src, float *psi, cudaStream_t st);
cudaError_t launch_adj_initial(const DeviceState &s, const float *M, const float *lam0, float *du0, cudaStream_t st);

}  // namespace mcg
