/*
 * mcg.h - C ABI of the B200 D3Q27 colour-gradient lattice Boltzmann step.
 *
 * This is the drop-in boundary for the per-time-step path of
 * Felipe-Aristi/Multicomponent_Color_Gradient.  That project has no FFI: its
 * de-facto operator boundary is the launcher set in launch.cuh:13-118 plus the
 * device-memory helpers in memory.cuh:58-133 and the mean-field runtime in
 * meanF/meanFieldsRT.cuh:132-381.  Each entry point below names the reference
 * interface it replaces.
 *
 * Conventions (kept identical to the reference so host buffers interoperate):
 *   - NX*NY*NZ counts the one-cell ghost shell (utilities/bounds.cuh:6-13);
 *   - node index id = x + NX*(y + NY*z), x fastest (utilities/indexing.cuh:10-13);
 *   - populations are structure-of-arrays, f[i*Ncells + id]
 *     (utilities/indexing.cuh:15-19), direction order of stencil_ct.cuh:9-16;
 *   - fields are float32, radial sums float64, radial counts uint64
 *     (utilities/types.cuh:6-11).
 *
 * Error behaviour: the reference prints and calls exit(1) on any CUDA error
 * (utilities/cudaUtilities.cuh:9-19).  Every function here instead returns an
 * mcg_status and never exits or traps; mcg_last_error_string() describes the
 * last failure of the calling thread.
 *
 * Threading: one handle is driven by one host thread at a time.  Work is
 * queued on the handle's stream (mcg_set_stream); functions that return host
 * data synchronise that stream first.
 */
#ifndef MCG_H
#define MCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCG_Q 27
#define MCG_ABI_VERSION 1

typedef enum mcg_status {
    MCG_OK = 0,
    MCG_ERR_INVALID_ARG = 1,  /* bad parameter, null pointer, size out of range */
    MCG_ERR_OOM = 2,          /* device or host allocation failed */
    MCG_ERR_CUDA = 3,         /* a CUDA runtime call or kernel launch failed */
    MCG_ERR_NONFINITE = 4,    /* NaN/Inf detected by mcg_check_finite */
    MCG_ERR_IO = 5,           /* file could not be created or fully written */
    MCG_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    MCG_ERR_STATE = 7,        /* call not valid in the handle's current state */
    MCG_ERR_UNSUPPORTED = 8,  /* option combination not implemented */
    MCG_ERR_NO_DEVICE = 9     /* no CUDA device visible */
} mcg_status;

/* Population storage in HBM.  Arithmetic is float32 in both cases. */
typedef enum mcg_storage {
    MCG_STORAGE_F32 = 0,  /* reference precision (utilities/types.cuh:6-11) */
    MCG_STORAGE_F16 = 1   /* offset by w_i*rho0, colour split as a fraction (extension) */
} mcg_storage;

/* What happens at the y ghost planes. */
typedef enum mcg_boundary {
    /* jet inlet at y=0 and convective outlet at y=NY-1
     * (jet/boundary_conditions.cuh:17-85,163-233) - the shipped driver main.cu */
    MCG_BOUNDARY_JET = 0,
    /* no boundary kernels: y ghost-plane populations are never rewritten and the
     * colour gradient reads the frozen ghost densities - what launch_bubble +
     * launch_Macros + launch_collistream alone do in the reference */
    MCG_BOUNDARY_CLOSED = 1,
    /* x, y and z periodic both for streaming and for the colour gradient
     * (extension: a true periodic box; the reference never wraps y) */
    MCG_BOUNDARY_PERIODIC = 2
} mcg_boundary;

/*
 * Case parameters.  Field names mirror constants.cuh:8-76 one-to-one so a
 * constants.cuh can be generated from them (mcg_write_constants_header).
 * mcg_params_default() fills the values shipped in constants.cuh;
 * mcg_params_derive() recomputes nu, taur, taub and sigma from Re, We and the
 * jet scales exactly as constants.cuh:59-76 does (float arithmetic).
 */
typedef struct mcg_params {
    int32_t NX, NY, NZ;                 /* constants.cuh:14-16 */
    int32_t NSTEP, NOUTPUT;             /* constants.cuh:8-9 */
    int32_t NSTATS_START_STEP;          /* constants.cuh:10 */
    int32_t write_vti_output;           /* constants.cuh:11 */
    int32_t sponge_cells;               /* constants.cuh:17 */
    float jet_radius, jet_x0, jet_z0, jet_velocity;              /* constants.cuh:32-35 */
    float bubble_radius, bubble_x0, bubble_y0, bubble_z0;        /* constants.cuh:38-41 */
    float rhor0, rhob0;                 /* constants.cuh:56-57 */
    float Re, We;                       /* constants.cuh:59,71 */
    float nu, taur, taub, sigma;        /* constants.cuh:60-64,73 */
    float beta_recolor;                 /* constants.cuh:74 */
    float sponge_K;                     /* utilities/mathUtilities.cuh:50 */
    /* ---- options with no counterpart in constants.cuh ---- */
    int32_t boundary;                   /* mcg_boundary */
    int32_t storage;                    /* mcg_storage */
    uint64_t seed;                      /* counter-based hash seed for all noise */
    float init_noise;                   /* relative amplitude of uniform noise on initial populations */
    float inlet_noise;                  /* relative amplitude of uniform noise on the inlet velocity */
    int32_t bubble_red_inside;          /* 0: blue sphere in red (bubble/bubbleIn.cuh:20-22); 1: red in blue */
    int32_t reserved[9];
} mcg_params;

typedef struct mcg_handle mcg_handle;

/* ---------------- parameters ---------------- */

/* Values of constants.cuh as shipped (128x400x128, Re 5000, We 2000, jet). */
mcg_status mcg_params_default(mcg_params *p);
/* nu = 2*R*U/Re, taur = taub = 0.5 + nu/cs2, sigma = rhob0*U^2*2R/We
 * (constants.cuh:60-73); jet_x0/z0 and bubble centres = (N-1)/2 (:33-34,39-41). */
mcg_status mcg_params_derive(mcg_params *p);
/* Sets taur = taub = tau and nu = (tau - 0.5)*cs2 directly (bubble cases that
 * are specified by tau and sigma rather than Re and We). */
mcg_status mcg_params_set_tau(mcg_params *p, float tau);
/* Writes a constants.cuh-compatible header (same names, same
 * `name = static_cast<T>(value)` text form that post/case_config.py:30-35 and
 * post/mean_profile_io.py:12-18 parse). */
mcg_status mcg_write_constants_header(const mcg_params *p, const char *path);

/* ---------------- lifetime (memory.cuh:58-133) ---------------- */

/* allocate_device_memory() + allocate_mean_fields_device() equivalent.
 * All device memory is owned by the handle and zero-filled like memory.cuh:79-95. */
mcg_status mcg_create(const mcg_params *p, mcg_handle **out);
/* free_device_memory() + free_mean_fields_runtime() equivalent. */
mcg_status mcg_destroy(mcg_handle *h);
/* cudaStream_t passed as void*; NULL selects the handle's own stream. */
mcg_status mcg_set_stream(mcg_handle *h, void *stream);
mcg_status mcg_synchronize(mcg_handle *h);
mcg_status mcg_get_params(const mcg_handle *h, mcg_params *out);
/* Bytes of device memory held by the handle. */
mcg_status mcg_device_bytes(const mcg_handle *h, uint64_t *out);

/* ---------------- initial conditions ---------------- */

/* launch_jetDensity + launch_Injet (launch.cuh:19-29 -> kernels.cu:29-56,
 * jet/jetIn.cuh:13-62): red at rest everywhere, blue disc on the y=0 plane. */
mcg_status mcg_init_jet(mcg_handle *h);
/* launch_bubble (launch.cuh:13-17 -> kernels.cu:13-27, bubble/bubbleIn.cuh:10-39). */
mcg_status mcg_init_bubble(mcg_handle *h);

/* ---------------- state transfer (host buffers, reference layout) ---------------- */

/* Populations f(t) in reference layout fr[i*Ncells+id], fb[...] (float32, Q*Ncells each).
 * set: every interior node's 27 populations plus the y-ghost-plane values that
 *      interior nodes receive from the boundary (slots no kernel rewrites keep them).
 * get: interior nodes as the reference's d.fir/d.fib hold them; ghost nodes are 0. */
mcg_status mcg_set_populations(mcg_handle *h, const float *fr, const float *fb);
mcg_status mcg_get_populations(mcg_handle *h, float *fr, float *fb);
/* Macroscopic fields, Ncells each, as d.rhor..d.uz hold them (memory.cuh:11-25),
 * ghost nodes included.  set_fields defines the ghost-node densities the colour
 * gradient reads and the outlet state (any of the pointers may be NULL). */
mcg_status mcg_set_fields(mcg_handle *h, const float *rhor, const float *rhob,
                          const float *ux, const float *uy, const float *uz);
mcg_status mcg_get_fields(mcg_handle *h, float *rhor, float *rhob,
                          float *ux, float *uy, float *uz);
/* Non-equilibrium stress Pixx,Pixy,Piyy,Piyz,Pizz,Pixz (6*Ncells, that order). */
mcg_status mcg_get_stress(mcg_handle *h, float *pi6);

/* ---------------- the per-step launch sequence (main.cu:52-104) ---------------- */

/* launch_Macros (launch.cuh:31-37 -> kernels.cu:60-76, lbm.cuh:82-165). */
mcg_status mcg_macros(mcg_handle *h);
/* launch_accumulate_radial_moments (launch.cuh:75-90 -> kernels.cu:188-233). */
mcg_status mcg_accumulate_radial_moments(mcg_handle *h);
/* launch_collistream (launch.cuh:92-99 -> kernels.cu:78-94, lbm.cuh:184-293).
 * Advances the step counter. */
mcg_status mcg_collistream(mcg_handle *h);
/* launch_inlet_bc (launch.cuh:101-108 -> kernels.cu:98-114,
 * jet/boundary_conditions.cuh:17-85).  Uses the moments of the last mcg_macros. */
mcg_status mcg_inlet_bc(mcg_handle *h);
/* launch_neumann_bc (launch.cuh:110-118 -> kernels.cu:116-132,
 * jet/boundary_conditions.cuh:163-233). */
mcg_status mcg_neumann_bc(mcg_handle *h);

/* nsteps iterations of main.cu:52-82 (macros, radial statistics once
 * step >= NSTATS_START_STEP as update_radial_statistics_start does
 * (meanF/meanFieldsRT.cuh:173-190), collision, inlet, outlet) through the fused
 * B200 kernels.  Same results as the granular sequence above.  No host sync. */
mcg_status mcg_step(mcg_handle *h, int32_t nsteps);
/* Same, but times the nsteps on the handle's stream with CUDA events and
 * returns the elapsed milliseconds (synchronises). */
mcg_status mcg_step_timed(mcg_handle *h, int32_t nsteps, float *ms);
/* Same steps with a CUDA event between consecutive launches: ms_total is the
 * whole span, ms_kernels[0] the summed device time of the fused step kernel,
 * ms_kernels[1] that of the boundary launch, ms_kernels[2] is 0
 * (bench/roofline instrumentation; ms_kernels has room for 3). */
mcg_status mcg_step_profiled(mcg_handle *h, int32_t nsteps, float *ms_total, float *ms_kernels);
/* Current step counter (number of completed collisions). */
mcg_status mcg_get_step(const mcg_handle *h, int64_t *step);
/* Kernel launches issued by this handle since creation. */
mcg_status mcg_launch_count(const mcg_handle *h, uint64_t *count);
/* Launch shape of the fused step (no counterpart in the reference, whose
 * launch configuration is fixed): out[0..7] = rows per tile, planes per
 * z chunk, threads per row, y tiles, z chunks, shared memory bytes per CTA,
 * march (0: k_fused, block-synchronous; 1: k_fused_pipe, pipelined;
 * 2: k_fused_bulk, pipelined with each pulled row staged in shared memory by
 * bulk copies; chosen only when the environment sets MCG_FUSED_BULK=1, as it
 * measured slower), row length the kernel is compiled for (0: runtime
 * geometry). */
#define MCG_TILING_FIELDS 8
mcg_status mcg_get_tiling(const mcg_handle *h, int32_t *out);
/* k_fused_bulk waits for each staged row at most `tries` times (about 1 us
 * each; default 2^20, about a second).  When a wait runs out, the kernel
 * finishes its march on stale rows and flags it; the next mcg_synchronize,
 * mcg_step_timed or mcg_step_profiled returns MCG_ERR_TIMEOUT and the state
 * must be set again.  tries = 0 makes every wait run out at once (testing
 * the error path).  No counterpart in the reference. */
mcg_status mcg_set_stage_wait_limit(mcg_handle *h, int32_t tries);

/* ---------------- mean fields and radial statistics (meanF/) ---------------- */

/* Forces statistics on (1) or off (0) regardless of NSTATS_START_STEP;
 * -1 restores the automatic start. */
mcg_status mcg_set_radial_statistics(mcg_handle *h, int32_t mode);
/* Device->host copies of the radial sums (meanF/meanFieldsRT.cuh:305-329):
 * five float64 arrays and one uint64 array of NY*NR_BINS, r fastest.
 * Any pointer may be NULL. */
mcg_status mcg_get_radial(mcg_handle *h, double *sum_uy, double *sum_uy2,
                          double *sum_ur, double *sum_ur2, double *sum_uruy,
                          uint64_t *count);
/* Radial-statistics state (meanF/memoryMeanFields.cuh:39-45). */
mcg_status mcg_get_radial_state(const mcg_handle *h, int32_t *started,
                                uint32_t *start_step, uint32_t *samples);
/* launch_compute_total_tke + launch_update_tke_average (main.cu:73-90,
 * kernels.cu:136-166): sum of 0.5|u|^2 over interior nodes (float64 on the
 * device, returned as the reference's float32) and its running average. */
mcg_status mcg_compute_tke(mcg_handle *h, int32_t step, float *tke_total, float *tke_avg);
/* launch_update_uy_average (launch.cuh:63-73 -> kernels.cu:168-186) - defined
 * but never launched by the reference; here it feeds mean_profiles/uy_avg.bin. */
mcg_status mcg_update_uy_average(mcg_handle *h);
mcg_status mcg_get_uy_average(mcg_handle *h, float *uy_avg, uint32_t *samples);

/* ---------------- diagnostics ---------------- */

/* Float64 sums over interior nodes of the current populations f(t):
 * out[0]=sum fr, out[1]=sum fb, out[2..4]=sum (fr+fb) c.  */
mcg_status mcg_conservation_sums(mcg_handle *h, double out[5]);
/* Scans fields and populations; MCG_ERR_NONFINITE if any NaN/Inf. */
mcg_status mcg_check_finite(mcg_handle *h);

/* No counterpart in the reference.  The float64 sums of mcg_conservation_sums
 * for callers that cannot let the library allocate: callers that own all
 * device memory themselves and allow no cudaMalloc/cudaFree inside their time
 * loop (HBM nearly full, where an allocation can fail and a free would
 * synchronise the device).  fr, fb: the caller's device arrays of Q*Ncells
 * floats each, direction-major, f[i*Ncells + id] with
 * id = x + NX*(y + NY*z) (ghost shell included); out5: the caller's device
 * array of 5 doubles (sum fr, sum fb, momentum x,y,z over interior nodes);
 * stream as a cudaStream_t or NULL.  Asynchronous; allocates nothing.  Scratch
 * is one static device array of MCG_STATIC_SCRATCH_PLANES*5 doubles (160 KiB,
 * held by every GPU that loads the library until exit): NZ-2 >
 * MCG_STATIC_SCRATCH_PLANES is rejected with MCG_ERR_INVALID_ARG.  The first
 * call on a device (and the first after a device reset) looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that
 * call before any stream capture.  All calls share the array: calls whose
 * kernels overlap on the GPU race and must be serialised. */
#define MCG_STATIC_SCRATCH_PLANES 4096
mcg_status mcg_conservation_sums_static(const float *fr, const float *fb, int32_t NX, int32_t NY, int32_t NZ,
                                        double *out5, void *stream);

/* ---------------- inlet profile (no counterpart in the reference) ---------------- */

#define MCG_INLET_BESSEL_MAX 8
/* Radial inlet profile around the top-hat: in jet columns the inlet velocity
 * U of jet/boundary_conditions.cuh:62 becomes U m(r) with
 *   m(r) = 1 + sum_{k=1..n} c_k J0(alpha_k r / R),
 * alpha_k the k-th zero of J0, r the distance of the column from the jet axis
 * (as in the inlet mask, utilities/mathUtilities.cuh:14-21), R = jet_radius.
 * n = 0 restores the top-hat (the reference's profile); n <= MCG_INLET_BESSEL_MAX.
 * The seeded perturbation (inlet_noise) multiplies on top. */
mcg_status mcg_set_inlet_bessel(mcg_handle *h, const float *coeffs, int32_t n);
/* The per-column multipliers m (NX*NZ floats, x fastest; 1 everywhere for the top-hat). */
mcg_status mcg_get_inlet_profile(mcg_handle *h, float *profile);

/* ---------------- discrete adjoint (no counterpart in the reference) ---------------- */

/* Initial state with a velocity field: every interior node gets, per colour,
 * the third-order equilibrium feq_i(rho_c, u) of lbm.cuh:16-35 (the
 * reference's bubble and jet initial states are the u = 0 case,
 * bubble/bubbleIn.cuh:25-39).  Host arrays of Ncells floats; resets the step
 * counter like mcg_init_bubble. */
mcg_status mcg_init_equilibrium(mcg_handle *h, const float *rhor, const float *rhob,
                                const float *ux, const float *uy, const float *uz);

/* Discrete adjoint of nsteps steps of the periodic box (boundary
 * MCG_BOUNDARY_PERIODIC, float32 storage) from the handle's current state S_0,
 * for J = sum over interior nodes of (psi_T - psi_target)^2, where psi_T is the
 * colour field of the populations after nsteps steps (what mcg_get_populations
 * returns then).  Reverse sweep with binomial checkpointing in device memory:
 * `snapshots` states are held (S_0 in the handle's own buffer, snapshots-1 more
 * allocated for the call), recomputing forward segments as Griewank's
 * treeverse schedule prescribes, its innermost segments reversed from a tape
 * of moment records (mcg_set_adjoint_tape, mcg_adjoint_plan_taped).  psi_target: host, Ncells floats (reference
 * node order).  Outputs (any may be NULL): J; dJ/dsigma and dJ/dtau (tau =
 * taur = taub, nu = (tau - 1/2) cs^2); dJ_du0: host, 3*Ncells floats (ux, uy,
 * uz planes, ghost nodes 0) - the gradient with respect to the velocity u0 of
 * an initial state made by mcg_init_equilibrium; forward_steps: fused steps run
 * (recomputation included); ms: device time of the call.  The handle's state,
 * fields and step counter are left as they were. */
mcg_status mcg_adjoint_run(mcg_handle *h, const float *psi_target, int32_t nsteps, int32_t snapshots,
                           double *J, double *dJ_dsigma, double *dJ_dtau, float *dJ_du0,
                           int64_t *forward_steps, float *ms);
/* Discrete adjoint of nsteps steps of the jet (MCG_BOUNDARY_JET) from the
 * handle's current state, boundary conditions included: the
 * inlet (jet/boundary_conditions.cuh:17-85) with its radial profile
 * (mcg_set_inlet_bessel) and the convective outlet with its carried state
 * (:163-233).  J = sum over steps t in [t_begin, t_end] of (1/2) sum of uy^2
 * over interior nodes with y >= y_obs, uy of the fields step t computes (the
 * velocity of the populations it pulls).  dJ_dc[MCG_INLET_BESSEL_MAX]: the
 * gradient with respect to the profile coefficients c_k (at the current ones,
 * for all k including unset ones).  Memory: with segment <= 0 or >= nsteps the
 * sweep keeps a tape of every step's moment record and outlet state (about
 * 48 B per node and step) and runs nsteps forward steps; with 0 < segment <
 * nsteps it keeps a snapshot (populations and outlet state, 216 B per node)
 * every `segment` steps and the tape of one segment, and runs about
 * 2*nsteps forward steps.  When device memory allows more segment tapes
 * (mcg_set_jet_adjoint_tapes), the first forward pass also records the last
 * segments it runs through, and those are reversed without running them
 * again.  The forward states keep the handle's storage: with
 * MCG_STORAGE_F16 the sweep is the float32 adjoint of the step taken at the
 * float16-stored forward states (snapshots then take 108 B per node).  The
 * handle's state is left as it was. */
mcg_status mcg_adjoint_jet_run(mcg_handle *h, int32_t nsteps, int32_t t_begin, int32_t t_end, int32_t y_obs,
                               int32_t segment, double *J, double *dJ_dc, int64_t *forward_steps, float *ms);
/* No counterpart in the reference.  The jet adjoint of mcg_adjoint_jet_run
 * for a misfit of time-averaged profiles: over the window steps t_begin..t_end
 * the radial statistics give the mean profile U(y, r) (the accumulation of
 * kernels.cu:188-233, averaged as post/mean_profile_io.py:182-212 does), its
 * centreline uc(y) = U(y, 0) and half-width r_half(y)
 * (post/plot_profiles.py:53-91), and
 *   J = 1/2 sum_{y_lo <= y <= y_hi} ((uc - uc_target)/U_jet)^2
 *                                  + ((r_half - rhalf_target)/D)^2,
 * each term where both of its values are defined (a NaN target drops it).
 * uc_target, rhalf_target: [NY] (mcg_jet_profile_metrics of a target run).
 * The sweep first runs the window forward for the averages, then reverses as
 * mcg_adjoint_jet_run does (about nsteps more forward steps with segments). */
mcg_status mcg_adjoint_jet_profile_run(mcg_handle *h, int32_t nsteps, int32_t t_begin, int32_t t_end, int32_t y_lo,
                                       int32_t y_hi, const float *uc_target, const float *rhalf_target, int32_t segment,
                                       double *J, double *dJ_dc, int64_t *forward_steps, float *ms);
/* No counterpart in the reference (post/plot_profiles.py forms the same
 * quantities from the files).  Centreline velocity uc[NY] and half-width
 * r_half[NY] (NaN where undefined) of the handle's radial statistics so far. */
mcg_status mcg_jet_profile_metrics(mcg_handle *h, float *uc, float *r_half);
/* The treeverse schedule without running it (host only, no device needed):
 * fused steps a reverse sweep over nsteps steps with `snapshots` held states
 * runs, and the recomputation depth r (least r with C(s + r, s) >= nsteps + 1,
 * s = min(snapshots, nsteps + 1)). */
mcg_status mcg_adjoint_plan(int32_t nsteps, int32_t snapshots, int64_t *forward_steps, int32_t *sweeps);
/* The schedule mcg_adjoint_run runs with an adjoint tape of `tape` records
 * (mcg_set_adjoint_tape): the treeverse splits, with every segment of at
 * most tape + 1 ops reversed from its held first state by one taped advance
 * (tape forward steps recording the states' moments, 48 B per node each).
 * tape = 0 is mcg_adjoint_plan. */
mcg_status mcg_adjoint_plan_taped(int32_t nsteps, int32_t snapshots, int32_t tape, int64_t *forward_steps,
                                  int32_t *sweeps);
/* Records of the taped segments of mcg_adjoint_run (default 20; 0: plain
 * treeverse, every op forming its record with the moments kernel). */
mcg_status mcg_set_adjoint_tape(mcg_handle *h, int32_t records);
/* Segment tapes of mcg_adjoint_jet_run / mcg_adjoint_jet_profile_run (each
 * segment * ~48 B per node): 0 (default) as many as fit while 5 % of device
 * memory (at least 4 GiB) stays free, n > 0 at most n.  One is always kept. */
mcg_status mcg_set_jet_adjoint_tapes(mcg_handle *h, int32_t tapes);

/* ---------------- output files (io/save_data.cuh, meanF/meanFieldsRT.cuh) ---------------- */

/* initialize_mean_fields_runtime (meanF/meanFieldsRT.cuh:132-162): creates
 * <root>/JET_VTK/Re<Re>_We<We>/{mean_profiles,vti_data}, opens tke_*.bin and
 * writes case_info.txt. */
mcg_status mcg_output_open(mcg_handle *h, const char *root_dir);
/* The NOUTPUT block of main.cu:73-103 for `step`: tke sample (stdout line +
 * tke_*.bin), radial outputs when statistics run, VTI when write_vti_output. */
mcg_status mcg_output_step(mcg_handle *h, int32_t step);
/* The same output step without stopping the GPU (no counterpart in the
 * reference): the solver's stream copies the fields and radial sums to a
 * device staging slot and sums the kinetic energy; a second stream and a
 * worker thread download them and write the same files as mcg_output_step, in
 * step order, while stepping continues.  Two slots: a third call waits for the
 * oldest.  Synchronous output and tke calls flush first. */
mcg_status mcg_output_step_async(mcg_handle *h, int32_t step);
/* Waits for every pending asynchronous output; returns the first write error. */
mcg_status mcg_output_flush(mcg_handle *h);
/* write_radial_profile_outputs (meanF/meanFieldsRT.cuh:297-336). */
mcg_status mcg_write_radial_outputs(mcg_handle *h);
/* write_vti (io/save_data.cuh:137-200) of the current fields to `path`. */
mcg_status mcg_write_vti(mcg_handle *h, const char *path);
/* mean_profiles/uy_avg.bin (float32, Ncells) read by post/binConversionVti.py:22-28. */
mcg_status mcg_write_uy_average(mcg_handle *h);
/* Paths chosen by mcg_output_open (empty strings before it). */
mcg_status mcg_output_dirs(const mcg_handle *h, char *case_dir, char *mean_dir,
                           char *vti_dir, size_t cap);
mcg_status mcg_output_close(mcg_handle *h);

/* ---------------- errors / introspection ---------------- */

const char *mcg_last_error_string(void);
const char *mcg_status_string(mcg_status s);
int32_t mcg_abi_version(void);
/* Number of CUDA devices (0 without a GPU; never fails). */
int32_t mcg_device_count(void);

#ifdef __cplusplus
}
#endif

#endif /* MCG_H */
