// adjoint.cu - discrete adjoint of the periodic-box step (mcg_adjoint_run and
// mcg_adjoint_plan in include/mcg.h).
//
// The reverse sweep visits the states S_T, S_{T-1}, ..., S_0 of a T-step run.
// Op t (t = T: terminal condition of J; t < T: one adjoint step
// lambda_{t+1} -> lambda_t) needs S_t, so a sweep is n = T + 1 ops over a
// chain whose states can only be made going forward.  The schedule is
// Griewank's binomial checkpointing (treeverse): with s held states (the
// segment's first included) and r recomputation sweeps, beta(s, r) =
// C(s + r, s) ops can be reversed.  A segment of n ops is split at m: advance
// m steps into a free slot, reverse the right part n - m with s - 1 held
// states, then the left part m with s.  r is least with beta(s, r) >= n and
// m = max(n - beta(s - 1, r), beta(s, r - 2), 1), the lower end of the range
// of splits that reach the fewest forward steps, r n - beta(s + 1, r - 1).
// With s >= n every state is made once (T forward steps).
//
// Segments of at most K + 1 ops (K = the handle's adjoint tape, 20 records
// by default) are reversed from their held first state by one taped advance
// instead: K forward steps in which the fused step records each state's
// moments as it pulls them, then the ops from the tape (the last state's
// record by the moments kernel).  The treeverse splits above them are
// unchanged.  On the 96^3 bubble with T = 400 and 20 held states this takes
// 834 forward steps and 28 moments launches instead of 950 and 401.
//
// An op reads its state only through the state's moment record (11 moment
// planes and psi, 48 B per node).  With a slot for every state (snapshots >
// nsteps) the sweep keeps no populations at all: one forward pass in which the
// fused step records each state's moments as it pulls them (a tape of
// (T + 1) records), then T + 1 ops.  With fewer slots the slots hold
// population buffers (216 B per node) as restart points, forward steps write
// straight into the next slot (or ping-pong through two work buffers for longer
// segments) so no state is ever copied, and each op first forms its record
// with the moments kernel.  The run's records live in their own buffers: the
// handle's state is left untouched.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.hpp"
#include "lattice.cuh"

using mcg::cuda_fail;
using mcg::fail;

namespace {

// beta(s, r) = C(s + r, s) (0 for r < 0), saturated well above any step count
int64_t beta(int64_t s, int64_t r) {
    if (r < 0) return 0;
    const int64_t cap = int64_t(1) << 40;
    int64_t b = 1;
    for (int64_t k = 1; k <= r; ++k) {
        b = b * (s + k) / k;  // C(s+k, k) = C(s+k-1, k-1) * (s+k) / k, exact
        if (b > cap) return cap;
    }
    return b;
}

// least r with beta(s, r) >= n, s >= 1 held states
int least_sweeps(int64_t n, int64_t s) {
    int r = 0;
    while (beta(s, r) < n) ++r;
    return r;
}

// One action of the schedule.
struct Action {
    enum Kind { kAdvance, kAdjoint, kTaped } kind;
    int src;      // slot holding the first state (kAdvance, kTaped) / the op's state (kAdjoint, -1: last advance's result)
    int dst;      // kAdvance: destination slot, -1 for a work buffer
    int64_t t0;   // time of the source state / of the op
    int64_t n;    // steps (kAdvance), ops (kTaped: states t0 .. t0+n-1)
};

void plan(std::vector<Action> &out, int64_t t0, int64_t n, int slot, int free_slots, int64_t tape) {
    if (n <= 0) return;
    if (n == 1) {
        out.push_back({Action::kAdjoint, slot, -1, t0, 0});
        return;
    }
    if (n <= tape + 1) {
        out.push_back({Action::kTaped, slot, -1, t0, n});
        return;
    }
    if (free_slots == 0) {
        for (int64_t k = n - 1; k >= 1; --k) {
            out.push_back({Action::kAdvance, slot, -1, t0, k});
            out.push_back({Action::kAdjoint, -1, -1, t0 + k, 0});
        }
        out.push_back({Action::kAdjoint, slot, -1, t0, 0});
        return;
    }
    const int64_t held = free_slots + 1;
    const int r = least_sweeps(n, held);
    int64_t m = std::max<int64_t>(std::max<int64_t>(n - beta(held - 1, r), beta(held, r - 2)), 1);
    if (m > n - 1) m = n - 1;
    out.push_back({Action::kAdvance, slot, slot + 1, t0, m});
    plan(out, t0 + m, n - m, slot + 1, free_slots - 1, tape);
    plan(out, t0, m, slot, free_slots, tape);
}

int64_t forward_steps_of(const std::vector<Action> &acts) {
    int64_t f = 0;
    for (const Action &a : acts) {
        if (a.kind == Action::kAdvance) f += a.n;
        if (a.kind == Action::kTaped) f += a.n - 1;
    }
    return f;
}

#define ADJ_CUDA(call, what)                                 \
    do {                                                     \
        cudaError_t e__ = (call);                            \
        if (e__ != cudaSuccess) return cuda_fail(e__, what); \
    } while (0)

#define ADJ_LAUNCH(h, call, what)                            \
    do {                                                     \
        cudaError_t e__ = (call);                            \
        if (e__ != cudaSuccess) return cuda_fail(e__, what); \
        ++(h)->launches;                                     \
    } while (0)

struct DeviceBuffers {
    cudaStream_t stream;  // the run's stream: buffers are cleared in its order
    std::vector<void *> ptrs;
    explicit DeviceBuffers(cudaStream_t st) : stream(st) {}
    ~DeviceBuffers() {
        if (!ptrs.empty()) cudaStreamSynchronize(stream);
        for (void *p : ptrs) cudaFree(p);
    }
    cudaError_t alloc(void **p, size_t bytes) {
        *p = nullptr;
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return e;
        ptrs.push_back(*p);
        return cudaMemsetAsync(*p, 0, bytes, stream);
    }
};

struct Run {
    mcg_handle *h = nullptr;
    mcg::DeviceState base{};   // the handle's state with the run's own moment / psi planes
    float *rec = nullptr;      // moment record of the op's state (checkpoint mode)
    std::vector<void *> slots; // slots[0] = S_0 (the handle's buffer)
    void *work[2] = {nullptr, nullptr};
    float *lam[2] = {nullptr, nullptr};
    int lc = 0;                // lam[lc]: adjoint of the latest state reached
    float *lmom = nullptr, *lf = nullptr;
    const float *target = nullptr;
    double *acc = nullptr;     // [0] J, [1] dJ/domega, [2] dJ/d(A/2)
    int64_t step0 = 0, T = 0;

    mcg::DeviceState with(void *from, void *to) const {
        mcg::DeviceState d = base;
        d.pops[0] = from;
        d.pops[1] = to;
        return d;
    }

    // S_{t0+n} from S_{t0} (in `src`) into `dst`, or into a work buffer when dst
    // is null; returns the buffer holding the result.
    mcg_status advance(void *src, void *dst, int64_t t0, int64_t n, void **result) {
        void *a = src;
        for (int64_t k = 0; k < n; ++k) {
            void *b = (k == n - 1 && dst) ? dst : work[k & 1];
            ADJ_LAUNCH(h, mcg::launch_fused(with(a, b), h->tiling, 0, step0 + t0 + k, false, h->stream),
                       "adjoint: forward step");
            a = b;
        }
        *result = a;
        return MCG_OK;
    }

    // op t with the moment record M of S_t
    const float *last_record = nullptr;  // the record the latest op read (op 0's, after a sweep)
    mcg_status op_record(const float *M, int64_t t) {
        last_record = M;
        if (t == T) {
            ADJ_LAUNCH(h, mcg::launch_adj_terminal(base, M, target, lam[lc], acc, h->stream), "adjoint: terminal");
        } else {
            ADJ_LAUNCH(h, mcg::launch_adj_step(base, M, lam[lc], lmom, lf, lam[lc ^ 1], acc + 1, h->stream),
                       "adjoint: step");
            h->launches += 1;  // two kernels
            lc ^= 1;
        }
        return MCG_OK;
    }

    // op t on the state held in `state` (its record formed first)
    mcg_status op(void *state, int64_t t) {
        ADJ_LAUNCH(h, mcg::launch_moments(with(state, nullptr), 0, step0 + t, false, h->stream), "adjoint: moments");
        return op_record(rec, t);
    }

    // Tape mode: one forward pass recording every state's moments into
    // tape[t] (t < T by the fused steps, T by the moments kernel), then the ops.
    mcg_status run_tape(float *tape, size_t record_floats) {
        void *a = slots[0];
        for (int64_t t = 0; t < T; ++t) {
            mcg::DeviceState d = with(a, work[t & 1]);
            d.tape = tape + size_t(t) * record_floats;
            ADJ_LAUNCH(h, mcg::launch_fused(d, h->tiling, 0, step0 + t, false, h->stream), "adjoint: forward step");
            a = work[t & 1];
        }
        {
            mcg::DeviceState d = with(a, nullptr);
            float *M = tape + size_t(T) * record_floats;
            d.mom = M;
            d.psi[0] = d.psi[1] = M + size_t(mcg::kTapePsi) * base.g.N;
            ADJ_LAUNCH(h, mcg::launch_moments(d, 0, step0 + T, false, h->stream), "adjoint: moments");
        }
        for (int64_t t = T; t >= 0; --t)
            if (mcg_status s = op_record(tape + size_t(t) * record_floats, t)) return s;
        return MCG_OK;
    }

    // States t0 .. t0+n-1 from the held state `src` (time t0): n-1 forward steps
    // that record the moments of S_t0 .. S_{t0+n-2} into `seg_tape`, then the
    // ops t0+n-1 (its record by the moments kernel) down to t0.
    float *seg_tape = nullptr;
    mcg_status taped(void *src, int64_t t0, int64_t n, size_t record_floats) {
        void *a = src;
        for (int64_t k = 0; k + 1 < n; ++k) {
            mcg::DeviceState d = with(a, work[k & 1]);
            d.tape = seg_tape + size_t(k) * record_floats;
            ADJ_LAUNCH(h, mcg::launch_fused(d, h->tiling, 0, step0 + t0 + k, false, h->stream), "adjoint: forward step");
            a = work[k & 1];
        }
        if (mcg_status s = op(a, t0 + n - 1)) return s;
        for (int64_t t = t0 + n - 2; t >= t0; --t)
            if (mcg_status s = op_record(seg_tape + size_t(t - t0) * record_floats, t)) return s;
        return MCG_OK;
    }

    mcg_status execute(const std::vector<Action> &acts, size_t record_floats) {
        void *last = nullptr;
        for (const Action &a : acts) {
            if (a.kind == Action::kTaped) {
                if (mcg_status s = taped(slots[size_t(a.src)], a.t0, a.n, record_floats)) return s;
                continue;
            }
            if (a.kind == Action::kAdvance) {
                void *dst = a.dst >= 0 ? slots[size_t(a.dst)] : nullptr;
                if (mcg_status s = advance(slots[size_t(a.src)], dst, a.t0, a.n, &last)) return s;
            } else {
                void *state = a.src >= 0 ? slots[size_t(a.src)] : last;
                if (mcg_status s = op(state, a.t0)) return s;
            }
        }
        return MCG_OK;
    }
};

}  // namespace

extern "C" {

mcg_status mcg_adjoint_plan_taped(int32_t nsteps, int32_t snapshots, int32_t tape, int64_t *forward_steps,
                                  int32_t *sweeps) {
    return mcg::guarded([&]() -> mcg_status {
        if (nsteps < 1) return fail(MCG_ERR_INVALID_ARG, "nsteps must be >= 1");
        if (snapshots < 1) return fail(MCG_ERR_INVALID_ARG, "snapshots must be >= 1");
        if (tape < 0) return fail(MCG_ERR_INVALID_ARG, "tape must be >= 0");
        const int free_slots = std::min<int64_t>(snapshots - 1, nsteps);
        std::vector<Action> acts;
        if (snapshots > nsteps)
            plan(acts, 0, int64_t(nsteps) + 1, 0, free_slots, 0);
        else
            plan(acts, 0, int64_t(nsteps) + 1, 0, free_slots, std::min<int64_t>(tape, nsteps));
        if (forward_steps) *forward_steps = forward_steps_of(acts);
        if (sweeps) *sweeps = least_sweeps(int64_t(nsteps) + 1, free_slots + 1);
        return MCG_OK;
    });
}

mcg_status mcg_adjoint_plan(int32_t nsteps, int32_t snapshots, int64_t *forward_steps, int32_t *sweeps) {
    return mcg_adjoint_plan_taped(nsteps, snapshots, 0, forward_steps, sweeps);
}

mcg_status mcg_set_jet_adjoint_tapes(mcg_handle *h, int32_t tapes) {
    return mcg::guarded([&]() -> mcg_status {
        if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
        if (tapes < 0) return fail(MCG_ERR_INVALID_ARG, "tapes must be >= 0");
        h->jet_adjoint_tapes = tapes;
        return MCG_OK;
    });
}

mcg_status mcg_set_adjoint_tape(mcg_handle *h, int32_t records) {
    return mcg::guarded([&]() -> mcg_status {
        if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
        if (records < 0) return fail(MCG_ERR_INVALID_ARG, "records must be >= 0");
        h->adjoint_tape = records;
        return MCG_OK;
    });
}

mcg_status mcg_adjoint_run(mcg_handle *h, const float *psi_target, int32_t nsteps, int32_t snapshots, double *J,
                           double *dJ_dsigma, double *dJ_dtau, float *dJ_du0, int64_t *forward_steps, float *ms) {
    return mcg::guarded([&]() -> mcg_status {
        if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
        if (!psi_target) return fail(MCG_ERR_INVALID_ARG, "psi_target is null");
        if (nsteps < 1) return fail(MCG_ERR_INVALID_ARG, "nsteps must be >= 1");
        if (snapshots < 1) return fail(MCG_ERR_INVALID_ARG, "snapshots must be >= 1");
        if (h->p.boundary != MCG_BOUNDARY_PERIODIC || h->p.storage != MCG_STORAGE_F32)
            return fail(MCG_ERR_UNSUPPORTED, "the adjoint covers the periodic box with float32 storage");
        if (h->p.sponge_K != 0.0f) return fail(MCG_ERR_UNSUPPORTED, "the adjoint needs a uniform relaxation rate");
        const mcg::Geometry &g = h->s.g;
        const size_t N = g.N;
        const size_t pop_bytes = size_t(2 * mcg::kQ) * N * sizeof(float);  // float32 populations or lambda
        const size_t record_floats = size_t(mcg::kTapePlanes) * N;
        const bool tape_mode = snapshots > nsteps;
        const int free_slots = tape_mode ? 0 : snapshots - 1;
        const int64_t seg = std::min<int64_t>(h->adjoint_tape, nsteps);  // records of a taped segment

        std::vector<Action> acts;
        if (!tape_mode) plan(acts, 0, int64_t(nsteps) + 1, 0, free_slots, seg);
        bool any_taped = false;
        for (const Action &a : acts) any_taped = any_taped || (a.kind == Action::kTaped && a.n > 1);

        DeviceBuffers buf(h->stream);
        Run run;
        run.h = h;
        run.base = h->s;
        run.step0 = h->step;
        run.T = nsteps;
        run.slots.assign(size_t(free_slots) + 1, nullptr);
        run.slots[0] = h->s.pops[h->cur];
        void *p = nullptr;
        for (int k = 1; k <= free_slots; ++k) {
            ADJ_CUDA(buf.alloc(&p, pop_bytes), "adjoint snapshot slots");
            run.slots[size_t(k)] = p;
        }
        for (int k = 0; k < 2; ++k) {
            ADJ_CUDA(buf.alloc(&p, pop_bytes), "adjoint work buffers");
            run.work[k] = p;
            ADJ_CUDA(buf.alloc(&p, pop_bytes), "adjoint lambda buffers");
            run.lam[k] = static_cast<float *>(p);
        }
        float *tape = nullptr;
        if (tape_mode) {
            ADJ_CUDA(buf.alloc(&p, (size_t(nsteps) + 1) * record_floats * sizeof(float)), "adjoint moment tape");
            tape = static_cast<float *>(p);
        } else {
            if (any_taped) {
                ADJ_CUDA(buf.alloc(&p, size_t(seg) * record_floats * sizeof(float)), "adjoint segment tape");
                run.seg_tape = static_cast<float *>(p);
            }
            ADJ_CUDA(buf.alloc(&p, record_floats * sizeof(float)), "adjoint moment record");
            run.rec = static_cast<float *>(p);
            // the moments kernel writes the record: 11 planes, then psi (ghost mirrors unused)
            run.base.mom = run.rec;
            run.base.psi[0] = run.base.psi[1] = run.rec + size_t(mcg::kTapePsi) * N;
        }
        ADJ_CUDA(buf.alloc(&p, size_t(mcg::kMomCount) * N * sizeof(float)), "adjoint moment adjoints");
        run.lmom = static_cast<float *>(p);
        ADJ_CUDA(buf.alloc(&p, 3 * N * sizeof(float)), "adjoint gradient adjoints");
        run.lf = static_cast<float *>(p);
        ADJ_CUDA(buf.alloc(&p, 3 * N * sizeof(float)), "adjoint du0");
        float *du0 = static_cast<float *>(p);
        ADJ_CUDA(buf.alloc(&p, N * sizeof(float)), "adjoint target");
        run.target = static_cast<const float *>(p);
        ADJ_CUDA(cudaMemcpyAsync(p, psi_target, N * sizeof(float), cudaMemcpyHostToDevice, h->stream), "upload target");
        ADJ_CUDA(buf.alloc(&p, 4 * sizeof(double)), "adjoint accumulators");
        run.acc = static_cast<double *>(p);

        ADJ_CUDA(cudaEventRecord(h->ev0, h->stream), "event");
        if (tape_mode) {
            if (mcg_status s = run.run_tape(tape, record_floats)) return s;
        } else {
            if (mcg_status s = run.execute(acts, record_floats)) return s;
        }
        // op 0 was the last: its record is S_0's (the moments kernel's, or a
        // taped segment's first)
        const float *M0 = tape_mode ? tape : run.last_record;
        ADJ_LAUNCH(h, mcg::launch_adj_initial(run.base, M0, run.lam[run.lc], du0, h->stream), "adjoint: initial state");
        ADJ_CUDA(cudaEventRecord(h->ev1, h->stream), "event");
        double acc[3] = {0, 0, 0};
        ADJ_CUDA(cudaMemcpyAsync(acc, run.acc, sizeof(acc), cudaMemcpyDeviceToHost, h->stream), "download J");
        if (dJ_du0)
            ADJ_CUDA(cudaMemcpyAsync(dJ_du0, du0, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
                     "download dJ/du0");
        ADJ_CUDA(cudaStreamSynchronize(h->stream), "adjoint run");
        float t_ms = 0.f;
        ADJ_CUDA(cudaEventElapsedTime(&t_ms, h->ev0, h->ev1), "event time");

        // omega = 1/(1/2 + nu/cs^2) = 1/tau; A/2 = sigma / (8 cs^4 taub)
        const double omega = h->s.ph.omega, Ah = h->s.ph.Ah;
        const double tau = h->p.taub;
        const double dAh_dsigma = 1.0 / (8.0 * double(mcg::kCs4) * tau);
        if (J) *J = acc[0];
        if (dJ_dsigma) *dJ_dsigma = acc[2] * dAh_dsigma;
        if (dJ_dtau) *dJ_dtau = acc[1] * (-omega * omega) + acc[2] * (-Ah / tau);
        if (forward_steps) *forward_steps = tape_mode ? int64_t(nsteps) : forward_steps_of(acts);
        if (ms) *ms = t_ms;
        return MCG_OK;
    });
}


namespace {
// J0(alpha_k r / R) of every column, k < kInletBesselMax (the inlet profile's basis).
std::vector<float> bessel_basis(const mcg_params &p) {
    const int NX = p.NX, NZ = p.NZ, nb = mcg::kInletBesselMax;
    std::vector<float> b(size_t(nb) * NX * NZ);
    for (int k = 0; k < nb; ++k) {
        double a = (double(k + 1) - 0.25) * M_PI;  // k-th zero of J0: Newton from McMahon's estimate
        for (int it = 0; it < 60; ++it) {
            const double dx = std::cyl_bessel_j(0.0, a) / -std::cyl_bessel_j(1.0, a);
            a -= dx;
            if (std::fabs(dx) < 1e-15 * a) break;
        }
        for (int z = 0; z < NZ; ++z)
            for (int x = 0; x < NX; ++x) {
                const double dx = double(float(x) - p.jet_x0), dz = double(float(z) - p.jet_z0);
                const double r = std::sqrt(dx * dx + dz * dz);
                b[(size_t(k) * NZ + z) * NX + x] = float(std::cyl_bessel_j(0.0, a * r / double(p.jet_radius)));
            }
    }
    return b;
}
}  // namespace

namespace {
// The objective of a jet adjoint run.  kind 0: J = sum over window steps of
// (1/2) sum uy^2 over interior nodes with y >= y_obs.  kind 1: the misfit of
// the window's time-averaged centreline velocity and half-width (see
// mcg_adjoint_jet_profile_run) against targets for y in [y_lo, y_hi].
struct JetObjective {
    int kind = 0;
    int y_obs = 0;
    int y_lo = 0, y_hi = -1;
    const float *uc_target = nullptr, *rh_target = nullptr;
};

mcg_status jet_adjoint(mcg_handle *h, int32_t nsteps, int32_t t_begin, int32_t t_end, int32_t segment,
                       const JetObjective &objective, double *J, double *dJ_dc, int64_t *forward_steps, float *ms) {
    if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
    if (nsteps < 1) return fail(MCG_ERR_INVALID_ARG, "nsteps must be >= 1");
    if (t_begin < 0 || t_end < t_begin || t_end >= nsteps)
        return fail(MCG_ERR_INVALID_ARG, "need 0 <= t_begin <= t_end < nsteps");
    if (h->p.boundary != MCG_BOUNDARY_JET) return fail(MCG_ERR_UNSUPPORTED, "the jet adjoint covers the jet boundary");
    if (h->p.sponge_K != 0.0f) return fail(MCG_ERR_UNSUPPORTED, "the adjoint needs a uniform relaxation rate");
    if (mcg_status st = mcg::async_flush(h)) return st;
    const mcg::Geometry &g = h->s.g;
    const size_t N = g.N, NP = size_t(g.NX) * g.NZ;
    const size_t NRB = size_t(g.NX / 2), M = size_t(g.NY) * NRB;
    // the forward states keep the handle's storage (float16 or float32); the
    // reverse sweep reads them only through their float32 moment records, and
    // its lambda arrays are float32 pairs
    const size_t state_bytes = g.storage == MCG_STORAGE_F16 ? size_t(mcg::kQ) * N * 4 : size_t(2 * mcg::kQ) * N * 4;
    const size_t lam_bytes = size_t(2 * mcg::kQ) * N * sizeof(float);
    const size_t rec_floats = size_t(mcg::kTapePlanes) * N + 5 * NP;  // moments, psi with ghosts, outlet state
    const int nb = mcg::kInletBesselMax;
    const bool profile = objective.kind == 1;

    DeviceBuffers buf(h->stream);
    void *p = nullptr;
    mcg::DeviceState run = h->s;
    void *work[2];
    for (int k = 0; k < 2; ++k) {
        ADJ_CUDA(buf.alloc(&p, state_bytes), "jet adjoint work buffers");
        work[k] = p;
    }
    // both buffers: slots no kernel rewrites carry their initial values in both
    ADJ_CUDA(cudaMemcpyAsync(work[0], h->s.pops[h->cur], state_bytes, cudaMemcpyDeviceToDevice, h->stream),
             "copy state");
    ADJ_CUDA(cudaMemcpyAsync(work[1], h->s.pops[h->cur ^ 1], state_bytes, cudaMemcpyDeviceToDevice, h->stream),
             "copy state");
    ADJ_CUDA(buf.alloc(&p, size_t(mcg::kMomCount) * N * sizeof(float)), "jet adjoint moment planes");
    run.mom = static_cast<float *>(p);
    ADJ_CUDA(cudaMemcpyAsync(run.mom, h->s.mom, size_t(mcg::kMomCount) * N * sizeof(float), cudaMemcpyDeviceToDevice,
                             h->stream),
             "copy moments");
    for (int k = 0; k < 2; ++k) {
        ADJ_CUDA(buf.alloc(&p, N * sizeof(float)), "jet adjoint psi planes");
        run.psi[k] = static_cast<float *>(p);
        ADJ_CUDA(cudaMemcpyAsync(run.psi[k], h->s.psi[k], N * sizeof(float), cudaMemcpyDeviceToDevice, h->stream),
                 "copy psi");
    }
    ADJ_CUDA(buf.alloc(&p, size_t(2) * g.NZ * mcg::kMomCount * g.NX * sizeof(float)), "jet adjoint bmom");
    run.bmom = static_cast<float *>(p);
    // the run's own radial sums (the profile objective's time averages)
    ADJ_CUDA(buf.alloc(&p, 5 * M * sizeof(double)), "jet adjoint radial sums");
    run.radial = static_cast<double *>(p);
    // segments of L steps: a snapshot (populations + outlet state) at the
    // start of each, and a tape of one segment's records
    const int64_t L = (segment <= 0 || segment >= nsteps) ? nsteps : segment;
    const int64_t nseg = (nsteps + L - 1) / L;
    std::vector<void *> snap(size_t(nseg), nullptr);
    std::vector<float *> snapB(size_t(nseg), nullptr);
    for (int64_t j = 0; j < nseg; ++j) {
        ADJ_CUDA(buf.alloc(&p, state_bytes), "jet adjoint snapshots");
        snap[size_t(j)] = p;
        ADJ_CUDA(buf.alloc(&p, 5 * NP * sizeof(float)), "jet adjoint snapshots");
        snapB[size_t(j)] = static_cast<float *>(p);
    }
    float *lam[2];
    for (int k = 0; k < 2; ++k) {
        ADJ_CUDA(buf.alloc(&p, lam_bytes), "jet adjoint lambda buffers");
        lam[k] = static_cast<float *>(p);
    }
    ADJ_CUDA(buf.alloc(&p, size_t(mcg::kMomCount) * N * sizeof(float)), "jet adjoint moment adjoints");
    float *lmom = static_cast<float *>(p);
    ADJ_CUDA(buf.alloc(&p, 3 * N * sizeof(float)), "jet adjoint gradient adjoints");
    float *lf = static_cast<float *>(p);
    float *LB[2];
    for (int k = 0; k < 2; ++k) {
        ADJ_CUDA(buf.alloc(&p, 5 * NP * sizeof(float)), "jet adjoint outlet adjoints");
        LB[k] = static_cast<float *>(p);
    }
    const std::vector<float> basis = bessel_basis(h->p);
    ADJ_CUDA(buf.alloc(&p, basis.size() * sizeof(float)), "jet adjoint profile basis");
    float *dbasis = static_cast<float *>(p);
    ADJ_CUDA(cudaMemcpyAsync(dbasis, basis.data(), basis.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream),
             "upload profile basis");
    ADJ_CUDA(buf.alloc(&p, (2 + size_t(nb)) * sizeof(double)), "jet adjoint accumulators");
    double *acc = static_cast<double *>(p);  // [0] J, [1] (unused), [2..] dJ/dc_k
    double *dacc_w = nullptr;
    ADJ_CUDA(buf.alloc(&p, 2 * sizeof(double)), "jet adjoint parameter partials");
    dacc_w = static_cast<double *>(p);
    float *table = nullptr;
    if (profile) {
        ADJ_CUDA(buf.alloc(&p, M * sizeof(float)), "jet adjoint profile source");
        table = static_cast<float *>(p);
    }
    // segment tapes, allocated last: tapes[0] serves every segment pass 2
    // re-runs; with more, pass 1 also records the last segments it runs
    // through into tapes[1..] (segment nseg-1-k into tapes[k]), and pass 2
    // reverses those without re-running them.  As many as fit with a margin
    // of device memory left free (h->jet_adjoint_tapes == 0), or that many.
    const size_t tape_bytes = size_t(L) * rec_floats * sizeof(float);
    int64_t ntapes = 1;
    {
        size_t free_b = 0, total_b = 0;
        ADJ_CUDA(cudaMemGetInfo(&free_b, &total_b), "device memory");
        const size_t margin = std::max<size_t>(size_t(4) << 30, total_b / 20);
        const int64_t fit = free_b > margin ? int64_t((free_b - margin) / tape_bytes) : 0;
        const int64_t want = h->jet_adjoint_tapes > 0 ? int64_t(h->jet_adjoint_tapes) : nseg;
        ntapes = std::max<int64_t>(1, std::min<int64_t>({want, nseg, fit}));
    }
    std::vector<float *> tapes(size_t(ntapes), nullptr);
    for (int64_t k = 0; k < ntapes; ++k) {
        ADJ_CUDA(buf.alloc(&p, tape_bytes), "jet adjoint moment tape");
        tapes[size_t(k)] = static_cast<float *>(p);
    }

    const int64_t step0 = h->step;
    ADJ_CUDA(cudaEventRecord(h->ev0, h->stream), "event");
    int64_t fwd = 0;
    // one forward step t of the run's state (work[t & 1] -> work[(t+1) & 1]),
    // recording into `rec` when given: its psi with the ghost values it reads,
    // the outlet state before its boundary, and (the fused step) its moments;
    // `stats` adds the step's radial statistics to the run's sums
    auto forward = [&](int64_t t, float *rec, bool stats) -> mcg_status {
        mcg::DeviceState d = run;
        d.pops[0] = work[t & 1];
        d.pops[1] = work[(t + 1) & 1];
        if (rec) {
            ADJ_CUDA(cudaMemcpyAsync(rec + size_t(mcg::kTapePsi) * N, run.psi[(step0 + t) & 1], N * sizeof(float),
                                     cudaMemcpyDeviceToDevice, h->stream),
                     "record psi");
            ADJ_LAUNCH(h, mcg::launch_copy_outlet_state(d, rec + size_t(mcg::kTapePlanes) * N, h->stream),
                       "jet adjoint: record outlet state");
            d.tape = rec;
        }
        ADJ_LAUNCH(h, mcg::launch_fused(d, h->tiling, 0, step0 + t, stats, h->stream), "jet adjoint: forward step");
        d.tape = nullptr;
        if (!h->tiling.boundary)
            ADJ_LAUNCH(h, mcg::launch_boundary(d, 1, step0 + t, -1, true, h->stream), "jet adjoint: boundary");
        ++fwd;
        return MCG_OK;
    };
    auto save = [&](int64_t j, int64_t t) -> mcg_status {
        ADJ_CUDA(cudaMemcpyAsync(snap[size_t(j)], work[t & 1], state_bytes, cudaMemcpyDeviceToDevice, h->stream),
                 "save snapshot");
        ADJ_LAUNCH(h, mcg::launch_copy_outlet_state(run, snapB[size_t(j)], h->stream), "jet adjoint: save outlet");
        return MCG_OK;
    };
    // ---- pass 1: snapshots at every segment start; the profile objective runs
    // at least through the window here, accumulating its radial statistics
    if (mcg_status st = save(0, 0)) return st;
    const int64_t pass1 = profile ? std::max<int64_t>(int64_t(t_end) + 1, (nseg - 1) * L) : (nseg - 1) * L;
    auto pass1_tape = [&](int64_t j) -> float * {  // segment j's pass-1 tape, or none
        const int64_t k = nseg - 1 - j;
        return k >= 0 && k < ntapes ? tapes[size_t(k)] : nullptr;
    };
    for (int64_t t = 0; t < pass1; ++t) {
        float *seg = pass1_tape(t / L);
        float *rec = seg ? seg + size_t(t - (t / L) * L) * rec_floats : nullptr;
        if (mcg_status st = forward(t, rec, profile && t >= t_begin && t <= t_end)) return st;
        if ((t + 1) % L == 0 && (t + 1) / L < nseg)
            if (mcg_status st = save((t + 1) / L, t + 1)) return st;
    }
    double J_host = 0.0;
    if (profile) {
        // J and its source dJ/duy per (y, radial bin) from the window's averages
        std::vector<double> sum_uy(M);
        ADJ_CUDA(cudaMemcpyAsync(sum_uy.data(), run.radial, M * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                 "download radial sums");
        ADJ_CUDA(cudaStreamSynchronize(h->stream), "jet adjoint forward pass");
        const uint32_t samples = uint32_t(t_end - t_begin + 1);
        std::vector<float> src(M, 0.0f);
        J_host = mcg::profile_objective(h, sum_uy.data(), samples, objective.y_lo, objective.y_hi, objective.uc_target,
                                        objective.rh_target, src.data());
        ADJ_CUDA(cudaMemcpyAsync(table, src.data(), M * sizeof(float), cudaMemcpyHostToDevice, h->stream),
                 "upload profile source");
        ADJ_CUDA(cudaStreamSynchronize(h->stream), "upload profile source");
    }
    // ---- pass 2: per segment from the last, restore, re-run recording, reverse
    int lc = 0, lb = 0;
    for (int64_t j = nseg - 1; j >= 0; --j) {
        const int64_t s0 = j * L, s1 = std::min<int64_t>(nsteps, s0 + L);
        float *tape = pass1_tape(j);
        if (!tape || pass1 < s1) {  // not recorded whole in pass 1: restore and re-run into tapes[0]
            tape = tapes[0];
            ADJ_CUDA(cudaMemcpyAsync(work[s0 & 1], snap[size_t(j)], state_bytes, cudaMemcpyDeviceToDevice,
                                     h->stream),
                     "restore snapshot");
            ADJ_LAUNCH(h,
                       mcg::launch_restore_outlet_state(run, snapB[size_t(j)], run.psi[(step0 + s0) & 1], h->stream),
                       "jet adjoint: restore outlet");
            for (int64_t t = s0; t < s1; ++t)
                if (mcg_status st = forward(t, tape + size_t(t - s0) * rec_floats, false)) return st;
        }
        for (int64_t t = s1 - 1; t >= s0; --t) {
            const float *rec = tape + size_t(t - s0) * rec_floats;
            const bool in_window = t >= t_begin && t <= t_end;
            mcg::AdjObjective obj{in_window && !profile ? 1.0f : 0.0f, objective.y_obs, profile ? nullptr : acc};
            if (profile && in_window) obj.table = table;
            ADJ_LAUNCH(h, mcg::launch_adj_collide(run, rec, lam[lc], lmom, lf, dacc_w, obj, h->stream),
                       "jet adjoint: collision");
            ADJ_LAUNCH(h,
                       mcg::launch_adj_boundary(run, step0 + t, rec, rec + size_t(mcg::kTapePlanes) * N, lam[lc], lf,
                                                lmom, LB[lb], LB[lb ^ 1], dbasis, nb, acc + 2, h->stream),
                       "jet adjoint: boundary");
            ADJ_LAUNCH(h, mcg::launch_adj_moments(run, rec, lmom, lf, lam[lc ^ 1], h->stream), "jet adjoint: moments");
            lc ^= 1;
            lb ^= 1;
        }
    }
    ADJ_CUDA(cudaEventRecord(h->ev1, h->stream), "event");
    std::vector<double> out(2 + size_t(nb));
    ADJ_CUDA(cudaMemcpyAsync(out.data(), acc, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
             "download J");
    ADJ_CUDA(cudaStreamSynchronize(h->stream), "jet adjoint run");
    float t_ms = 0.f;
    ADJ_CUDA(cudaEventElapsedTime(&t_ms, h->ev0, h->ev1), "event time");
    if (J) *J = profile ? J_host : out[0];
    if (dJ_dc)
        for (int k = 0; k < nb; ++k) dJ_dc[k] = out[2 + size_t(k)];
    if (forward_steps) *forward_steps = fwd;
    if (ms) *ms = t_ms;
    return MCG_OK;
}
}  // namespace

mcg_status mcg_adjoint_jet_run(mcg_handle *h, int32_t nsteps, int32_t t_begin, int32_t t_end, int32_t y_obs,
                               int32_t segment, double *J, double *dJ_dc, int64_t *forward_steps, float *ms) {
    return mcg::guarded([&]() -> mcg_status {
        JetObjective obj;
        obj.kind = 0;
        obj.y_obs = y_obs;
        return jet_adjoint(h, nsteps, t_begin, t_end, segment, obj, J, dJ_dc, forward_steps, ms);
    });
}

mcg_status mcg_adjoint_jet_profile_run(mcg_handle *h, int32_t nsteps, int32_t t_begin, int32_t t_end, int32_t y_lo,
                                       int32_t y_hi, const float *uc_target, const float *rhalf_target, int32_t segment,
                                       double *J, double *dJ_dc, int64_t *forward_steps, float *ms) {
    return mcg::guarded([&]() -> mcg_status {
        if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
        if (!uc_target || !rhalf_target) return fail(MCG_ERR_INVALID_ARG, "target profiles must not be null");
        if (y_lo < 1 || y_hi > h->p.NY - 2 || y_hi < y_lo)
            return fail(MCG_ERR_INVALID_ARG, "need 1 <= y_lo <= y_hi <= NY-2");
        JetObjective obj;
        obj.kind = 1;
        obj.y_lo = y_lo;
        obj.y_hi = y_hi;
        obj.uc_target = uc_target;
        obj.rh_target = rhalf_target;
        return jet_adjoint(h, nsteps, t_begin, t_end, segment, obj, J, dJ_dc, forward_steps, ms);
    });
}

mcg_status mcg_jet_profile_metrics(mcg_handle *h, float *uc, float *r_half) {
    return mcg::guarded([&]() -> mcg_status {
        if (!h) return fail(MCG_ERR_INVALID_ARG, "handle is null");
        if (!uc || !r_half) return fail(MCG_ERR_INVALID_ARG, "output arrays must not be null");
        if (mcg_status st = mcg::async_flush(h)) return st;
        if (!h->stats_started || h->stats_samples == 0)
            return fail(MCG_ERR_STATE, "no radial statistics have been accumulated");
        const size_t M = size_t(h->p.NY) * size_t(h->p.NX / 2);
        std::vector<double> sum_uy(M);
        ADJ_CUDA(cudaMemcpyAsync(sum_uy.data(), h->s.radial, M * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                 "download radial sums");
        ADJ_CUDA(cudaStreamSynchronize(h->stream), "profile metrics");
        mcg::profile_metrics(h, sum_uy.data(), h->stats_samples, uc, r_half);
        return MCG_OK;
    });
}

}  // extern "C"
