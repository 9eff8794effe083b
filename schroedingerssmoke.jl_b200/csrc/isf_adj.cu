// Reverse-mode entry points of libisf (isf_adj_*, include/isf.h): the
// adjoint of each operator of the ISF time step, of one whole step, and a
// checkpointed driver for the gradient of a particle loss over many steps.
//
// The step's forward is recomputed unfused for the reverse pass (Schroedinger
// flow without normalize, normalize, div -> Poisson -> q -> gauge, restrict,
// the second projection, one-form), keeping the five psi states and the two
// q fields in a tape; the reverse then runs the stage adjoints of
// k_adjoint.cu backwards.  The driver keeps psi every `checkpoint_every`
// steps and the particle positions of every step, and recomputes the psi
// states inside a segment from its checkpoint before reversing it.
#include <cstring>
#include <string>
#include <vector>

#include "isf_handle.h"

using namespace isf;

struct isf_adj_state {
    float* q = nullptr;     // q of a projection (N)
    float* qbar = nullptr;  // N
    float* fbar = nullptr;  // N
    float* ubar = nullptr;  // cotangent of the padded velocity planes (3 NP)
    double* acc = nullptr;  // 8 accumulators (jet adjoint, loss)
    float4* tape = nullptr;        // 5 psi states of one step: a (flowed), b (normalised), c, d, e
    float* tq = nullptr;           // q1 | q2 of one step (2 N)
    float* tparts = nullptr;       // particles after the step's emission
    long long tparts_cap = 0;
    // driver storage (grown on demand)
    float4* states = nullptr;      // work | checkpoints | init tape | segment states
    long long states_cap = 0;      // float4 elements
    float* positions = nullptr;    // particle positions of every step
    long long positions_cap = 0;   // floats
    float* lam = nullptr;          // particle cotangent
    long long lam_cap = 0;
};

namespace isf_int {

void adj_free(isf_handle* h) {
    isf_adj_state* a = h->adj;
    if (!a) return;
    cudaFree(a->q);
    cudaFree(a->qbar);
    cudaFree(a->fbar);
    cudaFree(a->ubar);
    cudaFree(a->acc);
    cudaFree(a->tape);
    cudaFree(a->tq);
    cudaFree(a->tparts);
    cudaFree(a->states);
    cudaFree(a->positions);
    cudaFree(a->lam);
    delete a;
    h->adj = nullptr;
}

}  // namespace isf_int

using namespace isf_int;

namespace {

int adj_ensure(isf_handle* h) {
    if (h->adj) return ISF_OK;
    isf_adj_state* a = new isf_adj_state();
    h->adj = a;
    const Grid& g = h->g;
    if (cudaMalloc(&a->q, sizeof(float) * g.N) != cudaSuccess || cudaMalloc(&a->qbar, sizeof(float) * g.N) != cudaSuccess ||
        cudaMalloc(&a->fbar, sizeof(float) * g.N) != cudaSuccess ||
        cudaMalloc(&a->ubar, sizeof(float) * 3 * g.NP) != cudaSuccess ||
        cudaMalloc(&a->acc, sizeof(double) * 8) != cudaSuccess ||
        cudaMalloc(&a->tape, sizeof(float4) * 5 * g.N) != cudaSuccess ||
        cudaMalloc(&a->tq, sizeof(float) * 2 * g.N) != cudaSuccess) {
        cudaGetLastError();
        adj_free(h);
        return fail(h, ISF_ERR_NOMEM, "adjoint work buffers: device allocation failed");
    }
    ISF_CUDA(h, cudaMemsetAsync(a->ubar, 0, sizeof(float) * 3 * g.NP, h->stream), "adjoint set-up");
    return ISF_OK;
}

// grows a float buffer to at least n elements (contents not kept)
template <class T>
int grow(isf_handle* h, T*& p, long long& cap, long long n, const char* what) {
    if (n <= cap) return ISF_OK;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, sizeof(T) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, ISF_ERR_NOMEM, std::string(what) + ": device allocation failed");
    }
    cap = n;
    return ISF_OK;
}

int copy_psi(isf_handle* h, void* dst, const void* src) {
    if (dst == src) return ISF_OK;
    ISF_CUDA(h, cudaMemcpyAsync(dst, src, sizeof(float4) * h->g.N, cudaMemcpyDeviceToDevice, h->stream), "psi copy");
    return ISF_OK;
}

// q = Poisson(div one-form(psi)) into q (real), psi unchanged
int projection_q(isf_handle* h, const float* psi, float* q) {
    StencilArgs sa = stargs(h, psi, h->f);
    ISF_LAUNCH(h, launch_stencil(ST_DIV, sa, h->stream), "adj projection div");
    XArgs xa = xargs(h);
    xa.rin = h->f;
    xa.rout = q;
    ISF_LAUNCH(h, launch_xreal(XR_FWD, xa, h->stream), "adj poisson x fwd");
    if (int rc = run_poisson_spectral(h, "adj poisson")) return rc;
    ISF_LAUNCH(h, launch_xreal(XR_INV_REAL, xa, h->stream), "adj poisson x inv");
    return ISF_OK;
}

// the real Poisson solve out = P in (P is symmetric: its own adjoint)
int poisson(isf_handle* h, const float* in, float* out) {
    XArgs xa = xargs(h);
    xa.rin = in;
    xa.rout = out;
    ISF_LAUNCH(h, launch_xreal(XR_FWD, xa, h->stream), "adj poisson x fwd");
    if (int rc = run_poisson_spectral(h, "adj poisson")) return rc;
    ISF_LAUNCH(h, launch_xreal(XR_INV_REAL, xa, h->stream), "adj poisson x inv");
    return ISF_OK;
}

// adjoint of psi_out = psi_in exp(-i q), q = P div W(psi_in)
int adj_projection(isf_handle* h, const float* psi_in, const float* q, float* bar) {
    isf_adj_state* a = h->adj;
    const float4* pin = reinterpret_cast<const float4*>(psi_in);
    float4* b = reinterpret_cast<float4*>(bar);
    ISF_LAUNCH(h, launch_adj_gauge(h->g, pin, q, b, a->qbar, h->stream), "adj gauge");
    if (int rc = poisson(h, a->qbar, a->fbar)) return rc;
    ISF_LAUNCH(h, launch_adj_oneform_div(h->g, pin, b, a->fbar, h->stream), "adj one-form (div)");
    return ISF_OK;
}

int adj_schroedinger(isf_handle* h, float* bar) {
    XArgs xa = xargs(h);
    xa.psi = reinterpret_cast<float4*>(bar);
    YZArgs mz = yzargs(h, bar, 2);
    mz.conj_mask = 1;  // IFFT conj(mask) FFT: the transpose of the unitary flow
    ISF_LAUNCH(h, launch_xpass(X_PSI_FWD, xa, h->stream), "adj schroedinger x fwd");
    ISF_LAUNCH(h, launch_yzpass_psi(YZ_FWD, yzargs(h, bar, 1), h->stream), "adj schroedinger y fwd");
    ISF_LAUNCH(h, launch_yzpass_psi(YZ_MASK, mz, h->stream), "adj schroedinger z mask");
    ISF_LAUNCH(h, launch_yzpass_psi(YZ_INV, yzargs(h, bar, 1), h->stream), "adj schroedinger y inv");
    ISF_LAUNCH(h, launch_xpass(X_PSI_INV, xa, h->stream), "adj schroedinger x inv");
    return ISF_OK;
}

int read_acc(isf_handle* h, double* out, int n) {
    ISF_CUDA(h, cudaMemcpyAsync(out, h->adj->acc, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream), "adjoint read");
    ISF_CUDA(h, cudaStreamSynchronize(h->stream), "adjoint read");
    return ISF_OK;
}

int clear_acc(isf_handle* h) {
    ISF_CUDA(h, cudaMemsetAsync(h->adj->acc, 0, sizeof(double) * 8, h->stream), "adjoint clear");
    return ISF_OK;
}

struct StepJet {
    bool jet = false;
    JetArgs j;
    EmitArgs e;
    long long emit_start = 0, emit_count = 0;
};

StepJet step_jet(const isf_step_args* s) {
    StepJet r;
    std::memset(&r.j, 0, sizeof(r.j));
    std::memset(&r.e, 0, sizeof(r.e));
    if (!s || !s->jet) return r;
    r.jet = true;
    r.j = make_jet(s->kvec, s->jetmask, s->nozzle_cen, s->nozzle_len, s->nozzle_rad, s->omega_t, s->phase_mode);
    for (int k = 0; k < 3; ++k) r.e.cen[k] = s->nozzle_cen[k];
    r.e.len = s->nozzle_len;
    r.e.rad = s->nozzle_rad;
    r.e.seed = s->seed;
    r.e.counter = s->counter;
    r.e.mode = s->emit_mode;
    r.emit_start = s->emit_start;
    r.emit_count = s->emit_count;
    return r;
}

// Forward of one step into a tape (psi a..e at T, q1 | q2 at tq) and, when
// the step emits, the particles after the emission into tparts.  The state
// after the step is tape e (c without a jet); psi_in is not modified.
int step_tape(isf_handle* h, const float* psi_in, const float* parts_in, long long np, const StepJet& sj, float4* T,
              float* tq, const float4** out_psi, const float** out_parts) {
    isf_adj_state* a = h->adj;
    const long long N = h->g.N;
    float4 *pa = T, *pb = T + N, *pc = T + 2 * N, *pd = T + 3 * N, *pe = T + 4 * N;
    if (int rc = copy_psi(h, pa, psi_in)) return rc;
    if (int rc = run_schroedinger(h, reinterpret_cast<float*>(pa), false)) return rc;
    ISF_LAUNCH(h, launch_normalize_to(h->g, pa, pb, h->stream), "adj tape normalize");
    if (int rc = projection_q(h, reinterpret_cast<const float*>(pb), tq)) return rc;
    ISF_LAUNCH(h, launch_gauge(h->g, pb, tq, pc, h->stream), "adj tape gauge");
    const float* parts = parts_in;
    if (sj.jet) {
        if (np > 0 && sj.emit_count > 0) {
            if (int rc = grow(h, a->tparts, a->tparts_cap, 3 * np, "adjoint particles")) return rc;
            ISF_CUDA(h, cudaMemcpyAsync(a->tparts, parts_in, sizeof(float) * 3 * np, cudaMemcpyDeviceToDevice, h->stream),
                     "adj tape particles");
            ISF_LAUNCH(h, launch_emit(a->tparts, np, sj.emit_start % np, sj.emit_count, sj.e, h->stream), "adj tape emit");
            parts = a->tparts;
        }
        ISF_LAUNCH(h, launch_restrict_to(h->g, pc, pd, sj.j, h->stream), "adj tape restrict");
        if (int rc = projection_q(h, reinterpret_cast<const float*>(pd), tq + N)) return rc;
        ISF_LAUNCH(h, launch_gauge(h->g, pd, tq + N, pe, h->stream), "adj tape gauge");
        *out_psi = pe;
    } else {
        *out_psi = pc;
    }
    *out_parts = parts;
    return ISF_OK;
}

// Reverse of one step given its tape: bar (psi cotangent after the step ->
// before it), lam (particle cotangent after -> before); the jet cotangent is
// added into acc[0..2] (kvec) and acc[3] (omega t times wscale).
int step_reverse(isf_handle* h, const float* parts_used, long long np, const StepJet& sj, const float4* T,
                 const float* tq, const float4* psi_out, float* bar, float* lam, float wscale) {
    isf_adj_state* a = h->adj;
    const long long N = h->g.N;
    // velocity of the step: one-form(hbar) + sharp of the state after the projections
    if (int rc = run_one_form(h, reinterpret_cast<const float*>(psi_out), h->g.hbar, 1, "adj tape one-form")) return rc;
    if (np > 0) {
        ISF_LAUNCH(h, launch_adj_advect(h->g, parts_used, lam, np, h->vel, a->ubar, h->stream), "adj advect");
        if (sj.jet && sj.emit_count > 0)
            ISF_LAUNCH(h, launch_zero_slots(lam, np, sj.emit_start, sj.emit_count, h->stream), "adj emitted slots");
    }
    float4* b = reinterpret_cast<float4*>(bar);
    ISF_LAUNCH(h, launch_adj_oneform_vel(h->g, psi_out, b, a->ubar, h->g.hbar, 1, h->stream), "adj one-form (velocity)");
    ISF_CUDA(h, cudaMemsetAsync(a->ubar, 0, sizeof(float) * 3 * h->g.NP, h->stream), "adj clear velocity cotangent");
    if (sj.jet) {
        if (int rc = adj_projection(h, reinterpret_cast<const float*>(T + 3 * N), tq + N, bar)) return rc;
        ISF_LAUNCH(h, launch_adj_restrict(h->g, T + 2 * N, b, sj.j, a->acc, wscale, h->stream), "adj restrict");
    }
    if (int rc = adj_projection(h, reinterpret_cast<const float*>(T + N), tq, bar)) return rc;
    ISF_LAUNCH(h, launch_adj_normalize(h->g, T, b, h->stream), "adj normalize");
    return adj_schroedinger(h, bar);
}

int check_problem(isf_handle* h, const isf_adj_problem* p, long long np, const char* who) {
    if (!p) return fail(h, ISF_ERR_INVALID, std::string(who) + ": null problem");
    if (p->nsteps < 1 || p->checkpoint_every < 1 || p->init_iters < 0)
        return fail(h, ISF_ERR_INVALID, std::string(who) + ": nsteps and checkpoint_every must be >= 1, init_iters >= 0");
    if (p->phase_mode != ISF_PHASE_REFERENCE_SUM && p->phase_mode != ISF_PHASE_DOT)
        return fail(h, ISF_ERR_INVALID, std::string(who) + ": bad phase_mode");
    if (np < 1 || np > kMaxParticles) return fail(h, ISF_ERR_INVALID, std::string(who) + ": bad particle count");
    return ISF_OK;
}

// jet of step n (1-based) of the problem: omega t = Float32(omega * Float32(n dt))
isf_step_args problem_step(const isf_adj_problem* p, float dt, int n, float* t_out) {
    isf_step_args s;
    std::memset(&s, 0, sizeof(s));
    s.jet = 1;
    s.phase_mode = p->phase_mode;
    const float t = (float)n * dt;
    for (int k = 0; k < 3; ++k) {
        s.kvec[k] = p->kvec[k];
        s.nozzle_cen[k] = p->nozzle_cen[k];
    }
    s.omega_t = (float)(p->omega * t);
    s.nozzle_len = p->nozzle_len;
    s.nozzle_rad = p->nozzle_rad;
    s.emit_mode = ISF_EMIT_DISC;
    s.jetmask = nullptr;
    if (t_out) *t_out = t;
    return s;
}

int init_jet_args(const isf_adj_problem* p, JetArgs& j) {
    j = make_jet(p->kvec, nullptr, p->nozzle_cen, p->nozzle_len, p->nozzle_rad, 0.f, p->phase_mode);
    return ISF_OK;
}

// psi after the problem's initialisation: init_iters x (restrict at
// omega t = 0, projection); the state before each iteration into init_tape
int problem_init(isf_handle* h, const isf_adj_problem* p, const float* psi0, float4* work, float4* init_tape) {
    const long long N = h->g.N;
    if (int rc = copy_psi(h, work, psi0)) return rc;
    JetArgs j0;
    init_jet_args(p, j0);
    for (int it = 0; it < p->init_iters; ++it) {
        if (init_tape)
            if (int rc = copy_psi(h, init_tape + it * N, work)) return rc;
        ISF_LAUNCH(h, launch_restrict(h->g, work, j0, h->stream), "adj init restrict");
        if (int rc = run_projection(h, reinterpret_cast<float*>(work), nullptr)) return rc;
    }
    return ISF_OK;
}

}  // namespace

extern "C" {

int isf_adj_schroedinger_flow(isf_handle* h, float* psibar) {
    ISF_ENTER(h);
    if (!psibar) return fail(h, ISF_ERR_INVALID, "isf_adj_schroedinger_flow: null argument");
    ISF_ALIGNED(h, psibar, 16, "psibar");
    return adj_schroedinger(h, psibar);
}

int isf_adj_normalize_psi(isf_handle* h, const float* psi_in, float* psibar) {
    ISF_ENTER(h);
    if (!psi_in || !psibar) return fail(h, ISF_ERR_INVALID, "isf_adj_normalize_psi: null argument");
    ISF_ALIGNED(h, psi_in, 16, "psi");
    ISF_ALIGNED(h, psibar, 16, "psibar");
    ISF_LAUNCH(h, launch_adj_normalize(h->g, reinterpret_cast<const float4*>(psi_in), reinterpret_cast<float4*>(psibar),
                                       h->stream),
               "adj normalize");
    return ISF_OK;
}

int isf_adj_pressure_project(isf_handle* h, const float* psi_in, float* psibar) {
    ISF_ENTER(h);
    if (!psi_in || !psibar) return fail(h, ISF_ERR_INVALID, "isf_adj_pressure_project: null argument");
    ISF_ALIGNED(h, psi_in, 16, "psi");
    ISF_ALIGNED(h, psibar, 16, "psibar");
    if (int rc = adj_ensure(h)) return rc;
    if (int rc = projection_q(h, psi_in, h->adj->q)) return rc;
    return adj_projection(h, psi_in, h->adj->q, psibar);
}

int isf_adj_restrict_velocity(isf_handle* h, const float* psi_in, float* psibar, const float kvec[3],
                              const uint8_t* jetmask, const float cen[3], float len, float rad, float omgterm,
                              int32_t phase_mode, double jetbar[4]) {
    ISF_ENTER(h);
    if (!psi_in || !psibar || !kvec || !cen || !jetbar)
        return fail(h, ISF_ERR_INVALID, "isf_adj_restrict_velocity: null argument");
    if (phase_mode != ISF_PHASE_REFERENCE_SUM && phase_mode != ISF_PHASE_DOT)
        return fail(h, ISF_ERR_INVALID, "isf_adj_restrict_velocity: bad phase_mode");
    ISF_ALIGNED(h, psi_in, 16, "psi");
    ISF_ALIGNED(h, psibar, 16, "psibar");
    if (int rc = adj_ensure(h)) return rc;
    if (int rc = clear_acc(h)) return rc;
    const JetArgs j = make_jet(kvec, jetmask, cen, len, rad, omgterm, phase_mode);
    ISF_LAUNCH(h, launch_adj_restrict(h->g, reinterpret_cast<const float4*>(psi_in), reinterpret_cast<float4*>(psibar), j,
                                      h->adj->acc, 1.f, h->stream),
               "adj restrict");
    return read_acc(h, jetbar, 4);
}

int isf_adj_velocity_one_form(isf_handle* h, const float* psi, float hbar, int32_t sharp, float* psibar) {
    ISF_ENTER(h);
    if (!psi || !psibar) return fail(h, ISF_ERR_INVALID, "isf_adj_velocity_one_form: null argument");
    ISF_ALIGNED(h, psi, 16, "psi");
    ISF_ALIGNED(h, psibar, 16, "psibar");
    if (int rc = adj_ensure(h)) return rc;
    ISF_LAUNCH(h, launch_adj_oneform_vel(h->g, reinterpret_cast<const float4*>(psi), reinterpret_cast<float4*>(psibar),
                                         h->adj->ubar, hbar, sharp ? 1 : 0, h->stream),
               "adj one-form (velocity)");
    ISF_CUDA(h, cudaMemsetAsync(h->adj->ubar, 0, sizeof(float) * 3 * h->g.NP, h->stream), "adj clear velocity cotangent");
    return ISF_OK;
}

int isf_adj_staggered_advect(isf_handle* h, const float* particles, float* particles_bar, int64_t np) {
    ISF_ENTER(h);
    if (np < 0 || (np > 0 && (!particles || !particles_bar)))
        return fail(h, ISF_ERR_INVALID, "isf_adj_staggered_advect: bad particles");
    if (np > kMaxParticles) return fail(h, ISF_ERR_INVALID, "isf_adj_staggered_advect: more than 715827882 particles");
    if (int rc = adj_ensure(h)) return rc;
    ISF_LAUNCH(h, launch_adj_advect(h->g, particles, particles_bar, np, h->vel, h->adj->ubar, h->stream), "adj advect");
    return ISF_OK;
}

int isf_adj_get_velocity_bar(isf_handle* h, float* aos) {
    ISF_ENTER(h);
    if (!aos) return fail(h, ISF_ERR_INVALID, "isf_adj_get_velocity_bar: null output");
    if (int rc = adj_ensure(h)) return rc;
    ISF_LAUNCH(h, launch_adj_fold(h->g, h->adj->ubar, h->stream), "adj fold");
    ISF_LAUNCH(h, launch_adj_to_aos(h->g, h->adj->ubar, aos, h->stream), "adj velocity cotangent to aos");
    return ISF_OK;
}

int isf_adj_set_velocity_bar(isf_handle* h, const float* aos) {
    ISF_ENTER(h);
    if (!aos) return fail(h, ISF_ERR_INVALID, "isf_adj_set_velocity_bar: null input");
    if (int rc = adj_ensure(h)) return rc;
    ISF_CUDA(h, cudaMemsetAsync(h->adj->ubar, 0, sizeof(float) * 3 * h->g.NP, h->stream), "adj clear velocity cotangent");
    ISF_LAUNCH(h, launch_adj_from_aos(h->g, aos, h->adj->ubar, h->stream), "adj velocity cotangent from aos");
    return ISF_OK;
}

int isf_adj_step(isf_handle* h, const float* psi_in, const float* particles_in, int64_t np, const isf_step_args* args,
                 float* psibar, float* particles_bar, double jetbar[4]) {
    ISF_ENTER(h);
    if (!psi_in || !psibar || !args || !jetbar) return fail(h, ISF_ERR_INVALID, "isf_adj_step: null argument");
    ISF_ALIGNED(h, psi_in, 16, "psi");
    ISF_ALIGNED(h, psibar, 16, "psibar");
    if (np < 0 || (np > 0 && (!particles_in || !particles_bar)))
        return fail(h, ISF_ERR_INVALID, "isf_adj_step: bad particles");
    if (np > kMaxParticles) return fail(h, ISF_ERR_INVALID, "isf_adj_step: more than 715827882 particles");
    if (args->jet && (args->emit_count < 0 || args->emit_start < 0 || (args->emit_count > 0 && args->emit_count > np)))
        return fail(h, ISF_ERR_INVALID, "isf_adj_step: bad emission range");
    if (int rc = adj_ensure(h)) return rc;
    if (int rc = clear_acc(h)) return rc;
    const StepJet sj = step_jet(args);
    const float4* out = nullptr;
    const float* parts = nullptr;
    if (int rc = step_tape(h, psi_in, particles_in, np, sj, h->adj->tape, h->adj->tq, &out, &parts)) return rc;
    if (int rc = step_reverse(h, parts, np, sj, h->adj->tape, h->adj->tq, out, psibar, particles_bar, 1.f)) return rc;
    return read_acc(h, jetbar, 4);
}

int isf_adj_loss(isf_handle* h, const isf_adj_problem* p, const float* psi0, const float* particles0, int64_t np,
                 const float* targets, double* loss) {
    ISF_ENTER(h);
    if (!psi0 || !particles0 || !targets || !loss) return fail(h, ISF_ERR_INVALID, "isf_adj_loss: null argument");
    ISF_ALIGNED(h, psi0, 16, "psi0");
    if (int rc = check_problem(h, p, np, "isf_adj_loss")) return rc;
    if (int rc = adj_ensure(h)) return rc;
    isf_adj_state* a = h->adj;
    if (int rc = grow(h, a->states, a->states_cap, h->g.N, "isf_adj_loss")) return rc;
    if (int rc = grow(h, a->positions, a->positions_cap, 3 * np, "isf_adj_loss")) return rc;
    if (int rc = grow(h, a->lam, a->lam_cap, 3 * np, "isf_adj_loss")) return rc;
    float4* work = a->states;
    if (int rc = problem_init(h, p, psi0, work, nullptr)) return rc;
    ISF_CUDA(h, cudaMemcpyAsync(a->positions, particles0, sizeof(float) * 3 * np, cudaMemcpyDeviceToDevice, h->stream),
             "isf_adj_loss: positions");
    for (int n = 1; n <= p->nsteps; ++n) {
        isf_step_args st = problem_step(p, h->g.dt, n, nullptr);
        if (int rc = isf_step(h, reinterpret_cast<float*>(work), a->positions, np, &st)) return rc;
        if (int rc = join(h)) return rc;  // the step's particles, on the handle's stream
    }
    if (int rc = clear_acc(h)) return rc;
    ISF_LAUNCH(h, launch_loss(a->positions, targets, a->lam, np, a->acc + 4, h->stream), "adj loss");
    double v[5];
    if (int rc = read_acc(h, v, 5)) return rc;
    *loss = v[4];
    return ISF_OK;
}

int isf_adj_gradient(isf_handle* h, const isf_adj_problem* p, const float* psi0, const float* particles0, int64_t np,
                     const float* targets, double* loss, float* psibar0, float* particles_bar0, double jetbar[4]) {
    ISF_ENTER(h);
    if (!psi0 || !particles0 || !targets || !loss || !psibar0 || !particles_bar0 || !jetbar)
        return fail(h, ISF_ERR_INVALID, "isf_adj_gradient: null argument");
    ISF_ALIGNED(h, psi0, 16, "psi0");
    ISF_ALIGNED(h, psibar0, 16, "psibar0");
    if (int rc = check_problem(h, p, np, "isf_adj_gradient")) return rc;
    if (int rc = adj_ensure(h)) return rc;
    isf_adj_state* a = h->adj;
    const long long N = h->g.N;
    const int T = p->nsteps, K = p->checkpoint_every < p->nsteps ? p->checkpoint_every : p->nsteps;
    const int nck = (T + K - 1) / K;
    // psi states: work | checkpoints (nck) | init tape (init_iters) | segment tapes (K x 5) ;
    // q fields: K x 2 N
    const long long nstates = 1 + nck + p->init_iters + 5LL * K;
    if (int rc = grow(h, a->states, a->states_cap, nstates * N, "isf_adj_gradient")) return rc;
    if (int rc = grow(h, a->positions, a->positions_cap, 3 * np * (long long)(T + 1) + 2 * N * K, "isf_adj_gradient"))
        return rc;
    float4* work = a->states;
    float4* ckpt = work + N;
    float4* itape = ckpt + nck * N;
    float4* tapes = itape + (long long)p->init_iters * N;
    float* pos = a->positions;
    float* tqs = pos + (size_t)3 * np * (T + 1);
    float* lam = particles_bar0;
    // forward: checkpoints and every step's particle positions; the last
    // segment records its tapes as it goes (it is reversed first)
    if (int rc = problem_init(h, p, psi0, work, itape)) return rc;
    ISF_CUDA(h, cudaMemcpyAsync(pos, particles0, sizeof(float) * 3 * np, cudaMemcpyDeviceToDevice, h->stream),
             "isf_adj_gradient: positions");
    const int last0 = (nck - 1) * K + 1;
    const float4* seg_in = nullptr;
    for (int n = 1; n <= T; ++n) {
        float* cur = pos + (size_t)3 * np * n;
        ISF_CUDA(h, cudaMemcpyAsync(cur, cur - 3 * np, sizeof(float) * 3 * np, cudaMemcpyDeviceToDevice, h->stream),
                 "isf_adj_gradient: positions");
        isf_step_args st = problem_step(p, h->g.dt, n, nullptr);
        if ((n - 1) % K == 0 && n < last0)
            if (int rc = copy_psi(h, ckpt + ((n - 1) / K) * N, work)) return rc;
        if (n < last0) {
            if (int rc = isf_step(h, reinterpret_cast<float*>(work), cur, np, &st)) return rc;
            if (int rc = join(h)) return rc;  // the step's particles, on the handle's stream
        } else {
            const StepJet sj = step_jet(&st);
            const float4* out = nullptr;
            const float* used = nullptr;
            const float* in = n == last0 ? reinterpret_cast<const float*>(work) : reinterpret_cast<const float*>(seg_in);
            if (int rc = step_tape(h, in, cur - 3 * np, np, sj, tapes + (long long)5 * (n - last0) * N,
                                   tqs + (size_t)2 * N * (n - last0), &out, &used))
                return rc;
            if (int rc = run_one_form(h, reinterpret_cast<const float*>(out), h->g.hbar, 1, "adj one-form")) return rc;
            ISF_LAUNCH(h, launch_advect(h->g, cur, np, h->vel, h->counters, h->stream), "adj advect forward");
            seg_in = out;
        }
    }
    if (int rc = clear_acc(h)) return rc;
    ISF_LAUNCH(h, launch_loss(pos + (size_t)3 * np * T, targets, lam, np, a->acc + 4, h->stream), "adj loss");
    ISF_CUDA(h, cudaMemsetAsync(psibar0, 0, sizeof(float4) * N, h->stream), "adj clear psibar");
    for (int s = nck - 1; s >= 0; --s) {
        const int n0 = s * K + 1, n1 = (s + 1) * K < T ? (s + 1) * K : T;
        if (s < nck - 1) {
            // the segment's tapes, recomputed from its checkpoint
            const float* in = reinterpret_cast<const float*>(ckpt + s * N);
            for (int n = n0; n <= n1; ++n) {
                isf_step_args st = problem_step(p, h->g.dt, n, nullptr);
                const StepJet sj = step_jet(&st);
                const float4* out = nullptr;
                const float* used = nullptr;
                if (int rc = step_tape(h, in, pos + (size_t)3 * np * (n - 1), np, sj, tapes + (long long)5 * (n - n0) * N,
                                       tqs + (size_t)2 * N * (n - n0), &out, &used))
                    return rc;
                in = reinterpret_cast<const float*>(out);
            }
        }
        for (int n = n1; n >= n0; --n) {
            float tn = 0.f;
            isf_step_args st = problem_step(p, h->g.dt, n, &tn);
            const StepJet sj = step_jet(&st);
            const float4* T5 = tapes + (long long)5 * (n - n0) * N;
            const float4* out = sj.jet ? T5 + 4 * N : T5 + 2 * N;
            if (int rc = step_reverse(h, pos + (size_t)3 * np * (n - 1), np, sj, T5, tqs + (size_t)2 * N * (n - n0), out,
                                      psibar0, lam, tn))
                return rc;
        }
    }
    // the jet initialisation, in reverse: restrict (omega t = 0), then projection
    JetArgs j0;
    init_jet_args(p, j0);
    for (int it = p->init_iters - 1; it >= 0; --it) {
        const float4* in = itape + (long long)it * N;
        ISF_LAUNCH(h, launch_restrict_to(h->g, in, work, j0, h->stream), "adj init restrict");
        if (int rc = projection_q(h, reinterpret_cast<const float*>(work), a->q)) return rc;
        if (int rc = adj_projection(h, reinterpret_cast<const float*>(work), a->q, psibar0)) return rc;
        ISF_LAUNCH(h, launch_adj_restrict(h->g, in, reinterpret_cast<float4*>(psibar0), j0, a->acc, 0.f, h->stream),
                   "adj init restrict");
    }
    double acc[5];
    if (int rc = read_acc(h, acc, 5)) return rc;
    *loss = acc[4];
    for (int k = 0; k < 4; ++k) jetbar[k] = acc[k];
    return ISF_OK;
}

}  // extern "C"
