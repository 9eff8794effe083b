// Batched ensemble: many independent ISF simulations of uneven grid sizes
// stepped together (C ABI in include/isf.h, isf_batch_*).
//
// Simulations with the same grid, torus, hbar, dt, particle slots, jet flag
// and emission count form a class.  A class's state is one array per field
// with the simulations back to back, and every pass of the time step is one
// launch over all of them (the simulation index is a grid dimension of the
// kernels).  Per-simulation jet and emission arguments live in device arrays
// that a prologue kernel rewrites from a device step counter, so one step of
// the whole ensemble is a fixed CUDA graph: prologue, then one branch per
// class (the branches run concurrently), replayed once per step.  Step k of
// simulation i is bit for bit isf_step with that simulation's arguments.
//
// Tile autotuner: for each class and each pass kind the batch times the
// pencil-group counts G = 1, 2, 4 the kernels are built for (on the class's
// own zeroed buffers, CUDA events on the batch stream) and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/isf.h"
#include "isf_launch.h"
#include "isf_passes.cuh"
#include "isf_persist.h"
#include "isf_stencil.cuh"

namespace isf {
namespace {

// Step counter and per-simulation jet / emission arguments of step it =
// counter + 1: omega t with t = Float32(it) * dt (every product rounded as
// the host computes it), Philox counter it, first ring slot (it-1)*count.
__global__ void k_batch_prologue(long long* __restrict__ step, const SimRT* __restrict__ rt,
                                 JetArgs* __restrict__ jets, EmitState* __restrict__ emits, int n) {
    const long long it = *step + 1;
    __syncthreads();  // every thread has read the counter before it moves
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const SimRT r = rt[s];
        jets[s].omgterm = __fmul_rn(r.omega, __fmul_rn((float)it, r.dt));
        emits[s].e.counter = (uint64_t)it;
        emits[s].start = r.nslots > 0 ? ((it - 1) * r.count) % r.nslots : 0;
    }
    if (threadIdx.x == 0) *step = it;
}

__global__ void k_fill(float* __restrict__ p, long long n, float v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

struct ClassKey {
    int n[3], L[3];
    float hbar, dt;
    long long nslots, emit;
    int jet;
    bool operator<(const ClassKey& o) const {
        return std::tie(n[0], n[1], n[2], L[0], L[1], L[2], hbar, dt, nslots, emit, jet) <
               std::tie(o.n[0], o.n[1], o.n[2], o.L[0], o.L[1], o.L[2], o.hbar, o.dt, o.nslots, o.emit, o.jet);
    }
};

}  // namespace
}  // namespace isf

using namespace isf;

struct BatchClass {
    ClassKey key;
    Grid g;
    int wp = 0;
    int nsim = 0;
    int first = 0;                 // index of its first simulation in class-major order
    float4* psi = nullptr;         // nsim x N
    float2* F = nullptr;           // nsim x wp*ny*nz
    float* f = nullptr;            // nsim x N
    float* vel = nullptr;          // nsim x kVelComp NP
    float* parts = nullptr;        // nsim x 3 nslots
    char* tables = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    int tiles[ISF_TILE_KINDS] = {1, 1, 1, 1, 1, 1};
    int kmajor = 0;  // k-major half spectrum, solved plane by plane
    long long bs_F() const { return (long long)wp * g.n[1] * g.n[2]; }
};

struct isf_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<BatchClass> cls;
    std::vector<int> sim_class, sim_index;  // per user simulation: class, index inside it
    std::vector<isf_sim_desc> desc;
    JetArgs* jets = nullptr;                // class-major, one per simulation
    EmitState* emits = nullptr;
    SimRT* rt = nullptr;
    long long* step = nullptr;
    unsigned long long* counters = nullptr;  // kCounterStride per simulation
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string err;
    // the persistent kernel (isf_batch_set_persistent): its phase table, one
    // CUDA graph per step count (zero the counters, one launch), the status
    int mode = 0;                  // ISF_PERSIST_* bits; 0: the per-step graph
    bool persist_ok = false;       // every class fits the persistent kernel
    std::string persist_why;
    std::vector<PPhase> phases;    // slot order
    std::vector<int> slot_start;   // items_per_step prefix
    PPhase* d_ph = nullptr;
    int* d_slot = nullptr;
    unsigned* d_done = nullptr;
    long long done_cap = 0;        // steps the done counters hold
    unsigned* d_ctl = nullptr;
    int* d_status = nullptr;
    long long spin_limit = 1LL << 22;
    int pgrid = 0, psmem = 0, psms = 0;  // persistent grid, its shared memory per block, the SMs it spans
    int dstride = 0, tiles_per_step = 0; // completion counters and tiles per step
    int preps = 1;                 // tuned: tiles per virtual CTA and item
    std::map<int, cudaGraphExec_t> pgraphs;
};

namespace {

thread_local std::string g_batch_create_error;

int bfail(isf_batch* b, int code, const std::string& msg) {
    if (b)
        b->err = msg;
    else
        g_batch_create_error = msg;
    return code;
}

int bcuda(isf_batch* b, cudaError_t e, const char* where) {
    return bfail(b, ISF_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define B_CUDA(b, expr, where)                          \
    do {                                                \
        cudaError_t e_ = (expr);                        \
        if (e_ != cudaSuccess) return bcuda(b, e_, where); \
    } while (0)

struct BDevice {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit BDevice(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~BDevice() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

#define B_ENTER(b)                                                        \
    if (!(b)) return bfail(nullptr, ISF_ERR_INVALID, "null batch");       \
    BDevice dev_(b->device);                                              \
    if (dev_.err != cudaSuccess) return bcuda(b, dev_.err, "cudaSetDevice")

// ---- the pass sequences of one class (the kernels of isf_step, batched)

XArgs bx(const BatchClass& c, int groups) {
    XArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = c.g;
    a.psi = c.psi;
    a.F = c.F;
    a.rin = c.f;
    a.wp = c.wp;
    a.nsim = c.nsim;
    a.bs_psi = c.g.N;
    a.bs_F = c.bs_F();
    a.bs_r = c.g.N;
    a.groups = groups;
    a.kmajor = c.kmajor;
    return a;
}

YZArgs byz(const BatchClass& c, bool half, int axis, int groups) {
    YZArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = c.g;
    a.axis = axis;
    a.nsim = c.nsim;
    a.groups = groups;
    if (half) {
        a.data = c.F;
        a.row = c.wp;
        a.kx_valid = c.g.n[0] / 2 + 1;
        a.bstride = c.bs_F();
    } else {
        a.data = c.psi;
        a.row = c.g.n[0];
        a.kx_valid = c.g.n[0];
        a.bstride = c.g.N;
    }
    return a;
}

StencilArgs bst(const BatchClass& c, float* out, long long bs_out) {
    StencilArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = c.g;
    a.psi = c.psi;
    a.out = out;
    a.nsim = c.nsim;
    a.bs_psi = c.g.N;
    a.bs_out = bs_out;
    return a;
}

cudaError_t class_schroedinger(const BatchClass& c, cudaStream_t s) {
    cudaError_t e;
    const XArgs xa = bx(c, c.tiles[ISF_TILE_X_PSI]);
    if ((e = launch_xpass(X_PSI_FWD, xa, s)) != cudaSuccess) return e;
    if ((e = launch_yzpass_psi(YZ_FWD, byz(c, false, 1, c.tiles[ISF_TILE_Y_PSI]), s)) != cudaSuccess) return e;
    if ((e = launch_yzpass_psi(YZ_MASK, byz(c, false, 2, c.tiles[ISF_TILE_Z_PSI]), s)) != cudaSuccess) return e;
    if ((e = launch_yzpass_psi(YZ_INV, byz(c, false, 1, c.tiles[ISF_TILE_Y_PSI]), s)) != cudaSuccess) return e;
    return launch_xpass(X_PSI_INV_NORM, xa, s);
}

cudaError_t class_projection(const BatchClass& c, const JetArgs* jets, cudaStream_t s) {
    cudaError_t e;
    StencilArgs sa = bst(c, c.f, c.g.N);
    XArgs xa = bx(c, c.tiles[ISF_TILE_X_REAL]);
    if (jets) {
        sa.use_jet = 1;
        sa.jets = jets;
        xa.use_jet = 1;
        xa.jets = jets;
    }
    if ((e = launch_stencil(ST_DIV, sa, s)) != cudaSuccess) return e;
    if ((e = launch_xreal(XR_FWD, xa, s)) != cudaSuccess) return e;
    if (c.kmajor) {
        if ((e = launch_poisson_plane(c.g, c.F, c.bs_F(), c.nsim, s)) != cudaSuccess) return e;
    } else {
        if ((e = launch_yzpass_c(YZ_FWD, byz(c, true, 1, c.tiles[ISF_TILE_Y_HALF]), s)) != cudaSuccess) return e;
        if ((e = launch_yzpass_c(YZ_FAC, byz(c, true, 2, c.tiles[ISF_TILE_Z_HALF]), s)) != cudaSuccess) return e;
        if ((e = launch_yzpass_c(YZ_INV, byz(c, true, 1, c.tiles[ISF_TILE_Y_HALF]), s)) != cudaSuccess) return e;
    }
    return launch_xreal(jets ? XR_INV_GAUGE_JET : XR_INV_GAUGE, xa, s);
}

// the simloop body of isf_step for every simulation of the class
cudaError_t class_step(const isf_batch* b, const BatchClass& c, cudaStream_t s) {
    cudaError_t e;
    if ((e = class_schroedinger(c, s)) != cudaSuccess) return e;
    if ((e = class_projection(c, nullptr, s)) != cudaSuccess) return e;
    if (c.key.jet) {
        if (c.key.emit > 0 && c.key.nslots > 0)
            if ((e = launch_emit_batch(c.parts, c.key.nslots, c.key.emit, c.nsim, b->emits + c.first, s)) !=
                cudaSuccess)
                return e;
        if ((e = class_projection(c, b->jets + c.first, s)) != cudaSuccess) return e;
    }
    StencilArgs va = bst(c, c.vel, kVelComp * c.g.NP);
    va.hbar = c.g.hbar;
    va.sharp = 1;
    if ((e = launch_stencil(ST_VEL, va, s)) != cudaSuccess) return e;
    if (c.key.nslots > 0)
        if ((e = launch_advect(c.g, c.parts, c.key.nslots, c.vel, b->counters + (size_t)c.first * kCounterStride, s,
                               c.nsim, kVelComp * c.g.NP)) != cudaSuccess)
            return e;
    return cudaSuccess;
}

// ---- autotuner

cudaError_t tune_launch(const BatchClass& c, int kind, int groups, cudaStream_t s) {
    switch (kind) {
        case ISF_TILE_X_PSI: return launch_xpass(X_PSI_FWD, bx(c, groups), s);
        case ISF_TILE_X_REAL: return launch_xreal(XR_FWD, bx(c, groups), s);
        case ISF_TILE_Y_PSI: return launch_yzpass_psi(YZ_FWD, byz(c, false, 1, groups), s);
        case ISF_TILE_Z_PSI: return launch_yzpass_psi(YZ_MASK, byz(c, false, 2, groups), s);
        case ISF_TILE_Y_HALF: return launch_yzpass_c(YZ_FWD, byz(c, true, 1, groups), s);
        case ISF_TILE_Z_HALF: return launch_yzpass_c(YZ_FAC, byz(c, true, 2, groups), s);
        default: return cudaErrorInvalidValue;
    }
}

int kind_len(const BatchClass& c, int kind) {
    return (kind == ISF_TILE_X_PSI || kind == ISF_TILE_X_REAL) ? c.g.n[0]
           : (kind == ISF_TILE_Y_PSI || kind == ISF_TILE_Y_HALF) ? c.g.n[1]
                                                                 : c.g.n[2];
}

// a G is a candidate when the kernels exist for it and it divides the work
bool tile_fits(const BatchClass& c, int kind, int G) {
    if (G == 1) return true;  // single-group tiles guard a partial last tile
    if (!grouped_tile_ok(kind_len(c, kind), G)) return false;
    // a k-major class runs its real x passes ungrouped and has no half-spectrum y / z passes
    if (c.kmajor && (kind == ISF_TILE_X_REAL || kind == ISF_TILE_Y_HALF || kind == ISF_TILE_Z_HALF)) return G == 1;
    const long long rows = (long long)c.g.n[1] * c.g.n[2];
    switch (kind) {
        case ISF_TILE_X_PSI: return rows % (8LL * G) == 0;
        case ISF_TILE_X_REAL: return rows % (32LL * G) == 0;
        case ISF_TILE_Y_PSI: case ISF_TILE_Y_HALF: return c.g.n[2] % G == 0;
        default: return c.g.n[1] % G == 0;
    }
}

int tune_class(isf_batch* b, BatchClass& c) {
    cudaEvent_t e0, e1;
    B_CUDA(b, cudaEventCreate(&e0), "tune event");
    B_CUDA(b, cudaEventCreate(&e1), "tune event");
    int rc = ISF_OK;
    for (int kind = 0; kind < ISF_TILE_KINDS && rc == ISF_OK; ++kind) {
        float best = 1e30f;
        int bestG = 1;
        if (c.kmajor && (kind == ISF_TILE_Y_HALF || kind == ISF_TILE_Z_HALF)) {
            c.tiles[kind] = 1;
            continue;
        }
        for (int G : {1, 2, 4}) {
            if (!tile_fits(c, kind, G)) continue;
            cudaError_t e = cudaSuccess;
            for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = tune_launch(c, kind, G, b->stream);
            if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
            for (int r = 0; r < 5 && e == cudaSuccess; ++r) e = tune_launch(c, kind, G, b->stream);
            if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                rc = bcuda(b, e, "isf_batch_create: tile autotuning");
                break;
            }
            if (ms < best * 0.97f) {  // prefer the smaller tile unless clearly faster
                best = ms;
                bestG = G;
            }
        }
        c.tiles[kind] = bestG;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

void free_persist(isf_batch* b);

void free_batch(isf_batch* b) {
    free_persist(b);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (BatchClass& c : b->cls) {
        cudaFree(c.psi);
        cudaFree(c.F);
        cudaFree(c.f);
        cudaFree(c.vel);
        cudaFree(c.parts);
        cudaFree(c.tables);
        if (c.stream) cudaStreamDestroy(c.stream);
        if (c.done) cudaEventDestroy(c.done);
    }
    cudaFree(b->jets);
    cudaFree(b->emits);
    cudaFree(b->rt);
    cudaFree(b->step);
    cudaFree(b->counters);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int capture_step(isf_batch* b) {
    if (b->exec) return ISF_OK;
    B_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "isf_batch_step: capture");
    cudaError_t e = cudaSuccess;
    const int n = (int)b->desc.size();
    k_batch_prologue<<<1, 256, 0, b->stream>>>(b->step, b->rt, b->jets, b->emits, n);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->stream);
    for (BatchClass& c : b->cls) {
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c.stream, b->fork, 0);
        if (e == cudaSuccess) e = class_step(b, c, c.stream);
        if (e == cudaSuccess) e = cudaEventRecord(c.done, c.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, c.done, 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return bcuda(b, e, "isf_batch_step: capturing the step graph");
    }
    e = cudaGraphInstantiate(&b->exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        b->exec = nullptr;
        return bcuda(b, e, "isf_batch_step: cudaGraphInstantiate");
    }
    b->graph = graph;
    return ISF_OK;
}

// ---- the persistent kernel: phase table, tuning, launch

void free_persist(isf_batch* b) {
    for (auto& kv : b->pgraphs) cudaGraphExecDestroy(kv.second);
    b->pgraphs.clear();
    cudaFree(b->d_ph);
    cudaFree(b->d_slot);
    cudaFree(b->d_done);
    cudaFree(b->d_ctl);
    cudaFree(b->d_status);
    b->d_ph = nullptr;
    b->d_slot = nullptr;
    b->d_done = nullptr;
    b->d_ctl = nullptr;
    b->d_status = nullptr;
    b->done_cap = 0;
}

PPhase new_phase(const BatchClass& c, int ci, int kind, int len, int gx, int gy, int gz) {
    PPhase p;
    std::memset(&p, 0, sizeof(p));
    p.kind = kind;
    p.cls = ci;
    p.len = len;
    p.gx = gx;
    p.gy = gy;
    p.tiles = gx * gy * gz;
    p.dep = p.dep_prev = -1;
    p.g = c.g;
    p.first = c.first;
    p.nsim = c.nsim;
    return p;
}

// the pass chain of class_step for class ci, one phase per launch of it
bool class_chain(const isf_batch* b, const BatchClass& c, int ci, std::vector<PPhase>& out, std::string& why) {
    const int nx = c.g.n[0], ny = c.g.n[1], nz = c.g.n[2], ns = c.nsim;
    if (!c.kmajor || !persist_plane_ok(ny) || !persist_len_ok(nx)) {
        why = "class " + std::to_string(ci) + " (" + std::to_string(nx) + "x" + std::to_string(ny) + "x" +
              std::to_string(nz) + "): the persistent kernel needs nx in {16,32,48,64,96,128} and ny = nz in "
              "{32,48,64,96}";
        return false;
    }
    const int rows = ny * nz;
    auto up = [](long long a, long long d) { return (int)((a + d - 1) / d); };
    out.push_back(new_phase(c, ci, PK_PROLOGUE, 0, 1, 1, 1));
    auto xphase = [&](int kind) {
        PPhase p = new_phase(c, ci, kind, nx, rows / 8, ns, 1);
        p.x = bx(c, 1);
        out.push_back(p);
    };
    auto yzphase = [&](int kind, int axis) {
        PPhase p = new_phase(c, ci, kind, axis == 1 ? ny : nz, nx / 8, axis == 1 ? nz : ny, ns);
        p.yz = byz(c, false, axis, 1);
        out.push_back(p);
    };
    xphase(PK_X_FWD);
    yzphase(PK_Y_FWD, 1);
    yzphase(PK_Z_MASK, 2);
    yzphase(PK_Y_INV, 1);
    xphase(PK_X_INV_NORM);
    auto projection = [&](const JetArgs* jets) {
        PPhase d = new_phase(c, ci, PK_DIV, 0, up(nx, st::BX), up(ny, st::BY), up(nz, st::planes_per_cta<ST_DIV>()) * ns);
        d.st = bst(c, c.f, c.g.N);
        PPhase f = new_phase(c, ci, PK_XR_FWD, nx, rows / 32, ns, 1);
        f.x = bx(c, 1);
        PPhase pl = new_phase(c, ci, PK_PLANE, ny, nx / 2 + 1, ns, 1);
        pl.pl.g = c.g;
        pl.pl.F = c.F;
        pl.pl.bs_F = c.bs_F();
        PPhase gi = new_phase(c, ci, PK_XR_INV_GAUGE, nx, rows / 32, ns, 1);
        gi.x = bx(c, 1);
        if (jets) {
            d.st.use_jet = 1;
            d.st.jets = jets;
            gi.x.use_jet = 1;
            gi.x.jets = jets;
        }
        out.push_back(d);
        out.push_back(f);
        out.push_back(pl);
        out.push_back(gi);
    };
    projection(nullptr);
    if (c.key.jet) {
        if (c.key.emit > 0 && c.key.nslots > 0) {
            PPhase e = new_phase(c, ci, PK_EMIT, 0, up(c.key.emit, kPersistThreads), ns, 1);
            e.parts = c.parts;
            e.nslots = c.key.nslots;
            e.count = c.key.emit;
            out.push_back(e);
        }
        projection(b->jets + c.first);
    }
    PPhase v = new_phase(c, ci, PK_VEL, 0, up(nx, st::BX), up(ny, st::BY), up(nz, st::planes_per_cta<ST_VEL>()) * ns);
    v.st = bst(c, c.vel, kVelComp * c.g.NP);
    v.st.hbar = c.g.hbar;
    v.st.sharp = 1;
    out.push_back(v);
    if (c.key.nslots > 0) {
        PPhase a = new_phase(c, ci, PK_ADVECT, 0, up(c.key.nslots, (long long)kPersistThreads * kAdvectSlots), ns, 1);
        a.parts = c.parts;
        a.nslots = c.key.nslots;
        a.vel = c.vel;
        a.bs_vel = kVelComp * c.g.NP;
        a.pow2 = c.g.d_pow2[0] && c.g.d_pow2[1] && c.g.d_pow2[2];
        a.normw = c.g.norm_w;
        out.push_back(a);
    }
    return true;
}

// The slot table: the classes' chains interleaved pass by pass, each phase
// waiting for its predecessor (the class's last phase of the previous step
// for the first one); an item is as many virtual CTAs as fit a block, each
// running `reps` tiles.
int build_plan(isf_batch* b, int reps, int blocks_per_sm_cap) {
    std::vector<std::vector<PPhase>> chains(b->cls.size());
    for (size_t ci = 0; ci < b->cls.size(); ++ci)
        if (!class_chain(b, b->cls[ci], (int)ci, chains[ci], b->persist_why))
            return bfail(b, ISF_ERR_INVALID, b->persist_why);
    size_t maxlen = 0, nslot = 0;
    for (auto& ch : chains) {
        maxlen = std::max(maxlen, ch.size());
        nslot += ch.size();
    }
    if (nslot > (size_t)kPersistMaxSlots)
        return bfail(b, ISF_ERR_INVALID, "persistent kernel: " + std::to_string(nslot) + " passes per step (" +
                                             std::to_string(b->cls.size()) + " classes); at most " +
                                             std::to_string(kPersistMaxSlots));
    std::vector<std::vector<int>> slot_of(chains.size());
    std::vector<PPhase> ph;
    for (size_t j = 0; j < maxlen; ++j)
        for (size_t ci = 0; ci < chains.size(); ++ci)
            if (j < chains[ci].size()) {
                slot_of[ci].push_back((int)ph.size());
                ph.push_back(chains[ci][j]);
            }
    // Dependencies: each pass waits for the pass before it in its class's
    // chain, and a few also wait for a pass of the previous step, so that
    // step n's advection runs beside step n+1's psi passes:
    //   prologue(n+1) after the last pass of step n that reads the jet and
    //     emission arguments it rewrites (the jet projection's gauge pass);
    //   x fwd(n+1), which transforms psi in place, after the one-form of step
    //     n, the last reader of psi;
    //   emission and one-form of step n+1, which write the particles and the
    //     velocity grid, after the advection of step n.
    for (size_t ci = 0; ci < chains.size(); ++ci) {
        const std::vector<PPhase>& ch = chains[ci];
        auto slot = [&](int kind, bool last) {
            int found = -1;
            for (size_t j = 0; j < ch.size(); ++j)
                if (ch[j].kind == kind) {
                    found = slot_of[ci][j];
                    if (!last) break;
                }
            return found;
        };
        const bool jet = b->cls[ci].key.jet;
        const int vel = slot(PK_VEL, true), adv = slot(PK_ADVECT, true);
        const int jet_gauge = jet ? slot(PK_XR_INV_GAUGE, true) : -1;
        for (size_t j = 0; j < ch.size(); ++j) {
            PPhase& p = ph[slot_of[ci][j]];
            p.dep = j > 0 ? slot_of[ci][j - 1] : -1;
            switch (p.kind) {
                case PK_PROLOGUE: p.dep_prev = jet_gauge; break;
                case PK_X_FWD: p.dep_prev = vel; break;
                case PK_EMIT: case PK_VEL: p.dep_prev = adv; break;
                default: p.dep_prev = -1; break;
            }
        }
    }
    int smem = 0, dstride = 0, tiles_per_step = 0;
    std::vector<int> start(1, 0);
    for (PPhase& p : ph) {
        // completion groups: the class's simulations when the tiles are
        // simulation-major (every pass but the prologue), else one
        p.nsg = (p.kind != PK_PROLOGUE && p.nsim > 1 && p.tiles % p.nsim == 0) ? p.nsim : 1;
        p.tps = p.tiles / p.nsg;
        p.doff = dstride;
        dstride += p.nsg;
        tiles_per_step += p.tiles;
        p.vblk = persist_vblk(p.kind, p.len);
        // a virtual CTA is whole warps (its named barrier counts threads in warps)
        if (p.vblk < 32 || p.vblk % 32 != 0 || p.vblk > kPersistThreads)
            return bfail(b, ISF_ERR_INVALID, "persistent kernel: pass kind " + std::to_string(p.kind) + " of length " +
                                                 std::to_string(p.len) + " has no virtual CTA shape");
        p.smem_v = persist_smem(p.kind, p.len);
        p.vper = std::max(1, kPersistThreads / p.vblk);
        p.reps = p.kind == PK_PROLOGUE ? 1 : reps;
        p.items = (p.tiles + p.vper * p.reps - 1) / (p.vper * p.reps);
        smem = std::max(smem, p.vper * p.smem_v);
        start.push_back(start.back() + p.items);
    }
    int bps = 0, sms = 0;
    B_CUDA(b, persist_setup(smem, &bps), "persistent kernel set-up");
    B_CUDA(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "persistent kernel set-up");
    if (bps < 1) return bfail(b, ISF_ERR_INVALID, "persistent kernel: no block fits an SM");
    bps = std::min(bps, blocks_per_sm_cap);
    free_persist(b);
    if (cudaMalloc(&b->d_ph, sizeof(PPhase) * ph.size()) != cudaSuccess ||
        cudaMalloc(&b->d_slot, sizeof(int) * start.size()) != cudaSuccess ||
        cudaMalloc(&b->d_ctl, 2 * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&b->d_status, 4 * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, ISF_ERR_NOMEM, "persistent kernel: device allocation failed");
    }
    B_CUDA(b, cudaMemcpy(b->d_ph, ph.data(), sizeof(PPhase) * ph.size(), cudaMemcpyHostToDevice), "persistent plan");
    B_CUDA(b, cudaMemcpy(b->d_slot, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice), "persistent plan");
    B_CUDA(b, cudaMemset(b->d_status, 0, 4 * sizeof(int)), "persistent plan");
    b->phases = ph;
    b->slot_start = start;
    b->dstride = dstride;
    b->tiles_per_step = tiles_per_step;
    b->psmem = smem;
    b->pgrid = sms * bps;
    b->psms = sms;
    b->preps = reps;
    return ISF_OK;
}

PPlan make_plan(const isf_batch* b, int nsteps) {
    PPlan p;
    std::memset(&p, 0, sizeof(p));
    p.ph = b->d_ph;
    p.slot_start = b->d_slot;
    p.nslot = (int)b->phases.size();
    p.items_per_step = b->slot_start.back();
    p.nsteps = nsteps;
    p.done = b->d_done;
    p.dstride = b->dstride;
    p.tiles_per_step = b->tiles_per_step;
    p.ctl = b->d_ctl;
    p.status = b->d_status;
    p.spin_limit = b->spin_limit;
    p.stall = (b->mode & ISF_PERSIST_STALL) ? 1 : 0;
    p.step = b->step;
    p.rt = b->rt;
    p.jets = b->jets;
    p.emits = b->emits;
    p.counters = b->counters;
    return p;
}

// queue nsteps persistent steps on s: zero the item counters, one launch
cudaError_t queue_persist(isf_batch* b, int nsteps, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(b->d_done, 0, sizeof(unsigned) * (size_t)b->dstride * nsteps, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_ctl, 0, 2 * sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status, 0, 4 * sizeof(int), s);
    if (e == cudaSuccess) e = launch_persist(make_plan(b, nsteps), b->pgrid, b->psmem, s);
    return e;
}

int ensure_done(isf_batch* b, long long nsteps) {
    if (b->done_cap >= nsteps) return ISF_OK;
    for (auto& kv : b->pgraphs) cudaGraphExecDestroy(kv.second);
    b->pgraphs.clear();
    cudaFree(b->d_done);
    b->d_done = nullptr;
    b->done_cap = 0;
    const long long cap = std::max<long long>(nsteps, 128);
    if (cudaMalloc(&b->d_done, sizeof(unsigned) * (size_t)b->dstride * cap) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, ISF_ERR_NOMEM, "persistent kernel: device allocation failed");
    }
    b->done_cap = cap;
    return ISF_OK;
}

// The persistent kernel's tile autotuner: tiles per virtual CTA and item
// (1, 2 or 4) and blocks per SM (as many as fit, or one), each timed over 3
// steps of the zeroed state; keeps the fastest.
int tune_persist(isf_batch* b, bool tune) {
    int best_reps = 1, best_bps = 2;
    if (tune) {
        cudaEvent_t e0, e1;
        B_CUDA(b, cudaEventCreate(&e0), "persistent tuning");
        B_CUDA(b, cudaEventCreate(&e1), "persistent tuning");
        float best = 1e30f;
        int rc = ISF_OK;
        for (int reps : {1, 2, 4}) {
            int tried = 0;  // blocks per SM already timed at this reps (the cap can clamp a candidate)
            for (int bps : {4, 3, 2, 1}) {
                if ((rc = build_plan(b, reps, bps)) != ISF_OK) break;
                const int eff = b->pgrid / std::max(1, b->psms);
                if (tried & (1 << eff)) continue;
                tried |= 1 << eff;
                if ((rc = ensure_done(b, 3)) != ISF_OK) break;
                cudaError_t e = queue_persist(b, 3, b->stream);  // warm-up
                if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
                if (e == cudaSuccess) e = queue_persist(b, 3, b->stream);
                if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                int st = 0;
                if (e == cudaSuccess) e = cudaMemcpy(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) {
                    rc = bcuda(b, e, "persistent kernel tuning");
                    break;
                }
                if (st != 0) {
                    rc = bfail(b, ISF_ERR_TIMEOUT, "persistent kernel tuning: a device-side wait ran out");
                    break;
                }
                if (ms < best * 0.97f) {
                    best = ms;
                    best_reps = reps;
                    best_bps = bps;
                }
            }
            if (rc != ISF_OK) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc != ISF_OK) return rc;
    }
    if (int rc = build_plan(b, best_reps, best_bps)) return rc;
    return ensure_done(b, 1);
}

int sim_ok(isf_batch* b, int32_t sim, const char* who) {
    if (sim < 0 || sim >= (int32_t)b->desc.size())
        return bfail(b, ISF_ERR_INVALID, std::string(who) + ": simulation index out of range");
    return ISF_OK;
}

JetArgs host_jet(const isf_sim_desc& d) {
    JetArgs j;
    std::memset(&j, 0, sizeof(j));
    for (int a = 0; a < 3; ++a) {
        j.kvec[a] = d.kvec[a];
        j.cen[a] = d.nozzle_cen[a];
    }
    j.len = d.nozzle_len;
    j.rad = d.nozzle_rad;
    j.omgterm = 0.f;
    j.phase_mode = d.phase_mode;
    j.mask = nullptr;
    return j;
}

}  // namespace

extern "C" {

int isf_batch_create(const isf_sim_desc* sims, int32_t nsims, int32_t device, int32_t tune, isf_batch** out) {
    if (!sims || !out || nsims <= 0) return bfail(nullptr, ISF_ERR_INVALID, "isf_batch_create: bad arguments");
    *out = nullptr;
    if (nsims > 65535) return bfail(nullptr, ISF_ERR_INVALID, "isf_batch_create: at most 65535 simulations");
    std::map<ClassKey, std::vector<int>> groups;
    for (int i = 0; i < nsims; ++i) {
        const isf_sim_desc& d = sims[i];
        isf_params p;
        std::memset(&p, 0, sizeof(p));
        for (int a = 0; a < 3; ++a) {
            p.grid_res[a] = d.grid_res[a];
            p.physical_size[a] = d.physical_size[a];
        }
        p.hbar = d.hbar;
        p.dt = d.dt;
        std::string why;
        const std::string who = "isf_batch_create: simulation " + std::to_string(i) + ": ";
        if (!check_params(&p, why)) return bfail(nullptr, ISF_ERR_INVALID, who + why);
        if (d.nslots < 0 || d.nslots > kMaxParticles)
            return bfail(nullptr, ISF_ERR_INVALID, who + "nslots must be in 0..715827882");
        if (d.jet != 0 && d.jet != 1) return bfail(nullptr, ISF_ERR_INVALID, who + "jet must be 0 or 1");
        if (d.jet) {
            if (d.phase_mode != ISF_PHASE_REFERENCE_SUM && d.phase_mode != ISF_PHASE_DOT)
                return bfail(nullptr, ISF_ERR_INVALID, who + "bad phase_mode");
            if (d.emit_per_step < 0 || d.emit_per_step > d.nslots)
                return bfail(nullptr, ISF_ERR_INVALID, who + "emit_per_step must be in 0..nslots");
            if (d.emit_per_step > 0 && (d.emit_mode < ISF_EMIT_RING || d.emit_mode > ISF_EMIT_RING_PLANE))
                return bfail(nullptr, ISF_ERR_INVALID, who + "bad emit_mode");
        }
        ClassKey k;
        for (int a = 0; a < 3; ++a) {
            k.n[a] = d.grid_res[a];
            k.L[a] = d.physical_size[a];
        }
        k.hbar = d.hbar;
        k.dt = d.dt;
        k.nslots = d.nslots;
        k.jet = d.jet;
        k.emit = d.jet ? d.emit_per_step : 0;
        groups[k].push_back(i);
    }
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess) return bcuda(nullptr, ce, "isf_batch_create: cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return bfail(nullptr, ISF_ERR_INVALID, "isf_batch_create: bad device ordinal");

    isf_batch* b = new isf_batch();
    b->device = device;
    BDevice dev(device);
    if (dev.err != cudaSuccess) {
        delete b;
        return bcuda(nullptr, dev.err, "isf_batch_create: cudaSetDevice");
    }
    auto fail_free = [&](int code, const std::string& msg) {
        free_batch(b);
        return bfail(nullptr, code, msg);
    };
    b->desc.assign(sims, sims + nsims);
    b->sim_class.assign(nsims, 0);
    b->sim_index.assign(nsims, 0);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return fail_free(ISF_ERR_CUDA, "isf_batch_create: stream / event creation failed");

    // classes in key order; per-simulation host records in class-major order
    std::vector<JetArgs> hjets;
    std::vector<EmitState> hemits;
    std::vector<SimRT> hrt;
    int first = 0;
    for (auto& kv : groups) {
        BatchClass c;
        c.key = kv.first;
        c.nsim = (int)kv.second.size();
        c.first = first;
        std::vector<char> host;
        fill_grid(c.key.n, c.key.L, c.key.hbar, c.key.dt, c.g, host);
        c.wp = half_spectrum_row(c.g.n[0]);
        c.kmajor = plane_supported(c.g.n) ? 1 : 0;
        const size_t ns = (size_t)c.nsim;
        if (cudaMalloc(&c.psi, sizeof(float4) * c.g.N * ns) != cudaSuccess ||
            cudaMalloc(&c.F, sizeof(float2) * c.bs_F() * ns) != cudaSuccess ||
            cudaMalloc(&c.f, sizeof(float) * c.g.N * ns) != cudaSuccess ||
            cudaMalloc(&c.vel, sizeof(float) * kVelComp * c.g.NP * ns) != cudaSuccess ||
            (c.key.nslots > 0 && cudaMalloc(&c.parts, sizeof(float) * 3 * c.key.nslots * ns) != cudaSuccess) ||
            cudaMalloc(&c.tables, host.size()) != cudaSuccess) {
            cudaGetLastError();
            b->cls.push_back(c);
            return fail_free(ISF_ERR_NOMEM, "isf_batch_create: device allocation failed");
        }
        const bool ok = cudaMemcpy(c.tables, host.data(), host.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
                        cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) == cudaSuccess &&
                        cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) == cudaSuccess;
        bind_tables(c.g, c.tables);
        b->cls.push_back(c);
        if (!ok) return fail_free(ISF_ERR_CUDA, "isf_batch_create: table upload / stream creation failed");
        for (int j = 0; j < c.nsim; ++j) {
            const int i = kv.second[j];
            b->sim_class[i] = (int)b->cls.size() - 1;
            b->sim_index[i] = j;
            const isf_sim_desc& d = sims[i];
            hjets.push_back(host_jet(d));
            EmitState es;
            std::memset(&es, 0, sizeof(es));
            for (int a = 0; a < 3; ++a) es.e.cen[a] = d.nozzle_cen[a];
            es.e.len = d.nozzle_len;
            es.e.rad = d.nozzle_rad;
            es.e.seed = d.seed;
            es.e.mode = d.emit_mode;
            hemits.push_back(es);
            hrt.push_back(SimRT{d.omega, d.dt, c.key.emit, d.nslots});
        }
        first += c.nsim;
    }
    if (cudaMalloc(&b->jets, sizeof(JetArgs) * nsims) != cudaSuccess ||
        cudaMalloc(&b->emits, sizeof(EmitState) * nsims) != cudaSuccess ||
        cudaMalloc(&b->rt, sizeof(SimRT) * nsims) != cudaSuccess || cudaMalloc(&b->step, sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&b->counters, sizeof(unsigned long long) * kCounterStride * nsims) != cudaSuccess) {
        cudaGetLastError();
        return fail_free(ISF_ERR_NOMEM, "isf_batch_create: device allocation failed");
    }
    cudaError_t e = cudaMemcpy(b->jets, hjets.data(), sizeof(JetArgs) * nsims, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->emits, hemits.data(), sizeof(EmitState) * nsims, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->rt, hrt.data(), sizeof(SimRT) * nsims, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->step, 0, sizeof(long long));
    if (e == cudaSuccess) e = cudaMemset(b->counters, 0, sizeof(unsigned long long) * kCounterStride * nsims);
    if (e != cudaSuccess) return fail_free(ISF_ERR_CUDA, std::string("isf_batch_create: upload: ") + cudaGetErrorString(e));
    // zero fields, dead particle slots
    auto clear = [&](const BatchClass& c) -> cudaError_t {
        const size_t ns = (size_t)c.nsim;
        cudaError_t r = cudaMemsetAsync(c.psi, 0, sizeof(float4) * c.g.N * ns, b->stream);
        if (r == cudaSuccess) r = cudaMemsetAsync(c.F, 0, sizeof(float2) * c.bs_F() * ns, b->stream);
        if (r == cudaSuccess) r = cudaMemsetAsync(c.f, 0, sizeof(float) * c.g.N * ns, b->stream);
        if (r == cudaSuccess) r = cudaMemsetAsync(c.vel, 0, sizeof(float) * kVelComp * c.g.NP * ns, b->stream);
        if (r == cudaSuccess && c.parts) {
            const long long n = 3 * c.key.nslots * (long long)ns;
            k_fill<<<(unsigned)std::min<long long>((n + 255) / 256, 148LL * 16), 256, 0, b->stream>>>(c.parts, n, -1.f);
            r = cudaGetLastError();
        }
        return r;
    };
    for (BatchClass& c : b->cls) {
        e = clear(c);
        if (e != cudaSuccess) return fail_free(ISF_ERR_CUDA, std::string("isf_batch_create: clear: ") + cudaGetErrorString(e));
        if (tune) {
            const int rc = tune_class(b, c);
            if (rc != ISF_OK) {
                const std::string m = b->err;
                free_batch(b);
                return bfail(nullptr, rc, m);
            }
        }
        // one eager step on the cleared state: every kernel of the class is
        // set up (shared-memory opt-ins) and launch-checked before capture
        e = class_step(b, c, b->stream);
        if (e != cudaSuccess) return fail_free(ISF_ERR_CUDA, std::string("isf_batch_create: warm-up step: ") + cudaGetErrorString(e));
        // the autotuner and the warm-up ran in place: clear again
        e = clear(c);
        if (e != cudaSuccess) return fail_free(ISF_ERR_CUDA, std::string("isf_batch_create: clear: ") + cudaGetErrorString(e));
    }
    // the persistent kernel's plan and tiles, when every class fits it (the
    // tuning runs in place on the cleared state: clear again after it)
    {
        std::vector<PPhase> probe;
        std::string pwhy;
        b->persist_ok = true;
        for (size_t ci = 0; ci < b->cls.size() && b->persist_ok; ++ci)
            b->persist_ok = class_chain(b, b->cls[ci], (int)ci, probe, pwhy);
        if (b->persist_ok && probe.size() > (size_t)kPersistMaxSlots) {
            b->persist_ok = false;
            pwhy = "the persistent kernel holds at most " + std::to_string(kPersistMaxSlots) +
                   " passes per step; these classes have " + std::to_string(probe.size());
        }
        b->persist_why = pwhy;
    }
    if (b->persist_ok && e == cudaSuccess) {
        e = cudaStreamSynchronize(b->stream);
        const int rc = e == cudaSuccess ? tune_persist(b, tune != 0) : ISF_OK;
        if (rc != ISF_OK) {
            const std::string m = b->err;
            free_batch(b);
            return bfail(nullptr, rc, "isf_batch_create: " + m);
        }
        for (BatchClass& c : b->cls)
            if (e == cudaSuccess) e = clear(c);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->step, 0, sizeof(long long), b->stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(b->counters, 0, sizeof(unsigned long long) * kCounterStride * nsims, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return fail_free(ISF_ERR_CUDA, std::string("isf_batch_create: ") + cudaGetErrorString(e));
    *out = b;
    return ISF_OK;
}

int isf_batch_destroy(isf_batch* b) {
    if (!b) return ISF_OK;
    BDevice dev(b->device);
    cudaStreamSynchronize(b->stream);
    free_batch(b);
    return ISF_OK;
}

const char* isf_batch_last_error(const isf_batch* b) {
    return b ? b->err.c_str() : g_batch_create_error.c_str();
}

static int batch_copy(isf_batch* b, int32_t sim, bool psi, bool to_batch, void* ptr, const char* who) {
    B_ENTER(b);
    if (int rc = sim_ok(b, sim, who)) return rc;
    if (!ptr) return bfail(b, ISF_ERR_INVALID, std::string(who) + ": null pointer");
    const BatchClass& c = b->cls[b->sim_class[sim]];
    const int j = b->sim_index[sim];
    size_t bytes;
    char* base;
    if (psi) {
        bytes = sizeof(float4) * (size_t)c.g.N;
        base = reinterpret_cast<char*>(c.psi) + bytes * j;
    } else {
        bytes = sizeof(float) * 3 * (size_t)c.key.nslots;
        if (bytes == 0) return ISF_OK;
        base = reinterpret_cast<char*>(c.parts) + bytes * j;
    }
    if (to_batch)
        B_CUDA(b, cudaMemcpyAsync(base, ptr, bytes, cudaMemcpyDefault, b->stream), who);
    else
        B_CUDA(b, cudaMemcpyAsync(ptr, base, bytes, cudaMemcpyDefault, b->stream), who);
    B_CUDA(b, cudaStreamSynchronize(b->stream), who);
    return ISF_OK;
}

int isf_batch_set_psi(isf_batch* b, int32_t sim, const float* psi) {
    return batch_copy(b, sim, true, true, const_cast<float*>(psi), "isf_batch_set_psi");
}
int isf_batch_get_psi(isf_batch* b, int32_t sim, float* psi) {
    return batch_copy(b, sim, true, false, psi, "isf_batch_get_psi");
}
int isf_batch_set_particles(isf_batch* b, int32_t sim, const float* parts) {
    return batch_copy(b, sim, false, true, const_cast<float*>(parts), "isf_batch_set_particles");
}
int isf_batch_get_particles(isf_batch* b, int32_t sim, float* parts) {
    return batch_copy(b, sim, false, false, parts, "isf_batch_get_particles");
}

int isf_batch_state(isf_batch* b, int32_t sim, float** psi, float** particles) {
    B_ENTER(b);
    if (int rc = sim_ok(b, sim, "isf_batch_state")) return rc;
    const BatchClass& c = b->cls[b->sim_class[sim]];
    const int j = b->sim_index[sim];
    if (psi) *psi = reinterpret_cast<float*>(c.psi + (size_t)c.g.N * j);
    if (particles) *particles = c.parts ? c.parts + (size_t)3 * c.key.nslots * j : nullptr;
    return ISF_OK;
}

int isf_batch_init_jet(isf_batch* b, int32_t iters) {
    B_ENTER(b);
    if (iters < 0) return bfail(b, ISF_ERR_INVALID, "isf_batch_init_jet: iters must be >= 0");
    // jet arguments at t = 0 (the prologue rewrites omega t every step)
    const int n = (int)b->desc.size();
    std::vector<JetArgs> hj(n);
    for (int i = 0; i < n; ++i) {
        const BatchClass& c = b->cls[b->sim_class[i]];
        hj[c.first + b->sim_index[i]] = host_jet(b->desc[i]);
    }
    B_CUDA(b, cudaMemcpyAsync(b->jets, hj.data(), sizeof(JetArgs) * n, cudaMemcpyHostToDevice, b->stream),
           "isf_batch_init_jet: upload");
    for (int it = 0; it < iters; ++it)
        for (const BatchClass& c : b->cls)
            if (c.key.jet) B_CUDA(b, class_projection(c, b->jets + c.first, b->stream), "isf_batch_init_jet");
    B_CUDA(b, cudaStreamSynchronize(b->stream), "isf_batch_init_jet");
    return ISF_OK;
}

int isf_batch_step(isf_batch* b, int32_t nsteps) {
    B_ENTER(b);
    if (nsteps < 0) return bfail(b, ISF_ERR_INVALID, "isf_batch_step: nsteps must be >= 0");
    if (b->mode & ISF_PERSIST_ON) {
        if (nsteps == 0) return ISF_OK;
        if (int rc = ensure_done(b, nsteps)) return rc;
        auto it = b->pgraphs.find(nsteps);
        if (it == b->pgraphs.end()) {
            // one graph per step count: zero the counters, one persistent launch
            B_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "isf_batch_step: capture");
            const cudaError_t e = queue_persist(b, nsteps, b->stream);
            cudaGraph_t graph = nullptr;
            const cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
            cudaGraphExec_t exec = nullptr;
            cudaError_t e3 = e != cudaSuccess ? e : e2;
            if (e3 == cudaSuccess) e3 = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e3 != cudaSuccess) {
                cudaGetLastError();
                return bcuda(b, e3, "isf_batch_step: capturing the persistent launch");
            }
            it = b->pgraphs.emplace(nsteps, exec).first;
        }
        B_CUDA(b, cudaGraphLaunch(it->second, b->stream), "isf_batch_step: cudaGraphLaunch");
        return ISF_OK;
    }
    if (int rc = capture_step(b)) return rc;
    for (int i = 0; i < nsteps; ++i) B_CUDA(b, cudaGraphLaunch(b->exec, b->stream), "isf_batch_step: cudaGraphLaunch");
    return ISF_OK;
}

int isf_batch_set_step(isf_batch* b, int64_t step) {
    B_ENTER(b);
    if (step < 0) return bfail(b, ISF_ERR_INVALID, "isf_batch_set_step: step must be >= 0");
    long long v = step;
    B_CUDA(b, cudaMemcpyAsync(b->step, &v, sizeof(v), cudaMemcpyHostToDevice, b->stream), "isf_batch_set_step");
    B_CUDA(b, cudaStreamSynchronize(b->stream), "isf_batch_set_step");
    return ISF_OK;
}

int isf_batch_get_stream(const isf_batch* b, void** stream) {
    if (!b || !stream) return bfail(const_cast<isf_batch*>(b), ISF_ERR_INVALID, "isf_batch_get_stream: null argument");
    *stream = b->stream;
    return ISF_OK;
}

int isf_batch_sync(isf_batch* b) {
    B_ENTER(b);
    B_CUDA(b, cudaStreamSynchronize(b->stream), "isf_batch_sync");
    if (b->d_status) {
        int st[3] = {0, 0, 0};
        B_CUDA(b, cudaMemcpy(st, b->d_status, sizeof(st), cudaMemcpyDeviceToHost), "isf_batch_sync: status");
        if (st[0] != 0) {
            const int slot = std::max(0, std::min(st[1], (int)b->phases.size() - 1));
            const PPhase& p = b->phases[(size_t)slot];
            return bfail(b, st[0], "isf_batch_sync: a device-side wait of the persistent kernel ran out (slot " +
                                       std::to_string(st[1]) + ": pass kind " + std::to_string(p.kind) + " of class " +
                                       std::to_string(p.cls) + ", step " + std::to_string(st[2]) +
                                       " of the launch); the ensemble state is partly stepped");
        }
    }
    return ISF_OK;
}

int isf_batch_set_persistent(isf_batch* b, int32_t mode, int64_t spin_limit) {
    B_ENTER(b);
    if (mode & ~(ISF_PERSIST_ON | ISF_PERSIST_STALL))
        return bfail(b, ISF_ERR_INVALID, "isf_batch_set_persistent: unknown mode bits");
    if ((mode & ISF_PERSIST_ON) && !b->persist_ok)
        return bfail(b, ISF_ERR_INVALID, "isf_batch_set_persistent: " + b->persist_why);
    B_CUDA(b, cudaStreamSynchronize(b->stream), "isf_batch_set_persistent");
    b->mode = mode;
    b->spin_limit = spin_limit > 0 ? spin_limit : (1LL << 22);
    for (auto& kv : b->pgraphs) cudaGraphExecDestroy(kv.second);
    b->pgraphs.clear();
    if (b->d_status) B_CUDA(b, cudaMemset(b->d_status, 0, 4 * sizeof(int)), "isf_batch_set_persistent");
    return ISF_OK;
}

int isf_batch_info(const isf_batch* b, int32_t* nclasses, int32_t* sim_class) {
    if (!b) return bfail(nullptr, ISF_ERR_INVALID, "null batch");
    if (nclasses) *nclasses = (int32_t)b->cls.size();
    if (sim_class)
        for (size_t i = 0; i < b->sim_class.size(); ++i) sim_class[i] = b->sim_class[i];
    return ISF_OK;
}

int isf_batch_tiles(const isf_batch* b, int32_t cls, int32_t tiles[6]) {
    if (!b) return bfail(nullptr, ISF_ERR_INVALID, "null batch");
    if (cls < 0 || cls >= (int32_t)b->cls.size() || !tiles)
        return bfail(const_cast<isf_batch*>(b), ISF_ERR_INVALID, "isf_batch_tiles: bad class index");
    for (int k = 0; k < ISF_TILE_KINDS; ++k) tiles[k] = b->cls[cls].tiles[k];
    return ISF_OK;
}

int isf_batch_counters(isf_batch* b, int32_t sim, uint64_t out[2], int32_t reset) {
    B_ENTER(b);
    if (int rc = sim_ok(b, sim, "isf_batch_counters")) return rc;
    if (!out) return bfail(b, ISF_ERR_INVALID, "isf_batch_counters: null output");
    const BatchClass& c = b->cls[b->sim_class[sim]];
    unsigned long long* p = b->counters + (size_t)(c.first + b->sim_index[sim]) * kCounterStride;
    unsigned long long tmp[2];
    B_CUDA(b, cudaMemcpyAsync(tmp, p, sizeof(tmp), cudaMemcpyDeviceToHost, b->stream), "isf_batch_counters");
    B_CUDA(b, cudaStreamSynchronize(b->stream), "isf_batch_counters");
    out[0] = tmp[0];
    out[1] = tmp[1];
    if (reset) {
        B_CUDA(b, cudaMemsetAsync(p, 0, sizeof(tmp), b->stream), "isf_batch_counters reset");
        B_CUDA(b, cudaStreamSynchronize(b->stream), "isf_batch_counters reset");
    }
    return ISF_OK;
}

}  // extern "C"
