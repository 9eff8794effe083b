// The ISF handle and the host-side helpers shared by the C ABI files
// (isf_abi.cu, isf_adj.cu); internal to libisf.
#pragma once
#include <string>
#include <vector>

#include "../../include/isf.h"
#include "isf_launch.h"
#include "isf_passes.cuh"

struct isf_adj_state;  // adjoint work buffers, allocated on first use (isf_adj.cu)

struct isf_handle {
    isf::Grid g;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    float2* F = nullptr;     // Poisson half spectrum (wp x ny x nz complex), N allocated
    int wp = 0;              // padded half-spectrum row: round_up(nx/2 + 1, 16)
    int flags = 0;           // ISF_FLAG_* of isf_create
    int kmajor = 0;          // the half spectrum is k-major and solved plane by plane (plane_supported)
    float* f = nullptr;      // divergence of the one-form (isf.f, parallel.jl:29), N
    float* vel = nullptr;    // the current padded velocity grid, float4 per cell (kVelComp NP floats): vel_buf[vcur]
    float* vel_buf[2] = {nullptr, nullptr};  // two velocity grids: a step writes one while the
    int vcur = 0;                            // previous step's advection may still read the other
    // isf_step runs its particle work (emission, advection) on `side`, so the
    // next step's psi passes overlap it; only for handles that own their stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_vel = nullptr;              // the step's velocity is written (main stream)
    cudaEvent_t ev_read[2] = {nullptr, nullptr};  // the advection that read vel_buf[i] is done (side)
    cudaEvent_t ev_side = nullptr;             // the last work queued on side
    bool side_pending = false;                 // side work the main stream has not waited for
    unsigned* keep_counts = nullptr;           // per-block counts of isf_keep_inside
    long long keep_cap = 0;
    void* tables = nullptr;  // twiddles, phase factors, Laplacian symbols
    unsigned long long* counters = nullptr;  // [0] clamp events, [1] live particles, [2..] ISF_CHECK record
    unsigned long long launches = 0;         // kernels launched by this handle
    std::string err;
    // optional per-launch-site event timing (isf_profile_*)
    struct Rec {
        int site;
        cudaEvent_t a, b;
    };
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<Rec> recs;
    std::vector<std::string> site_names;
    std::vector<double> site_ms;
    std::vector<long long> site_count;
    isf_adj_state* adj = nullptr;
    // cell order of the particle slots (isf_set_particle_order / isf_sort_particles)
    int order_every = 0;                 // isf_step re-sorts every order_every steps (0: storage order)
    int order_age = 0;                   // isf_step advections since the last sort
    long long order_n = 0;               // slots of the current permutation (0: none)
    const float* order_parts = nullptr;  // the slot array it was made for
    isf::OrderBufs ord = {};
    long long ord_cap = 0;               // slots the rank / order buffers hold
    // the tensor map of the TMA-staged z pass, for the psi it was encoded for
    isf::CUtensorMapStorage zmap = {};
    const float* zmap_psi = nullptr;
    bool zmap_ok = false;
};

namespace isf_int {

using namespace isf;

int fail(isf_handle* h, int code, const std::string& msg);
int cuda_fail(isf_handle* h, cudaError_t e, const char* where);
int prof_begin(isf_handle* h, const char* site, cudaStream_t st = nullptr);
void prof_end(isf_handle* h, int slot, cudaStream_t st = nullptr);
// make the main stream wait for the particle work isf_step queued on the side stream
int join(isf_handle* h);

// Make the handle's device current for the duration of a call.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};


// pass arguments of the handle's grid and work arrays
XArgs xargs(isf_handle* h);
YZArgs yzargs(isf_handle* h, void* data, int axis);
YZArgs yzhalf(isf_handle* h, int axis);
StencilArgs stargs(isf_handle* h, const float* psi, float* out);
JetArgs make_jet(const float kvec[3], const uint8_t* mask, const float cen[3], float len, float rad, float omgterm,
                 int mode);

// kernel sequences of the reference operators (isf_abi.cu)
int run_schroedinger(isf_handle* h, float* psi, bool norm);
int run_projection(isf_handle* h, float* psi, const JetArgs* jet);
int run_one_form(isf_handle* h, const float* psi, float hbar, int sharp, const char* site);
// the y / z transforms and the Laplacian multiply of the Poisson solve on h->F
int run_poisson_spectral(isf_handle* h, const char* site);

// the cell order of np slots on stream st (launch sites "<site> order count / scan / scatter")
int ensure_order(isf_handle* h, long long np);
int run_order(isf_handle* h, const float* parts, long long np, cudaStream_t st, const char* site);

// releases the adjoint work buffers (isf_adj.cu)
void adj_free(isf_handle* h);

}  // namespace isf_int

#define ISF_CHECK_HANDLE(h)                                                  \
    do {                                                                     \
        if (!(h)) return fail(nullptr, ISF_ERR_INVALID, "null isf handle");  \
    } while (0)

#define ISF_LAUNCH(h, expr, site)                                \
    do {                                                         \
        const int ps_ = prof_begin(h, site);                     \
        cudaError_t e_ = (expr);                                 \
        ++(h)->launches;                                         \
        prof_end(h, ps_);                                        \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, site);    \
    } while (0)

#define ISF_CUDA(h, expr, where)                      \
    do {                                              \
        cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, where); \
    } while (0)

// psi is read as float4 (16-byte) and complex work arrays as float2 (8-byte)
#define ISF_ALIGNED(h, ptr, a, name)                                                        \
    do {                                                                                    \
        if (((uintptr_t)(ptr)) % (a) != 0)                                                  \
            return fail(h, ISF_ERR_INVALID, std::string(name) + " must be " #a "-byte aligned"); \
    } while (0)

// Every entry point except isf_step and isf_counters_async first orders the
// handle's stream after the particle work earlier steps left on the side
// stream, so it sees their particles, counters and velocity reads finished.
#define ISF_ENTER_NOJOIN(h)                                   \
    ISF_CHECK_HANDLE(h);                                      \
    DeviceGuard guard_(h->device);                            \
    if (guard_.err != cudaSuccess) return cuda_fail(h, guard_.err, "cudaSetDevice")

#define ISF_ENTER(h)                                          \
    ISF_ENTER_NOJOIN(h);                                      \
    if (int rc_join_ = join(h)) return rc_join_

// a launch on another stream than the handle's (profiling events on it)
#define ISF_LAUNCH_ON(h, st, expr, site)                         \
    do {                                                         \
        const int ps_ = prof_begin(h, site, st);                 \
        cudaError_t e_ = (expr);                                 \
        ++(h)->launches;                                         \
        prof_end(h, ps_, st);                                    \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, site);    \
    } while (0)
