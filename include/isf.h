/*
 * libisf -- C ABI of the B200 (sm_100a) incompressible-Schroedinger-flow
 * (ISF) library.  Every entry point replaces one call of the reference
 * SchroedingersSmoke.jl API (paths inside the reference project are cited
 * beside each declaration); a Julia front-end reaches them through `ccall`.
 *
 * Conventions
 *   - Every function returns an int status: ISF_OK (0) or an ISF_ERR_* code;
 *     isf_last_error() gives the message.  Nothing aborts the process (the
 *     reference throws a Julia exception at the same places).
 *   - Arrays are device pointers with the reference's Julia layouts
 *     (column-major, x fastest):
 *       psi        4 floats per cell: re psi1, im psi1, re psi2, im psi2
 *                  (NTuple{2,ComplexF32}, examples/benchmark.jl:20)
 *       particles  3 floats per slot; a dead slot is (-1,-1,-1)
 *                  (src/parallel.jl:213-215)
 *       jetmask    1 byte per cell (Julia Bool array of isjet.(positions))
 *   - All work is asynchronous on the handle's stream until isf_sync(), like
 *     GPUArrays' launches (examples/benchmark.jl:66).  A handle is not
 *     thread-safe; separate handles are independent.
 *   - Grid sizes: each of nx, ny, nz in {8,12,16,20,24,32,40,48,50,56,64,80,
 *     96,100,112,128,160,192,200,256,384,512} (the FFT's radix plans: 2^a 3^b
 *     up to 512, and lengths with a factor 5 or 7; ISF_ERR_INVALID otherwise);
 *     the reference takes any dims (src/parallel.jl:41-79).  psi pointers
 *     16-byte aligned, complex arrays 8-byte aligned.
 */
#ifndef ISF_H
#define ISF_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ISF_API __attribute__((visibility("default")))
#else
#define ISF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ISF_OK = 0,
    ISF_ERR_INVALID = 1,     /* bad argument or unsupported size */
    ISF_ERR_CUDA = 2,        /* CUDA runtime error (message has the CUDA text) */
    ISF_ERR_NOMEM = 3,       /* device allocation failed */
    ISF_ERR_NAN = 4,         /* isf_step with ISF_FLAG_CHECK_NAN found a non-finite psi */
    ISF_ERR_TIMEOUT = 5,     /* a bounded device-side wait of the persistent batch kernel ran out */
};

/* isf_params.flags */
enum {
    /* staggered_velocity weights divided by d (parallel.jl:238 leaves them in
     * units of length, as does MatlabPort.jl:259-261): the interpolation
     * becomes the usual bilinear one */
    ISF_FLAG_NORMALIZED_WEIGHTS = 1,
    /* isf_step checks psi for non-finite values after the step (a
     * reduction and a synchronisation per step) and returns ISF_ERR_NAN */
    ISF_FLAG_CHECK_NAN = 2,
    /* the Schroedinger z pass copies its pencils into shared memory with the
     * TMA (double-buffered cp.async.bulk.tensor tiles) instead of loading
     * them into registers; same results, bitwise.  Off by default: on the
     * 256 x 128 x 128 step it measured 38.8 us against 37.6 us */
    ISF_FLAG_TMA_Z_PASS = 4,
    /* test switch of the TMA z pass: after its first tile has arrived, every
     * CTA also waits on a flag that nothing sets (counter 13, always 0), so
     * the bounded wait runs out.  Each CTA counts the timeout in counter 14,
     * waits (bounded) for its copy still in flight and returns: psi is left
     * partly transformed and the context stays usable.  Only with
     * ISF_FLAG_TMA_Z_PASS; for testing the timeout path. */
    ISF_FLAG_TMA_Z_STALL = 8,
};

/* jet phase: reference tuple_dot(k, x) = sum(k .+ x) (src/particles.jl:1,15)
 * or the dot product k . x (examples/matlabport/simple.jl:47,107) */
enum { ISF_PHASE_REFERENCE_SUM = 0, ISF_PHASE_DOT = 1 };

/* emission: reference ring (src/particles.jl:86-90), nozzle disc, nozzle
 * cylinder, and the MatlabPort driver's ring of 0.9 r in the plane x = cen.x
 * without jitter (examples/matlabport/simple.jl:112-115) */
enum { ISF_EMIT_RING = 0, ISF_EMIT_DISC = 1, ISF_EMIT_CYLINDER = 2, ISF_EMIT_RING_PLANE = 3 };

typedef struct isf_handle isf_handle;

/* ISF{ArrayType,UInt32,Float32}(physical_size, dims, hbar, dt) (src/parallel.jl:41) */
typedef struct isf_params {
    int32_t grid_res[3];      /* dims (nx, ny, nz) */
    int32_t physical_size[3]; /* torus size, integers as in src/parallel.jl:12,45 */
    float hbar;               /* reduced Planck constant */
    float dt;                 /* time step */
    int32_t device;           /* CUDA device ordinal */
    int32_t flags;            /* ISF_FLAG_* bits (0: the reference's semantics) */
    void* stream;             /* cudaStream_t to run on (cudaStreamLegacy included), or NULL: the handle makes its own */
} isf_params;

/* Arguments of one fused time step (the simloop body, examples/benchmark.jl:46-65). */
typedef struct isf_step_args {
    int32_t jet;              /* 0: no nozzle (one projection); 1: jet step */
    int32_t phase_mode;       /* ISF_PHASE_* */
    float kvec[3];            /* jet_velocity / hbar (examples/benchmark.jl:24) */
    float omega_t;            /* omega * t of this step (examples/benchmark.jl:58) */
    float nozzle_cen[3];
    float nozzle_len;
    float nozzle_rad;
    int32_t emit_mode;        /* ISF_EMIT_* */
    const uint8_t* jetmask;   /* device isjet array, or NULL to evaluate the nozzle analytically */
    int64_t emit_start;       /* first ring-buffer slot (0-based) of add_particles! */
    int64_t emit_count;       /* particles emitted this step (0: none) */
    uint64_t seed;            /* Philox key */
    uint64_t counter;         /* Philox stream counter (e.g. the step number) */
} isf_step_args;

/* ---- handle, memory, stream ------------------------------------------- */

/* ISF constructor (src/parallel.jl:41-98): tables and temporaries on the device. */
ISF_API int isf_create(const isf_params* params, isf_handle** out);
ISF_API int isf_destroy(isf_handle* h);
/* Message of the last failed call on h (or of the last failed isf_create when h is NULL). */
ISF_API const char* isf_last_error(const isf_handle* h);
/* The stream the handle's work runs on.  Without a caller stream, isf_create
 * makes a blocking stream, which is ordered with the legacy default stream,
 * and a second blocking stream for the particle work of isf_step (emission
 * and advection), which then overlaps the next step's psi passes.  Every
 * entry point except isf_step and isf_counters_async first orders the
 * handle's stream after that particle work; a caller that queues its own
 * work on the handle's stream right after isf_step calls isf_join first.
 * Work on the legacy default stream is ordered after both streams. */
ISF_API int isf_get_stream(const isf_handle* h, void** stream);
/* GPUArrays.synchronize (examples/benchmark.jl:66) */
ISF_API int isf_sync(isf_handle* h);
/* Order the handle's stream after the particle work of earlier isf_step
 * calls (no host wait). */
ISF_API int isf_join(isf_handle* h);
/* Device buffers for psi / particles / masks (the reference's ArrayType(...) uploads, src/parallel.jl:78-97) */
ISF_API int isf_malloc(isf_handle* h, void** dptr, size_t bytes);
ISF_API int isf_free(isf_handle* h, void* dptr);
/* Stream-ordered copies; host memory should be pinned for asynchrony. */
ISF_API int isf_memcpy_h2d(isf_handle* h, void* dst_dev, const void* src_host, size_t bytes);
ISF_API int isf_memcpy_d2h(isf_handle* h, void* dst_host, const void* src_dev, size_t bytes);
/* grid facts: n[3], d[3] (Float32(physical_size ./ grid_res), src/parallel.jl:46) */
ISF_API int isf_grid_info(const isf_handle* h, int32_t n_out[3], float d_out[3]);

/* ---- operators (exported API of src/parallel.jl:264-266, src/particles.jl:97) */

/* schroedinger_flow!(isf, psi)            src/parallel.jl:176-187 */
ISF_API int isf_schroedinger_flow(isf_handle* h, float* psi);
/* psi .= normalize_psi.(psi)             src/parallel.jl:162-165, examples/benchmark.jl:50 */
ISF_API int isf_normalize_psi(isf_handle* h, float* psi);
/* pressure_project!(isf, psi)             src/parallel.jl:155-160 */
ISF_API int isf_pressure_project(isf_handle* h, float* psi);
/* velocity_one_form!(isf, psi, hbar)      src/parallel.jl:115-122 (into the handle's velocity) */
ISF_API int isf_velocity_one_form(isf_handle* h, const float* psi, float hbar);
/* velocity .*= 1 ./ d (staggered sharp)   examples/benchmark.jl:61-63 */
ISF_API int isf_staggered_sharp(isf_handle* h);
/* isf.velocity as AoS float3 per cell     src/parallel.jl:14, 66 (copy into a device buffer) */
ISF_API int isf_get_velocity(isf_handle* h, float* vel_aos_dev);
ISF_API int isf_set_velocity(isf_handle* h, const float* vel_aos_dev);
/* isjet.(isf.positions, cen, len, rad)    src/particles.jl:6-10, examples/benchmark.jl:26 */
ISF_API int isf_isjet(isf_handle* h, uint8_t* jetmask_dev, const float cen[3], float len, float rad);
/* restrict_velocity!(isf, psi, kvec, isjetarr, omgterm)   src/particles.jl:25-27
 * jetmask_dev may be NULL: the nozzle (cen, len, rad) is then evaluated per cell. */
ISF_API int isf_restrict_velocity(isf_handle* h, float* psi, const float kvec[3], const uint8_t* jetmask_dev,
                          const float cen[3], float len, float rad, float omgterm, int32_t phase_mode);
/* The jet set-up loop (examples/benchmark.jl:28-31): iters times
 * restrict_velocity!(isf, psi, kvec, isjetarr, 0) then pressure_project!(isf, psi),
 * in one call.  jetmask_dev may be NULL: the nozzle is evaluated per cell. */
ISF_API int isf_init_jet(isf_handle* h, float* psi, int32_t iters, const float kvec[3], const uint8_t* jetmask_dev,
                         const float cen[3], float len, float rad, int32_t phase_mode);
/* add_particles!(particles, start:start+count-1, cen, rad)   src/particles.jl:60-94
 * slots wrap modulo nslots; seeded Philox stream (seed, counter). */
ISF_API int isf_add_particles(isf_handle* h, float* particles, int64_t nslots, int64_t start, int64_t count,
                      const float cen[3], float len, float rad, uint64_t seed, uint64_t counter,
                      int32_t mode);
/* staggered_advect!(particles, isf)       src/parallel.jl:248-261 (uses the handle's velocity) */
ISF_API int isf_staggered_advect(isf_handle* h, float* particles, int64_t nparticles);
/* One fused time step: the simloop body examples/benchmark.jl:46-65. */
ISF_API int isf_step(isf_handle* h, float* psi, float* particles, int64_t nparticles, const isf_step_args* args);

/* Cell-sorted traversal of the particle slots.  staggered_advect!
 * (src/parallel.jl:248-261) advects every slot of the buffer in storage
 * order, dead ones included.  With every > 0, isf_step advects through a
 * permutation of the slots instead: live particles grouped by 2 x 2 x 2 cell
 * tile, so a warp's velocity gathers share cells, and dead slots last, so
 * they share warps.  Slots never move (a slot stays a particle's identity)
 * and each particle's arithmetic is unchanged, so the positions are bitwise
 * those of storage order.  The permutation is rebuilt every `every` steps on
 * the particle stream (launch sites "step order count / scan / scatter"),
 * and whenever the slot array or its length changes; particles emitted in
 * between keep their slot's place in it.  every = 0 restores storage order. */
ISF_API int isf_set_particle_order(isf_handle* h, int32_t every);
/* Build the permutation of np slots now, on the handle's stream; the next
 * isf_step with these particles uses it if ordering is on. */
ISF_API int isf_sort_particles(isf_handle* h, const float* particles, int64_t nparticles);
/* *n = the length of the current permutation (0: none); with order non-NULL,
 * copies it into that device buffer (cap entries), stream-ordered on the
 * handle's stream. */
ISF_API int isf_get_particle_order(isf_handle* h, int32_t* order, int64_t cap, int64_t* n);

/* ---- diagnostics (internal stages of the reference, exposed for parity checks) */

/* isf.f from the handle's velocity: div!(isf)   src/parallel.jl:144-152 */
ISF_API int isf_div(isf_handle* h, float* f_dev);
/* real part of poisson_solve with isf.f := f   src/parallel.jl:168-174 */
ISF_API int isf_poisson_solve(isf_handle* h, const float* f_dev, float* q_dev);
/* in-place 3D complex FFT of interleaved complex64 data, sign -1 forward
 * (unnormalised), +1 inverse (1/N): the plan_fft! / plan_ifft! of src/parallel.jl:79 */
ISF_API int isf_fft3(isf_handle* h, float* data_dev, int32_t sign);
/* First n (<= 16) counters of the advections since the last reset: [0] clamp
 * events (staggered_velocity index rounded to n+1), [1] live particles; in a
 * bounds-checking build (-DISF_CHECK) [2] rejected gather indices, [3] the
 * first of them and [4..11] its cell indices, two neighbour indices and strides;
 * [13] always 0 (the flag ISF_FLAG_TMA_Z_STALL waits on);
 * [14] waits of the TMA-staged Schroedinger z pass (ISF_FLAG_TMA_Z_PASS)
 * that ran out (its CTA then stops; 0 unless a copy stalled for about half
 * a second, or ISF_FLAG_TMA_Z_STALL); [15] non-finite
 * psi cells after the last isf_step of a handle made with ISF_FLAG_CHECK_NAN.
 * Synchronises the handle's stream. */
ISF_API int isf_counters(isf_handle* h, uint64_t* out, int32_t n, int32_t reset);
/* The same counters copied asynchronously: the copy of the first n (1..16)
 * into host_out (pinned host memory for a truly asynchronous copy) is queued
 * on the handle's stream after the work already queued, and the reset after
 * it; host_out is valid once the stream is synchronised. */
ISF_API int isf_counters_async(isf_handle* h, uint64_t* host_out, int32_t n, int32_t reset);

/* ---- allocation-free entry point (no counterpart in the reference) -------
 * The real part of poisson_solve (the same result as isf_poisson_solve) for
 * callers that cannot let the library allocate device memory: a host runtime
 * whose own pool owns all device memory, a hard memory cap, or a loop that
 * must not allocate after set-up.  It needs no handle and calls no cudaMalloc
 * / cudaFree: its workspace is a file-scope device array of 262144 complex64
 * values (2 MiB, held by every GPU that loads libisf until exit), so
 * round_up(nx/2 + 1, 16) * ny * nz must not exceed 262144 (ISF_ERR_INVALID
 * otherwise; e.g. 64 x 64 x 64 fits).  Runs on params->stream (NULL: the
 * legacy default stream) of params->device; f and q are device arrays of N
 * floats.  All calls share the workspace: calls that overlap on the GPU race,
 * so serialise them.  The first call on a device looks up the workspace
 * address; make it before any stream capture.  The grid tables are uploaded
 * from host memory when (grid_res, physical_size, hbar, dt) differ from the
 * previous call's on that device; a call that needs such an upload while
 * params->stream is being captured returns ISF_ERR_INVALID and queues
 * nothing.  Errors: isf_static_last_error(). */
ISF_API int isf_poisson_solve_static(const isf_params* params, const float* f_dev, float* q_dev);
ISF_API const char* isf_static_last_error(void);

/* ---- adjoint (reverse mode; the reference has no derivatives) -----------
 * Each isf_adj_* call maps the cotangent of an operator's output to that of
 * its input at the forward input passed (psi as 4 reals per cell: for every
 * complex component the cotangent holds dL/dRe, dL/dIm).  Cotangent arrays
 * are updated in place.  What is differentiated is the reference's own
 * arithmetic: the angle's branch cut, the unnormalised staggered weights'
 * jumps at cell faces and the death of particles leaving the box carry no
 * derivative, so the derivative exists almost everywhere.  The projected
 * velocity does not change under a phase common to both components of psi
 * (a gauge), so the jet kvec / omega and such phases have zero gradient
 * almost everywhere. */

/* schroedinger_flow! transpose (src/parallel.jl:176-187): the flow with conj(mask) */
ISF_API int isf_adj_schroedinger_flow(isf_handle* h, float* psibar);
/* normalize_psi (src/parallel.jl:162-165) at psi_in */
ISF_API int isf_adj_normalize_psi(isf_handle* h, const float* psi_in, float* psibar);
/* pressure_project! (src/parallel.jl:155-160) at psi_in */
ISF_API int isf_adj_pressure_project(isf_handle* h, const float* psi_in, float* psibar);
/* restrict_velocity! (src/particles.jl:12-27) at psi_in; jetbar = cotangents
 * of (kvec[0], kvec[1], kvec[2], omgterm) */
ISF_API int isf_adj_restrict_velocity(isf_handle* h, const float* psi_in, float* psibar, const float kvec[3],
                                      const uint8_t* jetmask_dev, const float cen[3], float len, float rad,
                                      float omgterm, int32_t phase_mode, double jetbar[4]);
/* velocity_one_form!(isf, psi, hbar) [+ staggered sharp] (src/parallel.jl:115-122,
 * examples/benchmark.jl:61-63): consumes the handle's velocity cotangent
 * (from isf_adj_staggered_advect or isf_adj_set_velocity_bar), adds into
 * psibar and clears it */
ISF_API int isf_adj_velocity_one_form(isf_handle* h, const float* psi, float hbar, int32_t sharp, float* psibar);
/* staggered_advect! (src/parallel.jl:197-261) from `particles` with the
 * handle's current velocity: particles_bar (after -> before, in place); the
 * velocity cotangent is added into the handle's */
ISF_API int isf_adj_staggered_advect(isf_handle* h, const float* particles, float* particles_bar, int64_t np);
/* the handle's velocity cotangent as / from AoS float3 per cell */
ISF_API int isf_adj_get_velocity_bar(isf_handle* h, float* vel_aos_dev);
ISF_API int isf_adj_set_velocity_bar(isf_handle* h, const float* vel_aos_dev);
/* One whole isf_step, reversed at (psi_in, particles_in): psibar and
 * particles_bar go from after the step to before it; jetbar = cotangents of
 * (kvec[0..2], omega_t).  Recomputes the step's forward internally. */
ISF_API int isf_adj_step(isf_handle* h, const float* psi_in, const float* particles_in, int64_t np,
                         const isf_step_args* args, float* psibar, float* particles_bar, double jetbar[4]);

/* A jet run whose particle loss is differentiated by isf_adj_gradient:
 * psi0 -> init_iters x (restrict_velocity! at omega t = 0, pressure_project!)
 * (examples/benchmark.jl:28-31) -> nsteps jet steps n = 1.. with
 * omega_t = Float32(omega * Float32(n dt)) and no emission ->
 * L = sum over particles alive at the end of |x - target|^2. */
typedef struct isf_adj_problem {
    int32_t nsteps;
    int32_t checkpoint_every;  /* psi kept every k steps; the others are recomputed in the reverse pass */
    int32_t init_iters;
    int32_t phase_mode;        /* ISF_PHASE_* */
    float kvec[3];
    float omega;
    float nozzle_cen[3];
    float nozzle_len;
    float nozzle_rad;
} isf_adj_problem;

/* L only (the forward of isf_adj_gradient) */
ISF_API int isf_adj_loss(isf_handle* h, const isf_adj_problem* p, const float* psi0, const float* particles0,
                         int64_t np, const float* targets, double* loss);
/* L and its gradient: psibar0 (N float4), particles_bar0 (np float3),
 * jetbar = dL/d(kvec[0], kvec[1], kvec[2], omega).  Device arrays; psi0 and
 * particles0 are not modified. */
ISF_API int isf_adj_gradient(isf_handle* h, const isf_adj_problem* p, const float* psi0, const float* particles0,
                             int64_t np, const float* targets, double* loss, float* psibar0, float* particles_bar0,
                             double jetbar[4]);

/* ---- batched ensemble (no single counterpart in the reference: many
 * independent ISF{...} instances of uneven grid sizes, each driven by the
 * simloop of examples/benchmark.jl:46-65, stepped together on one GPU) ------
 *
 * Simulations with the same grid_res, physical_size, hbar, dt, nslots, jet
 * flag and emission count share a class; every pass of a step is one launch
 * per class, and one step of the whole batch is one CUDA graph (replayed per
 * step) whose class branches run concurrently.  Step k of simulation i is
 * exactly isf_step on that simulation's psi and particles with
 *   omega_t    = Float32(omega * Float32(k * dt))   (every product in float),
 *   emit_start = (k-1) * emit_per_step mod nslots,  counter = k,
 *   the other isf_step_args fields from its isf_sim_desc (jetmask NULL).
 * The batch owns all state; psi starts at 0 and every particle slot dead. */
typedef struct isf_batch isf_batch;

typedef struct isf_sim_desc {
    int32_t grid_res[3];
    int32_t physical_size[3];
    float hbar, dt;
    int64_t nslots;           /* particle slots (0: no particles) */
    int32_t jet;              /* 0: plain step (one projection); 1: jet step */
    int32_t phase_mode;       /* ISF_PHASE_* */
    float kvec[3];            /* jet_velocity / hbar */
    float omega;              /* jet frequency: phase k.x - omega t */
    float nozzle_cen[3];
    float nozzle_len, nozzle_rad;
    int32_t emit_mode;        /* ISF_EMIT_* */
    int64_t emit_per_step;    /* particles emitted per jet step (<= nslots) */
    uint64_t seed;            /* Philox key of the emission */
} isf_sim_desc;

/* pass kinds with an autotuned tile (pencil groups per CTA, 1, 2 or 4) */
enum {
    ISF_TILE_X_PSI = 0,   /* x passes of psi */
    ISF_TILE_X_REAL = 1,  /* real-to-complex / complex-to-real x passes of the Poisson solve */
    ISF_TILE_Y_PSI = 2,   /* y passes of psi */
    ISF_TILE_Z_PSI = 3,   /* z pass of psi with the Schroedinger phase */
    ISF_TILE_Y_HALF = 4,  /* y passes of the Poisson half spectrum */
    ISF_TILE_Z_HALF = 5,  /* z pass of the half spectrum with the inverse Laplacian */
    ISF_TILE_KINDS = 6
};

/* Allocate and set up nsims simulations on `device`; tune != 0 runs the tile
 * autotuner per class (otherwise every tile is 1).  Errors of a failed
 * create: isf_batch_last_error(NULL). */
ISF_API int isf_batch_create(const isf_sim_desc* sims, int32_t nsims, int32_t device, int32_t tune, isf_batch** out);
ISF_API int isf_batch_destroy(isf_batch* b);
ISF_API const char* isf_batch_last_error(const isf_batch* b);
/* Copy simulation sim's psi (N float4) or particles (nslots float3) in or out;
 * the pointer may be host or device memory.  Synchronous. */
ISF_API int isf_batch_set_psi(isf_batch* b, int32_t sim, const float* psi);
ISF_API int isf_batch_get_psi(isf_batch* b, int32_t sim, float* psi);
ISF_API int isf_batch_set_particles(isf_batch* b, int32_t sim, const float* particles);
ISF_API int isf_batch_get_particles(isf_batch* b, int32_t sim, float* particles);
/* Device pointers of simulation sim's psi and particles (owned by the batch). */
ISF_API int isf_batch_state(isf_batch* b, int32_t sim, float** psi, float** particles);
/* The jet initialisation of examples/benchmark.jl:28-31 for every jet simulation:
 * iters x (restrict_velocity! at omega t = 0, pressure_project!). */
ISF_API int isf_batch_init_jet(isf_batch* b, int32_t iters);
/* nsteps whole time steps of every simulation (asynchronous). */
ISF_API int isf_batch_step(isf_batch* b, int32_t nsteps);
/* Set the step counter (the number of the last completed step; 0 after create). */
ISF_API int isf_batch_set_step(isf_batch* b, int64_t step);
ISF_API int isf_batch_get_stream(const isf_batch* b, void** stream);
ISF_API int isf_batch_sync(isf_batch* b);

/* The persistent batch kernel.  With mode ISF_PERSIST_ON, isf_batch_step(b,
 * k) runs all k ensemble steps as one launch of one persistent kernel
 * (captured in a CUDA graph per k, after a zeroing of its work counters).
 * Its blocks take work items in order from one counter: an item is a few
 * CTAs' worth of one pass of one class (the passes of isf_step, the same
 * arithmetic, so results are bitwise those of the per-step graph and of
 * isf_step).  A pass waits on the device, per simulation, for the pass
 * before it in its class's chain (and a few passes for one of the previous
 * step, so that a step's advection overlaps the next step's psi passes)
 * with a bounded poll: after spin_limit polls (<= 0: the
 * default, 2^22, about a second) the kernel records ISF_ERR_TIMEOUT, every
 * block stops at its next item, and isf_batch_sync returns ISF_ERR_TIMEOUT
 * naming the pass; the state is then partly stepped.  ISF_PERSIST_STALL adds
 * a wait on a flag that nothing sets to every dependent pass, so the timeout
 * path can be exercised without a fault.  Needs every class to have nx in
 * {16,32,48,64,96,128} and ny = nz in {32,48,64,96}, and at most 255 passes
 * per ensemble step in all (about a dozen classes; ISF_ERR_INVALID
 * otherwise).  Mode 0 returns to the per-step graph.  Reference: the
 * ensemble is new; each simulation's step is examples/benchmark.jl:46-65. */
enum { ISF_PERSIST_ON = 1, ISF_PERSIST_STALL = 2 };
ISF_API int isf_batch_set_persistent(isf_batch* b, int32_t mode, int64_t spin_limit);
/* number of classes, and the class of every simulation (nsims entries, may be NULL) */
ISF_API int isf_batch_info(const isf_batch* b, int32_t* nclasses, int32_t* sim_class);
/* the autotuned tile of each pass kind (ISF_TILE_*) of class cls */
ISF_API int isf_batch_tiles(const isf_batch* b, int32_t cls, int32_t tiles[6]);
/* [0] clamp events, [1] live particles of simulation sim's advections since the last reset */
ISF_API int isf_batch_counters(isf_batch* b, int32_t sim, uint64_t out[2], int32_t reset);

/* ---- tracing (no reference counterpart beyond @time, examples/benchmark.jl:70) */

/* Per-launch-site CUDA-event timing: between start and stop every kernel
 * launch of h is bracketed by an event pair on h's stream; stop synchronises
 * and accumulates the elapsed time per launch site (e.g. "proj y fwd"). */
ISF_API int isf_profile_start(isf_handle* h);
ISF_API int isf_profile_stop(isf_handle* h);
ISF_API int isf_profile_sites(const isf_handle* h, int32_t* n);
ISF_API int isf_profile_get(const isf_handle* h, int32_t i, char* name, size_t cap, double* total_ms,
                            int64_t* launches);
/* kernels launched by h since isf_create */
ISF_API int isf_launch_count(const isf_handle* h, uint64_t* out);

/* ---- FP64 structure-of-arrays front-end (src/MatlabPort.jl)
 *
 * MatlabPort.jl is the reference's second formulation of the same operators
 * (MatlabPort.jl:38-273): separate Complex{Float64} arrays psi1 and psi2,
 * Float64 velocity components vx, vy, vz and scalar fields, all column-major
 * with x fastest, and a Particles type holding Float32 x, y, z vectors and a
 * list of active slots.  These entry points convert between that layout and
 * the handle's FP32 layouts on the device, so the MatlabPort API runs on the
 * kernels above (FP32 arithmetic inside).  Complex128 arrays are interleaved
 * (re, im) and 16-byte aligned; slot lists are int64, 0-based, at most
 * 2^31 - 1 long, and their slots distinct.  A slot outside [0, nslots) is
 * skipped and counted in counter [12] (isf_counters). */

/* psi (float4 per cell) from / to psi1, psi2 (complex128 per cell) */
ISF_API int isf_psi_from_f64(isf_handle* h, const double* psi1, const double* psi2, float* psi);
ISF_API int isf_psi_to_f64(isf_handle* h, const float* psi, double* psi1, double* psi2);
/* the handle's velocity from / to vx, vy, vz (float64 per cell) */
ISF_API int isf_velocity_from_f64(isf_handle* h, const double* vx, const double* vy, const double* vz);
ISF_API int isf_velocity_to_f64(isf_handle* h, double* vx, double* vy, double* vz);
/* dst[i] = (float)(scale * src[i * stride]), i < n: a real field, or the real
 * (src) or imaginary (src + 1) part of a complex128 array with stride 2 */
ISF_API int isf_real_from_f64(isf_handle* h, const double* src, int64_t stride, double scale, float* dst, int64_t n);
/* dst[i] = (double)src[i], i < n */
ISF_API int isf_real_to_f64(isf_handle* h, const float* src, double* dst, int64_t n);
/* dst[i] = re[i] + i im[i] as complex128, i < n (im may be NULL: 0) */
ISF_API int isf_complex_to_f64(isf_handle* h, const float* re, const float* im, double* dst, int64_t n);
/* psi .= gauge_transform.(psi, q) with complex q = q_re + i q_im (q_im may be
 * NULL): psi * exp(-i q) per cell        src/parallel.jl:125-129
 * (GaugeTransform of MatlabPort.jl:139-144 multiplies by exp(+i q): pass -q) */
ISF_API int isf_gauge_transform(isf_handle* h, float* psi, const float* q_re, const float* q_im);
/* isf_add_particles into x, y, z vectors (the slots of a Particles) */
ISF_API int isf_add_particles_soa(isf_handle* h, float* x, float* y, float* z, int64_t nslots, int64_t start,
                                  int64_t count, const float cen[3], float len, float rad, uint64_t seed,
                                  uint64_t counter, int32_t mode);
/* StaggeredVelocity(px, py, pz, torus, vx, vy, vz) at n points on the
 * handle's velocity                       src/MatlabPort.jl:238-273 */
ISF_API int isf_staggered_velocity(isf_handle* h, const float* x, const float* y, const float* z, int64_t n,
                                   float* ux, float* uy, float* uz);
/* StaggeredAdvect(p, torus, vx, vy, vz, dt) on the handle's velocity: RK4
 * for the slots active[0..n) (NULL: slots 0..n-1) with no box test; points
 * wrap by mod inside the interpolation only   src/MatlabPort.jl:200-222 */
ISF_API int isf_advect_active(isf_handle* h, float* x, float* y, float* z, int64_t nslots, const int64_t* active,
                              int64_t n, float dt);
/* removethedead! (examples/matlabport/simple.jl:67-74): the slots of
 * active[0..n) (NULL: 0..n-1) whose position is strictly inside the box, in
 * order, into out_active; their number into *out_n, a device int64.
 * out_active must not overlap active. */
ISF_API int isf_keep_inside(isf_handle* h, const float* x, const float* y, const float* z, int64_t nslots,
                            const int64_t* active, int64_t n, int64_t* out_active, int64_t* out_n);
/* Keep(particle, ind): ox[i] = x[ind[i]] etc., i < n   src/MatlabPort.jl:228-233
 * (a slot outside [0, nslots) gives -1) */
ISF_API int isf_gather_particles(isf_handle* h, const float* x, const float* y, const float* z, int64_t nslots,
                                 const int64_t* ind, int64_t n, float* ox, float* oy, float* oz);

#ifdef __cplusplus
}
#endif
#endif /* ISF_H */
