// The persistent batch kernel: K steps of a whole ensemble in one launch
// (internal to libisf; the host side is in isf_batch.cu).
//
// The ensemble's classes (simulations sharing a grid, see isf_batch.cu) each
// run the pass chain of isf_step.  A phase is one pass of one class: its
// tiles are the CTAs the pass kernel would be launched with.  The kernel's
// blocks take work items, in order, from one counter; an item is `vper`
// tiles of one phase, each run by `vblk` threads of the block (a virtual CTA
// with its own named barrier).  Items are numbered step by step, and inside a
// step pass by pass with the classes interleaved, so a phase's predecessor
// in its class's chain always has smaller item numbers: a block that waits
// for it waits only on items already taken by running blocks, which never
// wait on later ones.  A phase's tiles are simulation-major and the
// simulations are independent, so completion is counted per (step, slot,
// simulation): an item waits only for the simulations its tiles belong to.  Every wait is bounded: after `spin_limit` polls the
// block records ISF_ERR_TIMEOUT, the slot and the step in the status word,
// and every block stops at its next item.
#pragma once
#include "isf_launch.h"
#include "isf_passes.cuh"

namespace isf {

// per-simulation run-time constants of a step's jet / emission arguments
struct SimRT {
    float omega, dt;
    long long count, nslots;
};

enum PKind : int {
    PK_PROLOGUE = 0,    // this step's omega t, emission counter and ring slot per simulation
    PK_X_FWD,           // schroedinger x fwd
    PK_Y_FWD,           // schroedinger y fwd
    PK_Z_MASK,          // schroedinger z fwd * mask / N, z inv
    PK_Y_INV,           // schroedinger y inv
    PK_X_INV_NORM,      // schroedinger x inv + normalize
    PK_DIV,             // projection div stencil (restricted with the step's jets when use_jet)
    PK_XR_FWD,          // projection x fwd (real, k-major half spectrum)
    PK_PLANE,           // projection (y, z) planes
    PK_XR_INV_GAUGE,    // projection x inv + gauge (restricted when use_jet)
    PK_EMIT,            // add_particles! into the step's ring slots
    PK_VEL,             // one-form stencil (hbar, sharp)
    PK_ADVECT,          // staggered_advect!
};

struct PPhase {
    int kind, cls;
    int len;            // pencil length of an FFT pass
    int vblk, vper;     // threads per virtual CTA, virtual CTAs per item
    int reps;           // tiles a virtual CTA runs one after another in an item
    int tiles, items;   // tiles of the pass, items = ceil(tiles / (vper reps))
    int gx, gy;         // tile t -> block (t % gx, (t / gx) % gy, t / (gx gy))
    int dep;            // slot of the same step this phase waits for (-1: none)
    int dep_prev;       // slot of the previous step it waits for (-1: none)
    int nsg, tps;       // completion groups (the class's simulations; 1 for the prologue) and tiles per group
    int doff;           // first completion counter of this slot within a step
    int smem_v;         // shared memory bytes of one virtual CTA
    int pow2, normw;    // advection variants
    // arguments of the pass (the member of its kind)
    XArgs x;
    YZArgs yz;
    StencilArgs st;
    PlaneArgs pl;
    Grid g;                      // PROLOGUE / EMIT / ADVECT
    int first, nsim;             // the class's simulations (class-major index of the first)
    float* parts;                // EMIT / ADVECT: nsim x 3 nslots
    long long nslots, count;     // slots per simulation, emitted per step
    const float* vel;            // ADVECT: the class's velocity grids
    long long bs_vel;
};

struct PPlan {
    const PPhase* ph;        // nslot phases, in slot order
    const int* slot_start;   // nslot + 1: first item of each slot within a step
    int nslot, items_per_step, nsteps;
    int dstride;             // completion counters per step (the slots' nsg summed)
    int tiles_per_step;      // tiles of all slots of one step
    unsigned* done;          // nsteps x dstride tiles finished per (slot, simulation) (zeroed before the launch)
    unsigned* ctl;           // [0] next item, [1] tiles finished in the last step (zeroed before the launch)
    int* status;             // [0] error code, [1] slot, [2] step, [3] a flag nothing sets (zeroed)
    long long spin_limit;    // polls of one wait before it gives up
    int stall;               // 1: the first dependent item also waits for status[3] (a timeout by construction)
    long long* step;         // the ensemble's step counter: read by the prologues, advanced by nsteps at the end
    const SimRT* rt;
    JetArgs* jets;           // class-major, one per simulation
    EmitState* emits;
    unsigned long long* counters;  // kCounterStride per simulation
};

constexpr int kPersistThreads = 256;
// slots (passes of all classes in one step) the kernel's shared slot table holds
constexpr int kPersistMaxSlots = 255;
// slots an advection thread steps per work item
constexpr int kAdvectSlots = 4;
// x pencil lengths and (y, z) plane sizes the persistent kernel is built for
bool persist_len_ok(int n);
bool persist_plane_ok(int n);
// threads and shared memory of one virtual CTA of a phase's pass
int persist_vblk(int kind, int len);
int persist_smem(int kind, int len);
// the persistent kernel's dynamic shared memory opt-in and blocks per SM
cudaError_t persist_setup(int smem_bytes, int* blocks_per_sm);
cudaError_t launch_persist(const PPlan& p, int grid, int smem_bytes, cudaStream_t s);

}  // namespace isf
