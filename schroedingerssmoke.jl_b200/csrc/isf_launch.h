// Host-side launchers of the ISF kernels (internal to libisf).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/isf.h"
#include "isf_common.cuh"

namespace isf {

// Launch with programmatic stream serialization: the kernel (which must call
// pdl_enter before touching global memory) may be scheduled while the
// previous kernel on the stream drains.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// grid set-up shared by isf_create and the allocation-free entry points (isf_abi.cu)
bool check_params(const isf_params* p, std::string& why);
bool valid_grid(const int n[3], std::string& why);
int half_spectrum_row(int nx);
size_t table_bytes(const int n[3]);
void fill_grid(const int n[3], const int L[3], float hbar, float dt, Grid& g, std::vector<char>& host);
void bind_tables(Grid& g, const char* dev_tables);

struct XArgs;
struct YZArgs;

bool supported_len(int n);
// a tile of `groups` pencil groups per CTA is available for pencil length n
bool grouped_tile_ok(int n, int groups);

cudaError_t launch_xpass(int op, const XArgs& a, cudaStream_t s);
cudaError_t launch_xreal(int op, const XArgs& a, cudaStream_t s);
cudaError_t launch_yzpass_psi(int op, const YZArgs& a, cudaStream_t s);
cudaError_t launch_yzpass_c(int op, const YZArgs& a, cudaStream_t s);
// the (y, z) plane Poisson solver of a k-major half spectrum (ny == nz in
// {32, 48, 64, 96, 128}); nsim simulations bs_F elements apart
bool plane_supported(const int n[3]);
cudaError_t launch_poisson_plane(const Grid& g, float2* F, long long bs_F, int nsim, cudaStream_t s);

// The Schroedinger z pass with TMA-staged pencils (k_ztma.cu): the storage
// of a CUtensorMap (128 bytes) describing psi, encoded for psi's address;
// err counts mbarrier waits that ran out (the CTA then returns)
struct alignas(64) CUtensorMapStorage {
    unsigned long long q[16];
};
bool zmask_tma_len(int n);
bool encode_psi_zmap(CUtensorMapStorage* out, const float* psi, const Grid& g);
// stall: null, or a counter that nothing sets, which every CTA also waits on
// after its first tile (the timeout test)
cudaError_t launch_zmask_tma(const CUtensorMapStorage& map, const YZArgs& a, long long limit, unsigned long long* err,
                             const unsigned long long* stall, cudaStream_t s);

// z-marching stencils of the one-form (k_stencil.cu)
enum StOp { ST_DIV = 0, ST_VEL = 1 };
struct StencilArgs {
    Grid g;
    const float4* psi;
    float* out;  // ST_DIV: f[N]; ST_VEL: padded velocity grid, float4 (vx, vy, vz, 0) per cell (kVelComp NP floats)
    JetArgs jet;
    int use_jet;
    float hbar;
    int sharp;
    // a batch of nsim simulations of this grid (0 or 1: a single one):
    // simulation s reads psi + s * bs_psi, writes out + s * bs_out and, with
    // jets != null, restricts with jets[s] instead of jet
    int nsim;
    long long bs_psi, bs_out;
    const JetArgs* jets;
};
cudaError_t launch_stencil(int op, const StencilArgs& a, cudaStream_t s);

// pointwise kernels (k_point.cu)
cudaError_t launch_normalize(const Grid& g, float4* psi, cudaStream_t s);
cudaError_t launch_restrict(const Grid& g, float4* psi, const JetArgs& j, cudaStream_t s);
cudaError_t launch_isjet(const Grid& g, uint8_t* out, const float* cen, float len, float rad, cudaStream_t s);
cudaError_t launch_sharp(const Grid& g, float* vel, cudaStream_t s);
cudaError_t launch_div(const Grid& g, const float* vel, float* f, cudaStream_t s);
cudaError_t launch_vel_to_aos(const Grid& g, const float* vel, float* aos, cudaStream_t s);
cudaError_t launch_vel_from_aos(const Grid& g, const float* aos, float* vel, cudaStream_t s);
cudaError_t launch_scale_c(const Grid& g, float2* a, float s, cudaStream_t st);
cudaError_t launch_count_nonfinite(const Grid& g, const float4* psi, unsigned long long* count, cudaStream_t s);

// particles (k_particles.cu); slot indices are 32-bit: 3 * np < 2^31
constexpr long long kMaxParticles = 715827882LL;
struct EmitArgs {
    float cen[3];
    float len, rad;
    uint64_t seed, counter;
    int mode;
};
// per-simulation emission of a batch: the arguments and the first ring slot
struct EmitState {
    EmitArgs e;
    long long start;
};
cudaError_t launch_emit(float* parts, long long nslots, long long start, long long count, const EmitArgs& e,
                        cudaStream_t s);
// one launch for nsim simulations: simulation s emits count particles with
// emits[s] into parts + s * 3 * nslots
cudaError_t launch_emit_batch(float* parts, long long nslots, long long count, int nsim, const EmitState* emits,
                              cudaStream_t s);
// counters: 8 entries per simulation (clamp events, live particles, check records)
constexpr int kCounterStride = 8;
// order: null (storage order) or a permutation of the np slots to traverse them in
cudaError_t launch_advect(const Grid& g, float* parts, long long np, const float* vel,
                          unsigned long long* counters, cudaStream_t s, int nsim = 1, long long bs_vel = 0,
                          const int* order = nullptr);

// Cell order of the particle slots (k_particles.cu): a permutation of the np
// slots, live ones grouped by 2 x 2 x 2 cell tile (tiles x fastest), dead
// ones last.  Three steps on one stream: count (ranks within each key), scan
// (the key counts to offsets), scatter (the permutation).
struct OrderGeom {
    float L[3], dinv[3];
    int n[3], t[3];  // cells and tiles per axis
    int nkeys;       // tiles + 1 (the dead slots' key)
};
struct OrderBufs {
    unsigned* hist;   // order_keys(g) counts, then offsets
    unsigned* rank;   // np: each slot's rank within its key
    unsigned* sums;   // order_sums(g): per-tile sums of the scan
    long long* total; // the scan's total (np)
    int* order;       // np: the permutation
};
long long order_keys(const Grid& g);
long long order_sums(const Grid& g);
cudaError_t launch_order_count(const Grid& g, const float* parts, long long np, const OrderBufs& b, cudaStream_t s);
cudaError_t launch_order_scan(const Grid& g, const OrderBufs& b, cudaStream_t s);
cudaError_t launch_order_scatter(const Grid& g, const float* parts, long long np, const OrderBufs& b,
                                 cudaStream_t s);

// the Particles type of MatlabPort.jl: x, y, z vectors and active slot lists (k_particles.cu)
cudaError_t launch_emit_soa(float* x, float* y, float* z, long long nslots, long long start, long long count,
                            const EmitArgs& e, cudaStream_t s);
// counters: [0] clamp events, [1] advected slots, [12] slots outside [0, nslots)
cudaError_t launch_advect_active(const Grid& g, float* x, float* y, float* z, long long nslots, const long long* active,
                                 long long n, float dt, const float* vel, unsigned long long* counters, cudaStream_t s);
cudaError_t launch_sample_velocity(const Grid& g, const float* x, const float* y, const float* z, long long n,
                                   const float* vel, float* ux, float* uy, float* uz, unsigned long long* counters,
                                   cudaStream_t s);
// block count of the keep-inside filter of n items (the size of its counts scratch)
long long keep_blocks(long long n);
cudaError_t launch_keep_inside(const Grid& g, const float* x, const float* y, const float* z, long long nslots,
                               const long long* active, long long n, unsigned* counts, long long* out,
                               long long* out_n, cudaStream_t s);
cudaError_t launch_gather3(const float* x, const float* y, const float* z, long long nslots, const long long* ind,
                           long long n, float* ox, float* oy, float* oz, unsigned long long* counters, cudaStream_t s);

// FP64 structure-of-arrays conversions and the complex gauge (k_soa.cu)
cudaError_t launch_psi_from_f64(const double* a, const double* b, float* psi, long long n, cudaStream_t s);
cudaError_t launch_psi_to_f64(const float* psi, double* a, double* b, long long n, cudaStream_t s);
cudaError_t launch_vel_from_f64(const Grid& g, const double* vx, const double* vy, const double* vz, float* vel,
                                cudaStream_t s);
cudaError_t launch_vel_to_f64(const Grid& g, const float* vel, double* vx, double* vy, double* vz, cudaStream_t s);
cudaError_t launch_real_from_f64(const double* src, long long stride, double scale, float* dst, long long n,
                                 cudaStream_t s);
cudaError_t launch_real_to_f64(const float* src, double* dst, long long n, cudaStream_t s);
cudaError_t launch_complex_to_f64(const float* re, const float* im, double* dst, long long n, cudaStream_t s);
cudaError_t launch_gauge_complex(float* psi, const float* qre, const float* qim, long long n, cudaStream_t s);

// adjoint kernels (k_adjoint.cu)
cudaError_t launch_gauge(const Grid& g, const float4* in, const float* q, float4* out, cudaStream_t s);
cudaError_t launch_normalize_to(const Grid& g, const float4* in, float4* out, cudaStream_t s);
cudaError_t launch_restrict_to(const Grid& g, const float4* in, float4* out, const JetArgs& j, cudaStream_t s);
cudaError_t launch_adj_normalize(const Grid& g, const float4* psi_in, float4* bar, cudaStream_t s);
cudaError_t launch_adj_gauge(const Grid& g, const float4* psi_in, const float* q, float4* bar, float* qbar,
                             cudaStream_t s);
cudaError_t launch_adj_oneform_div(const Grid& g, const float4* psi, float4* bar, const float* fbar, cudaStream_t s);
// folds the padded copies of ubar, then adds the one-form transpose (scale hbar [/ d])
cudaError_t launch_adj_oneform_vel(const Grid& g, const float4* psi, float4* bar, float* ubar, float hbar, int sharp,
                                   cudaStream_t s);
cudaError_t launch_adj_fold(const Grid& g, float* ubar, cudaStream_t s);
cudaError_t launch_adj_from_aos(const Grid& g, const float* aos, float* ubar, cudaStream_t s);
cudaError_t launch_adj_to_aos(const Grid& g, const float* ubar, float* aos, cudaStream_t s);
// acc[0..2] += cotangent of kvec, acc[3] += cotangent of omega t times wscale
cudaError_t launch_adj_restrict(const Grid& g, const float4* psi_in, float4* bar, const JetArgs& j, double* acc,
                                float wscale, cudaStream_t s);
cudaError_t launch_adj_advect(const Grid& g, const float* parts, float* lam, long long np, const float* vel,
                              float* ubar, cudaStream_t s);
cudaError_t launch_loss(const float* x, const float* y, float* lam, long long np, double* loss, cudaStream_t s);
cudaError_t launch_zero_slots(float* lam, long long nslots, long long start, long long count, cudaStream_t s);

}  // namespace isf
