// Particle kernels: seeded emission (add_particles!) and RK4 advection on the
// staggered velocity (staggered_advect!).
#include <cstdlib>
#include <type_traits>

#include "isf_launch.h"
#include "isf_particles.cuh"

namespace isf {

// Particles of slot array(s) parts; a batch launch (emits != null) handles
// simulation s = blockIdx.y with emits[s] and its own slots parts + s * 3 * nslots.
__global__ void k_emit(float* __restrict__ parts, long long nslots, long long start, long long count, EmitArgs e,
                       const EmitState* __restrict__ emits) {
    pdl_enter();
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= count) return;
    if (emits) {
        const EmitState& st = emits[blockIdx.y];
        e = st.e;
        start = st.start;
        parts += blockIdx.y * 3 * nslots;
    }
    const float3 p = emit_point(j, e);
    long long s = (start + j) % nslots;
    parts[3 * s + 0] = p.x;
    parts[3 * s + 1] = p.y;
    parts[3 * s + 2] = p.z;
}

// the same stream into separate x, y, z vectors (the Particles type of MatlabPort.jl:178-196)
__global__ void k_emit_soa(float* __restrict__ x, float* __restrict__ y, float* __restrict__ z, long long nslots,
                           long long start, long long count, EmitArgs e) {
    pdl_enter();
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= count) return;
    const float3 p = emit_point(j, e);
    const long long s = (start + j) % nslots;
    x[s] = p.x;
    y[s] = p.y;
    z[s] = p.z;
}

// staggered_advect! (parallel.jl:197-216, 248-261): classical RK4 for every
// slot inside the open box 0 < p < L, (-1,-1,-1) otherwise (a slot that holds
// (-1,-1,-1) already is not stored again).
// counters[0] accumulates clamp events, counters[1] live particles.
// A batch launch advects simulation s = blockIdx.y: slots parts + s * 3 np,
// velocity vel + s * bs_vel, counters + s * kCounterStride.
// With `order` (a permutation of the np slots, cell-sorted by k_order_*),
// thread t advects slot order[t]: the arithmetic of every slot is the same,
// only the traversal changes.  FIDX: a padded grid of at most 2^24 cells
// (the base cell index formed in float).
// ISF_ADV_MINB: resident CTAs per SM the advection is compiled for (caps its
// registers; 0: ptxas chooses).  At 5 (48 registers, no spills) it runs 409
// instructions per particle against 427 at the 56 ptxas picks alone.
#ifndef ISF_ADV_MINB
#define ISF_ADV_MINB 5
#endif
#if ISF_ADV_MINB > 0
#define ISF_ADV_BOUNDS __launch_bounds__(256, ISF_ADV_MINB)
#else
#define ISF_ADV_BOUNDS __launch_bounds__(256)
#endif
template <bool POW2, bool NORMW, bool FIDX, bool ORD>
__global__ void ISF_ADV_BOUNDS k_advect(Grid g, float* __restrict__ parts, int np,
                                                const float* __restrict__ vel,
                                                unsigned long long* __restrict__ counters, long long bs_vel,
                                                const int* __restrict__ order) {
    pdl_enter();
    const int sim = blockIdx.y;
    parts += sim * 3LL * np;
    if (counters) counters += sim * kCounterStride;
    const AdvConst kc = adv_const(g, vel + sim * bs_vel);
    unsigned clamps = 0, live = 0;
    unsigned long long* chk = counters ? counters + 2 : nullptr;  // ISF_CHECK records
    const float dt = g.dt, s6 = g.dt / 6.0f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x)
        advect_slot<POW2, NORMW, CtaBar, FIDX>(kc, parts, ORD ? __ldg(order + t) : t, dt, s6, clamps, live, chk);
    if (counters) {
        // block-aggregated counters: one atomic per CTA and counter
        __shared__ unsigned red[2][8];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            clamps += __shfl_down_sync(0xffffffffu, clamps, o);
            live += __shfl_down_sync(0xffffffffu, live, o);
        }
        if ((threadIdx.x & 31) == 0) {
            red[0][threadIdx.x >> 5] = clamps;
            red[1][threadIdx.x >> 5] = live;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long c = 0, l = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                c += red[0][w];
                l += red[1][w];
            }
            if (c) atomicAdd(&counters[0], c);
            if (l) atomicAdd(&counters[1], l);
        }
    }
}

// ---- the Particles type of MatlabPort.jl (x, y, z vectors and a list of
// active slots) on the same interpolation

// block-aggregated counter increments: one atomic per CTA
__device__ __forceinline__ void block_add(unsigned long long* ctr, unsigned v) {
    __shared__ unsigned red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        if (t) atomicAdd(ctr, t);
    }
    __syncthreads();
}

// StaggeredAdvect (MatlabPort.jl:200-222): RK4 for the slots active[j]
// (j < n; slot j itself when active is null) with no box test, sample points
// wrapped by mod inside the interpolation.  Slots outside [0, nslots) are
// skipped and counted in counters[12]; counters[0] accumulates clamp events,
// counters[1] advected slots.
template <bool POW2, bool NORMW>
__global__ void __launch_bounds__(256) k_advect_active(Grid g, float* __restrict__ x, float* __restrict__ y,
                                                       float* __restrict__ z, long long nslots,
                                                       const long long* __restrict__ active, long long n, float dt,
                                                       const float* __restrict__ vel,
                                                       unsigned long long* __restrict__ counters) {
    pdl_enter();
    const AdvConst kc = adv_const(g, vel);
    unsigned clamps = 0, moved = 0, bad = 0;
    unsigned long long* chk = counters + 2;
    const float s6 = dt / 6.0f;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const long long k = active ? active[j] : j;
        if (k < 0 || k >= nslots) {
            ++bad;
            continue;
        }
        ++moved;
        float3 p = make_float3(x[k], y[k], z[k]);
        const float3 k1 = stag_vel<POW2, NORMW>(kc, p, clamps, chk);
        float3 q = make_float3(p.x + k1.x * dt * 0.5f, p.y + k1.y * dt * 0.5f, p.z + k1.z * dt * 0.5f);
        const float3 k2 = stag_vel<POW2, NORMW>(kc, q, clamps, chk);
        q = make_float3(p.x + k2.x * dt * 0.5f, p.y + k2.y * dt * 0.5f, p.z + k2.z * dt * 0.5f);
        const float3 k3 = stag_vel<POW2, NORMW>(kc, q, clamps, chk);
        q = make_float3(p.x + k3.x * dt, p.y + k3.y * dt, p.z + k3.z * dt);
        const float3 k4 = stag_vel<POW2, NORMW>(kc, q, clamps, chk);
        x[k] = p.x + s6 * (k1.x + 2.f * k2.x + 2.f * k3.x + k4.x);
        y[k] = p.y + s6 * (k1.y + 2.f * k2.y + 2.f * k3.y + k4.y);
        z[k] = p.z + s6 * (k1.z + 2.f * k2.z + 2.f * k3.z + k4.z);
    }
    block_add(&counters[0], clamps);
    block_add(&counters[1], moved);
    block_add(&counters[12], bad);
}

// StaggeredVelocity (MatlabPort.jl:238-273) at n points
template <bool POW2, bool NORMW>
__global__ void __launch_bounds__(256) k_sample_vel(Grid g, const float* __restrict__ x, const float* __restrict__ y,
                                                    const float* __restrict__ z, long long n,
                                                    const float* __restrict__ vel, float* __restrict__ ux,
                                                    float* __restrict__ uy, float* __restrict__ uz,
                                                    unsigned long long* __restrict__ counters) {
    pdl_enter();
    const AdvConst kc = adv_const(g, vel);
    unsigned clamps = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const float3 u = stag_vel<POW2, NORMW>(kc, make_float3(x[j], y[j], z[j]), clamps, counters + 2);
        ux[j] = u.x;
        uy[j] = u.y;
        uz[j] = u.z;
    }
    block_add(&counters[0], clamps);
}

// Order-preserving filter of the active slots whose position is strictly
// inside the box (removethedead!, examples/matlabport/simple.jl:67-74, with
// the open-box test of its isinside): per-block counts, one scan, scatter.
constexpr int KEEP_T = 256, KEEP_V = 4, KEEP_ITEMS = KEEP_T * KEEP_V;

__device__ __forceinline__ bool keep_item(const float* x, const float* y, const float* z, long long nslots,
                                          const long long* active, long long n, long long j, float L0, float L1,
                                          float L2, long long* slot) {
    if (j >= n) return false;
    const long long k = active ? active[j] : j;
    *slot = k;
    if (k < 0 || k >= nslots) return false;
    const float px = x[k], py = y[k], pz = z[k];
    return (px > 0.f && px < L0) && (py > 0.f && py < L1) && (pz > 0.f && pz < L2);
}

__global__ void __launch_bounds__(KEEP_T) k_keep_count(const float* __restrict__ x, const float* __restrict__ y,
                                                       const float* __restrict__ z, long long nslots,
                                                       const long long* __restrict__ active, long long n, float L0,
                                                       float L1, float L2, unsigned* __restrict__ counts) {
    pdl_enter();
    const long long base = (long long)blockIdx.x * KEEP_ITEMS + (long long)threadIdx.x * KEEP_V;
    unsigned c = 0;
    long long slot;
#pragma unroll
    for (int v = 0; v < KEEP_V; ++v) c += keep_item(x, y, z, nslots, active, n, base + v, L0, L1, L2, &slot) ? 1u : 0u;
    __shared__ unsigned red[KEEP_T / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < KEEP_T / 32; ++w) t += red[w];
        counts[blockIdx.x] = t;
    }
}

// exclusive scan of nb block counts in place (one CTA of 1024 threads, each
// summing a contiguous run), the total into *out_n
__global__ void __launch_bounds__(1024) k_keep_scan(unsigned* __restrict__ counts, long long nb,
                                                    long long* __restrict__ out_n) {
    pdl_enter();
    __shared__ unsigned long long part[1024];
    const long long per = (nb + 1023) / 1024;
    const long long b0 = threadIdx.x * per, b1 = min(b0 + per, nb);
    unsigned long long s = 0;
    for (long long b = b0; b < b1; ++b) s += counts[b];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // Hillis-Steele inclusive scan of the runs
        const unsigned long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0ull;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = part[threadIdx.x] - s;
    for (long long b = b0; b < b1; ++b) {
        const unsigned c = counts[b];
        counts[b] = (unsigned)run;
        run += c;
    }
    if (threadIdx.x == 1023) *out_n = (long long)part[1023];
}

__global__ void __launch_bounds__(KEEP_T) k_keep_scatter(const float* __restrict__ x, const float* __restrict__ y,
                                                         const float* __restrict__ z, long long nslots,
                                                         const long long* __restrict__ active, long long n, float L0,
                                                         float L1, float L2, const unsigned* __restrict__ offsets,
                                                         long long* __restrict__ out) {
    pdl_enter();
    const long long base = (long long)blockIdx.x * KEEP_ITEMS + (long long)threadIdx.x * KEEP_V;
    bool f[KEEP_V];
    long long slot[KEEP_V];
    unsigned c = 0;
#pragma unroll
    for (int v = 0; v < KEEP_V; ++v) {
        f[v] = keep_item(x, y, z, nslots, active, n, base + v, L0, L1, L2, &slot[v]);
        c += f[v] ? 1u : 0u;
    }
    // exclusive prefix of c over the block: warp inclusive scan, then warp totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    __shared__ unsigned wsum[KEEP_T / 32];
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    unsigned wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += wsum[w];
    long long pos = (long long)offsets[blockIdx.x] + wbase + inc - c;
#pragma unroll
    for (int v = 0; v < KEEP_V; ++v)
        if (f[v]) out[pos++] = slot[v];
}

// Keep(particle, ind) (MatlabPort.jl:228-233): o[i] = p[ind[i]]; an index
// outside [0, nslots) gives (-1, -1, -1) and is counted in counters[12]
__global__ void __launch_bounds__(256) k_gather3(const float* __restrict__ x, const float* __restrict__ y,
                                                 const float* __restrict__ z, long long nslots,
                                                 const long long* __restrict__ ind, long long n,
                                                 float* __restrict__ ox, float* __restrict__ oy,
                                                 float* __restrict__ oz, unsigned long long* __restrict__ counters) {
    pdl_enter();
    unsigned bad = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const long long k = ind[j];
        const bool ok = k >= 0 && k < nslots;
        bad += ok ? 0u : 1u;
        ox[j] = ok ? x[k] : -1.f;
        oy[j] = ok ? y[k] : -1.f;
        oz[j] = ok ? z[k] : -1.f;
    }
    block_add(&counters[12], bad);
}

// ---- cell order of the particle slots: the traversal of k_advect.
// A slot's key is the 2 x 2 x 2 cell tile holding it (tiles x fastest), or
// nkeys - 1 for a slot outside the open box (dead), so live particles come
// out grouped by tile and the dead ones last.  Counting sort: k_order_count
// takes each slot's rank within its key with an atomic (the order inside a
// key is whatever the atomics give; every slot still appears exactly once),
// an exclusive scan turns the key counts into offsets, k_order_scatter
// places each slot.
__device__ __forceinline__ int order_key(const OrderGeom& o, const float* __restrict__ parts, int s) {
    const float x = parts[3 * s], y = parts[3 * s + 1], z = parts[3 * s + 2];
    const bool inside = (x > 0.f && x < o.L[0]) && (y > 0.f && y < o.L[1]) && (z > 0.f && z < o.L[2]);
    if (!inside) return o.nkeys - 1;
    const int cx = min((int)(x * o.dinv[0]), o.n[0] - 1) >> 1;
    const int cy = min((int)(y * o.dinv[1]), o.n[1] - 1) >> 1;
    const int cz = min((int)(z * o.dinv[2]), o.n[2] - 1) >> 1;
    return cx + o.t[0] * (cy + o.t[1] * cz);
}

__global__ void __launch_bounds__(256) k_order_count(OrderGeom o, const float* __restrict__ parts, int np,
                                                     unsigned* __restrict__ hist, unsigned* __restrict__ rank) {
    pdl_enter();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < np; s += gridDim.x * blockDim.x)
        rank[s] = atomicAdd(&hist[order_key(o, parts, s)], 1u);
}

__global__ void __launch_bounds__(256) k_order_scatter(OrderGeom o, const float* __restrict__ parts, int np,
                                                       const unsigned* __restrict__ offs,
                                                       const unsigned* __restrict__ rank, int* __restrict__ order) {
    pdl_enter();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < np; s += gridDim.x * blockDim.x)
        order[offs[order_key(o, parts, s)] + rank[s]] = s;
}

// exclusive scan of n counts in place, in tiles of SCAN_ITEMS: per-tile sums,
// a scan of the sums (k_keep_scan), then each tile's scan plus its offset
constexpr int SCAN_T = 1024, SCAN_V = 4, SCAN_ITEMS = SCAN_T * SCAN_V;

__device__ __forceinline__ unsigned block_exclusive(unsigned v) {
    __shared__ unsigned wsum[SCAN_T / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const unsigned w = wsum[lane];
        unsigned wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        wsum[lane] = wi - w;
    }
    __syncthreads();
    return wsum[warp] + inc - v;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(const unsigned* __restrict__ a, long long n,
                                                       unsigned* __restrict__ sums) {
    pdl_enter();
    const long long base = (long long)blockIdx.x * SCAN_ITEMS + (long long)threadIdx.x * SCAN_V;
    unsigned v = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k)
        if (base + k < n) v += a[base + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __shared__ unsigned red[SCAN_T / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned t = red[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(SCAN_T) k_scan_apply(unsigned* __restrict__ a, long long n,
                                                       const unsigned* __restrict__ offs) {
    pdl_enter();
    const long long base = (long long)blockIdx.x * SCAN_ITEMS + (long long)threadIdx.x * SCAN_V;
    unsigned v[SCAN_V];
    unsigned t = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        v[k] = base + k < n ? a[base + k] : 0u;
        t += v[k];
    }
    unsigned run = offs[blockIdx.x] + block_exclusive(t);
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        if (base + k < n) a[base + k] = run;
        run += v[k];
    }
}

long long order_scan_tiles(long long nkeys) { return (nkeys + SCAN_ITEMS - 1) / SCAN_ITEMS; }

OrderGeom order_geom(const Grid& g) {
    OrderGeom o;
    long long nk = 1;
    for (int a = 0; a < 3; ++a) {
        o.L[a] = g.L[a];
        o.dinv[a] = g.dinv[a];
        o.n[a] = g.n[a];
        o.t[a] = (g.n[a] + 1) >> 1;
        nk *= o.t[a];
    }
    o.nkeys = (int)(nk + 1);
    return o;
}

namespace {
unsigned grid_for(long long n, int blk) {
    long long b = (n + blk - 1) / blk;
    if (b > 148LL * 64) b = 148LL * 64;
    return (unsigned)(b > 0 ? b : 1);
}
}  // namespace

cudaError_t launch_emit_soa(float* x, float* y, float* z, long long nslots, long long start, long long count,
                            const EmitArgs& e, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int blk = 256;
    return launch_pdl(k_emit_soa, dim3((unsigned)((count + blk - 1) / blk)), dim3(blk), 0, s, x, y, z, nslots, start,
                      count, e);
}

cudaError_t launch_advect_active(const Grid& g, float* x, float* y, float* z, long long nslots, const long long* active,
                                 long long n, float dt, const float* vel, unsigned long long* counters, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const dim3 grid(grid_for(n, 256));
    const bool pow2 = g.d_pow2[0] && g.d_pow2[1] && g.d_pow2[2];
    if (g.norm_w)
        return pow2 ? launch_pdl(k_advect_active<true, true>, grid, dim3(256), 0, s, g, x, y, z, nslots, active, n, dt,
                                 vel, counters)
                    : launch_pdl(k_advect_active<false, true>, grid, dim3(256), 0, s, g, x, y, z, nslots, active, n, dt,
                                 vel, counters);
    return pow2 ? launch_pdl(k_advect_active<true, false>, grid, dim3(256), 0, s, g, x, y, z, nslots, active, n, dt,
                             vel, counters)
                : launch_pdl(k_advect_active<false, false>, grid, dim3(256), 0, s, g, x, y, z, nslots, active, n, dt,
                             vel, counters);
}

cudaError_t launch_sample_velocity(const Grid& g, const float* x, const float* y, const float* z, long long n,
                                   const float* vel, float* ux, float* uy, float* uz, unsigned long long* counters,
                                   cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const dim3 grid(grid_for(n, 256));
    const bool pow2 = g.d_pow2[0] && g.d_pow2[1] && g.d_pow2[2];
    if (g.norm_w)
        return pow2 ? launch_pdl(k_sample_vel<true, true>, grid, dim3(256), 0, s, g, x, y, z, n, vel, ux, uy, uz, counters)
                    : launch_pdl(k_sample_vel<false, true>, grid, dim3(256), 0, s, g, x, y, z, n, vel, ux, uy, uz,
                                 counters);
    return pow2 ? launch_pdl(k_sample_vel<true, false>, grid, dim3(256), 0, s, g, x, y, z, n, vel, ux, uy, uz, counters)
                : launch_pdl(k_sample_vel<false, false>, grid, dim3(256), 0, s, g, x, y, z, n, vel, ux, uy, uz, counters);
}

long long keep_blocks(long long n) { return (n + KEEP_ITEMS - 1) / KEEP_ITEMS; }

cudaError_t launch_keep_inside(const Grid& g, const float* x, const float* y, const float* z, long long nslots,
                               const long long* active, long long n, unsigned* counts, long long* out,
                               long long* out_n, cudaStream_t s) {
    const long long nb = keep_blocks(n);
    if (nb == 0) return cudaMemsetAsync(out_n, 0, sizeof(long long), s);
    const float L0 = g.L[0], L1 = g.L[1], L2 = g.L[2];
    cudaError_t e = launch_pdl(k_keep_count, dim3((unsigned)nb), dim3(KEEP_T), 0, s, x, y, z, nslots, active, n, L0, L1,
                               L2, counts);
    if (e == cudaSuccess) e = launch_pdl(k_keep_scan, dim3(1), dim3(1024), 0, s, counts, nb, out_n);
    if (e == cudaSuccess)
        e = launch_pdl(k_keep_scatter, dim3((unsigned)nb), dim3(KEEP_T), 0, s, x, y, z, nslots, active, n, L0, L1, L2,
                       (const unsigned*)counts, out);
    return e;
}

cudaError_t launch_gather3(const float* x, const float* y, const float* z, long long nslots, const long long* ind,
                           long long n, float* ox, float* oy, float* oz, unsigned long long* counters, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    return launch_pdl(k_gather3, dim3(grid_for(n, 256)), dim3(256), 0, s, x, y, z, nslots, ind, n, ox, oy, oz,
                      counters);
}

cudaError_t launch_emit(float* parts, long long nslots, long long start, long long count, const EmitArgs& e,
                        cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int blk = 256;
    return launch_pdl(k_emit, dim3((unsigned)((count + blk - 1) / blk)), dim3(blk), 0, s, parts, nslots, start, count, e,
                      (const EmitState*)nullptr);
}

cudaError_t launch_emit_batch(float* parts, long long nslots, long long count, int nsim, const EmitState* emits,
                              cudaStream_t s) {
    if (count <= 0 || nsim <= 0) return cudaSuccess;
    if (count > nslots || !emits) return cudaErrorInvalidValue;
    const int blk = 256;
    const dim3 grid((unsigned)((count + blk - 1) / blk), (unsigned)nsim);
    return launch_pdl(k_emit, grid, dim3(blk), 0, s, parts, nslots, 0LL, count, EmitArgs{}, emits);
}

#ifndef ISF_ADVECT_WAVES
#define ISF_ADVECT_WAVES 1
#endif

cudaError_t launch_advect(const Grid& g, float* parts, long long np, const float* vel, unsigned long long* counters,
                          cudaStream_t s, int nsim, long long bs_vel, const int* order) {
    if (np <= 0 || nsim <= 0) return cudaSuccess;
    if (np > kMaxParticles) return cudaErrorInvalidValue;
    const int blk = 256;
    // ISF_ADVECT_WAVES resident waves (0: one CTA per 256 slots), grid-stride over the slots
    static int resident = 0;  // CTAs per SM of either instantiation (the same registers)
    if (resident == 0) {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_advect<false, false, true, false>, blk, 0) !=
                cudaSuccess ||
            per < 1)
            return cudaErrorInvalidValue;
        resident = sms * per;
    }
    long long b = (np + blk - 1) / blk;
    if (ISF_ADVECT_WAVES > 0 && b > (long long)ISF_ADVECT_WAVES * resident) b = (long long)ISF_ADVECT_WAVES * resident;
    const dim3 grid((unsigned)b, (unsigned)nsim);
    const bool pow2 = g.d_pow2[0] && g.d_pow2[1] && g.d_pow2[2];
    // the float base-cell index needs the padded grid below 2^24 cells; the
    // environment variable ISF_ADVECT_INT_INDEX (read once) forces the
    // integer index, so tests can compare the two paths on one grid
    static const bool force_int = std::getenv("ISF_ADVECT_INT_INDEX") != nullptr;
    const bool fidx = !force_int && g.NP <= (1LL << 24);
    auto go = [&](auto kernel) {
        return launch_pdl(kernel, grid, dim3(blk), 0, s, g, parts, (int)np, vel, counters, bs_vel, order);
    };
    // the traversal through a slot permutation is its own instantiation, so
    // the storage-order loop carries no test of it
    auto pick = [&](auto p2, auto nw) {
        constexpr bool P2 = decltype(p2)::value, NW = decltype(nw)::value;
        if (order) return fidx ? go(k_advect<P2, NW, true, true>) : go(k_advect<P2, NW, false, true>);
        return fidx ? go(k_advect<P2, NW, true, false>) : go(k_advect<P2, NW, false, false>);
    };
    using T = std::true_type;
    using F = std::false_type;
    if (g.norm_w) return pow2 ? pick(T(), T()) : pick(F(), T());
    return pow2 ? pick(T(), F()) : pick(F(), F());
}

cudaError_t launch_order_count(const Grid& g, const float* parts, long long np, const OrderBufs& b, cudaStream_t s) {
    if (np <= 0) return cudaSuccess;
    if (np > kMaxParticles) return cudaErrorInvalidValue;
    const OrderGeom o = order_geom(g);
    cudaError_t e = cudaMemsetAsync(b.hist, 0, sizeof(unsigned) * (size_t)o.nkeys, s);
    if (e != cudaSuccess) return e;
    return launch_pdl(k_order_count, dim3(grid_for(np, 256)), dim3(256), 0, s, o, parts, (int)np, b.hist, b.rank);
}

cudaError_t launch_order_scan(const Grid& g, const OrderBufs& b, cudaStream_t s) {
    const OrderGeom o = order_geom(g);
    const long long ntiles = order_scan_tiles(o.nkeys);
    cudaError_t e = launch_pdl(k_scan_tiles, dim3((unsigned)ntiles), dim3(SCAN_T), 0, s, (const unsigned*)b.hist,
                               (long long)o.nkeys, b.sums);
    if (e == cudaSuccess) e = launch_pdl(k_keep_scan, dim3(1), dim3(1024), 0, s, b.sums, ntiles, b.total);
    if (e == cudaSuccess)
        e = launch_pdl(k_scan_apply, dim3((unsigned)ntiles), dim3(SCAN_T), 0, s, b.hist, (long long)o.nkeys,
                       (const unsigned*)b.sums);
    return e;
}

cudaError_t launch_order_scatter(const Grid& g, const float* parts, long long np, const OrderBufs& b,
                                 cudaStream_t s) {
    if (np <= 0) return cudaSuccess;
    const OrderGeom o = order_geom(g);
    return launch_pdl(k_order_scatter, dim3(grid_for(np, 256)), dim3(256), 0, s, o, parts, (int)np,
                      (const unsigned*)b.hist, (const unsigned*)b.rank, b.order);
}

long long order_keys(const Grid& g) { return order_geom(g).nkeys; }
long long order_sums(const Grid& g) { return order_scan_tiles(order_geom(g).nkeys); }

}  // namespace isf
