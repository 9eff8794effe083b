// Particle kernels: seeded emission (add_particles!) and RK4 advection on the
// staggered velocity (staggered_advect!).
#include "isf_launch.h"
#include "isf_particles.cuh"

namespace isf {

// Philox4x32-10 (Salmon et al., SC'11): ten rounds of two 32x32->64-bit
// multiplies, round keys bumped by the Weyl constants after each round.
struct U4 {
    uint32_t v[4];
};
__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.v[0]), lo0 = M0 * c.v[0];
        const uint32_t hi1 = __umulhi(M1, c.v[2]), lo1 = M1 * c.v[2];
        U4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// add_particles! (particles.jl:30-94) with a seeded counter-based stream.
// Stream: counter = (j, counter_lo, counter_hi, 0x15F0015F), key = seed.
// mode 0: the reference ring (0.9 r around (x - 0.1) with +-0.05 jitter,
//         particles.jl:86-90); 1: uniform in the nozzle disc at x = cen.x;
//         2: uniform in the nozzle cylinder; 3: the MatlabPort driver's ring
//         (0.9 r in the plane x = cen.x, no jitter,
//         examples/matlabport/simple.jl:112-115).
__device__ __forceinline__ float3 emit_point(long long j, const EmitArgs& e) {
    U4 c = {{(uint32_t)j, (uint32_t)e.counter, (uint32_t)(e.counter >> 32), 0x15F0015Fu}};
    const U4 r = philox4x32_10(c, (uint32_t)e.seed, (uint32_t)(e.seed >> 32));
    const float u0 = u01(r.v[0]), u1 = u01(r.v[1]), u2 = u01(r.v[2]), u3 = u01(r.v[3]);
    const float pi = 3.14159265358979323846f;
    float p0, p1, p2;
    if (e.mode == 0 || e.mode == 3) {
        const float rt = __fmul_rn(__fmul_rn(u0, 2.0f), pi);
        const float rr = __fmul_rn(0.9f, e.rad);
        if (e.mode == 3) {
            p0 = e.cen[0];
            p1 = __fadd_rn(e.cen[1], __fmul_rn(rr, cosf(rt)));
            p2 = __fadd_rn(e.cen[2], __fmul_rn(rr, sinf(rt)));
        } else {
            const float o0 = __fsub_rn(__fmul_rn(u1, 0.1f), 0.05f);
            const float o1 = __fsub_rn(__fmul_rn(u2, 0.1f), 0.05f);
            const float o2 = __fsub_rn(__fmul_rn(u3, 0.1f), 0.05f);
            p0 = __fadd_rn(__fsub_rn(e.cen[0], 0.1f), o0);
            p1 = __fadd_rn(__fadd_rn(e.cen[1], __fmul_rn(rr, cosf(rt))), o1);
            p2 = __fadd_rn(__fadd_rn(e.cen[2], __fmul_rn(rr, sinf(rt))), o2);
        }
    } else {
        const float th = __fmul_rn(__fmul_rn(u0, 2.0f), pi);
        const float rho = __fmul_rn(e.rad, sqrtf(u1));
        p0 = (e.mode == 1) ? e.cen[0] : __fadd_rn(e.cen[0], __fmul_rn(__fsub_rn(u2, 0.5f), e.len));
        p1 = __fadd_rn(e.cen[1], __fmul_rn(rho, cosf(th)));
        p2 = __fadd_rn(e.cen[2], __fmul_rn(rho, sinf(th)));
    }
    return make_float3(p0, p1, p2);
}

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

#ifdef ISF_CHECK
// debug builds: validate a gather index, record the first bad one, read cell 0
__device__ __forceinline__ int checked(const AdvConst& k, int c, unsigned long long* chk, const int i[3]) {
    if (c < 0 || (long long)c >= k.NP) {
        if (chk && atomicAdd(&chk[0], 1ull) == 0) {
            chk[1] = (unsigned long long)(unsigned)c;
            for (int a = 0; a < 3; ++a) chk[2 + a] = (unsigned long long)(unsigned)i[a];
        }
        return 0;
    }
    return c;
}
#define ISF_IDX(c) checked(k, (c), chk, i)
#else
#define ISF_IDX(c) (c)
#endif

// staggered_velocity (parallel.jl:219-246) on the handle's padded velocity
// grid: seven 16-byte gathers (the cells whose components the reference's
// twelve samples need).  Interpolation weights are the reference's unnormalised
// w = p - (i-1) d.  An index that rounds to n (p rounded up to L by mod) is
// clamped to the last cell and counted.
template <bool POW2, bool NORMW>
__device__ __forceinline__ float3 stag_vel(const AdvConst& k, float3 pt, unsigned& clamps, unsigned long long* chk) {
    float P[3] = {pt.x, pt.y, pt.z};
    // mod.(point, ph_size): identity for points inside the box (the common case)
    const bool inbox = (pt.x >= 0.f && pt.x < k.L[0]) && (pt.y >= 0.f && pt.y < k.L[1]) &&
                       (pt.z >= 0.f && pt.z < k.L[2]);
    if (!inbox) {
#pragma unroll
        for (int a = 0; a < 3; ++a) P[a] = jl_mod_box(P[a], k.L[a]);
    }
    int i[3];
    float w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // the cell floor, its clamp and the weight stay in float (integer
        // values, exact); a NaN point clamps to cell 0 as an int floor would
        float fl = cell_floor_f<POW2>(P[a], k.dinv[a], k.d[a], k.feps[a]);
        clamps += (fl > k.nmf[a]) ? 1u : 0u;  // mod rounded up to L
        fl = fminf(fmaxf(fl, 0.f), k.nmf[a]);
        i[a] = __float2int_rz(fl);
        w[a] = __fsub_rn(P[a], __fmul_rn(fl, k.d[a]));
        if (NORMW) w[a] = __fdiv_rn(w[a], k.d[a]);
    }
    (void)chk;
    // the +1 neighbour mod(i, res) + 1 is the padded plane's next cell
    const int sy = k.pnx, sz = k.pnxy;
    const int c000 = i[0] + sy * i[1] + sz * i[2];
    const int c100 = c000 + 1, c010 = c000 + sy, c001 = c000 + sz;
    // the reference's 12 samples (parallel.jl:224-234) from 7 cells
    const float4 a000 = __ldg(k.v + ISF_IDX(c000)), a100 = __ldg(k.v + ISF_IDX(c100));
    const float4 a010 = __ldg(k.v + ISF_IDX(c010)), a001 = __ldg(k.v + ISF_IDX(c001));
    const float4 a011 = __ldg(k.v + ISF_IDX(c010 + sz)), a101 = __ldg(k.v + ISF_IDX(c100 + sz));
    const float4 a110 = __ldg(k.v + ISF_IDX(c100 + sy));
    const float x00 = a000.x, x10 = a010.x, x01 = a001.x, x11 = a011.x;
    const float y00 = a000.y, y10 = a100.y, y01 = a001.y, y11 = a101.y;
    const float z00 = a000.z, z10 = a100.z, z01 = a010.z, z11 = a110.z;
    const float wx = w[0], wy = w[1], wz = w[2];
    float3 u;
    // u_x bilinear in (y, z), u_y in (x, z), u_z in (x, y) (parallel.jl:230-245)
    u.x = (1.f - wz) * ((1.f - wy) * x00 + wy * x10) + wz * ((1.f - wy) * x01 + wy * x11);
    u.y = (1.f - wz) * ((1.f - wx) * y00 + wx * y10) + wz * ((1.f - wx) * y01 + wx * y11);
    u.z = (1.f - wy) * ((1.f - wx) * z00 + wx * z10) + wy * ((1.f - wx) * z01 + wx * z11);
    return u;
}
#undef ISF_IDX

// staggered_advect! (parallel.jl:197-216, 248-261): classical RK4 for every
// slot inside the open box 0 < p < L, (-1,-1,-1) otherwise (a slot that holds
// (-1,-1,-1) already is not stored again).
// counters[0] accumulates clamp events, counters[1] live particles.
// A batch launch advects simulation s = blockIdx.y: slots parts + s * 3 np,
// velocity vel + s * bs_vel, counters + s * kCounterStride.
// With `order` (a permutation of the np slots, cell-sorted by k_order_*),
// thread t advects slot order[t]: the arithmetic of every slot is the same,
// only the traversal changes.
template <bool POW2, bool NORMW>
__global__ void __launch_bounds__(256) k_advect(Grid g, float* __restrict__ parts, int np,
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
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x) {
        const int k = order ? __ldg(order + t) : t;
        float3 p = make_float3(parts[3 * k], parts[3 * k + 1], parts[3 * k + 2]);
        const bool inside = (p.x > 0.f && p.x < kc.L[0]) && (p.y > 0.f && p.y < kc.L[1]) &&
                            (p.z > 0.f && p.z < kc.L[2]);
        if (inside) {
            ++live;
            // k2 = p .+ k1 .* dt .* 0.5f0 etc. (parallel.jl:201-212)
            const float3 k1 = stag_vel<POW2, NORMW>(kc, p, clamps, chk);
            float3 q = make_float3(p.x + k1.x * dt * 0.5f, p.y + k1.y * dt * 0.5f, p.z + k1.z * dt * 0.5f);
            const float3 k2 = stag_vel<POW2, NORMW>(kc, q, clamps, chk);
            q = make_float3(p.x + k2.x * dt * 0.5f, p.y + k2.y * dt * 0.5f, p.z + k2.z * dt * 0.5f);
            const float3 k3 = stag_vel<POW2, NORMW>(kc, q, clamps, chk);
            q = make_float3(p.x + k3.x * dt, p.y + k3.y * dt, p.z + k3.z * dt);
            const float3 k4 = stag_vel<POW2, NORMW>(kc, q, clamps, chk);
            p.x = p.x + s6 * (k1.x + 2.f * k2.x + 2.f * k3.x + k4.x);
            p.y = p.y + s6 * (k1.y + 2.f * k2.y + 2.f * k3.y + k4.y);
            p.z = p.z + s6 * (k1.z + 2.f * k2.z + 2.f * k3.z + k4.z);
        } else {
            if (p.x == -1.f && p.y == -1.f && p.z == -1.f) continue;  // dead already
            p = make_float3(-1.f, -1.f, -1.f);
        }
        parts[3 * k] = p.x;
        parts[3 * k + 1] = p.y;
        parts[3 * k + 2] = p.z;
    }
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
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_advect<false, false>, blk, 0) != cudaSuccess || per < 1)
            return cudaErrorInvalidValue;
        resident = sms * per;
    }
    long long b = (np + blk - 1) / blk;
    if (ISF_ADVECT_WAVES > 0 && b > (long long)ISF_ADVECT_WAVES * resident) b = (long long)ISF_ADVECT_WAVES * resident;
    const dim3 grid((unsigned)b, (unsigned)nsim);
    const bool pow2 = g.d_pow2[0] && g.d_pow2[1] && g.d_pow2[2];
    if (g.norm_w)
        return pow2 ? launch_pdl(k_advect<true, true>, grid, dim3(blk), 0, s, g, parts, (int)np, vel, counters, bs_vel,
                                 order)
                    : launch_pdl(k_advect<false, true>, grid, dim3(blk), 0, s, g, parts, (int)np, vel, counters, bs_vel,
                                 order);
    return pow2 ? launch_pdl(k_advect<true, false>, grid, dim3(blk), 0, s, g, parts, (int)np, vel, counters, bs_vel,
                             order)
                : launch_pdl(k_advect<false, false>, grid, dim3(blk), 0, s, g, parts, (int)np, vel, counters, bs_vel,
                             order);
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
