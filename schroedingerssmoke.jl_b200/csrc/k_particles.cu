// Particle kernels: seeded emission (add_particles!) and RK4 advection on the
// staggered velocity (staggered_advect!).
#include "isf_launch.h"

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
//         2: uniform in the nozzle cylinder.
__global__ void k_emit(float* __restrict__ parts, long long nslots, long long start, long long count, EmitArgs e) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= count) return;
    U4 c = {{(uint32_t)j, (uint32_t)e.counter, (uint32_t)(e.counter >> 32), 0x15F0015Fu}};
    const U4 r = philox4x32_10(c, (uint32_t)e.seed, (uint32_t)(e.seed >> 32));
    const float u0 = u01(r.v[0]), u1 = u01(r.v[1]), u2 = u01(r.v[2]), u3 = u01(r.v[3]);
    const float pi = 3.14159265358979323846f;
    float p0, p1, p2;
    if (e.mode == 0) {
        const float rt = __fmul_rn(__fmul_rn(u0, 2.0f), pi);
        const float o0 = __fsub_rn(__fmul_rn(u1, 0.1f), 0.05f);
        const float o1 = __fsub_rn(__fmul_rn(u2, 0.1f), 0.05f);
        const float o2 = __fsub_rn(__fmul_rn(u3, 0.1f), 0.05f);
        const float rr = __fmul_rn(0.9f, e.rad);
        p0 = __fadd_rn(__fsub_rn(e.cen[0], 0.1f), o0);
        p1 = __fadd_rn(__fadd_rn(e.cen[1], __fmul_rn(rr, cosf(rt))), o1);
        p2 = __fadd_rn(__fadd_rn(e.cen[2], __fmul_rn(rr, sinf(rt))), o2);
    } else {
        const float th = __fmul_rn(__fmul_rn(u0, 2.0f), pi);
        const float rho = __fmul_rn(e.rad, sqrtf(u1));
        p0 = (e.mode == 1) ? e.cen[0] : __fadd_rn(e.cen[0], __fmul_rn(__fsub_rn(u2, 0.5f), e.len));
        p1 = __fadd_rn(e.cen[1], __fmul_rn(rho, cosf(th)));
        p2 = __fadd_rn(e.cen[2], __fmul_rn(rho, sinf(th)));
    }
    long long s = (start + j) % nslots;
    parts[3 * s + 0] = p0;
    parts[3 * s + 1] = p1;
    parts[3 * s + 2] = p2;
}

// Julia's mod(x, y) for floats (sign of y; r + y rounded)
__device__ __forceinline__ float jl_modf(float x, float y) {
    float r = fmodf(x, y);
    if (r == 0.f) return copysignf(0.f, y);
    if ((r > 0.f) != (y > 0.f)) r += y;
    return r;
}

// staggered_velocity (parallel.jl:219-246).  Interpolation weights are the
// reference's unnormalised w = p - (i-1) d.  An index that rounds to n (p
// rounded up to L by mod) is clamped to the last cell and counted.
__device__ __forceinline__ float3 stag_vel(const Grid& g, const float* __restrict__ vx,
                                           const float* __restrict__ vy, const float* __restrict__ vz, float3 pt,
                                           unsigned& clamps) {
    const float P[3] = {pt.x, pt.y, pt.z};
    int i[3], ip[3];
    float w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // mod(x, L) is x itself inside [0, L): skip the fmod there
        const float p = (P[a] >= 0.f && P[a] < g.L[a]) ? P[a] : jl_modf(P[a], g.L[a]);
        const float qd = g.d_pow2[a] ? p * g.dinv[a] : __fdiv_rn(p, g.d[a]);
        int ii = (int)floorf(qd);
        if (ii >= g.n[a]) {
            ii = g.n[a] - 1;
            ++clamps;
        }
        if (ii < 0) ii = 0;
        i[a] = ii;
        ip[a] = (ii + 1 == g.n[a]) ? 0 : ii + 1;
        w[a] = __fsub_rn(p, __fmul_rn((float)ii, g.d[a]));
    }
    const long long nx = g.n[0], nxy = (long long)g.n[0] * g.n[1];
    const long long i0 = i[0], j0 = (long long)i[1] * nx, k0 = (long long)i[2] * nxy;
    const long long i1 = ip[0], j1 = (long long)ip[1] * nx, k1 = (long long)ip[2] * nxy;
    // u_x: bilinear in (y, z) over x-edge samples
    const float x00 = __ldg(&vx[i0 + j0 + k0]), x10 = __ldg(&vx[i0 + j1 + k0]);
    const float x01 = __ldg(&vx[i0 + j0 + k1]), x11 = __ldg(&vx[i0 + j1 + k1]);
    // u_y: bilinear in (x, z)
    const float y00 = __ldg(&vy[i0 + j0 + k0]), y10 = __ldg(&vy[i1 + j0 + k0]);
    const float y01 = __ldg(&vy[i0 + j0 + k1]), y11 = __ldg(&vy[i1 + j0 + k1]);
    // u_z: bilinear in (x, y)
    const float z00 = __ldg(&vz[i0 + j0 + k0]), z10 = __ldg(&vz[i1 + j0 + k0]);
    const float z01 = __ldg(&vz[i0 + j1 + k0]), z11 = __ldg(&vz[i1 + j1 + k0]);
    float3 u;
    u.x = (1.f - w[2]) * ((1.f - w[1]) * x00 + w[1] * x10) + w[2] * ((1.f - w[1]) * x01 + w[1] * x11);
    u.y = (1.f - w[2]) * ((1.f - w[0]) * y00 + w[0] * y10) + w[2] * ((1.f - w[0]) * y01 + w[0] * y11);
    u.z = (1.f - w[1]) * ((1.f - w[0]) * z00 + w[0] * z10) + w[1] * ((1.f - w[0]) * z01 + w[0] * z11);
    return u;
}

// staggered_advect! (parallel.jl:197-216, 248-261): classical RK4 for every
// slot inside the open box 0 < p < L, (-1,-1,-1) otherwise.
// counters[0] accumulates clamp events, counters[1] live particles.
__global__ void k_advect(Grid g, float* __restrict__ parts, long long np, const float* __restrict__ vel,
                         unsigned long long* __restrict__ counters) {
    const long long N = g.N;
    const float* vx = vel;
    const float* vy = vel + N;
    const float* vz = vel + 2 * N;
    unsigned clamps = 0, live = 0;
    const float dt = g.dt;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < np; k += (long long)gridDim.x * blockDim.x) {
        float3 p = make_float3(parts[3 * k], parts[3 * k + 1], parts[3 * k + 2]);
        const bool inside = (p.x > 0.f && p.x < g.L[0]) && (p.y > 0.f && p.y < g.L[1]) && (p.z > 0.f && p.z < g.L[2]);
        if (inside) {
            ++live;
            const float3 k1 = stag_vel(g, vx, vy, vz, p, clamps);
            float3 q = make_float3(p.x + k1.x * dt * 0.5f, p.y + k1.y * dt * 0.5f, p.z + k1.z * dt * 0.5f);
            const float3 k2 = stag_vel(g, vx, vy, vz, q, clamps);
            q = make_float3(p.x + k2.x * dt * 0.5f, p.y + k2.y * dt * 0.5f, p.z + k2.z * dt * 0.5f);
            const float3 k3 = stag_vel(g, vx, vy, vz, q, clamps);
            q = make_float3(p.x + k3.x * dt, p.y + k3.y * dt, p.z + k3.z * dt);
            const float3 k4 = stag_vel(g, vx, vy, vz, q, clamps);
            const float s = dt / 6.0f;
            p.x = p.x + s * (k1.x + 2.f * k2.x + 2.f * k3.x + k4.x);
            p.y = p.y + s * (k1.y + 2.f * k2.y + 2.f * k3.y + k4.y);
            p.z = p.z + s * (k1.z + 2.f * k2.z + 2.f * k3.z + k4.z);
        } else {
            p = make_float3(-1.f, -1.f, -1.f);
        }
        parts[3 * k] = p.x;
        parts[3 * k + 1] = p.y;
        parts[3 * k + 2] = p.z;
    }
    if (counters) {
        // warp-aggregated counters
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            clamps += __shfl_down_sync(0xffffffffu, clamps, o);
            live += __shfl_down_sync(0xffffffffu, live, o);
        }
        if ((threadIdx.x & 31) == 0) {
            if (clamps) atomicAdd(&counters[0], (unsigned long long)clamps);
            if (live) atomicAdd(&counters[1], (unsigned long long)live);
        }
    }
}

cudaError_t launch_emit(float* parts, long long nslots, long long start, long long count, const EmitArgs& e,
                        cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int blk = 256;
    k_emit<<<(unsigned)((count + blk - 1) / blk), blk, 0, s>>>(parts, nslots, start, count, e);
    return cudaGetLastError();
}

cudaError_t launch_advect(const Grid& g, float* parts, long long np, const float* vel, unsigned long long* counters,
                          cudaStream_t s) {
    if (np <= 0) return cudaSuccess;
    const int blk = 256;
    long long b = (np + blk - 1) / blk;
    if (b > 148LL * 64) b = 148LL * 64;
    k_advect<<<(unsigned)b, blk, 0, s>>>(g, parts, np, vel, counters);
    return cudaGetLastError();
}

}  // namespace isf
