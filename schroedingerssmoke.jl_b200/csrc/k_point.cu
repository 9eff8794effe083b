// Pointwise and nearest-neighbour kernels of the ISF API that are not fused
// into an FFT pass or a stencil: the standalone forms of normalize_psi,
// restrict_velocity!, isjet, the staggered sharp and div! (from the velocity
// grid), and layout conversions of the handle's padded velocity grid.
#include "isf_launch.h"

namespace isf {

static inline unsigned grid_for(long long n, int block) {
    long long b = (n + block - 1) / block;
    const long long cap = 148LL * 32;  // grid-stride beyond 32 CTAs per SM
    return (unsigned)(b < cap ? b : cap);
}

// normalize_psi broadcast (parallel.jl:162-165, examples/benchmark.jl:50)
__global__ void k_normalize(float4* __restrict__ psi, long long N) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x)
        psi[c] = normalize4(psi[c]);
}

// restrict_velocity! (particles.jl:25-27 -> restrict_kernel :12-20)
__global__ void k_restrict(Grid g, float4* __restrict__ psi, JetArgs j) {
    const long long N = g.N;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % g.n[0]);
        const long long r = c / g.n[0];
        const int y = (int)(r % g.n[1]), z = (int)(r / g.n[1]);
        float4 v = psi[c];
        if (restrict_cell(g, j, x, y, z, c, v)) psi[c] = v;
    }
}

// isjet.(isf.positions, ...) (particles.jl:6-10, examples/benchmark.jl:26)
__global__ void k_isjet(Grid g, uint8_t* __restrict__ out, float c0, float c1, float c2, float len, float rad) {
    const float cen[3] = {c0, c1, c2};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % g.n[0]);
        const long long r = c / g.n[0];
        const int y = (int)(r % g.n[1]), z = (int)(r / g.n[1]);
        const float px = __fmul_rn((float)x, g.d[0]), py = __fmul_rn((float)y, g.d[1]), pz = __fmul_rn((float)z, g.d[2]);
        out[c] = isjet_f32(px, py, pz, cen, len, rad) ? 1 : 0;
    }
}

// staggered sharp on the handle's padded velocity grid (examples/benchmark.jl:61-63)
__global__ void k_sharp(Grid g, float4* __restrict__ vel) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.NP; c += (long long)gridDim.x * blockDim.x) {
        float4 v = vel[c];
        v.x = __fmul_rn(v.x, g.dinv[0]);
        v.y = __fmul_rn(v.y, g.dinv[1]);
        v.z = __fmul_rn(v.z, g.dinv[2]);
        vel[c] = v;
    }
}

__device__ __forceinline__ void decode(const Grid& g, long long c, int& x, int& y, int& z) {
    x = (int)(c % g.n[0]);
    const long long r = c / g.n[0];
    y = (int)(r % g.n[1]);
    z = (int)(r / g.n[1]);
}

// div! (parallel.jl:131-152) from the padded velocity grid
__global__ void k_div(Grid g, const float4* __restrict__ vel, float* __restrict__ f) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(g, c, x, y, z);
        const int xm = (x == 0) ? g.n[0] - 1 : x - 1;
        const int ym = (y == 0) ? g.n[1] - 1 : y - 1;
        const int zm = (z == 0) ? g.n[2] - 1 : z - 1;
        const float4 v = vel[pcell(g, x, y, z)];
        const float t0 = (v.x - vel[pcell(g, xm, y, z)].x) * g.inv_d2[0];
        const float t1 = (v.y - vel[pcell(g, x, ym, z)].y) * g.inv_d2[1];
        const float t2 = (v.z - vel[pcell(g, x, y, zm)].z) * g.inv_d2[2];
        f[c] = (t0 + t1) + t2;
    }
}

__global__ void k_vel_to_aos(Grid g, const float4* __restrict__ vel, float* __restrict__ aos) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(g, c, x, y, z);
        const float4 v = vel[pcell(g, x, y, z)];
        aos[3 * c + 0] = v.x;
        aos[3 * c + 1] = v.y;
        aos[3 * c + 2] = v.z;
    }
}

__global__ void k_vel_from_aos(Grid g, const float* __restrict__ aos, float4* __restrict__ vel) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(g, c, x, y, z);
        pstore(g, vel, x, y, z, make_float3(aos[3 * c + 0], aos[3 * c + 1], aos[3 * c + 2]));
    }
}

__global__ void k_scale_c(float2* __restrict__ a, long long N, float s) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x)
        a[c] = cscale(a[c], s);
}

// cells of psi with a non-finite component, added into *count
__global__ void k_count_nonfinite(const float4* __restrict__ psi, long long N, unsigned long long* __restrict__ count) {
    unsigned n = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
        const float4 v = psi[c];
        n += (isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w)) ? 0u : 1u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, (unsigned long long)n);
}

cudaError_t launch_count_nonfinite(const Grid& g, const float4* psi, unsigned long long* count, cudaStream_t s) {
    k_count_nonfinite<<<grid_for(g.N, 256), 256, 0, s>>>(psi, g.N, count);
    return cudaGetLastError();
}

cudaError_t launch_scale_c(const Grid& g, float2* a, float s, cudaStream_t st) {
    k_scale_c<<<grid_for(g.N, 256), 256, 0, st>>>(a, g.N, s);
    return cudaGetLastError();
}
cudaError_t launch_normalize(const Grid& g, float4* psi, cudaStream_t s) {
    k_normalize<<<grid_for(g.N, 256), 256, 0, s>>>(psi, g.N);
    return cudaGetLastError();
}
cudaError_t launch_restrict(const Grid& g, float4* psi, const JetArgs& j, cudaStream_t s) {
    k_restrict<<<grid_for(g.N, 256), 256, 0, s>>>(g, psi, j);
    return cudaGetLastError();
}
cudaError_t launch_isjet(const Grid& g, uint8_t* out, const float* cen, float len, float rad, cudaStream_t s) {
    k_isjet<<<grid_for(g.N, 256), 256, 0, s>>>(g, out, cen[0], cen[1], cen[2], len, rad);
    return cudaGetLastError();
}
cudaError_t launch_sharp(const Grid& g, float* vel, cudaStream_t s) {
    k_sharp<<<grid_for(g.NP, 256), 256, 0, s>>>(g, reinterpret_cast<float4*>(vel));
    return cudaGetLastError();
}
cudaError_t launch_div(const Grid& g, const float* vel, float* f, cudaStream_t s) {
    k_div<<<grid_for(g.N, 256), 256, 0, s>>>(g, reinterpret_cast<const float4*>(vel), f);
    return cudaGetLastError();
}
cudaError_t launch_vel_to_aos(const Grid& g, const float* vel, float* aos, cudaStream_t s) {
    k_vel_to_aos<<<grid_for(g.N, 256), 256, 0, s>>>(g, reinterpret_cast<const float4*>(vel), aos);
    return cudaGetLastError();
}
cudaError_t launch_vel_from_aos(const Grid& g, const float* aos, float* vel, cudaStream_t s) {
    k_vel_from_aos<<<grid_for(g.N, 256), 256, 0, s>>>(g, aos, reinterpret_cast<float4*>(vel));
    return cudaGetLastError();
}

}  // namespace isf
