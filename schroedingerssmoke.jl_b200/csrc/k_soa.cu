// Layout conversions between the FP64 structure-of-arrays fields of
// MatlabPort.jl (separate Complex{Float64} psi1, psi2; Float64 vx, vy, vz and
// scalar fields, column-major with x fastest, src/MatlabPort.jl:38-273) and
// the handle's FP32 layouts, plus the standalone gauge transform with a
// complex q (src/parallel.jl:125-129).  Grid-stride elementwise kernels with
// 16-byte accesses where the layout allows.
#include "isf_launch.h"

namespace isf {

namespace {
constexpr int kBlk = 256;
unsigned blocks(long long n) {
    long long b = (n + kBlk - 1) / kBlk;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b > 0 ? b : 1);
}
}  // namespace

// psi (float4 per cell) <- psi1, psi2 (complex128 per cell)
__global__ void k_psi_from_f64(const double2* __restrict__ a, const double2* __restrict__ b, float4* __restrict__ psi,
                               long long n) {
    pdl_enter();
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const double2 u = a[c], v = b[c];
        psi[c] = make_float4((float)u.x, (float)u.y, (float)v.x, (float)v.y);
    }
}

__global__ void k_psi_to_f64(const float4* __restrict__ psi, double2* __restrict__ a, double2* __restrict__ b,
                             long long n) {
    pdl_enter();
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const float4 p = psi[c];
        a[c] = make_double2(p.x, p.y);
        b[c] = make_double2(p.z, p.w);
    }
}

// padded velocity grid (with its periodic +face copies) <- vx, vy, vz
__global__ void k_vel_from_f64(Grid g, const double* __restrict__ vx, const double* __restrict__ vy,
                               const double* __restrict__ vz, float4* __restrict__ vel) {
    pdl_enter();
    const int nx = g.n[0], ny = g.n[1];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % nx);
        const long long r = c / nx;
        const int y = (int)(r % ny), z = (int)(r / ny);
        pstore(g, vel, x, y, z, make_float3((float)vx[c], (float)vy[c], (float)vz[c]));
    }
}

__global__ void k_vel_to_f64(Grid g, const float4* __restrict__ vel, double* __restrict__ vx, double* __restrict__ vy,
                             double* __restrict__ vz) {
    pdl_enter();
    const int nx = g.n[0], ny = g.n[1];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % nx);
        const long long r = c / nx;
        const int y = (int)(r % ny), z = (int)(r / ny);
        const float4 v = vel[pcell(g, x, y, z)];
        vx[c] = v.x;
        vy[c] = v.y;
        vz[c] = v.z;
    }
}

// dst[i] = (float)(scale * src[i * stride])
__global__ void k_real_from_f64(const double* __restrict__ src, long long stride, double scale, float* __restrict__ dst,
                                long long n) {
    pdl_enter();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)(scale * src[i * stride]);
}

__global__ void k_real_to_f64(const float* __restrict__ src, double* __restrict__ dst, long long n) {
    pdl_enter();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// dst[i] = re[i] + i im[i] (im null: 0) as complex128
__global__ void k_complex_to_f64(const float* __restrict__ re, const float* __restrict__ im, double2* __restrict__ dst,
                                 long long n) {
    pdl_enter();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = make_double2(re[i], im ? (double)im[i] : 0.0);
}

// gauge_transform (parallel.jl:125-129): psi * exp(i (-q)) with complex
// q = a + i b, i.e. psi * exp(b) * (cos a - i sin a)
__global__ void k_gauge_complex(float4* __restrict__ psi, const float* __restrict__ qre, const float* __restrict__ qim,
                                long long n) {
    pdl_enter();
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        float4 v = gauge4(psi[c], qre[c]);
        if (qim) v = cscale(v, expf(qim[c]));
        psi[c] = v;
    }
}

cudaError_t launch_psi_from_f64(const double* a, const double* b, float* psi, long long n, cudaStream_t s) {
    return launch_pdl(k_psi_from_f64, dim3(blocks(n)), dim3(kBlk), 0, s, reinterpret_cast<const double2*>(a),
                      reinterpret_cast<const double2*>(b), reinterpret_cast<float4*>(psi), n);
}

cudaError_t launch_psi_to_f64(const float* psi, double* a, double* b, long long n, cudaStream_t s) {
    return launch_pdl(k_psi_to_f64, dim3(blocks(n)), dim3(kBlk), 0, s, reinterpret_cast<const float4*>(psi),
                      reinterpret_cast<double2*>(a), reinterpret_cast<double2*>(b), n);
}

cudaError_t launch_vel_from_f64(const Grid& g, const double* vx, const double* vy, const double* vz, float* vel,
                                cudaStream_t s) {
    return launch_pdl(k_vel_from_f64, dim3(blocks(g.N)), dim3(kBlk), 0, s, g, vx, vy, vz, reinterpret_cast<float4*>(vel));
}

cudaError_t launch_vel_to_f64(const Grid& g, const float* vel, double* vx, double* vy, double* vz, cudaStream_t s) {
    return launch_pdl(k_vel_to_f64, dim3(blocks(g.N)), dim3(kBlk), 0, s, g, reinterpret_cast<const float4*>(vel), vx, vy,
                      vz);
}

cudaError_t launch_real_from_f64(const double* src, long long stride, double scale, float* dst, long long n,
                                 cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    return launch_pdl(k_real_from_f64, dim3(blocks(n)), dim3(kBlk), 0, s, src, stride, scale, dst, n);
}

cudaError_t launch_real_to_f64(const float* src, double* dst, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    return launch_pdl(k_real_to_f64, dim3(blocks(n)), dim3(kBlk), 0, s, src, dst, n);
}

cudaError_t launch_complex_to_f64(const float* re, const float* im, double* dst, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    return launch_pdl(k_complex_to_f64, dim3(blocks(n)), dim3(kBlk), 0, s, re, im, reinterpret_cast<double2*>(dst), n);
}

cudaError_t launch_gauge_complex(float* psi, const float* qre, const float* qim, long long n, cudaStream_t s) {
    return launch_pdl(k_gauge_complex, dim3(blocks(n)), dim3(kBlk), 0, s, reinterpret_cast<float4*>(psi), qre, qim, n);
}

}  // namespace isf
