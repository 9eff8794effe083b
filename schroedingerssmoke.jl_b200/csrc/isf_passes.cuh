// FFT pass kernels of the ISF step with their fused pointwise work.
//
// A 3D transform is three axis passes over the array in HBM; each pass is in
// place and moves every element once (read + write).  Fusions:
//   Schroedinger step  x fwd | y fwd | z fwd * mask/N, z inv | y inv | x inv + normalize
//   Poisson solve      x fwd of f = div(one-form(psi)) computed from psi on the fly
//                      | y fwd | z fwd * fac/N, z inv | y inv | x inv + gauge of psi
// so the reference's split/merge broadcasts (parallel.jl:179-180, 185), the
// complex(f) copy (:169) and the mask / fac multiplies (:171, :182-183) never
// touch HBM on their own, and velocity and f of the projection are never stored.
#pragma once
#include <type_traits>

#include "isf_fft.cuh"

namespace isf {

// ------------------------------------------------------------------ x pass
enum XOp {
    X_PSI_FWD = 0,       // psi rows, forward
    X_PSI_INV = 1,       // psi rows, inverse
    X_PSI_INV_NORM = 2,  // psi rows, inverse, then normalize_psi
    X_C_FWD = 3,         // complex work array F, forward
    X_C_INV = 4,         // complex work array F, inverse
    X_STENCIL_FWD = 5,   // f = div(one-form(psi)) (optionally of the nozzle-restricted psi) -> F, forward
    X_GAUGE_INV = 6,     // F inverse -> q = Re; psi = gauge(psi (restricted), q)
    X_REAL_FWD = 7,      // real input array -> F, forward
    X_REAL_INV = 8,      // F inverse -> real part to a real output array
};

struct XArgs {
    Grid g;
    float4* psi;
    float2* F;
    const float* rin;
    float* rout;
    JetArgs jet;
    int use_jet;
};

template <int OP>
struct XTraits {
    static constexpr bool psi_elems = (OP == X_PSI_FWD || OP == X_PSI_INV || OP == X_PSI_INV_NORM);
    using T = typename std::conditional<psi_elems, float4, float2>::type;
    static constexpr int C = 128 / (int)sizeof(T);
    static constexpr int S =
        (OP == X_PSI_FWD || OP == X_C_FWD || OP == X_STENCIL_FWD || OP == X_REAL_FWD) ? -1 : +1;
};

__device__ __forceinline__ float4 load_psi_restricted(const XArgs& a, int x, int y, int z) {
    const long long c = cell(a.g, x, y, z);
    float4 v = __ldg(&a.psi[c]);
    if (a.use_jet) restrict_cell(a.g, a.jet, x, y, z, c, v);
    return v;
}

// div(velocity_one_form(psi, 1)) at cell (x,y,z): parallel.jl:100-152
__device__ __forceinline__ float stencil_f(const XArgs& a, int x, int y, int z) {
    const int nx = a.g.n[0], ny = a.g.n[1], nz = a.g.n[2];
    const int xp = (x + 1 == nx) ? 0 : x + 1, xm = (x == 0) ? nx - 1 : x - 1;
    const int yp = (y + 1 == ny) ? 0 : y + 1, ym = (y == 0) ? ny - 1 : y - 1;
    const int zp = (z + 1 == nz) ? 0 : z + 1, zm = (z == 0) ? nz - 1 : z - 1;
    const float4 c0 = load_psi_restricted(a, x, y, z);
    const float4 cxp = load_psi_restricted(a, xp, y, z);
    const float4 cxm = load_psi_restricted(a, xm, y, z);
    const float4 cyp = load_psi_restricted(a, x, yp, z);
    const float4 cym = load_psi_restricted(a, x, ym, z);
    const float4 czp = load_psi_restricted(a, x, y, zp);
    const float4 czm = load_psi_restricted(a, x, y, zm);
    const float vx = pair_angle(c0, cxp), vxm = pair_angle(cxm, c0);
    const float vy = pair_angle(c0, cyp), vym = pair_angle(cym, c0);
    const float vz = pair_angle(c0, czp), vzm = pair_angle(czm, c0);
    const float t0 = (vx - vxm) * a.g.inv_d2[0];
    const float t1 = (vy - vym) * a.g.inv_d2[1];
    const float t2 = (vz - vzm) * a.g.inv_d2[2];
    return (t0 + t1) + t2;
}

template <int N, int OP>
__global__ void __launch_bounds__(Threads<N, XTraits<OP>::C>::block) k_xpass(XArgs a) {
    using Tr = XTraits<OP>;
    using T = typename Tr::T;
    constexpr int C = Tr::C;
    constexpr int BLK = Threads<N, C>::block;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* A = reinterpret_cast<T*>(smraw);
    T* B = A + N * C;
    const long long row0 = (long long)blockIdx.x * C;
    const int tid = threadIdx.x;
    const int ny = a.g.n[1];

#pragma unroll 1
    for (int e = tid; e < N * C; e += BLK) {
        const int q = e / N, j = e - q * N;
        const long long row = row0 + q;
        const long long c = row * N + j;
        T v;
        if constexpr (Tr::psi_elems) {
            v = a.psi[c];
        } else if constexpr (OP == X_C_FWD || OP == X_C_INV || OP == X_GAUGE_INV) {
            v = a.F[c];
        } else if constexpr (OP == X_REAL_FWD) {
            v = make_float2(a.rin[c], 0.f);
        } else {  // X_STENCIL_FWD
            const int y = (int)(row % ny), z = (int)(row / ny);
            v = make_float2(stencil_f(a, j, y, z), 0.f);
        }
        A[sidx<C>(j, q)] = v;
    }
    __syncthreads();
    T* R = fft_pencils<N, C, Tr::S>(A, B, a.g.tw[0], tid % C, tid / C);

#pragma unroll 1
    for (int e = tid; e < N * C; e += BLK) {
        const int q = e / N, j = e - q * N;
        const long long row = row0 + q;
        const long long c = row * N + j;
        T v = R[sidx<C>(j, q)];
        if constexpr (OP == X_PSI_FWD || OP == X_PSI_INV) {
            a.psi[c] = v;
        } else if constexpr (OP == X_PSI_INV_NORM) {
            a.psi[c] = normalize4(v);
        } else if constexpr (OP == X_C_FWD || OP == X_C_INV || OP == X_STENCIL_FWD || OP == X_REAL_FWD) {
            a.F[c] = v;
        } else if constexpr (OP == X_REAL_INV) {
            a.rout[c] = v.x;
        } else {  // X_GAUGE_INV
            float4 p = a.psi[c];
            if (a.use_jet) {
                const int y = (int)(row % ny), z = (int)(row / ny);
                restrict_cell(a.g, a.jet, j, y, z, c, p);
            }
            a.psi[c] = gauge4(p, v.x);
        }
    }
}

// -------------------------------------------------------------- y / z pass
enum YZOp {
    YZ_FWD = 0,
    YZ_INV = 1,
    YZ_MASK = 2,  // forward, * mask(k)/N (Schroedinger phase), inverse
    YZ_FAC = 3,   // forward, * fac(k)/N (inverse torus Laplacian), inverse
};

struct YZArgs {
    Grid g;
    void* data;
    int axis;  // 1 (y) or 2 (z)
};

// exp(i (th_x + th_y + th_z)) / N in double, rounded to float: the
// reference's Float32(exp(i lambda dt / 2)) (parallel.jl:58-62) up to the
// double rounding of the product.
__device__ __forceinline__ float2 mask_value(const Grid& g, int kx, int ky, int kz) {
    const double2 a = g.mtab[0][kx], b = g.mtab[1][ky], c = g.mtab[2][kz];
    const double abx = a.x * b.x - a.y * b.y, aby = a.x * b.y + a.y * b.x;
    const double mx = abx * c.x - aby * c.y, my = abx * c.y + aby * c.x;
    return make_float2((float)(mx * g.invN), (float)(my * g.invN));
}

// fac(k) / N, fac = -0.25 / sum_a (sin(pi k_a / n_a) / d_a)^2, fac(0) = 0
// (parallel.jl:53-55, 63)
__device__ __forceinline__ float fac_value(const Grid& g, int kx, int ky, int kz) {
    if ((kx | ky | kz) == 0) return 0.f;
    const double den = g.s2[0][kx] + g.s2[1][ky] + g.s2[2][kz];
    return (float)(-0.25 / den * g.invN);
}

template <int N, class T, int OP>
__global__ void __launch_bounds__(Threads<N, 128 / (int)sizeof(T)>::block) k_yzpass(YZArgs a) {
    constexpr int C = 128 / (int)sizeof(T);
    constexpr int BLK = Threads<N, C>::block;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* A = reinterpret_cast<T*>(smraw);
    T* B = A + N * C;
    const int tid = threadIdx.x;
    const int nx = a.g.n[0], ny = a.g.n[1];
    const int x0 = blockIdx.x * C;
    const int o = blockIdx.y;
    long long stride, base;
    if (a.axis == 1) {
        stride = nx;
        base = x0 + (long long)o * nx * ny;
    } else {
        stride = (long long)nx * ny;
        base = x0 + (long long)o * nx;
    }
    T* data = reinterpret_cast<T*>(a.data);
    const float2* tw = a.g.tw[a.axis];

#pragma unroll 1
    for (int e = tid; e < N * C; e += BLK) {
        const int j = e / C, q = e - j * C;
        A[sidx<C>(j, q)] = data[base + j * stride + q];
    }
    __syncthreads();
    T* R;
    if constexpr (OP == YZ_INV) {
        R = fft_pencils<N, C, +1>(A, B, tw, tid % C, tid / C);
    } else {
        R = fft_pencils<N, C, -1>(A, B, tw, tid % C, tid / C);
    }
    if constexpr (OP == YZ_MASK || OP == YZ_FAC) {
#pragma unroll 1
        for (int e = tid; e < N * C; e += BLK) {
            const int j = e / C, q = e - j * C;
            const int kx = x0 + q;
            const int ky = (a.axis == 1) ? j : o;
            const int kz = (a.axis == 1) ? o : j;
            T v = R[sidx<C>(j, q)];
            if constexpr (OP == YZ_MASK) {
                v = cmul(v, mask_value(a.g, kx, ky, kz));
            } else {
                v = cscale(v, fac_value(a.g, kx, ky, kz));
            }
            R[sidx<C>(j, q)] = v;
        }
        __syncthreads();
        T* other = (R == A) ? B : A;
        R = fft_pencils<N, C, +1>(R, other, tw, tid % C, tid / C);
    }
#pragma unroll 1
    for (int e = tid; e < N * C; e += BLK) {
        const int j = e / C, q = e - j * C;
        data[base + j * stride + q] = R[sidx<C>(j, q)];
    }
}

}  // namespace isf
