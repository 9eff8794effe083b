// FFT pass kernels of the ISF step with their fused pointwise work.
//
// A 3D transform is three axis passes over the array in HBM; each pass is in
// place and moves every element once (read + write).  Fusions:
//   Schroedinger step  x fwd | y fwd | z fwd * mask/N, z inv | y inv | x inv + normalize
//   Poisson solve      x fwd of the real divergence f | y fwd | z fwd * fac/N, z inv
//                      | y inv | x inv + gauge of psi (+ the nozzle restriction)
// so the reference's split/merge broadcasts (parallel.jl:179-180, 185), the
// complex(f) copy (:169), the mask / fac multiplies (:171, :182-183) and the
// gauge broadcast (:159) never touch HBM on their own.
//
// x pass: lanes run along the row (coalesced 512-byte row segments); y / z
// passes: lanes run across C consecutive x columns (128-byte segments).
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
    static constexpr int S = (OP == X_PSI_FWD || OP == X_C_FWD || OP == X_REAL_FWD) ? -1 : +1;
};

template <int N, int OP>
struct XShape {
    static constexpr int C = XTraits<OP>::C;
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = C * NT;
    static constexpr size_t SMEM = (size_t)N * C * sizeof(typename XTraits<OP>::T);
};

template <int N, int OP>
__global__ void __launch_bounds__(XShape<N, OP>::BLK) k_xpass(XArgs a) {
    using Tr = XTraits<OP>;
    using T = typename Tr::T;
    constexpr int C = Tr::C;
    constexpr int NT = Plan<N>::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int t = threadIdx.x % NT, q = threadIdx.x / NT;
    const long long row = (long long)blockIdx.x * C + q;
    const long long rb = row * N;
    T x[Plan<N>::EMAX];

    auto src = [&](int j) -> T {
        if constexpr (Tr::psi_elems) {
            return a.psi[rb + j];
        } else if constexpr (OP == X_REAL_FWD) {
            return make_float2(__ldg(&a.rin[rb + j]), 0.f);
        } else {
            return a.F[rb + j];
        }
    };
    auto dst = [&](int j, const T& v) {
        if constexpr (OP == X_PSI_FWD || OP == X_PSI_INV) {
            a.psi[rb + j] = v;
        } else if constexpr (OP == X_PSI_INV_NORM) {
            a.psi[rb + j] = normalize4(v);
        } else if constexpr (OP == X_C_FWD || OP == X_C_INV || OP == X_REAL_FWD) {
            a.F[rb + j] = v;
        } else if constexpr (OP == X_REAL_INV) {
            a.rout[rb + j] = v.x;
        } else {
            static_assert(OP == X_GAUGE_INV, "unhandled x-pass op");
            float4 p = a.psi[rb + j];
            if (a.use_jet) {
                const int ny = a.g.n[1];
                restrict_cell(a.g, a.jet, j, (int)(row % ny), (int)(row / ny), rb + j, p);
            }
            a.psi[rb + j] = gauge4(p, v.x);
        }
    };
    Plan<N>::template run<C, Tr::S, false>(x, t, q, sm, a.g.tw[0], src, dst);
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

template <int N, class T>
struct YZShape {
    static constexpr int C = 128 / (int)sizeof(T);
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = C * NT;
    static constexpr size_t SMEM = (size_t)N * C * sizeof(T);
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <int N, class T, int OP>
__global__ void __launch_bounds__(YZShape<N, T>::BLK) k_yzpass(YZArgs a) {
    constexpr int C = YZShape<N, T>::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int q = threadIdx.x % C, t = threadIdx.x / C;
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
    T* __restrict__ data = reinterpret_cast<T*>(a.data);
    const float2* tw = a.g.tw[a.axis];
    T x[Plan<N>::EMAX];

    auto gsrc = [&](int j) -> T { return data[base + j * stride + q]; };
    auto gdst = [&](int j, const T& v) { data[base + j * stride + q] = v; };

    if constexpr (OP == YZ_FWD) {
        Plan<N>::template run<C, -1, false>(x, t, q, sm, tw, gsrc, gdst);
    } else if constexpr (OP == YZ_INV) {
        Plan<N>::template run<C, +1, false>(x, t, q, sm, tw, gsrc, gdst);
    } else {
        // spectral multiply between the forward and the inverse transform of
        // this pencil; k along the pass axis is the pencil position j
        const int kx = x0 + q;
        const int other = a.axis == 1 ? 2 : 1;
        if constexpr (OP == YZ_MASK) {
            // exp(i (th_x + th_y + th_z)) / N in double, rounded to float: the
            // reference's Float32(exp(i lambda dt / 2)) (parallel.jl:58-62) up
            // to the double rounding of the product
            const double2 cxo = zmul(a.g.mtab[0][kx], a.g.mtab[other][o]);
            const double2* __restrict__ mt = a.g.mtab[a.axis];
            const double invN = a.g.invN;
            auto mdst = [&](int j, const T& v) {
                const double2 m = zmul(cxo, mt[j]);
                sm[sidx<C>(j, q)] = cmul(v, make_float2((float)(m.x * invN), (float)(m.y * invN)));
            };
            Plan<N>::template run<C, -1, false>(x, t, q, sm, tw, gsrc, mdst);
        } else {
            static_assert(OP == YZ_FAC, "unhandled y/z op");
            // fac(k)/N, fac = -0.25 / sum_a (sin(pi k_a / n_a) / d_a)^2, fac(0) = 0
            // (parallel.jl:53-55, 63)
            const double dxo = a.g.s2[0][kx] + a.g.s2[other][o];
            const bool zero_line = (kx == 0) && (o == 0);
            const double* __restrict__ s2 = a.g.s2[a.axis];
            const double sc = -0.25 * a.g.invN;
            auto fdst = [&](int j, const T& v) {
                const float f = (zero_line && j == 0) ? 0.f : (float)(sc / (dxo + s2[j]));
                sm[sidx<C>(j, q)] = cscale(v, f);
            };
            Plan<N>::template run<C, -1, false>(x, t, q, sm, tw, gsrc, fdst);
        }
        __syncthreads();
        auto ssrc = [&](int j) -> T { return sm[sidx<C>(j, q)]; };
        Plan<N>::template run<C, +1, true>(x, t, q, sm, tw, ssrc, gdst);
    }
}

}  // namespace isf
