// FFT pass kernels of the ISF step with their fused pointwise work.
//
// A 3D transform is three axis passes over the array in HBM; each pass is in
// place and moves every element once (read + write).  Fusions:
//   Schroedinger step  x fwd | y fwd | z fwd * mask/N, z inv | y inv | x inv + normalize
//   Poisson solve      real-to-complex x fwd of the divergence f | y fwd on the half
//                      spectrum | z fwd * fac/N, z inv | y inv | complex-to-real x inv
//                      + gauge of psi (+ the nozzle restriction)
// so the reference's split/merge broadcasts (parallel.jl:179-180, 185), the
// complex(f) copy (:169), the mask / fac multiplies (:171, :182-183) and the
// gauge broadcast (:159) never touch HBM on their own.
//
// x pass: lanes run along the row (coalesced 512-byte row segments); y / z
// passes: lanes run across C consecutive x columns (128-byte segments).
//
// Tile shape: a CTA runs G independent groups of C pencils (G = 1, 2 or 4),
// each with its own [N][C] shared tile, so short pencils (N = 32: 4 threads
// per pencil) still make CTAs of 128+ threads.  G is chosen per grid by the
// batch autotuner (isf_batch.cu); single simulations use G = 1.  G changes
// which pencils share a CTA, never the arithmetic of a pencil.
#pragma once
#include <type_traits>

#include "isf_fft.cuh"

namespace isf {

// ------------------------------------------------------------------ x pass
enum XOp {
    X_PSI_FWD = 0,       // psi rows, forward
    X_PSI_INV = 1,       // psi rows, inverse
    X_PSI_INV_NORM = 2,  // psi rows, inverse, then normalize_psi
    X_C_FWD = 3,         // complex array, forward
    X_C_INV = 4,         // complex array, inverse
};

struct XArgs {
    Grid g;
    float4* psi;
    float2* F;
    const float* rin;
    float* rout;
    JetArgs jet;
    int use_jet;
    int wp;  // row stride (complex elements) of the half spectrum of real data
    // a batch of nsim simulations of this grid (blockIdx.y = simulation;
    // 0 or 1: a single one): element strides between simulations of psi, F
    // and the real rows, and per-simulation jets (null: jet)
    int nsim;
    long long bs_psi, bs_F, bs_r;
    const JetArgs* jets;
    int groups;  // pencil groups per CTA (0 or 1: one)
};

template <int OP>
struct XTraits {
    static constexpr bool psi_elems = (OP == X_PSI_FWD || OP == X_PSI_INV || OP == X_PSI_INV_NORM);
    using T = typename std::conditional<psi_elems, float4, float2>::type;
    static constexpr int C = 128 / (int)sizeof(T);
    static constexpr int S = (OP == X_PSI_FWD || OP == X_C_FWD) ? -1 : +1;
};

template <int N, int OP, int G = 1>
struct XShape {
    static constexpr int C = XTraits<OP>::C;
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = G * C * NT;
    static constexpr size_t SMEM = (size_t)G * N * C * sizeof(typename XTraits<OP>::T);
};

template <int N, int OP, int G>
__global__ void __launch_bounds__(XShape<N, OP, G>::BLK) k_xpass(XArgs a) {
    pdl_enter();
    using Tr = XTraits<OP>;
    using T = typename Tr::T;
    constexpr int C = Tr::C;
    constexpr int NT = Plan<N>::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int grp = threadIdx.x / (C * NT), lt = threadIdx.x % (C * NT);
    T* sm = reinterpret_cast<T*>(smraw) + grp * (N * C);
    const int t = lt % NT, q = lt / NT;
    const long long row = ((long long)blockIdx.x * G + grp) * C + q;
    const long long rb = row * N;
    float4* __restrict__ psi = a.psi + blockIdx.y * a.bs_psi;
    float2* __restrict__ F = a.F + blockIdx.y * a.bs_F;
    T x[Plan<N>::EMAX];

    auto src = [&](int j) -> T {
        if constexpr (Tr::psi_elems) {
            return psi[rb + j];
        } else {
            return F[rb + j];
        }
    };
    auto dst = [&](int j, const T& v) {
        if constexpr (OP == X_PSI_FWD || OP == X_PSI_INV) {
            psi[rb + j] = v;
        } else if constexpr (OP == X_PSI_INV_NORM) {
            psi[rb + j] = normalize4(v);
        } else {
            static_assert(OP == X_C_FWD || OP == X_C_INV, "unhandled x-pass op");
            F[rb + j] = v;
        }
    };
    Plan<N>::template run<C, Tr::S, false>(x, t, q, sm, a.g.tw[0], src, dst);
}

// ------------------------------------------- x pass of real data (Poisson)
// Two real rows r0 = 2m, r1 = 2m+1 travel as one complex pencil a + i b.
//   XR_FWD        f rows -> half spectra A[k], B[k], k = 0..N/2, with
//                 A = (Z_k + conj Z_{N-k}) / 2 and B = (Z_k - conj Z_{N-k}) / 2i
//   XR_INV_GAUGE  Z_j = A_j + i B_j (Hermitian extension for j > N/2) ->
//                 inverse -> q rows (Re, Im) -> psi = gauge(psi (restricted), q)
//   XR_INV_REAL   the same inverse, q rows to a real output array
// The half spectrum of row r starts at F + r * wp (wp >= N/2 + 1, padded to
// whole 16-column tiles for the y / z passes).
enum XROp { XR_FWD = 0, XR_INV_GAUGE = 1, XR_INV_REAL = 2 };

template <int N, int G = 1>
struct XRShape {
    static constexpr int C = 16;
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = G * C * NT;
    static constexpr size_t SMEM = (size_t)G * N * C * sizeof(float2);
};

template <int N, int OP, int G>
__global__ void __launch_bounds__(XRShape<N, G>::BLK) k_xreal(XArgs a) {
    pdl_enter();
    using T = float2;
    constexpr int C = 16;
    constexpr int NT = Plan<N>::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int grp = threadIdx.x / (C * NT), lt = threadIdx.x % (C * NT);
    T* sm = reinterpret_cast<T*>(smraw) + grp * (N * C);
    const int t = lt % NT, q = lt / NT;
    const long long r0 = 2 * (((long long)blockIdx.x * G + grp) * C + q);
    const int wp = a.wp;
    const int sim = blockIdx.y;
    float2* __restrict__ Fs = a.F + sim * a.bs_F;
    T x[Plan<N>::EMAX];
    if constexpr (OP == XR_FWD) {
        const float* __restrict__ f0 = a.rin + sim * a.bs_r + r0 * N;
        const float* __restrict__ f1 = f0 + N;
        auto src = [&](int j) -> T { return make_float2(__ldg(&f0[j]), __ldg(&f1[j])); };
        auto sdst = [&](int j, const T& v) { sm[sidx<C>(j, q)] = v; };
        Plan<N>::template run<C, -1, false>(x, t, q, sm, a.g.tw[0], src, sdst);
        __syncthreads();
        float2* __restrict__ A = Fs + r0 * wp;
        float2* __restrict__ B = A + wp;
#pragma unroll 1
        for (int k = t; k <= N / 2; k += NT) {
            const float2 zk = sm[sidx<C>(k, q)];
            const float2 zn = sm[sidx<C>(k == 0 ? 0 : N - k, q)];
            A[k] = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
            B[k] = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
        }
    } else {
        const float2* __restrict__ A = Fs + r0 * wp;
        const float2* __restrict__ B = A + wp;
        float* __restrict__ rout = a.rout + sim * a.bs_r;
        float4* __restrict__ psi = a.psi + sim * a.bs_psi;
        const bool use_jet = a.use_jet != 0;
        const JetArgs jet = a.jets ? a.jets[sim] : a.jet;
        auto src = [&](int j) -> T {
            if (j <= N / 2) {
                const float2 u = A[j], v = B[j];
                return make_float2(u.x - v.y, u.y + v.x);
            }
            const float2 u = A[N - j], v = B[N - j];
            return make_float2(u.x + v.y, v.x - u.y);
        };
        const long long b0 = r0 * N, b1 = b0 + N;
        auto dst = [&](int j, const T& v) {
            if constexpr (OP == XR_INV_REAL) {
                rout[b0 + j] = v.x;
                rout[b1 + j] = v.y;
            } else {
                static_assert(OP == XR_INV_GAUGE, "unhandled real x-pass op");
                float4 p0 = psi[b0 + j], p1 = psi[b1 + j];
                if (use_jet) {
                    const int ny = a.g.n[1];
                    restrict_cell(a.g, jet, j, (int)(r0 % ny), (int)(r0 / ny), b0 + j, p0);
                    restrict_cell(a.g, jet, j, (int)((r0 + 1) % ny), (int)((r0 + 1) / ny), b1 + j, p1);
                }
                psi[b0 + j] = gauge4(p0, v.x);
                psi[b1 + j] = gauge4(p1, v.y);
            }
        };
        Plan<N>::template run<C, +1, false>(x, t, q, sm, a.g.tw[0], src, dst);
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
    int axis;      // 1 (y) or 2 (z)
    int row;       // elements per x row of data (nx, or the padded half-spectrum width)
    int kx_valid;  // columns holding spectrum data; the others are padding
    int nsim;            // simulations in a batch (blockIdx.z; 0 or 1: one)
    long long bstride;   // elements between simulations
    int groups;          // pencil groups per CTA along the other axis (0 or 1: one)
    int conj_mask;       // YZ_MASK: multiply by conj(mask) (the adjoint step, dt -> -dt)
};

// minimum resident threads per SM the y / z passes are compiled for (caps
// their registers); the spectral ones hold the FP64 symbol products as well
#ifndef ISF_YZ_MIN_THREADS
#define ISF_YZ_MIN_THREADS 768
#endif
#ifndef ISF_YZ_SPECTRAL_MIN_THREADS
#define ISF_YZ_SPECTRAL_MIN_THREADS 768
#endif
// the psi (float4) spectral pass holds twice the data per element: fewer
// resident threads, more registers (no spills)
#ifndef ISF_YZ_PSI_SPECTRAL_MIN_THREADS
#define ISF_YZ_PSI_SPECTRAL_MIN_THREADS 512
#endif

template <int N, class T, int OP = 0, int G = 1>
struct YZShape {
    static constexpr int C = 128 / (int)sizeof(T);
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = G * C * NT;
    static constexpr size_t SMEM = (size_t)G * N * C * sizeof(T);
    static constexpr int MINT = (OP < 2) ? ISF_YZ_MIN_THREADS
                                : (sizeof(T) == 16 ? ISF_YZ_PSI_SPECTRAL_MIN_THREADS : ISF_YZ_SPECTRAL_MIN_THREADS);
    static constexpr int MINB = (MINT / BLK) > 1 ? (MINT / BLK) : 1;
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <int N, class T, int OP, int G>
__global__ void __launch_bounds__(YZShape<N, T, OP, G>::BLK, YZShape<N, T, OP, G>::MINB) k_yzpass(YZArgs a) {
    pdl_enter();
    constexpr int C = YZShape<N, T>::C;
    constexpr int NT = Plan<N>::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int grp = threadIdx.x / (C * NT), lt = threadIdx.x % (C * NT);
    T* sm = reinterpret_cast<T*>(smraw) + grp * (N * C);
    const int q = lt % C, t = lt / C;
    const int rl = a.row, ny = a.g.n[1];
    const int x0 = blockIdx.x * C;
    const int o = blockIdx.y * G + grp;
    long long stride, base;
    if (a.axis == 1) {
        stride = rl;
        base = x0 + (long long)o * rl * ny;
    } else {
        stride = (long long)rl * ny;
        base = x0 + (long long)o * rl;
    }
    T* __restrict__ data = reinterpret_cast<T*>(a.data) + blockIdx.z * a.bstride;
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
            double2 cxo = zmul(a.g.mtab[0][kx], a.g.mtab[other][o]);
            cxo.x *= a.g.invN;
            cxo.y *= a.g.invN;
            const double2* __restrict__ mt = a.g.mtab[a.axis];
            const double msign = a.conj_mask ? -1.0 : 1.0;
            auto mmul = [&](int j, const T& v) -> T {
                double2 m = zmul(cxo, __ldg(&mt[j]));
                m.y *= msign;
                return cmul(v, make_float2((float)m.x, (float)m.y));
            };
            Plan<N>::template run_spectral<C>(x, t, q, sm, tw, gsrc, mmul, gdst);
        } else {
            static_assert(OP == YZ_FAC, "unhandled y/z op");
            // fac(k)/N, fac = -0.25 / sum_a (sin(pi k_a / n_a) / d_a)^2, fac(0) = 0
            // (parallel.jl:53-55, 63)
            const bool pad = kx >= a.kx_valid;  // padding column of a half spectrum
            const double dxo = (pad ? 0.0 : a.g.s2[0][kx]) + a.g.s2[other][o];
            const bool zero_line = (kx == 0) && (o == 0);
            const double* __restrict__ s2 = a.g.s2[a.axis];
            const double sc = -0.25 * a.g.invN;
            auto fmul = [&](int j, const T& v) -> T {
                const float f = (pad || (zero_line && j == 0)) ? 0.f : (float)(sc * __drcp_rn(dxo + __ldg(&s2[j])));
                return cscale(v, f);
            };
            Plan<N>::template run_spectral<C>(x, t, q, sm, tw, gsrc, fmul, gdst);
        }
    }
}

}  // namespace isf
