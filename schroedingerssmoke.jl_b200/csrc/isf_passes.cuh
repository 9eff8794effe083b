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
    int kmajor;  // real x passes: the half spectrum is k-major (see k_xreal)
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

// FULL: the launch has whole tiles only (the row count a multiple of C G), so
// no pencil needs the past-the-end guard
template <int N, int OP, int G, bool FULL = false, class BarT = CtaBar>
__device__ __forceinline__ void xpass_body(const XArgs a, const Blk bk, unsigned char* smraw,
                                           const BarT& bar = BarT()) {
    using Tr = XTraits<OP>;
    using T = typename Tr::T;
    constexpr int C = Tr::C;
    constexpr int NT = Plan<N>::NT;
    const int grp = bk.tid / (C * NT), lt = bk.tid % (C * NT);
    T* sm = reinterpret_cast<T*>(smraw) + grp * (N * C);
    const int t = lt % NT, q = lt / NT;
    const long long row = ((long long)bk.x * G + grp) * C + q;
    const long long rb = row * N;
    // the last CTA of a grid whose row count is not a multiple of C holds
    // pencils past the end: they read zeros and store nothing
    const bool valid = FULL || row < (long long)a.g.n[1] * a.g.n[2];
    float4* __restrict__ psi = a.psi + bk.y * a.bs_psi;
    float2* __restrict__ F = a.F + bk.y * a.bs_F;
    T x[Plan<N>::EMAX];

    auto src = [&](int j) -> T {
        if (!valid) return T{};
        if constexpr (Tr::psi_elems) {
            return psi[rb + j];
        } else {
            return F[rb + j];
        }
    };
    auto dst = [&](int j, const T& v) {
        if (!valid) return;
        if constexpr (OP == X_PSI_FWD || OP == X_PSI_INV) {
            psi[rb + j] = v;
        } else if constexpr (OP == X_PSI_INV_NORM) {
            psi[rb + j] = normalize4(v);
        } else {
            static_assert(OP == X_C_FWD || OP == X_C_INV, "unhandled x-pass op");
            F[rb + j] = v;
        }
    };
    Plan<N>::template run<C, Tr::S, false>(x, t, q, sm, a.g.tw[0], src, dst, pencil_bar<NT, C>(bar));
}

template <int N, int OP, int G, bool FULL = false>
__global__ void __launch_bounds__(XShape<N, OP, G>::BLK) k_xpass(XArgs a) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    xpass_body<N, OP, G, FULL>(a, launch_blk(), smraw);
}

// ------------------------------------------- x pass of real data (Poisson)
// Two real rows r0 = 2m, r1 = 2m+1 travel as one complex pencil a + i b.
//   XR_FWD        f rows -> half spectra A[k], B[k], k = 0..N/2, with
//                 A = (Z_k + conj Z_{N-k}) / 2 and B = (Z_k - conj Z_{N-k}) / 2i
//   XR_INV_GAUGE  Z_j = A_j + i B_j (Hermitian extension for j > N/2) ->
//                 inverse -> q rows (Re, Im) -> psi = gauge(psi (restricted), q)
//   XR_INV_REAL   the same inverse, q rows to a real output array
// Half-spectrum layouts:
//   row-major (KM = false)  row r's spectrum at F + r * wp (wp >= N/2 + 1,
//                           padded to whole 16-column tiles for the y / z passes)
//   k-major   (KM = true)   element (k, y, z) at F + (k nz + z) ny + y: one
//                           contiguous (y, z) plane per k for the plane solver
//                           (k_poisson_plane); A and B of a row pair are
//                           neighbours, moved as one 16-byte vector, with the
//                           lanes running over row pairs.
//   XR_INV_GAUGE_JET  the gauge with psi restricted in the nozzle first (use_jet):
//                 a separate op so that the plain gauge carries none of the
//                 restriction's code
enum XROp { XR_FWD = 0, XR_INV_GAUGE = 1, XR_INV_REAL = 2, XR_INV_GAUGE_JET = 3 };

template <int N, int G = 1, bool KM = false>
struct XRShape {
    static constexpr int C = 16;
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = G * C * NT;
    // the k-major inverse stages (A, B) of N/2 + 1 k per row pair in the tile
    static constexpr size_t TILE = (size_t)N * C * sizeof(float2);
    static constexpr size_t STAGE = (size_t)(N / 2 + 1) * C * sizeof(float4);
    static constexpr size_t SMEM = (size_t)G * (KM && STAGE > TILE ? STAGE : TILE);
};

template <int N, int OP, int G, bool KM = false, class BarT = CtaBar>
__device__ __forceinline__ void xreal_body(const XArgs a, const Blk bk, unsigned char* smraw,
                                           const BarT& bar = BarT()) {
    using T = float2;
    constexpr int C = 16;
    constexpr int NT = Plan<N>::NT;
    const int grp = bk.tid / (C * NT), lt = bk.tid % (C * NT);
    T* sm = reinterpret_cast<T*>(smraw + grp * XRShape<N, G, KM>::SMEM / G);
    const int t = lt % NT, q = lt / NT;
    const long long rbase = 2 * ((long long)bk.x * G + grp) * C;  // first row of the group
    const long long r0 = rbase + 2 * q;
    const int wp = a.wp;
    const int ny = a.g.n[1], nz = a.g.n[2];
    const int sim = bk.y;
    float2* __restrict__ Fs = a.F + sim * a.bs_F;
    T x[Plan<N>::EMAX];
    // row pairs past the last row (a row count that is not a multiple of
    // 2 C) read zeros and store nothing; the k-major layout has none
    const long long rows = (long long)ny * nz;
    const bool v0 = KM || r0 < rows, v1 = KM || r0 + 1 < rows;
    if constexpr (OP == XR_FWD) {
        const float* __restrict__ f0 = a.rin + sim * a.bs_r + r0 * N;
        const float* __restrict__ f1 = f0 + N;
        auto src = [&](int j) -> T {
            return make_float2(v0 ? ldm<BarT>(&f0[j]) : 0.f, v1 ? ldm<BarT>(&f1[j]) : 0.f);
        };
        auto sdst = [&](int j, const T& v) { sm[sidx<C>(j, q)] = v; };
        Plan<N>::template run<C, -1, false>(x, t, q, sm, a.g.tw[0], src, sdst, pencil_bar<NT, C>(bar));
        bar.sync();
        if constexpr (KM) {
            // lanes over the row pairs of the group: 16 x 16 B per k
            float4* __restrict__ F4 = reinterpret_cast<float4*>(Fs);
            for (int idx = lt; idx < (N / 2 + 1) * C; idx += C * NT) {
                const int qq = idx % C, k = idx / C;
                const float2 zk = sm[sidx<C>(k, qq)];
                const float2 zn = sm[sidx<C>(k == 0 ? 0 : N - k, qq)];
                const long long r = rbase + 2 * qq;
                const int y = (int)(r % ny), z = (int)(r / ny);
                F4[(((long long)k * nz + z) * ny + y) >> 1] =
                    make_float4(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y), 0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
            }
        } else {
            float2* __restrict__ A = Fs + r0 * wp;
            float2* __restrict__ B = A + wp;
#pragma unroll 1
            for (int k = t; k <= N / 2; k += NT) {
                const float2 zk = sm[sidx<C>(k, q)];
                const float2 zn = sm[sidx<C>(k == 0 ? 0 : N - k, q)];
                if (v0) A[k] = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
                if (v1) B[k] = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
            }
        }
    } else {
        const float2* __restrict__ A = Fs + r0 * wp;
        const float2* __restrict__ B = A + wp;
        // k-major: (A_k, B_k) of every row pair staged in the tile first
        // (swizzled: conflict free for the lanes over row pairs that fill it
        // and for the lanes over k that read it)
        float4* stg = reinterpret_cast<float4*>(sm);
        if constexpr (KM) {
            const float4* __restrict__ F4 = reinterpret_cast<const float4*>(Fs);
            for (int idx = lt; idx < (N / 2 + 1) * C; idx += C * NT) {
                const int qq = idx % C, k = idx / C;
                const long long r = rbase + 2 * qq;
                const int y = (int)(r % ny), z = (int)(r / ny);
                stg[k * C + (qq ^ (k & (C - 1)))] = F4[(((long long)k * nz + z) * ny + y) >> 1];
            }
            bar.sync();
        }
        float* __restrict__ rout = a.rout + sim * a.bs_r;
        float4* __restrict__ psi = a.psi + sim * a.bs_psi;
        constexpr bool kJet = OP == XR_INV_GAUGE_JET;
        JetArgs jet;
        if constexpr (kJet) jet = a.jets ? a.jets[sim] : a.jet;
        auto src = [&](int j) -> T {
            const int k = j <= N / 2 ? j : N - j;
            float2 u, v;
            if constexpr (KM) {
                const float4 s = stg[k * C + (q ^ (k & (C - 1)))];
                u = make_float2(s.x, s.y);
                v = make_float2(s.z, s.w);
            } else {
                u = v0 ? A[k] : make_float2(0.f, 0.f);
                v = v1 ? B[k] : make_float2(0.f, 0.f);
            }
            if (j <= N / 2) return make_float2(u.x - v.y, u.y + v.x);
            return make_float2(u.x + v.y, v.x - u.y);
        };
        const long long b0 = r0 * N, b1 = b0 + N;
        auto dst = [&](int j, const T& v) {
            if constexpr (OP == XR_INV_REAL) {
                if (v0) rout[b0 + j] = v.x;
                if (v1) rout[b1 + j] = v.y;
            } else {
                static_assert(OP == XR_INV_GAUGE || OP == XR_INV_GAUGE_JET, "unhandled real x-pass op");
                // both rows' psi loaded before either is stored (two loads in flight)
                float4 p0 = v0 ? psi[b0 + j] : make_float4(0.f, 0.f, 0.f, 0.f);
                float4 p1 = v1 ? psi[b1 + j] : make_float4(0.f, 0.f, 0.f, 0.f);
                if constexpr (kJet) {
                    if (v0) restrict_cell(a.g, jet, j, (int)(r0 % ny), (int)(r0 / ny), b0 + j, p0);
                    if (v1) restrict_cell(a.g, jet, j, (int)((r0 + 1) % ny), (int)((r0 + 1) / ny), b1 + j, p1);
                }
                if (v0) psi[b0 + j] = gauge4(p0, v.x);
                if (v1) psi[b1 + j] = gauge4(p1, v.y);
            }
        };
        // k-major: the staging aliases the tile, so the first gather must
        // complete before the first stage writes the tile
        Plan<N>::template run<C, +1, KM>(x, t, q, sm, a.g.tw[0], src, dst, pencil_bar<NT, C>(bar));
    }
}

template <int N, int OP, int G, bool KM = false>
__global__ void __launch_bounds__(XRShape<N, G, KM>::BLK) k_xreal(XArgs a) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    xreal_body<N, OP, G, KM>(a, launch_blk(), smraw);
}

// The same pass compiled for 3 resident CTAs per SM (at most 42 registers),
// launched for rows of at least 256 cells: the gauge pass at 256x128x128 ran
// 35.4 -> 34.6 us.  The ensembles' short rows keep k_xreal; capped, their
// batched step was 5 % slower.
template <int N, int OP, int G, bool KM = false>
__global__ void __launch_bounds__(XRShape<N, G, KM>::BLK, 3) k_xreal_long(XArgs a) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    xreal_body<N, OP, G, KM>(a, launch_blk(), smraw);
}

// ------------------------------------------- Poisson solve on (y, z) planes
// With the k-major half spectrum, the y and z transforms of one kx are a
// contiguous N x N plane (ny = nz = N).  One CTA holds the plane in shared
// memory and runs y forward -> z forward * fac/N, z inverse (register
// hand-off, Plan::run_spectral) -> y inverse on it, so the plane crosses HBM
// / L2 once instead of three times.  GROUPS pencil groups of C pencils work
// side by side, each with its own [N][C] tile; every group runs the same
// number of rounds (idle in the last one if N / C is not a multiple), so the
// barriers inside the transforms stay uniform.
struct PlaneArgs {
    Grid g;
    float2* F;       // k-major half spectrum
    long long bs_F;  // elements between simulations of a batch
};

#ifndef ISF_PLANE_MAX_THREADS
#define ISF_PLANE_MAX_THREADS 1024
#endif
// the 128 x 128 plane's radix-16 pencils hold twice the registers per thread
#ifndef ISF_PLANE128_MAX_THREADS
#define ISF_PLANE128_MAX_THREADS 512
#endif
template <int N>
constexpr int plane_max_threads() { return N == 128 ? ISF_PLANE128_MAX_THREADS : ISF_PLANE_MAX_THREADS; }

template <int N, int MAXT = plane_max_threads<N>()>
struct PlaneShape {
    static constexpr int C = 16;
    static constexpr int NT = PlanPlane<N>::NT;
    static constexpr int GT = C * NT;  // threads of one pencil group
    static constexpr int GMAX = MAXT / GT > 0 ? MAXT / GT : 1;
    static constexpr int GROUPS = GMAX < (N / C) ? GMAX : (N / C);
    static constexpr int BLK = GROUPS * GT;
    static constexpr int ROUNDS = (N / C + GROUPS - 1) / GROUPS;
    static constexpr size_t SMEM = (size_t)N * N * sizeof(float2) + (size_t)GROUPS * N * C * sizeof(float2);
    static_assert(N % C == 0, "plane width");
};

template <int N, class Sh = PlaneShape<N>, class BarT = CtaBar>
__device__ __forceinline__ void plane_body(const PlaneArgs a, const Blk bk, unsigned char* smraw,
                                           const BarT& bar = BarT()) {
    constexpr int C = Sh::C, NT = Sh::NT, GT = Sh::GT;
    float2* plane = reinterpret_cast<float2*>(smraw);
    const int grp = bk.tid / GT, lt = bk.tid % GT;
    float2* tile = plane + N * N + grp * (N * C);
    const int kx = bk.x;
    float2* __restrict__ Fp = a.F + bk.y * a.bs_F + (long long)kx * N * N;
    float2 x[PlanPlane<N>::EMAX];
    const float2 zero = make_float2(0.f, 0.f);
    // every group's pencils exist in every round when the groups divide the
    // pencils evenly (N = 128: 4 groups, 2 rounds): no guard is compiled then
    constexpr bool kAllOn = (N / C) % Sh::GROUPS == 0;
    // y transforms: pencil = row z of the plane, lanes along y.  The forward
    // one reads its rows straight from HBM into registers and leaves them in
    // shared memory; the inverse one reads shared memory and writes HBM.  A
    // pencil's lanes are consecutive, so where they fit in one warp its stage
    // exchanges are ordered by the warp (pencil_bar); the z transforms'
    // lanes run across pencils and keep the CTA barrier.
    auto ysweep = [&](auto sign) {
        constexpr int S = decltype(sign)::value;
        const int t = lt % NT, q = lt / NT;
#pragma unroll 1
        for (int round = 0; round < Sh::ROUNDS; ++round) {
            const int z = (round * Sh::GROUPS + grp) * C + q;
            const bool on = kAllOn || z < N;
            auto src = [&](int j) -> float2 {
                if (S < 0) return on ? Fp[z * N + j] : zero;
                return on ? plane[z * N + j] : zero;
            };
            auto dst = [&](int j, const float2& v) {
                if (!on) return;
                if (S < 0)
                    plane[z * N + j] = v;
                else
                    Fp[z * N + j] = v;
            };
            PlanPlane<N>::template run<C, S, false>(x, t, q, tile, a.g.tw[1], src, dst, pencil_bar<NT, C>(bar));
            bar.sync();
        }
    };
    ysweep(std::integral_constant<int, -1>());
    // z: forward, * fac(kx, ky, kz) / N, inverse; pencil = column ky, lanes across ky
    {
        const int q = lt % C, t = lt / C;
        const double sx = a.g.s2[0][kx];
        const double sc = -0.25 * a.g.invN;
        const double* __restrict__ s2z = a.g.s2[2];
#pragma unroll 1
        for (int round = 0; round < Sh::ROUNDS; ++round) {
            const int ky = (round * Sh::GROUPS + grp) * C + q;
            const bool on = kAllOn || ky < N;
            const int kyc = on ? ky : 0;
            const double dxo = sx + a.g.s2[1][kyc];
            const bool zero_line = (kx == 0) && (kyc == 0);
            auto src = [&](int j) -> float2 { return on ? plane[j * N + ky] : zero; };
            auto dst = [&](int j, const float2& v) {
                if (on) plane[j * N + ky] = v;
            };
            // fac(k)/N, fac = -0.25 / sum_a (sin(pi k_a / n_a) / d_a)^2, fac(0) = 0
            // (parallel.jl:53-55, 63), as in the y/z pass YZ_FAC
            auto fmul = [&](int j, const float2& v) -> float2 {
                const float f = (zero_line && j == 0) ? 0.f : (float)(sc * __drcp_rn(dxo + __ldg(&s2z[j])));
                return cscale(v, f);
            };
            PlanPlane<N>::template run_spectral<C>(x, t, q, tile, a.g.tw[2], src, fmul, dst, bar);
            bar.sync();
        }
    }
    ysweep(std::integral_constant<int, +1>());
}

template <int N>
__global__ void __launch_bounds__(PlaneShape<N>::BLK) k_poisson_plane(PlaneArgs a) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    plane_body<N>(a, launch_blk(), smraw);
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
    // at least 1, at most the 32 resident CTAs an SM takes (short pencils
    // make small CTAs)
    static constexpr int MINB = (MINT / BLK) > 32 ? 32 : ((MINT / BLK) > 1 ? (MINT / BLK) : 1);
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// FULL: the row length is a multiple of C, so no column needs the past-the-end guard
template <int N, class T, int OP, int G, bool FULL = false, class BarT = CtaBar>
__device__ __forceinline__ void yzpass_body(const YZArgs a, const Blk bk, unsigned char* smraw,
                                            const BarT& bar = BarT()) {
    constexpr int C = YZShape<N, T>::C;
    constexpr int NT = Plan<N>::NT;
    const int grp = bk.tid / (C * NT), lt = bk.tid % (C * NT);
    T* sm = reinterpret_cast<T*>(smraw) + grp * (N * C);
    const int q = lt % C, t = lt / C;
    const int rl = a.row, ny = a.g.n[1];
    const int x0 = bk.x * C;
    const int o = bk.y * G + grp;
    long long stride, base;
    if (a.axis == 1) {
        stride = rl;
        base = x0 + (long long)o * rl * ny;
    } else {
        stride = (long long)rl * ny;
        base = x0 + (long long)o * rl;
    }
    T* __restrict__ data = reinterpret_cast<T*>(a.data) + bk.z * a.bstride;
    const float2* tw = a.g.tw[a.axis];
    T x[Plan<N>::EMAX];

    // columns past the row's end (a row length that is not a multiple of
    // C) read zeros and store nothing
    const bool valid = FULL || x0 + q < rl;
    auto gsrc = [&](int j) -> T { return valid ? data[base + j * stride + q] : T{}; };
    auto gdst = [&](int j, const T& v) {
        if (valid) data[base + j * stride + q] = v;
    };

    if constexpr (OP == YZ_FWD) {
        Plan<N>::template run<C, -1, false>(x, t, q, sm, tw, gsrc, gdst, bar);
    } else if constexpr (OP == YZ_INV) {
        Plan<N>::template run<C, +1, false>(x, t, q, sm, tw, gsrc, gdst, bar);
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
            Plan<N>::template run_spectral<C>(x, t, q, sm, tw, gsrc, mmul, gdst, bar);
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
            Plan<N>::template run_spectral<C>(x, t, q, sm, tw, gsrc, fmul, gdst, bar);
        }
    }
}

template <int N, class T, int OP, int G, bool FULL = false>
__global__ void __launch_bounds__(YZShape<N, T, OP, G>::BLK, YZShape<N, T, OP, G>::MINB) k_yzpass(YZArgs a) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    yzpass_body<N, T, OP, G, FULL>(a, launch_blk(), smraw);
}

}  // namespace isf
