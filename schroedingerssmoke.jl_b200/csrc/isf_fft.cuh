// Register-staged Stockham FFT engine for batches of pencils.
//
// A CTA transforms C pencils of length N.  Each pencil is worked by NT
// threads; in a stage of radix R every thread owns NBT = ceil(N/R / NT)
// butterflies and keeps their R inputs in registers:
//
//   butterfly i in [0, N/R), span p = product of the earlier radices,
//   k = i mod p,  x_r = in[i + r N/R] * w^(r k),  w = exp(S 2 pi i / (p R)),
//   y = DFT_R(x),  out[(i - k) R + k + r p] = y_r.
//
// The first stage gathers its inputs straight from the caller's source
// (global memory, with all loads of a thread issued back to back) and the
// last stage scatters straight to the caller's sink, so only the stage
// boundaries in between go through shared memory: one [N][C] tile per CTA,
// in place (a barrier after every gather and after every scatter).  The
// tile stores element (j, q) of pencil q at j*C + (q ^ ((j ^ (j >> 3)) mod C)):
// row-wise accesses (y/z passes: lanes over q) are conflict free for any
// swizzle since C * sizeof(T) is 128 bytes; this one also keeps the
// column-wise stage accesses of the x pass (lanes over j, strides 1, R and
// the grouped p-strides) within 1.04 x the ideal wavefront count for every
// radix plan (simulated per quarter / half warp for 16- / 8-byte elements).
//
// Forward transforms use S = -1 (unnormalised), inverse S = +1 (the 1/N of
// the reference's ifft is folded into the spectral multiply by the callers).
#pragma once
#include <initializer_list>

#include "isf_common.cuh"

namespace isf {

template <int C>
__device__ __forceinline__ int sidx(int j, int q) {
    static_assert(C == 8 || C == 16, "tile width");
    return j * C + (q ^ ((j ^ (j >> 3)) & (C - 1)));
}

// --------------------------------------------------------------- radix DFTs
template <int S, class T>
__device__ __forceinline__ void dft2(T& a, T& b) {
    T t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int S, class T>
__device__ __forceinline__ void dft4(T& x0, T& x1, T& x2, T& x3) {
    T a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), e = mul_si<S>(csub(x1, x3));
    x0 = cadd(a, c);
    x1 = cadd(b, e);
    x2 = csub(a, c);
    x3 = csub(b, e);
}

template <int S, class T>
__device__ __forceinline__ void dft3(T& x0, T& x1, T& x2) {
    const float h = 0.8660254037844386f;  // sin(pi/3)
    T t = cadd(x1, x2);
    T u = cscale(mul_si<S>(csub(x1, x2)), h);
    T m = csub(x0, cscale(t, 0.5f));
    x0 = cadd(x0, t);
    x1 = cadd(m, u);
    x2 = csub(m, u);
}

template <int S, class T>
__device__ __forceinline__ void dft8(T* x) {
    // even / odd radix-4 halves, then combine with w8^s, w8 = exp(S 2 pi i / 8)
    dft4<S>(x[0], x[2], x[4], x[6]);
    dft4<S>(x[1], x[3], x[5], x[7]);
    const float r = 0.70710678118654752f;
    T o1 = cscale(cadd(x[3], mul_si<S>(x[3])), r);  // w8^1 * O1
    T o2 = mul_si<S>(x[5]);                          // w8^2 * O2
    T o3 = cscale(csub(mul_si<S>(x[7]), x[7]), r);   // w8^3 * O3
    T e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6], o0 = x[1];
    x[0] = cadd(e0, o0);
    x[4] = csub(e0, o0);
    x[1] = cadd(e1, o1);
    x[5] = csub(e1, o1);
    x[2] = cadd(e2, o2);
    x[6] = csub(e2, o2);
    x[3] = cadd(e3, o3);
    x[7] = csub(e3, o3);
}

// Odd prime radix R = 2M + 1 from the symmetric pairs a_q = x_q + x_{R-q},
// b_q = x_q - x_{R-q} (q = 1..M):
//   y_k     = x_0 + sum_q cos(2 pi q k / R) a_q + S i sum_q sin(2 pi q k / R) b_q
//   y_{R-k} = x_0 + sum_q cos(2 pi q k / R) a_q - S i sum_q sin(2 pi q k / R) b_q
// for k = 1..M, with cos / sin of 2 pi m / R taken from the first M angles by
// the symmetries of m mod R.
template <int R, int S, class T>
__device__ __forceinline__ void dft_odd(T* x, const float* c, const float* sn) {
    constexpr int M = R / 2;
    T a[M], b[M];
#pragma unroll
    for (int q = 1; q <= M; ++q) {
        a[q - 1] = cadd(x[q], x[R - q]);
        b[q - 1] = csub(x[q], x[R - q]);
    }
    T y0 = x[0];
#pragma unroll
    for (int q = 0; q < M; ++q) y0 = cadd(y0, a[q]);
    T yk[R];
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        T re = x[0], im = cscale(b[0], 0.f);
#pragma unroll
        for (int q = 1; q <= M; ++q) {
            const int m = (q * k) % R;                 // angle 2 pi m / R
            const int mm = m <= M ? m : R - m;         // cos(2 pi m / R) = c[mm - 1]
            const float sg = m <= M ? 1.f : -1.f;      // sin(2 pi m / R) = sg * sn[mm - 1]
            re = cadd(re, cscale(a[q - 1], c[mm - 1]));
            im = cadd(im, cscale(b[q - 1], sg * sn[mm - 1]));
        }
        const T u = mul_si<S>(im);
        yk[k] = cadd(re, u);
        yk[R - k] = csub(re, u);
    }
    x[0] = y0;
#pragma unroll
    for (int k = 1; k < R; ++k) x[k] = yk[k];
}

template <int S, class T>
__device__ __forceinline__ void dft5(T* x) {
    // cos / sin of 2 pi / 5 and 4 pi / 5
    const float c[2] = {0.30901699437494742f, -0.80901699437494742f};
    const float sn[2] = {0.95105651629515357f, 0.58778525229247313f};
    dft_odd<5, S>(x, c, sn);
}

template <int S, class T>
__device__ __forceinline__ void dft7(T* x) {
    // cos / sin of 2 pi k / 7, k = 1, 2, 3
    const float c[3] = {0.62348980185873353f, -0.22252093395631440f, -0.90096886790241913f};
    const float sn[3] = {0.78183148246802981f, 0.97492791218182361f, 0.43388373911755812f};
    dft_odd<7, S>(x, c, sn);
}

// 16 = 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2;
//   X[k1 + 4 k2] = sum_n2 w4^(n2 k2) w16^(n2 k1) sum_n1 w4^(n1 k1) x[4 n1 + n2]
template <int S, class T>
__device__ __forceinline__ void dft16(T* x) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<S>(x[n2], x[4 + n2], x[8 + n2], x[12 + n2]);
    // twiddles w16^(n2 k1) on y[n2][k1] = x[4 k1 + n2], w16 = exp(S 2 pi i / 16)
    const float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
    const float Sf = S < 0 ? -1.f : 1.f;
    x[5] = cmul(x[5], make_float2(c1, Sf * s1));    // n2 = 1, k1 = 1: w^1
    x[9] = cmul(x[9], make_float2(h, Sf * h));      // n2 = 1, k1 = 2: w^2
    x[13] = cmul(x[13], make_float2(s1, Sf * c1));  // n2 = 1, k1 = 3: w^3
    x[6] = cmul(x[6], make_float2(h, Sf * h));      // n2 = 2, k1 = 1: w^2
    x[10] = mul_si<S>(x[10]);                       // n2 = 2, k1 = 2: w^4
    x[14] = cmul(x[14], make_float2(-h, Sf * h));   // n2 = 2, k1 = 3: w^6
    x[7] = cmul(x[7], make_float2(s1, Sf * c1));    // n2 = 3, k1 = 1: w^3
    x[11] = cmul(x[11], make_float2(-h, Sf * h));   // n2 = 3, k1 = 2: w^6
    x[15] = cmul(x[15], make_float2(-c1, -Sf * s1));  // n2 = 3, k1 = 3: w^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<S>(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3]);
    // x[4 k1 + k2] holds X[k1 + 4 k2]: transpose the 4 x 4 block
    T t;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = a + 1; b < 4; ++b) {
            t = x[4 * a + b];
            x[4 * a + b] = x[4 * b + a];
            x[4 * b + a] = t;
        }
}

template <int R, int S, class T>
__device__ __forceinline__ void dft(T* x) {
    if constexpr (R == 2) dft2<S>(x[0], x[1]);
    else if constexpr (R == 3) dft3<S>(x[0], x[1], x[2]);
    else if constexpr (R == 4) dft4<S>(x[0], x[1], x[2], x[3]);
    else if constexpr (R == 5) dft5<S>(x);
    else if constexpr (R == 7) dft7<S>(x);
    else if constexpr (R == 8) dft8<S>(x);
    else if constexpr (R == 16) dft16<S>(x);
    else static_assert(R == 2, "unsupported radix");
}

// ------------------------------------------------------------ stage pieces
template <int N, int NT, int R>
struct Stage {
    static constexpr int NB = N / R;
    static constexpr int NBT = (NB + NT - 1) / NT;
    static constexpr int E = NBT * R;
};

// x[b*R + r] := input r of butterfly i = t + b*NT, read through src(j)
template <int N, int NT, int R, class T, class Src>
__device__ __forceinline__ void gather(T* x, int t, const Src& src) {
    constexpr int NB = Stage<N, NT, R>::NB, NBT = Stage<N, NT, R>::NBT;
#pragma unroll
    for (int b = 0; b < NBT; ++b) {
        const int i = t + b * NT;
        if (NB % NT == 0 || i < NB) {
#pragma unroll
            for (int r = 0; r < R; ++r) x[b * R + r] = src(i + r * NB);
        }
    }
}

template <int N, int NT, int R, int P, int S, class T>
__device__ __forceinline__ void butterflies(T* x, int t, const float2* __restrict__ tw) {
    constexpr int NB = Stage<N, NT, R>::NB, NBT = Stage<N, NT, R>::NBT;
    static_assert(N % (P * R) == 0, "bad radix plan");
    constexpr int TS = N / (P * R);  // twiddle table stride
#pragma unroll
    for (int b = 0; b < NBT; ++b) {
        const int i = t + b * NT;
        if (NB % NT == 0 || i < NB) {
            if constexpr (P > 1) {
                const int k = i % P;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = __ldg(&tw[r * k * TS]);  // r*k*TS < N
                    if (S > 0) w.y = -w.y;
                    x[b * R + r] = cmul(x[b * R + r], w);
                }
            }
            dft<R, S>(x + b * R);
        }
    }
}

// dst(j, v) for every output j = (i - k) R + k + r P of this thread's butterflies
template <int N, int NT, int R, int P, class T, class Dst>
__device__ __forceinline__ void scatter(const T* x, int t, const Dst& dst) {
    constexpr int NB = Stage<N, NT, R>::NB, NBT = Stage<N, NT, R>::NBT;
#pragma unroll
    for (int b = 0; b < NBT; ++b) {
        const int i = t + b * NT;
        if (NB % NT == 0 || i < NB) {
            const int k = i % P;
            const int base = (i - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst(base + r * P, x[b * R + r]);
        }
    }
}

template <int A, int... B>
struct First {
    static constexpr int value = A;
};

// Runs stages (P, R), Rest... on x, which holds the inputs of stage (P, R);
// intermediate results go through the shared tile sm (pencil q), the final
// outputs to dst.  Ends without a barrier after the final scatter.
template <int N, int NT, int C, int S, class T, class Dst, class B, int P, int R, int... Rest>
__device__ __forceinline__ void pipeline(T* x, int t, int q, T* sm, const float2* __restrict__ tw, const Dst& dst,
                                         const B& bar) {
    butterflies<N, NT, R, P, S>(x, t, tw);
    if constexpr (sizeof...(Rest) == 0) {
        scatter<N, NT, R, P>(x, t, dst);
    } else {
        scatter<N, NT, R, P>(x, t, [&](int j, const T& v) { sm[sidx<C>(j, q)] = v; });
        bar.xsync();
        constexpr int R2 = First<Rest...>::value;
        gather<N, NT, R2>(x, t, [&](int j) { return sm[sidx<C>(j, q)]; });
        bar.xsync();
        pipeline<N, NT, C, S, T, Dst, B, P * R, Rest...>(x, t, q, sm, tw, dst, bar);
    }
}

// Like pipeline, but the last stage's outputs stay in x: butterfly
// i = t + b NT (i < N / R) holds output i + r P at x[b R + r].  That is
// exactly the input layout of a first stage of radix R with N / R
// butterflies, so an inverse transform whose radices run in the reverse
// order can start from these registers without a pass through shared memory.
template <int N, int NT, int C, int S, class T, class B, int P, int R, int... Rest>
__device__ __forceinline__ void pipeline_keep(T* x, int t, int q, T* sm, const float2* __restrict__ tw, const B& bar) {
    butterflies<N, NT, R, P, S>(x, t, tw);
    if constexpr (sizeof...(Rest) > 0) {
        scatter<N, NT, R, P>(x, t, [&](int j, const T& v) { sm[sidx<C>(j, q)] = v; });
        bar.xsync();
        constexpr int R2 = First<Rest...>::value;
        gather<N, NT, R2>(x, t, [&](int j) { return sm[sidx<C>(j, q)]; });
        bar.xsync();
        pipeline_keep<N, NT, C, S, T, B, P * R, Rest...>(x, t, q, sm, tw, bar);
    }
}

// --------------------------------------------------------------- radix plans
constexpr int isf_emax(int N, int NT, std::initializer_list<int> rs) {
    int m = 0;
    for (int r : rs) {
        const int nb = N / r;
        const int e = ((nb + NT - 1) / NT) * r;
        m = e > m ? e : m;
    }
    return m;
}

#define ISF_UNPAREN(...) __VA_ARGS__

// Supported pencil lengths: 2^a 3^b with 8 <= N <= 512, and 20, 40, 50, 56,
// 80, 100, 112, 160, 200 (radices 5 and 7).  NT = N / (first radix).
// FWD lists the radices in stage order, REV the same radices reversed (the
// inverse of run_spectral).
template <int N>
struct Plan;
#define ISF_PLAN(NN, R0, FWD, REV) ISF_PLAN_NAMED(Plan, NN, R0, FWD, REV)
#define ISF_PLAN_NAMED(NAME, NN, R0, FWD, REV)                                                              \
    template <>                                                                                             \
    struct NAME<NN> {                                                                                       \
        static constexpr int first = R0;                                                                    \
        static constexpr int NT = NN / R0;                                                                  \
        static constexpr int EMAX = isf_emax(NN, NN / R0, {ISF_UNPAREN FWD});                              \
        /* SYNC: barrier after the first gather (needed when src reads the tile) */                       \
        template <int C, int S, bool SYNC, class T, class Src, class Dst, class B = CtaBar>                 \
        static __device__ __forceinline__ void run(T* x, int t, int q, T* sm, const float2* __restrict__ tw, \
                                                   const Src& src, const Dst& dst, const B& bar = B()) {    \
            gather<NN, NN / R0, R0>(x, t, src);                                                             \
            if constexpr (SYNC) bar.sync();                                                                 \
            pipeline<NN, NN / R0, C, S, T, Dst, B, 1, ISF_UNPAREN FWD>(x, t, q, sm, tw, dst, bar);          \
        }                                                                                                   \
        /* forward transform, mul(j, v) on every output j in registers, inverse transform */               \
        /* (SYNC: barrier after the first gather, when src reads the tile)  */                             \
        template <int C, bool SYNC = false, class T, class Src, class Mul, class Dst, class B = CtaBar>     \
        static __device__ __forceinline__ void run_spectral(T* x, int t, int q, T* sm,                      \
                                                            const float2* __restrict__ tw, const Src& src,  \
                                                            const Mul& mul, const Dst& dst,                 \
                                                            const B& bar = B()) {                           \
            constexpr int NTh = NN / R0;                                                                    \
            gather<NN, NTh, R0>(x, t, src);                                                                 \
            if constexpr (SYNC) bar.sync();                                                                 \
            pipeline_keep<NN, NTh, C, -1, T, B, 1, ISF_UNPAREN FWD>(x, t, q, sm, tw, bar);                  \
            constexpr int RL = First<ISF_UNPAREN REV>::value, PL = NN / RL;                                 \
            constexpr int NBT = Stage<NN, NTh, RL>::NBT;                                                    \
            _Pragma("unroll") for (int b = 0; b < NBT; ++b) {                                               \
                const int i = t + b * NTh;                                                                  \
                if (PL % NTh == 0 || i < PL) {                                                              \
                    _Pragma("unroll") for (int r = 0; r < RL; ++r) x[b * RL + r] = mul(i + r * PL, x[b * RL + r]); \
                }                                                                                           \
            }                                                                                               \
            pipeline<NN, NTh, C, +1, T, Dst, B, 1, ISF_UNPAREN REV>(x, t, q, sm, tw, dst, bar);             \
        }                                                                                                   \
    };

ISF_PLAN(8, 8, (8), (8))
ISF_PLAN(12, 4, (4, 3), (3, 4))
ISF_PLAN(16, 4, (4, 4), (4, 4))
ISF_PLAN(24, 8, (8, 3), (3, 8))
ISF_PLAN(32, 8, (8, 4), (4, 8))
ISF_PLAN(48, 4, (4, 4, 3), (3, 4, 4))
ISF_PLAN(64, 8, (8, 8), (8, 8))
ISF_PLAN(96, 8, (8, 4, 3), (3, 4, 8))
ISF_PLAN(128, 8, (8, 4, 4), (4, 4, 8))
ISF_PLAN(192, 8, (8, 8, 3), (3, 8, 8))
ISF_PLAN(256, 8, (8, 8, 4), (4, 8, 8))
ISF_PLAN(384, 8, (8, 4, 4, 3), (3, 4, 4, 8))
ISF_PLAN(512, 8, (8, 8, 8), (8, 8, 8))
// lengths with factors 5 and 7
ISF_PLAN(20, 4, (4, 5), (5, 4))
ISF_PLAN(40, 8, (8, 5), (5, 8))
ISF_PLAN(50, 5, (5, 5, 2), (2, 5, 5))
ISF_PLAN(56, 8, (8, 7), (7, 8))
ISF_PLAN(80, 4, (4, 4, 5), (5, 4, 4))
ISF_PLAN(100, 4, (4, 5, 5), (5, 5, 4))
ISF_PLAN(112, 4, (4, 4, 7), (7, 4, 4))
ISF_PLAN(160, 8, (8, 4, 5), (5, 4, 8))
ISF_PLAN(200, 8, (8, 5, 5), (5, 5, 8))
#undef ISF_PLAN

// Plans of the (y, z) plane Poisson solver: Plan<N>, except N = 128 in two
// stages (16, 8), one shared-memory exchange per transform instead of two.
// The plane kernel keeps its pencils in shared memory, so its time follows
// the exchanges; the radix-16 butterfly's 16 complex registers per thread
// fit its float2 data (the psi passes keep Plan<128>).
#ifndef ISF_PLANE128_RADIX16
#define ISF_PLANE128_RADIX16 1
#endif
template <int N>
struct PlanPlane : Plan<N> {};
#if ISF_PLANE128_RADIX16
ISF_PLAN_NAMED(PlanPlane, 128, 16, (16, 8), (8, 16))
#endif
#undef ISF_PLAN_NAMED

}  // namespace isf
