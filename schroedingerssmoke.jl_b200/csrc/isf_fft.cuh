// Shared-memory Stockham FFT engine for batches of pencils.
//
// One CTA holds C pencils of length N in shared memory as a [N][C] tile of
// elements T (float2: one complex value; float4: the two psi components,
// transformed together with shared twiddles).  C * sizeof(T) == 128 bytes,
// so every pencil position j is one 128-byte shared-memory row and every
// stage access touches whole rows (bank-conflict free).  The pencil index is
// XOR-swizzled with the low bits of j so that the transposing global loads of
// the x pass (lanes walking along j) are conflict free as well.
//
// Each stage is a radix-R Stockham step between two buffers (ping-pong):
//   butterfly i in [0, N/R), span p = product of the earlier radices,
//   k = i mod p,  x_r = in[i + r N/R] * w^(r k),  w = exp(S 2 pi i / (p R)),
//   y = DFT_R(x),  out[(i - k) R + k + r p] = y_r.
// Forward transforms use S = -1 (unnormalised), inverse S = +1 (the 1/N of
// the reference's ifft is folded into the spectral multiply by the callers).
#pragma once
#include "isf_common.cuh"

namespace isf {

template <int C>
__device__ __forceinline__ int sidx(int j, int q) {
    return j * C + (q ^ (j & (C - 1)));
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

template <int R, int S, class T>
__device__ __forceinline__ void dft(T* x) {
    if constexpr (R == 2) dft2<S>(x[0], x[1]);
    else if constexpr (R == 3) dft3<S>(x[0], x[1], x[2]);
    else if constexpr (R == 4) dft4<S>(x[0], x[1], x[2], x[3]);
    else if constexpr (R == 8) dft8<S>(x);
    else static_assert(R == 2, "unsupported radix");
}

// --------------------------------------------------------------- one stage
template <int N, int C, int NT, int R, int P, int S, class T>
__device__ __forceinline__ void fft_stage(const T* __restrict__ in, T* __restrict__ out,
                                          const float2* __restrict__ tw, int q, int t) {
    constexpr int NB = N / R;
    static_assert(N % (P * R) == 0, "bad radix plan");
    constexpr int TS = N / (P * R);  // twiddle table stride
#pragma unroll 1
    for (int i = t; i < NB; i += NT) {
        const int k = i % P;
        T x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = in[sidx<C>(i + r * NB, q)];
        if constexpr (P > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(&tw[r * k * TS]);  // r*k*TS < N
                if (S > 0) w.y = -w.y;
                x[r] = cmul(x[r], w);
            }
        }
        dft<R, S>(x);
        const int base = (i - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[sidx<C>(base + r * P, q)] = x[r];
    }
}

template <int N, int C, int NT, int S, class T, int P, int R, int... Rest>
__device__ __forceinline__ T* run_stages(T* a, T* b, const float2* __restrict__ tw, int q, int t) {
    fft_stage<N, C, NT, R, P, S, T>(a, b, tw, q, t);
    __syncthreads();
    if constexpr (sizeof...(Rest) == 0) {
        return b;
    } else {
        return run_stages<N, C, NT, S, T, P * R, Rest...>(b, a, tw, q, t);
    }
}

// Radix plans for the supported pencil lengths (2^a 3^b, 8 <= N <= 512).
template <int N>
struct Plan;
#define ISF_PLAN(NN, FIRST, ...)                                                                  \
    template <>                                                                                   \
    struct Plan<NN> {                                                                             \
        static constexpr int first = FIRST;                                                       \
        template <int C, int NT, int S, class T>                                                  \
        static __device__ __forceinline__ T* run(T* a, T* b, const float2* __restrict__ tw, int q, \
                                                 int t) {                                         \
            return run_stages<NN, C, NT, S, T, 1, __VA_ARGS__>(a, b, tw, q, t);                   \
        }                                                                                         \
    };
ISF_PLAN(8, 8, 8)
ISF_PLAN(12, 4, 4, 3)
ISF_PLAN(16, 4, 4, 4)
ISF_PLAN(24, 8, 8, 3)
ISF_PLAN(32, 8, 8, 4)
ISF_PLAN(48, 4, 4, 4, 3)
ISF_PLAN(64, 8, 8, 8)
ISF_PLAN(96, 8, 8, 4, 3)
ISF_PLAN(128, 8, 8, 4, 4)
ISF_PLAN(192, 8, 8, 8, 3)
ISF_PLAN(256, 8, 8, 8, 4)
ISF_PLAN(384, 8, 8, 4, 4, 3)
ISF_PLAN(512, 8, 8, 8, 8)
#undef ISF_PLAN

// threads per pencil: the butterfly count of the first stage, capped so that
// a CTA of C pencils stays within 1024 threads
template <int N, int C>
struct Threads {
    static constexpr int raw = N / Plan<N>::first;
    static constexpr int NT = (raw * C > 1024) ? 1024 / C : raw;
    static constexpr int block = NT * C;
};

template <int N, int C, int S, class T>
__device__ __forceinline__ T* fft_pencils(T* a, T* b, const float2* __restrict__ tw, int q, int t) {
    return Plan<N>::template run<C, Threads<N, C>::NT, S, T>(a, b, tw, q, t);
}

}  // namespace isf
