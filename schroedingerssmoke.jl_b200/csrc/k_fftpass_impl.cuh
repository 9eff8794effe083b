// Launch templates of the FFT pass kernels, shared by k_fftpass.cu (G = 1 and
// the size / op / tile dispatch) and k_fftpass_g2.cu / k_fftpass_g4.cu (the
// grouped tiles, compiled in parallel).
#pragma once
#include <atomic>

#include "isf_launch.h"
#include "isf_passes.cuh"

namespace isf {

// pencil lengths that have grouped-tile (G = 2, 4) instantiations
constexpr int kMaxGroupedN = 128;
#define ISF_GROUPED_SIZES(M) M(8) M(12) M(16) M(24) M(32) M(48) M(64) M(96) M(128)
constexpr bool grouped_size(int n) {
    return n == 8 || n == 12 || n == 16 || n == 24 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128;
}

// Kernels needing more than 48 KB of dynamic shared memory must opt in once
// per device.
template <class K>
cudaError_t ensure_smem(K kernel, size_t smem, std::atomic<unsigned long long>& done) {
    if (smem <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

inline unsigned batch_dim(int nsim) { return (unsigned)(nsim > 1 ? nsim : 1); }

template <int N, int OP, int G, bool FULL = false>
cudaError_t launch_x_ng(const XArgs& a, cudaStream_t s) {
    using Sh = XShape<N, OP, G>;
    static std::atomic<unsigned long long> done{0};
    const long long rows = (long long)a.g.n[1] * a.g.n[2];
    // grouped tiles (and the FULL variant) need whole tiles; single groups
    // guard a partial last one
    if ((G > 1 || FULL) && rows % (Sh::C * G) != 0) return cudaErrorInvalidValue;
    cudaError_t e = ensure_smem(k_xpass<N, OP, G, FULL>, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((rows + Sh::C * G - 1) / (Sh::C * G)), batch_dim(a.nsim));
    return launch_pdl(k_xpass<N, OP, G, FULL>, grid, dim3(Sh::BLK), Sh::SMEM, s, a);
}

template <int N, int OP, int G, bool KM = false>
cudaError_t launch_xr_ng(const XArgs& a, cudaStream_t s) {
    using Sh = XRShape<N, G, KM>;
    static std::atomic<unsigned long long> done{0};
    const long long rows = (long long)a.g.n[1] * a.g.n[2];
    if ((G > 1 || KM) && rows % (2 * Sh::C * G) != 0) return cudaErrorInvalidValue;
    constexpr auto kern = [] {
        if constexpr (N >= 256) return k_xreal_long<N, OP, G, KM>;
        else return k_xreal<N, OP, G, KM>;
    }();
    cudaError_t e = ensure_smem(kern, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((rows + 2 * Sh::C * G - 1) / (2 * Sh::C * G)), batch_dim(a.nsim));
    return launch_pdl(kern, grid, dim3(Sh::BLK), Sh::SMEM, s, a);
}

template <int N, class T, int OP, int G, bool FULL = false>
cudaError_t launch_yz_ng(const YZArgs& a, cudaStream_t s) {
    using Sh = YZShape<N, T, OP, G>;
    static std::atomic<unsigned long long> done{0};
    const int other = (a.axis == 1) ? a.g.n[2] : a.g.n[1];
    if (other % G != 0 || ((G > 1 || FULL) && a.row % Sh::C != 0)) return cudaErrorInvalidValue;
    cudaError_t e = ensure_smem(k_yzpass<N, T, OP, G, FULL>, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((a.row + Sh::C - 1) / Sh::C), (unsigned)(other / G), batch_dim(a.nsim));
    return launch_pdl(k_yzpass<N, T, OP, G, FULL>, grid, dim3(Sh::BLK), Sh::SMEM, s, a);
}

// every supported pencil length, each case expanding MACRO(n)
#define ISF_SIZE_SWITCH(n, MACRO)                  \
    switch (n) {                                   \
        case 8: MACRO(8);                          \
        case 12: MACRO(12);                        \
        case 16: MACRO(16);                        \
        case 24: MACRO(24);                        \
        case 32: MACRO(32);                        \
        case 48: MACRO(48);                        \
        case 64: MACRO(64);                        \
        case 96: MACRO(96);                        \
        case 128: MACRO(128);                      \
        case 192: MACRO(192);                      \
        case 256: MACRO(256);                      \
        case 384: MACRO(384);                      \
        case 512: MACRO(512);                      \
        case 20: MACRO(20);                        \
        case 40: MACRO(40);                        \
        case 50: MACRO(50);                        \
        case 56: MACRO(56);                        \
        case 80: MACRO(80);                        \
        case 100: MACRO(100);                      \
        case 112: MACRO(112);                      \
        case 160: MACRO(160);                      \
        case 200: MACRO(200);                      \
        default: return cudaErrorInvalidValue;     \
    }

// whole-tile launchers of the psi passes (k_fftpass_full.cu): the x passes
// X_PSI_* with the row count a multiple of 8, the y / z passes YZ_FWD /
// YZ_INV / YZ_MASK on float4 with the row length a multiple of 8
cudaError_t launch_xpass_full(int op, const XArgs& a, cudaStream_t s);
cudaError_t launch_yzpass_psi_full(int op, const YZArgs& a, cudaStream_t s);

// the grouped instantiations compiled in k_fftpass_g2.cu / k_fftpass_g4.cu:
// the ops the batch runs (EXT is empty there and `extern` in k_fftpass.cu)
#define ISF_GROUPED_DECLS(EXT, NN, G)                                                            \
    EXT template cudaError_t launch_x_ng<NN, X_PSI_FWD, G>(const XArgs&, cudaStream_t);          \
    EXT template cudaError_t launch_x_ng<NN, X_PSI_INV_NORM, G>(const XArgs&, cudaStream_t);     \
    EXT template cudaError_t launch_xr_ng<NN, XR_FWD, G>(const XArgs&, cudaStream_t);            \
    EXT template cudaError_t launch_xr_ng<NN, XR_INV_GAUGE, G>(const XArgs&, cudaStream_t);      \
    EXT template cudaError_t launch_xr_ng<NN, XR_INV_GAUGE_JET, G>(const XArgs&, cudaStream_t);  \
    EXT template cudaError_t launch_yz_ng<NN, float4, YZ_FWD, G>(const YZArgs&, cudaStream_t);   \
    EXT template cudaError_t launch_yz_ng<NN, float4, YZ_INV, G>(const YZArgs&, cudaStream_t);   \
    EXT template cudaError_t launch_yz_ng<NN, float4, YZ_MASK, G>(const YZArgs&, cudaStream_t);  \
    EXT template cudaError_t launch_yz_ng<NN, float2, YZ_FWD, G>(const YZArgs&, cudaStream_t);   \
    EXT template cudaError_t launch_yz_ng<NN, float2, YZ_INV, G>(const YZArgs&, cudaStream_t);   \
    EXT template cudaError_t launch_yz_ng<NN, float2, YZ_FAC, G>(const YZArgs&, cudaStream_t);

// is the op one of the grouped ones (x pass / real x pass / y-z pass)?
constexpr bool grouped_x_op(int op) { return op == X_PSI_FWD || op == X_PSI_INV_NORM; }
constexpr bool grouped_xr_op(int op) { return op == XR_FWD || op == XR_INV_GAUGE || op == XR_INV_GAUGE_JET; }
constexpr bool grouped_yz_op(int op, bool psi) { return psi ? (op == YZ_FWD || op == YZ_INV || op == YZ_MASK)
                                                            : (op == YZ_FWD || op == YZ_INV || op == YZ_FAC); }

}  // namespace isf
