// Instantiations and launchers of the FFT pass kernels for every supported
// pencil length (2^a 3^b, 8 <= n <= 512).
#include <atomic>

#include "isf_launch.h"
#include "isf_passes.cuh"

namespace isf {

bool supported_len(int n) {
    switch (n) {
        case 8: case 12: case 16: case 24: case 32: case 48: case 64:
        case 96: case 128: case 192: case 256: case 384: case 512:
            return true;
        default:
            return false;
    }
}

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
        default: return cudaErrorInvalidValue;     \
    }

// Kernels needing more than 48 KB of dynamic shared memory must opt in once
// per device.
template <class K>
static cudaError_t ensure_smem(K kernel, size_t smem, std::atomic<unsigned long long>& done) {
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

template <int N, int OP>
static cudaError_t launch_x_n(const XArgs& a, cudaStream_t s) {
    using Sh = XShape<N, OP>;
    static std::atomic<unsigned long long> done{0};
    cudaError_t e = ensure_smem(k_xpass<N, OP>, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const long long rows = (long long)a.g.n[1] * a.g.n[2];
    k_xpass<N, OP><<<(unsigned)(rows / Sh::C), Sh::BLK, Sh::SMEM, s>>>(a);
    return cudaGetLastError();
}

template <int OP>
static cudaError_t launch_x_op(const XArgs& a, cudaStream_t s) {
#define ISF_X(NN) return launch_x_n<NN, OP>(a, s)
    ISF_SIZE_SWITCH(a.g.n[0], ISF_X)
#undef ISF_X
}

cudaError_t launch_xpass(int op, const XArgs& a, cudaStream_t s) {
    switch (op) {
        case X_PSI_FWD: return launch_x_op<X_PSI_FWD>(a, s);
        case X_PSI_INV: return launch_x_op<X_PSI_INV>(a, s);
        case X_PSI_INV_NORM: return launch_x_op<X_PSI_INV_NORM>(a, s);
        case X_C_FWD: return launch_x_op<X_C_FWD>(a, s);
        case X_C_INV: return launch_x_op<X_C_INV>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int N, int OP>
static cudaError_t launch_xr_n(const XArgs& a, cudaStream_t s) {
    using Sh = XRShape<N>;
    static std::atomic<unsigned long long> done{0};
    cudaError_t e = ensure_smem(k_xreal<N, OP>, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const long long rows = (long long)a.g.n[1] * a.g.n[2];
    k_xreal<N, OP><<<(unsigned)(rows / (2 * Sh::C)), Sh::BLK, Sh::SMEM, s>>>(a);
    return cudaGetLastError();
}

template <int OP>
static cudaError_t launch_xr_op(const XArgs& a, cudaStream_t s) {
#define ISF_XR(NN) return launch_xr_n<NN, OP>(a, s)
    ISF_SIZE_SWITCH(a.g.n[0], ISF_XR)
#undef ISF_XR
}

cudaError_t launch_xreal(int op, const XArgs& a, cudaStream_t s) {
    switch (op) {
        case XR_FWD: return launch_xr_op<XR_FWD>(a, s);
        case XR_INV_GAUGE: return launch_xr_op<XR_INV_GAUGE>(a, s);
        case XR_INV_REAL: return launch_xr_op<XR_INV_REAL>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int N, class T, int OP>
static cudaError_t launch_yz_n(const YZArgs& a, cudaStream_t s) {
    using Sh = YZShape<N, T>;
    static std::atomic<unsigned long long> done{0};
    cudaError_t e = ensure_smem(k_yzpass<N, T, OP>, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const int other = (a.axis == 1) ? a.g.n[2] : a.g.n[1];
    dim3 grid((unsigned)(a.row / Sh::C), (unsigned)other);
    k_yzpass<N, T, OP><<<grid, Sh::BLK, Sh::SMEM, s>>>(a);
    return cudaGetLastError();
}

template <class T, int OP>
static cudaError_t launch_yz_op(const YZArgs& a, cudaStream_t s) {
#define ISF_YZ(NN) return launch_yz_n<NN, T, OP>(a, s)
    ISF_SIZE_SWITCH(a.g.n[a.axis], ISF_YZ)
#undef ISF_YZ
}

cudaError_t launch_yzpass_psi(int op, const YZArgs& a, cudaStream_t s) {
    switch (op) {
        case YZ_FWD: return launch_yz_op<float4, YZ_FWD>(a, s);
        case YZ_INV: return launch_yz_op<float4, YZ_INV>(a, s);
        case YZ_MASK: return launch_yz_op<float4, YZ_MASK>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_yzpass_c(int op, const YZArgs& a, cudaStream_t s) {
    switch (op) {
        case YZ_FWD: return launch_yz_op<float2, YZ_FWD>(a, s);
        case YZ_INV: return launch_yz_op<float2, YZ_INV>(a, s);
        case YZ_FAC: return launch_yz_op<float2, YZ_FAC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace isf
