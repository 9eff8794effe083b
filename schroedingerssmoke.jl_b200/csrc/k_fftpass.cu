// Instantiations and launchers of the FFT pass kernels for every supported
// pencil length (2^a 3^b with 8 <= n <= 512, and 20, 40, 50, 56, 80, 100,
// 112, 160, 200), and the dispatch over the tile shape (pencil groups per
// CTA) chosen by the caller.
#include "k_fftpass_impl.cuh"

namespace isf {

bool supported_len(int n) {
    switch (n) {
        case 8: case 12: case 16: case 24: case 32: case 48: case 64:
        case 96: case 128: case 192: case 256: case 384: case 512:
        case 20: case 40: case 50: case 56: case 80: case 100: case 112: case 160: case 200:
            return true;
        default:
            return false;
    }
}

// the grouped instantiations live in k_fftpass_g2.cu / k_fftpass_g4.cu
#define ISF_EXT2(NN) ISF_GROUPED_DECLS(extern, NN, 2)
#define ISF_EXT4(NN) ISF_GROUPED_DECLS(extern, NN, 4)
ISF_GROUPED_SIZES(ISF_EXT2)
ISF_GROUPED_SIZES(ISF_EXT4)
#undef ISF_EXT2
#undef ISF_EXT4

bool grouped_tile_ok(int n, int groups) {
    return groups <= 1 || ((groups == 2 || groups == 4) && grouped_size(n));
}


template <int N, int OP>
static cudaError_t launch_x_n(const XArgs& a, cudaStream_t s) {
    if constexpr (grouped_size(N) && grouped_x_op(OP)) {
        if (a.groups == 2) return launch_x_ng<N, OP, 2>(a, s);
        if (a.groups == 4) return launch_x_ng<N, OP, 4>(a, s);
    }
    if (a.groups > 1) return cudaErrorInvalidValue;
    return launch_x_ng<N, OP, 1>(a, s);
}

template <int OP>
static cudaError_t launch_x_op(const XArgs& a, cudaStream_t s) {
#define ISF_X(NN) return launch_x_n<NN, OP>(a, s)
    ISF_SIZE_SWITCH(a.g.n[0], ISF_X)
#undef ISF_X
}

cudaError_t launch_xpass(int op, const XArgs& a, cudaStream_t s) {
    const bool psi_op = op == X_PSI_FWD || op == X_PSI_INV || op == X_PSI_INV_NORM;
    if (psi_op && a.groups <= 1 && ((long long)a.g.n[1] * a.g.n[2]) % XTraits<X_PSI_FWD>::C == 0)
        return launch_xpass_full(op, a, s);
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
    if (a.kmajor) {
        if (a.groups > 1) return cudaErrorInvalidValue;
        return launch_xr_ng<N, OP, 1, true>(a, s);
    }
    if constexpr (grouped_size(N) && grouped_xr_op(OP)) {
        if (a.groups == 2) return launch_xr_ng<N, OP, 2>(a, s);
        if (a.groups == 4) return launch_xr_ng<N, OP, 4>(a, s);
    }
    if (a.groups > 1) return cudaErrorInvalidValue;
    return launch_xr_ng<N, OP, 1>(a, s);
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
        case XR_INV_GAUGE_JET: return launch_xr_op<XR_INV_GAUGE_JET>(a, s);
        case XR_INV_REAL: return launch_xr_op<XR_INV_REAL>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int N, class T, int OP>
static cudaError_t launch_yz_n(const YZArgs& a, cudaStream_t s) {
    constexpr bool psi = sizeof(T) == sizeof(float4);
    if constexpr (grouped_size(N) && grouped_yz_op(OP, psi)) {
        if (a.groups == 2) return launch_yz_ng<N, T, OP, 2>(a, s);
        if (a.groups == 4) return launch_yz_ng<N, T, OP, 4>(a, s);
    }
    if (a.groups > 1) return cudaErrorInvalidValue;
    return launch_yz_ng<N, T, OP, 1>(a, s);
}

template <class T, int OP>
static cudaError_t launch_yz_op(const YZArgs& a, cudaStream_t s) {
#define ISF_YZ(NN) return launch_yz_n<NN, T, OP>(a, s)
    ISF_SIZE_SWITCH(a.g.n[a.axis], ISF_YZ)
#undef ISF_YZ
}

cudaError_t launch_yzpass_psi(int op, const YZArgs& a, cudaStream_t s) {
    if (a.groups <= 1 && a.row % YZShape<8, float4>::C == 0) return launch_yzpass_psi_full(op, a, s);
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

// ---- the (y, z) plane Poisson solver of the k-major half spectrum

bool plane_supported(const int n[3]) {
    if (n[1] != n[2]) return false;
    switch (n[1]) {
        case 32: case 48: case 64: case 96: case 128:
            return true;
        default:
            return false;
    }
}

template <int N>
static cudaError_t launch_plane_n(const PlaneArgs& a, int nsim, cudaStream_t s) {
    using Sh = PlaneShape<N>;
    static std::atomic<unsigned long long> done{0};
    cudaError_t e = ensure_smem(k_poisson_plane<N>, Sh::SMEM, done);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)(a.g.n[0] / 2 + 1), batch_dim(nsim));
    return launch_pdl(k_poisson_plane<N>, grid, dim3(Sh::BLK), Sh::SMEM, s, a);
}

cudaError_t launch_poisson_plane(const Grid& g, float2* F, long long bs_F, int nsim, cudaStream_t s) {
    if (!plane_supported(g.n)) return cudaErrorInvalidValue;
    PlaneArgs a;
    a.g = g;
    a.F = F;
    a.bs_F = bs_F;
    switch (g.n[1]) {
        case 32: return launch_plane_n<32>(a, nsim, s);
        case 48: return launch_plane_n<48>(a, nsim, s);
        case 64: return launch_plane_n<64>(a, nsim, s);
        case 96: return launch_plane_n<96>(a, nsim, s);
        case 128: return launch_plane_n<128>(a, nsim, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace isf
