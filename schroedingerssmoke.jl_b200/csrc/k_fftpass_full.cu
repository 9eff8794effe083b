// Whole-tile instantiations of the psi passes (the Schroedinger step's x and
// y / z transforms): the launches whose rows (x) or row length (y / z) are a
// multiple of the tile, so the kernels carry no past-the-end guard.  The
// arithmetic of a pencil is that of the guarded kernels.
#include "k_fftpass_impl.cuh"

namespace isf {

namespace {

template <int OP>
cudaError_t x_full(const XArgs& a, cudaStream_t s) {
#define ISF_X(NN) return launch_x_ng<NN, OP, 1, true>(a, s)
    ISF_SIZE_SWITCH(a.g.n[0], ISF_X)
#undef ISF_X
}

template <int OP>
cudaError_t yz_full(const YZArgs& a, cudaStream_t s) {
#define ISF_YZ(NN) return launch_yz_ng<NN, float4, OP, 1, true>(a, s)
    ISF_SIZE_SWITCH(a.g.n[a.axis], ISF_YZ)
#undef ISF_YZ
}

}  // namespace

cudaError_t launch_xpass_full(int op, const XArgs& a, cudaStream_t s) {
    switch (op) {
        case X_PSI_FWD: return x_full<X_PSI_FWD>(a, s);
        case X_PSI_INV: return x_full<X_PSI_INV>(a, s);
        case X_PSI_INV_NORM: return x_full<X_PSI_INV_NORM>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_yzpass_psi_full(int op, const YZArgs& a, cudaStream_t s) {
    switch (op) {
        case YZ_FWD: return yz_full<YZ_FWD>(a, s);
        case YZ_INV: return yz_full<YZ_INV>(a, s);
        case YZ_MASK: return yz_full<YZ_MASK>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace isf
