// z-marching stencil kernels of the velocity one-form (the body is in
// isf_stencil.cuh): k_stencil for the one-form, k_stencil_div for the
// divergence.
#include "isf_stencil.cuh"

namespace isf {

// Both stencils are compiled for 4 resident CTAs per SM (at most 64
// registers).  The one-form stencil: 60 registers and 185 instructions per
// cell left to ptxas (35.9 us at 256x128x128), 64 and 181 capped (34.6 us).
template <int OP, bool JET, bool SHARP = false>
__global__ void __launch_bounds__(st::BX* st::TY, 4) k_stencil(StencilArgs a) {
    pdl_enter();
    __shared__ StencilSmem<OP> sm;
    stencil_body<OP, JET, SHARP>(a, launch_blk(), sm);
}

// The div stencil: 48 registers and 235 instructions per cell left to
// ptxas (40.9 us at 256x128x128), 64 and 200 capped (37.9 us).
template <bool JET>
__global__ void __launch_bounds__(st::BX* st::TY, 4) k_stencil_div(StencilArgs a) {
    pdl_enter();
    __shared__ StencilSmem<ST_DIV> sm;
    stencil_body<ST_DIV, JET>(a, launch_blk(), sm);
}

cudaError_t launch_stencil(int op, const StencilArgs& a, cudaStream_t s) {
    const int nsim = a.nsim > 1 ? a.nsim : 1;
    const int sz = op == ST_DIV ? st::planes_per_cta<ST_DIV>() : st::planes_per_cta<ST_VEL>();
    dim3 grid((unsigned)((a.g.n[0] + st::BX - 1) / st::BX), (unsigned)((a.g.n[1] + st::BY - 1) / st::BY),
              (unsigned)(((a.g.n[2] + sz - 1) / sz) * nsim));
    const dim3 blk(st::BX * st::TY);
    const bool jet = a.use_jet != 0;
    if (op == ST_DIV)
        return jet ? launch_pdl(k_stencil_div<true>, grid, blk, 0, s, a)
                   : launch_pdl(k_stencil_div<false>, grid, blk, 0, s, a);
    if (op == ST_VEL) {
        if (a.sharp)
            return jet ? launch_pdl(k_stencil<ST_VEL, true, true>, grid, blk, 0, s, a)
                       : launch_pdl(k_stencil<ST_VEL, false, true>, grid, blk, 0, s, a);
        return jet ? launch_pdl(k_stencil<ST_VEL, true>, grid, blk, 0, s, a)
                   : launch_pdl(k_stencil<ST_VEL, false>, grid, blk, 0, s, a);
    }
    return cudaErrorInvalidValue;
}

}  // namespace isf
