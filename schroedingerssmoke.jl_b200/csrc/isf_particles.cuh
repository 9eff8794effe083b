// Device helpers of the particle kernels shared by the advection
// (k_particles.cu) and its adjoint (k_adjoint.cu): Julia's periodic mod, the
// exact cell floor and the grid constants of the staggered interpolation.
#pragma once
#include "isf_common.cuh"

namespace isf {

// Julia's mod(x, L) for floats and L > 0 (rem, then + L when negative, the
// addition rounded).  RK sample points lie within one box length of [0, L)
// in practice, where the result needs no fmod: for x in [L, 2L), fmod(x, L) =
// x - L is exact (Sterbenz); for x in (-L, 0), fmod(x, L) = x and the
// reference adds L.  Other values take the general path.
__device__ __forceinline__ float jl_mod_box(float x, float L) {
    if (x >= 0.f && x < L) return x;
    if (x >= L && x < 2.f * L) return x - L;
    if (x < 0.f && x > -L) return x + L;
    float r = fmodf(x, L);
    if (r == 0.f) return 0.f;  // copysign(0, L)
    if (r < 0.f) r += L;
    return r;
}

// floor(fl(p / d)) for p in [0, L]: with d a power of two p * (1/d) is exact;
// otherwise p * fl(1/d) differs from fl(p / d) by at most 3 ulp(p / d), so
// when it lies more than eps = 4 ulp(n) from an integer both have the same
// floor, and near an integer the IEEE quotient decides.
template <bool POW2>
__device__ __forceinline__ int cell_floor(float p, float dinv, float d, float eps) {
    const float q1 = p * dinv;
    if (POW2) return __float2int_rd(q1);
    const float f1 = floorf(q1);
    const float fr = q1 - f1;
    return (fr > eps && fr < 1.f - eps) ? (int)f1 : __float2int_rd(__fdiv_rn(p, d));
}

// The same floor as a float (an integer value): the advection clamps it,
// forms its weights and converts it once, with no int -> float round trip.
template <bool POW2>
__device__ __forceinline__ float cell_floor_f(float p, float dinv, float d, float eps) {
    const float q1 = p * dinv;
    const float f1 = floorf(q1);
    if (POW2) return f1;
    const float fr = q1 - f1;
    return (fr > eps && fr < 1.f - eps) ? f1 : floorf(__fdiv_rn(p, d));
}

// The grid constants the advection needs, copied once into registers (the
// kernel parameter is otherwise re-read at every RK stage).
struct AdvConst {
    float L[3], d[3], dinv[3], feps[3];
    float nmf[3];  // n - 1 as a float
    int nm[3];  // n - 1
    int pnx, pnxy;
    const float4* __restrict__ v;  // (vx, vy, vz, 0) per padded cell
    long long NP;
};

__device__ __forceinline__ AdvConst adv_const(const Grid& g, const float* vel) {
    AdvConst c;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        c.L[a] = g.L[a];
        c.d[a] = g.d[a];
        c.dinv[a] = g.dinv[a];
        c.feps[a] = g.feps[a];
        c.nm[a] = g.n[a] - 1;
        c.nmf[a] = (float)(g.n[a] - 1);
    }
    c.pnx = g.pnx;
    c.pnxy = g.pnxy;
    c.v = reinterpret_cast<const float4*>(vel);
    c.NP = g.NP;
    return c;
}

}  // namespace isf
