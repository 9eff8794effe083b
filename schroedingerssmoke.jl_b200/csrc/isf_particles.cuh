// Device helpers of the particle kernels shared by the advection and the
// emission (k_particles.cu), their adjoint (k_adjoint.cu) and the persistent
// batch kernel: Julia's periodic mod, the exact cell floor, the grid
// constants of the staggered interpolation, the interpolation itself, one
// slot's RK4 step, and the seeded emission stream.
#pragma once
#include "isf_launch.h"

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
    if (__builtin_expect(fr > eps && fr < 1.f - eps, 1)) return f1;
    return floorf(__fdiv_rn(p, d));
}

// The grid constants the advection needs, copied once into registers (the
// kernel parameter is otherwise re-read at every RK stage).
struct AdvConst {
    float L[3], d[3], dinv[3], feps[3];
    float nmf[3];  // n - 1 as a float
    int nm[3];  // n - 1
    int pnx, pnxy;
    float pnxf, pnxyf;  // the padded strides as floats (cell indices below 2^24 are exact)
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
    c.pnxf = (float)g.pnx;
    c.pnxyf = (float)g.pnxy;
    c.v = reinterpret_cast<const float4*>(vel);
    c.NP = g.NP;
    return c;
}

// Philox4x32-10 (Salmon et al., SC'11): ten rounds of two 32x32->64-bit
// multiplies, round keys bumped by the Weyl constants after each round.
struct U4 {
    uint32_t v[4];
};
__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.v[0]), lo0 = M0 * c.v[0];
        const uint32_t hi1 = __umulhi(M1, c.v[2]), lo1 = M1 * c.v[2];
        U4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// add_particles! (particles.jl:30-94) with a seeded counter-based stream.
// Stream: counter = (j, counter_lo, counter_hi, 0x15F0015F), key = seed.
// mode 0: the reference ring (0.9 r around (x - 0.1) with +-0.05 jitter,
//         particles.jl:86-90); 1: uniform in the nozzle disc at x = cen.x;
//         2: uniform in the nozzle cylinder; 3: the MatlabPort driver's ring
//         (0.9 r in the plane x = cen.x, no jitter,
//         examples/matlabport/simple.jl:112-115).
__device__ __forceinline__ float3 emit_point(long long j, const EmitArgs& e) {
    U4 c = {{(uint32_t)j, (uint32_t)e.counter, (uint32_t)(e.counter >> 32), 0x15F0015Fu}};
    const U4 r = philox4x32_10(c, (uint32_t)e.seed, (uint32_t)(e.seed >> 32));
    const float u0 = u01(r.v[0]), u1 = u01(r.v[1]), u2 = u01(r.v[2]), u3 = u01(r.v[3]);
    const float pi = 3.14159265358979323846f;
    float p0, p1, p2;
    if (e.mode == 0 || e.mode == 3) {
        const float rt = __fmul_rn(__fmul_rn(u0, 2.0f), pi);
        const float rr = __fmul_rn(0.9f, e.rad);
        if (e.mode == 3) {
            p0 = e.cen[0];
            p1 = __fadd_rn(e.cen[1], __fmul_rn(rr, cosf(rt)));
            p2 = __fadd_rn(e.cen[2], __fmul_rn(rr, sinf(rt)));
        } else {
            const float o0 = __fsub_rn(__fmul_rn(u1, 0.1f), 0.05f);
            const float o1 = __fsub_rn(__fmul_rn(u2, 0.1f), 0.05f);
            const float o2 = __fsub_rn(__fmul_rn(u3, 0.1f), 0.05f);
            p0 = __fadd_rn(__fsub_rn(e.cen[0], 0.1f), o0);
            p1 = __fadd_rn(__fadd_rn(e.cen[1], __fmul_rn(rr, cosf(rt))), o1);
            p2 = __fadd_rn(__fadd_rn(e.cen[2], __fmul_rn(rr, sinf(rt))), o2);
        }
    } else {
        const float th = __fmul_rn(__fmul_rn(u0, 2.0f), pi);
        const float rho = __fmul_rn(e.rad, sqrtf(u1));
        p0 = (e.mode == 1) ? e.cen[0] : __fadd_rn(e.cen[0], __fmul_rn(__fsub_rn(u2, 0.5f), e.len));
        p1 = __fadd_rn(e.cen[1], __fmul_rn(rho, cosf(th)));
        p2 = __fadd_rn(e.cen[2], __fmul_rn(rho, sinf(th)));
    }
    return make_float3(p0, p1, p2);
}

#ifdef ISF_CHECK
// debug builds: validate a gather index, record the first bad one, read cell 0
__device__ __forceinline__ int checked(const AdvConst& k, int c, unsigned long long* chk, const int i[3]) {
    if (c < 0 || (long long)c >= k.NP) {
        if (chk && atomicAdd(&chk[0], 1ull) == 0) {
            chk[1] = (unsigned long long)(unsigned)c;
            for (int a = 0; a < 3; ++a) chk[2 + a] = (unsigned long long)(unsigned)i[a];
        }
        return 0;
    }
    return c;
}
#define ISF_IDX(c) checked(k, (c), chk, i)
#else
#define ISF_IDX(c) (c)
#endif

// mod.(point, L) for a sample point outside [0, L)^3: out of line, so the
// common in-box path carries none of its instructions
static __device__ __noinline__ float3 wrap_box(float3 p, float L0, float L1, float L2) {
    return make_float3(jl_mod_box(p.x, L0), jl_mod_box(p.y, L1), jl_mod_box(p.z, L2));
}

// staggered_velocity (parallel.jl:219-246) on the handle's padded velocity
// grid: seven 16-byte gathers (the cells whose components the reference's
// twelve samples need).  Interpolation weights are the reference's unnormalised
// w = p - (i-1) d.  An index that rounds to n (p rounded up to L by mod) is
// clamped to the last cell and counted.  INBOX: the caller knows the point
// lies in [0, L)^3 (the first RK stage of a live particle).  FIDX: the
// padded grid has at most 2^24 cells, so the base cell index is formed
// exactly in float from the floors and converted once.
template <bool POW2, bool NORMW, class B = CtaBar, bool INBOX = false, bool FIDX = false>
__device__ __forceinline__ float3 stag_vel(const AdvConst& k, float3 pt, unsigned& clamps, unsigned long long* chk) {
    if (!INBOX) {
        // mod.(point, ph_size): the identity for points inside the box.  For
        // x >= +0 and L > 0 the float order is the order of the bit patterns,
        // so x in [0, L) is one unsigned compare; -0 (in the box as a float)
        // takes the wrap, which returns it unchanged.
        const bool inbox = (__float_as_uint(pt.x) < __float_as_uint(k.L[0])) &&
                           (__float_as_uint(pt.y) < __float_as_uint(k.L[1])) &&
                           (__float_as_uint(pt.z) < __float_as_uint(k.L[2]));
        if (__builtin_expect(!inbox, 0)) pt = wrap_box(pt, k.L[0], k.L[1], k.L[2]);
    }
    const float P[3] = {pt.x, pt.y, pt.z};
    // The cell floor, its clamp and the weight stay in float (integer values,
    // exact).  The common case takes p * (1/d) away from an integer and below
    // n on all three axes, tested together with one branch; otherwise every
    // axis takes the exact floor (the IEEE quotient near an integer) and the
    // upper clamp.  P lies in [0, L] here, so the floor is >= 0 and only the
    // upper clamp can act; a NaN point keeps a NaN floor, which converts to
    // cell 0 and gives NaN weights as the clamped floor did.
    float fl[3];
    bool fast = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float q1 = P[a] * k.dinv[a];
        fl[a] = floorf(q1);
        if (!POW2) {
            const float fr = q1 - fl[a];
            fast = fast && fr > k.feps[a] && fr < 1.f - k.feps[a];
        }
        fast = fast && !(fl[a] > k.nmf[a]);
    }
    if (__builtin_expect(!fast, 0)) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            fl[a] = cell_floor_f<POW2>(P[a], k.dinv[a], k.d[a], k.feps[a]);
            if (fl[a] > k.nmf[a]) {  // mod rounded up to L
                ++clamps;
                fl[a] = k.nmf[a];
            }
        }
    }
    float w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        w[a] = __fsub_rn(P[a], __fmul_rn(fl[a], k.d[a]));
        if (NORMW) w[a] = __fdiv_rn(w[a], k.d[a]);
    }
    (void)chk;
    // the +1 neighbour mod(i, res) + 1 is the padded plane's next cell; the
    // seven cells as offsets from one base pointer
    const int sy = k.pnx, sz = k.pnxy;
#if defined(ISF_CHECK)
    constexpr bool kFloatIndex = false;
#else
    constexpr bool kFloatIndex = FIDX;
#endif
    int c000;
    int i[3];
    if constexpr (kFloatIndex) {
        c000 = __float2int_rz(__fmaf_rn(k.pnxyf, fl[2], __fmaf_rn(k.pnxf, fl[1], fl[0])));
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) i[a] = __float2int_rz(fl[a]);
        c000 = i[0] + sy * i[1] + sz * i[2];
    }
    (void)i;
#ifdef ISF_CHECK
    const float4* v = k.v;
    const float4 a000 = ldm<B>(v + ISF_IDX(c000)), a100 = ldm<B>(v + ISF_IDX(c000 + 1));
    const float4 a010 = ldm<B>(v + ISF_IDX(c000 + sy)), a001 = ldm<B>(v + ISF_IDX(c000 + sz));
    const float4 a011 = ldm<B>(v + ISF_IDX(c000 + sy + sz)), a101 = ldm<B>(v + ISF_IDX(c000 + 1 + sz));
    const float4 a110 = ldm<B>(v + ISF_IDX(c000 + 1 + sy));
#else
    // the reference's 12 samples (parallel.jl:224-234) from 7 cells
    const float4* b0 = k.v + c000;
    const float4* by = b0 + sy;
    const float4* bz = b0 + sz;
    const float4 a000 = ldm<B>(b0), a100 = ldm<B>(b0 + 1);
    const float4 a010 = ldm<B>(by), a001 = ldm<B>(bz);
    const float4 a011 = ldm<B>(by + sz), a101 = ldm<B>(bz + 1);
    const float4 a110 = ldm<B>(by + 1);
#endif
    const float x00 = a000.x, x10 = a010.x, x01 = a001.x, x11 = a011.x;
    const float y00 = a000.y, y10 = a100.y, y01 = a001.y, y11 = a101.y;
    const float z00 = a000.z, z10 = a100.z, z01 = a010.z, z11 = a110.z;
    const float wx = w[0], wy = w[1], wz = w[2];
    float3 u;
    // u_x bilinear in (y, z), u_y in (x, z), u_z in (x, y) (parallel.jl:230-245)
    u.x = (1.f - wz) * ((1.f - wy) * x00 + wy * x10) + wz * ((1.f - wy) * x01 + wy * x11);
    u.y = (1.f - wz) * ((1.f - wx) * y00 + wx * y10) + wz * ((1.f - wx) * y01 + wx * y11);
    u.z = (1.f - wy) * ((1.f - wx) * z00 + wx * z10) + wy * ((1.f - wx) * z01 + wx * z11);
    return u;
}


// staggered_advect (parallel.jl:197-216) of slot k: classical RK4 if the
// particle is inside the open box 0 < p < L, (-1,-1,-1) otherwise (a slot
// that holds (-1,-1,-1) already is not stored again).
template <bool POW2, bool NORMW, class B = CtaBar, bool FIDX = false>
__device__ __forceinline__ void advect_slot(const AdvConst& kc, float* __restrict__ parts, int k, float dt, float s6,
                                            unsigned& clamps, unsigned& live, unsigned long long* chk) {
    float3 p = make_float3(parts[3 * k], parts[3 * k + 1], parts[3 * k + 2]);
    const bool inside = (p.x > 0.f && p.x < kc.L[0]) && (p.y > 0.f && p.y < kc.L[1]) && (p.z > 0.f && p.z < kc.L[2]);
    if (inside) {
        ++live;
        // k2 = p .+ k1 .* dt .* 0.5f0 etc. (parallel.jl:201-212)
        const float3 k1 = stag_vel<POW2, NORMW, B, true, FIDX>(kc, p, clamps, chk);
        float3 q = make_float3(p.x + k1.x * dt * 0.5f, p.y + k1.y * dt * 0.5f, p.z + k1.z * dt * 0.5f);
        const float3 k2 = stag_vel<POW2, NORMW, B, false, FIDX>(kc, q, clamps, chk);
        q = make_float3(p.x + k2.x * dt * 0.5f, p.y + k2.y * dt * 0.5f, p.z + k2.z * dt * 0.5f);
        const float3 k3 = stag_vel<POW2, NORMW, B, false, FIDX>(kc, q, clamps, chk);
        q = make_float3(p.x + k3.x * dt, p.y + k3.y * dt, p.z + k3.z * dt);
        const float3 k4 = stag_vel<POW2, NORMW, B, false, FIDX>(kc, q, clamps, chk);
        p.x = p.x + s6 * (k1.x + 2.f * k2.x + 2.f * k3.x + k4.x);
        p.y = p.y + s6 * (k1.y + 2.f * k2.y + 2.f * k3.y + k4.y);
        p.z = p.z + s6 * (k1.z + 2.f * k2.z + 2.f * k3.z + k4.z);
    } else {
        if (p.x == -1.f && p.y == -1.f && p.z == -1.f) return;  // dead already
        p = make_float3(-1.f, -1.f, -1.f);
    }
    parts[3 * k] = p.x;
    parts[3 * k + 1] = p.y;
    parts[3 * k + 2] = p.z;
}
#undef ISF_IDX

}  // namespace isf
