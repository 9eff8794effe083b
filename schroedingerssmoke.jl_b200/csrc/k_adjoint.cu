// Adjoint (reverse-mode) kernels of the ISF time step.
//
// Convention: psi is treated as 4 reals per cell; for a complex component z
// the adjoint zbar holds (dL/dRe z, dL/dIm z), so dL = Re(conj(zbar) dz)
// summed over components.  Each kernel maps the adjoint of a stage's output
// to the adjoint of its input (and of its parameters) at the forward input
// the caller passes; none of them is the reference's, which has no
// derivatives -- they differentiate its operators:
//   normalize_psi          parallel.jl:162-165
//   gauge_transform        parallel.jl:125-129 (real q)
//   velocity_one_form/div  parallel.jl:100-152 (angle derivative
//                          d angle(z) = Im(conj(z) dz) / |z|^2)
//   restrict_kernel        particles.jl:12-20
//   staggered_advect       parallel.jl:197-246 (RK4 and the unnormalised
//                          staggered interpolation, differentiated inside a
//                          cell; the jumps at cell faces carry no derivative)
#include "isf_launch.h"
#include "isf_particles.cuh"

namespace isf {

namespace {

inline unsigned grid_n(long long n, int block) {
    long long b = (n + block - 1) / block;
    const long long cap = 148LL * 32;
    return (unsigned)(b < cap ? b : cap);
}

__device__ __forceinline__ void decode_cell(const Grid& g, long long c, int& x, int& y, int& z) {
    x = (int)(c % g.n[0]);
    const long long r = c / g.n[0];
    y = (int)(r % g.n[1]);
    z = (int)(r / g.n[1]);
}

// z = conj(a1) b1 + conj(a2) b2 for psi pairs (the one-form's argument)
__device__ __forceinline__ float2 zpair(float4 a, float4 b) {
    return make_float2(a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w, a.x * b.y - a.y * b.x + a.z * b.w - a.w * b.z);
}

// block-wide sum of n doubles into acc[] (one atomicAdd per value per block)
template <int NV>
__device__ __forceinline__ void block_sum_add(double (&v)[NV], double* acc) {
    __shared__ double red[NV][32];
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nw ? red[k][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0 && s != 0.0) atomicAdd(&acc[k], s);
        }
    }
}

}  // namespace

// out = in exp(-i q) with a real q per cell (the forward gauge on its own)
__global__ void k_gauge(const float4* __restrict__ in, const float* __restrict__ q, float4* __restrict__ out,
                        long long N) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x)
        out[c] = gauge4(in[c], q[c]);
}

// out = normalize_psi(in)
__global__ void k_normalize_to(const float4* __restrict__ in, float4* __restrict__ out, long long N) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x)
        out[c] = normalize4(in[c]);
}

// out = restrict_velocity(in) (every cell written)
__global__ void k_restrict_to(Grid g, const float4* __restrict__ in, float4* __restrict__ out, JetArgs j) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode_cell(g, c, x, y, z);
        float4 v = in[c];
        restrict_cell(g, j, x, y, z, c, v);
        out[c] = v;
    }
}

// normalize: out = v / |v| (4 reals); bar_in = (bar_out - b (b . bar_out)) / |v|
__global__ void k_adj_normalize(const float4* __restrict__ psi_in, float4* __restrict__ bar, long long N) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
        const float4 v = psi_in[c];
        const float r = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w);
        if (!(r > 0.f)) {
            bar[c] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const float ir = 1.0f / r;
        const float4 b = make_float4(v.x * ir, v.y * ir, v.z * ir, v.w * ir);
        const float4 g = bar[c];
        const float d = b.x * g.x + b.y * g.y + b.z * g.z + b.w * g.w;
        bar[c] = make_float4((g.x - b.x * d) * ir, (g.y - b.y * d) * ir, (g.z - b.z * d) * ir, (g.w - b.w * d) * ir);
    }
}

// gauge: out = in exp(-i q).  qbar = sum_k Im(conj(bar_k) out_k);
// bar_in = bar_out exp(+i q)
__global__ void k_adj_gauge(const float4* __restrict__ psi_in, const float* __restrict__ q, float4* __restrict__ bar,
                            float* __restrict__ qbar, long long N) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
        const float qc = q[c];
        const float4 o = gauge4(psi_in[c], qc);
        const float4 g = bar[c];
        qbar[c] = (g.x * o.y - g.y * o.x) + (g.z * o.w - g.w * o.z);
        float s, co;
        sincosf(qc, &s, &co);
        bar[c] = make_float4(g.x * co - g.y * s, g.x * s + g.y * co, g.z * co - g.w * s, g.z * s + g.w * co);
    }
}

// Transpose of the one-form at psi, added into bar.  The one-form's cotangent
// per edge (cell i, axis a) is
//   mode 0: wbar_a[i] = s_a (fbar[i] - fbar[i + e_a])   (through div, s_a = 1/d_a^2)
//   mode 1: wbar_a[i] = s_a ubar_a[i]                    (velocity planes, s_a = hbar / d_a)
// and w_a[i] = angle(z), z = sum_k conj(psi_k[i]) psi_k[i+e_a], contributes
//   bar_k[i]     += wbar (-i conj(z) psi_k[i+e_a]) / |z|^2
//   bar_k[i+e_a] += wbar ( i z psi_k[i]) / |z|^2
// gathered here per cell from the edges i and i - e_a.
struct AdjOneFormArgs {
    Grid g;
    const float4* psi;
    float4* bar;
    const float* fbar;  // mode 0
    const float* ubar;  // mode 1: padded planes (copies folded into the cells they repeat)
    float s[3];
    int mode;
};

__global__ void k_adj_oneform(AdjOneFormArgs A) {
    const Grid& g = A.g;
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode_cell(g, c, x, y, z);
        const float4 p0 = A.psi[c];
        float4 acc = A.bar[c];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int xp = x, yp = y, zp = z, xm = x, ym = y, zm = z;
            if (a == 0) {
                xp = (x + 1 == nx) ? 0 : x + 1;
                xm = (x == 0) ? nx - 1 : x - 1;
            } else if (a == 1) {
                yp = (y + 1 == ny) ? 0 : y + 1;
                ym = (y == 0) ? ny - 1 : y - 1;
            } else {
                zp = (z + 1 == nz) ? 0 : z + 1;
                zm = (z == 0) ? nz - 1 : z - 1;
            }
            const long long cp = cell(g, xp, yp, zp), cm = cell(g, xm, ym, zm);
            float wh, wp;
            if (A.mode == 0) {
                const float f0 = A.fbar[c];
                wh = A.s[a] * (f0 - A.fbar[cp]);
                wp = A.s[a] * (A.fbar[cm] - f0);
            } else {
                const float* u = A.ubar + a * g.NP;
                wh = A.s[a] * u[pcell(g, x, y, z)];
                wp = A.s[a] * u[pcell(g, xm, ym, zm)];
            }
            const float4 pp = A.psi[cp], pm = A.psi[cm];
            const float2 z1 = zpair(p0, pp);
            const float n1 = z1.x * z1.x + z1.y * z1.y;
            if (n1 > 0.f && wh != 0.f) {
                const float t = wh / n1;
                // -i conj(z1) pp_k
                float mx = z1.x * pp.x + z1.y * pp.y, my = z1.x * pp.y - z1.y * pp.x;
                acc.x += t * my;
                acc.y -= t * mx;
                mx = z1.x * pp.z + z1.y * pp.w;
                my = z1.x * pp.w - z1.y * pp.z;
                acc.z += t * my;
                acc.w -= t * mx;
            }
            const float2 z2 = zpair(pm, p0);
            const float n2 = z2.x * z2.x + z2.y * z2.y;
            if (n2 > 0.f && wp != 0.f) {
                const float t = wp / n2;
                // i z2 pm_k
                float mx = z2.x * pm.x - z2.y * pm.y, my = z2.x * pm.y + z2.y * pm.x;
                acc.x -= t * my;
                acc.y += t * mx;
                mx = z2.x * pm.z - z2.y * pm.w;
                my = z2.x * pm.w + z2.y * pm.z;
                acc.z -= t * my;
                acc.w += t * mx;
            }
        }
        A.bar[c] = acc;
    }
}

// restrict_kernel: in the nozzle out_k = |in_k| exp(i phi), phi = phase(k, x)
// - omega t.  bar_in,k = Re(conj(bar_k) e^{i phi}) in_k / |in_k|; phibar =
// -sum_k Im(conj(bar_k) out_k); acc[0..2] += phibar dphi/dk_a, acc[3] +=
// -phibar wscale (the adjoint of omega t times wscale: t for the adjoint of
// omega itself).
__global__ void k_adj_restrict(Grid g, const float4* __restrict__ psi_in, float4* __restrict__ bar, JetArgs j,
                               double* __restrict__ acc, float wscale) {
    double v4[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode_cell(g, c, x, y, z);
        const float px = __fmul_rn((float)x, g.d[0]);
        const float py = __fmul_rn((float)y, g.d[1]);
        const float pz = __fmul_rn((float)z, g.d[2]);
        const bool jet = j.mask ? (j.mask[c] != 0) : isjet_f32(px, py, pz, j.cen, j.len, j.rad);
        if (!jet) continue;
        float ph;
        if (j.phase_mode == 0)
            ph = __fadd_rn(__fadd_rn(__fadd_rn(j.kvec[0], px), __fadd_rn(j.kvec[1], py)), __fadd_rn(j.kvec[2], pz));
        else
            ph = j.kvec[0] * px + j.kvec[1] * py + j.kvec[2] * pz;
        ph = ph - j.omgterm;
        float s, co;
        sincosf(ph, &s, &co);
        const float4 v = psi_in[c];
        const float a1 = hypotf(v.x, v.y), a2 = hypotf(v.z, v.w);
        const float4 o = make_float4(a1 * co, a1 * s, a2 * co, a2 * s);
        const float4 gb = bar[c];
        const float phb = -((gb.x * o.y - gb.y * o.x) + (gb.z * o.w - gb.w * o.z));
        const float r1 = gb.x * co + gb.y * s, r2 = gb.z * co + gb.w * s;
        const float i1 = a1 > 0.f ? r1 / a1 : 0.f, i2 = a2 > 0.f ? r2 / a2 : 0.f;
        bar[c] = make_float4(i1 * v.x, i1 * v.y, i2 * v.z, i2 * v.w);
        if (j.phase_mode == 0) {
            v4[0] += phb;
            v4[1] += phb;
            v4[2] += phb;
        } else {
            v4[0] += (double)phb * px;
            v4[1] += (double)phb * py;
            v4[2] += (double)phb * pz;
        }
        v4[3] -= (double)phb * wscale;
    }
    block_sum_add<4>(v4, acc);
}

// Add the padded planes' periodic copies (x = nx, y = ny or z = nz) into the
// cells they repeat and clear them: the cotangent of the one-form's stores.
__global__ void k_adj_fold(Grid g, float* __restrict__ ubar) {
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.NP; c += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(c % g.pnx);
        const long long r = c / g.pnx;
        const int y = (int)(r % (ny + 1)), z = (int)(r / (ny + 1));
        if (x > nx || !(x == nx || y == ny || z == nz)) continue;
        const int o = pcell(g, x == nx ? 0 : x, y == ny ? 0 : y, z == nz ? 0 : z);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float* u = ubar + a * g.NP;
            const float v = u[c];
            if (v != 0.f) atomicAdd(&u[o], v);
            u[c] = 0.f;
        }
    }
}

namespace {

// one staggered sample with everything its adjoint needs
struct Sample {
    int c000;
    float w[3];
    float v[12];  // x00 x10 x01 x11 | y00 y10 y01 y11 | z00 z10 z01 z11
    float3 u;
};

template <bool POW2, bool NORMW>
__device__ __forceinline__ void stag_sample(const AdvConst& k, float3 pt, Sample& S) {
    float P[3] = {pt.x, pt.y, pt.z};
    const bool inbox = (pt.x >= 0.f && pt.x < k.L[0]) && (pt.y >= 0.f && pt.y < k.L[1]) &&
                       (pt.z >= 0.f && pt.z < k.L[2]);
    if (!inbox) {
#pragma unroll
        for (int a = 0; a < 3; ++a) P[a] = jl_mod_box(P[a], k.L[a]);
    }
    int i[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int ii = cell_floor<POW2>(P[a], k.dinv[a], k.d[a], k.feps[a]);
        ii = max(min(ii, k.nm[a]), 0);
        i[a] = ii;
        S.w[a] = __fsub_rn(P[a], __fmul_rn((float)ii, k.d[a]));
        if (NORMW) S.w[a] = __fdiv_rn(S.w[a], k.d[a]);
    }
    const int sy = k.pnx, sz = k.pnxy;
    const int c000 = i[0] + sy * i[1] + sz * i[2];
    S.c000 = c000;
    const int c100 = c000 + 1, c010 = c000 + sy, c001 = c000 + sz;
    const float4 a000 = __ldg(k.v + c000), a100 = __ldg(k.v + c100), a010 = __ldg(k.v + c010);
    const float4 a001 = __ldg(k.v + c001), a011 = __ldg(k.v + c010 + sz), a101 = __ldg(k.v + c100 + sz);
    const float4 a110 = __ldg(k.v + c100 + sy);
    S.v[0] = a000.x;
    S.v[1] = a010.x;
    S.v[2] = a001.x;
    S.v[3] = a011.x;
    S.v[4] = a000.y;
    S.v[5] = a100.y;
    S.v[6] = a001.y;
    S.v[7] = a101.y;
    S.v[8] = a000.z;
    S.v[9] = a100.z;
    S.v[10] = a010.z;
    S.v[11] = a110.z;
    const float wx = S.w[0], wy = S.w[1], wz = S.w[2];
    S.u.x = (1.f - wz) * ((1.f - wy) * S.v[0] + wy * S.v[1]) + wz * ((1.f - wy) * S.v[2] + wy * S.v[3]);
    S.u.y = (1.f - wz) * ((1.f - wx) * S.v[4] + wx * S.v[5]) + wz * ((1.f - wx) * S.v[6] + wx * S.v[7]);
    S.u.z = (1.f - wy) * ((1.f - wx) * S.v[8] + wx * S.v[9]) + wy * ((1.f - wx) * S.v[10] + wx * S.v[11]);
}

// adjoint of one sample: ub = cotangent of u; returns the cotangent of the
// sample point and scatters ub times the weights into the velocity cotangent planes
template <bool NORMW>
__device__ __forceinline__ float3 stag_sample_adj(const AdvConst& k, const Sample& S, float3 ub, float* ubx, float* uby,
                                                  float* ubz) {
    const float wx = S.w[0], wy = S.w[1], wz = S.w[2];
    const float* v = S.v;
    // d u / d w (the weights are unnormalised: dw/dp = 1)
    const float dux_dwy = (1.f - wz) * (v[1] - v[0]) + wz * (v[3] - v[2]);
    const float dux_dwz = ((1.f - wy) * v[2] + wy * v[3]) - ((1.f - wy) * v[0] + wy * v[1]);
    const float duy_dwx = (1.f - wz) * (v[5] - v[4]) + wz * (v[7] - v[6]);
    const float duy_dwz = ((1.f - wx) * v[6] + wx * v[7]) - ((1.f - wx) * v[4] + wx * v[5]);
    const float duz_dwx = (1.f - wy) * (v[9] - v[8]) + wy * (v[11] - v[10]);
    const float duz_dwy = ((1.f - wx) * v[10] + wx * v[11]) - ((1.f - wx) * v[8] + wx * v[9]);
    float3 pb;
    pb.x = ub.y * duy_dwx + ub.z * duz_dwx;
    pb.y = ub.x * dux_dwy + ub.z * duz_dwy;
    pb.z = ub.x * dux_dwz + ub.y * duy_dwz;
    if (NORMW) {  // w = (p - i d) / d
        pb.x *= k.dinv[0];
        pb.y *= k.dinv[1];
        pb.z *= k.dinv[2];
    }
    const int sy = k.pnx, sz = k.pnxy;
    const int c000 = S.c000, c100 = c000 + 1, c010 = c000 + sy, c001 = c000 + sz;
    if (ub.x != 0.f) {
        atomicAdd(ubx + c000, ub.x * (1.f - wz) * (1.f - wy));
        atomicAdd(ubx + c010, ub.x * (1.f - wz) * wy);
        atomicAdd(ubx + c001, ub.x * wz * (1.f - wy));
        atomicAdd(ubx + c010 + sz, ub.x * wz * wy);
    }
    if (ub.y != 0.f) {
        atomicAdd(uby + c000, ub.y * (1.f - wz) * (1.f - wx));
        atomicAdd(uby + c100, ub.y * (1.f - wz) * wx);
        atomicAdd(uby + c001, ub.y * wz * (1.f - wx));
        atomicAdd(uby + c100 + sz, ub.y * wz * wx);
    }
    if (ub.z != 0.f) {
        atomicAdd(ubz + c000, ub.z * (1.f - wy) * (1.f - wx));
        atomicAdd(ubz + c100, ub.z * (1.f - wy) * wx);
        atomicAdd(ubz + c010, ub.z * wy * (1.f - wx));
        atomicAdd(ubz + c100 + sy, ub.z * wy * wx);
    }
    return pb;
}

__device__ __forceinline__ float3 f3add(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 f3scale(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }

}  // namespace

// Reverse of one RK4 advection (staggered_advect!, parallel.jl:197-216):
// lam holds the cotangent of the positions after the step and becomes that
// of the positions before it (parts, the positions the forward step started
// from); the cotangent of the velocity planes is added into ubar.  A slot
// outside the open box was set to (-1,-1,-1): its cotangent is 0.
template <bool POW2, bool NORMW>
__global__ void __launch_bounds__(256) k_adj_advect(Grid g, const float* __restrict__ parts, float* __restrict__ lam,
                                                    int np, const float* __restrict__ vel, float* __restrict__ ubar) {
    const AdvConst kc = adv_const(g, vel);
    float* ubx = ubar;
    float* uby = ubar + g.NP;
    float* ubz = ubar + 2 * g.NP;
    const float dt = g.dt, s6 = g.dt / 6.0f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        const float3 p = make_float3(parts[3 * k], parts[3 * k + 1], parts[3 * k + 2]);
        const bool inside = (p.x > 0.f && p.x < kc.L[0]) && (p.y > 0.f && p.y < kc.L[1]) &&
                            (p.z > 0.f && p.z < kc.L[2]);
        if (!inside) {
            lam[3 * k] = lam[3 * k + 1] = lam[3 * k + 2] = 0.f;
            continue;
        }
        Sample S1, S2, S3, S4;
        stag_sample<POW2, NORMW>(kc, p, S1);
        const float3 k1 = S1.u;
        float3 q = make_float3(p.x + k1.x * dt * 0.5f, p.y + k1.y * dt * 0.5f, p.z + k1.z * dt * 0.5f);
        stag_sample<POW2, NORMW>(kc, q, S2);
        const float3 k2 = S2.u;
        q = make_float3(p.x + k2.x * dt * 0.5f, p.y + k2.y * dt * 0.5f, p.z + k2.z * dt * 0.5f);
        stag_sample<POW2, NORMW>(kc, q, S3);
        const float3 k3 = S3.u;
        q = make_float3(p.x + k3.x * dt, p.y + k3.y * dt, p.z + k3.z * dt);
        stag_sample<POW2, NORMW>(kc, q, S4);
        // reverse of p' = p + dt/6 (k1 + 2 k2 + 2 k3 + k4)
        const float3 L = make_float3(lam[3 * k], lam[3 * k + 1], lam[3 * k + 2]);
        float3 pb = L;
        float3 kb1 = f3scale(L, s6), kb2 = f3scale(L, 2.f * s6), kb3 = f3scale(L, 2.f * s6);
        const float3 kb4 = f3scale(L, s6);
        float3 qb = stag_sample_adj<NORMW>(kc, S4, kb4, ubx, uby, ubz);  // q4 = p + dt k3
        pb = f3add(pb, qb);
        kb3 = f3add(kb3, f3scale(qb, dt));
        qb = stag_sample_adj<NORMW>(kc, S3, kb3, ubx, uby, ubz);  // q3 = p + dt/2 k2
        pb = f3add(pb, qb);
        kb2 = f3add(kb2, f3scale(qb, 0.5f * dt));
        qb = stag_sample_adj<NORMW>(kc, S2, kb2, ubx, uby, ubz);  // q2 = p + dt/2 k1
        pb = f3add(pb, qb);
        kb1 = f3add(kb1, f3scale(qb, 0.5f * dt));
        qb = stag_sample_adj<NORMW>(kc, S1, kb1, ubx, uby, ubz);  // k1 at p
        pb = f3add(pb, qb);
        lam[3 * k] = pb.x;
        lam[3 * k + 1] = pb.y;
        lam[3 * k + 2] = pb.z;
    }
}

// L = sum over slots alive in x (x >= 0) of |x - y|^2 (into loss[0], double);
// lam = dL/dx = 2 (x - y), 0 for dead slots
__global__ void k_loss(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ lam, int np,
                       double* __restrict__ loss) {
    double v[1] = {0.0};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        const bool alive = x[3 * k] >= 0.f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float d = alive ? x[3 * k + a] - y[3 * k + a] : 0.f;
            v[0] += (double)d * d;
            lam[3 * k + a] = 2.f * d;
        }
    }
    block_sum_add<1>(v, loss);
}

// velocity-plane cotangent from AoS float3 per cell: the cells themselves
// only (the periodic copies stay 0)
__global__ void k_adj_from_aos(Grid g, const float* __restrict__ aos, float* __restrict__ ubar) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode_cell(g, c, x, y, z);
        const int pc = pcell(g, x, y, z);
        ubar[pc] = aos[3 * c];
        ubar[g.NP + pc] = aos[3 * c + 1];
        ubar[2 * g.NP + pc] = aos[3 * c + 2];
    }
}

// the velocity cotangent (three padded planes, folded) as AoS float3 per cell
__global__ void k_adj_to_aos(Grid g, const float* __restrict__ ubar, float* __restrict__ aos) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.N; c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode_cell(g, c, x, y, z);
        const int pc = pcell(g, x, y, z);
        aos[3 * c] = ubar[pc];
        aos[3 * c + 1] = ubar[g.NP + pc];
        aos[3 * c + 2] = ubar[2 * g.NP + pc];
    }
}

// cotangent 0 for the ring slots an emission overwrote
__global__ void k_zero_slots(float* __restrict__ lam, long long nslots, long long start, long long count) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= count) return;
    const long long s = (start + j) % nslots;
    lam[3 * s] = lam[3 * s + 1] = lam[3 * s + 2] = 0.f;
}

// ---------------------------------------------------------------- launchers

cudaError_t launch_gauge(const Grid& g, const float4* in, const float* q, float4* out, cudaStream_t s) {
    k_gauge<<<grid_n(g.N, 256), 256, 0, s>>>(in, q, out, g.N);
    return cudaGetLastError();
}
cudaError_t launch_normalize_to(const Grid& g, const float4* in, float4* out, cudaStream_t s) {
    k_normalize_to<<<grid_n(g.N, 256), 256, 0, s>>>(in, out, g.N);
    return cudaGetLastError();
}
cudaError_t launch_restrict_to(const Grid& g, const float4* in, float4* out, const JetArgs& j, cudaStream_t s) {
    k_restrict_to<<<grid_n(g.N, 256), 256, 0, s>>>(g, in, out, j);
    return cudaGetLastError();
}
cudaError_t launch_adj_normalize(const Grid& g, const float4* psi_in, float4* bar, cudaStream_t s) {
    k_adj_normalize<<<grid_n(g.N, 256), 256, 0, s>>>(psi_in, bar, g.N);
    return cudaGetLastError();
}
cudaError_t launch_adj_gauge(const Grid& g, const float4* psi_in, const float* q, float4* bar, float* qbar,
                             cudaStream_t s) {
    k_adj_gauge<<<grid_n(g.N, 256), 256, 0, s>>>(psi_in, q, bar, qbar, g.N);
    return cudaGetLastError();
}
cudaError_t launch_adj_oneform_div(const Grid& g, const float4* psi, float4* bar, const float* fbar, cudaStream_t s) {
    AdjOneFormArgs a;
    a.g = g;
    a.psi = psi;
    a.bar = bar;
    a.fbar = fbar;
    a.ubar = nullptr;
    for (int k = 0; k < 3; ++k) a.s[k] = g.inv_d2[k];
    a.mode = 0;
    k_adj_oneform<<<grid_n(g.N, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_adj_oneform_vel(const Grid& g, const float4* psi, float4* bar, float* ubar, float hbar, int sharp,
                                   cudaStream_t s) {
    k_adj_fold<<<grid_n(g.NP, 256), 256, 0, s>>>(g, ubar);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    AdjOneFormArgs a;
    a.g = g;
    a.psi = psi;
    a.bar = bar;
    a.fbar = nullptr;
    a.ubar = ubar;
    for (int k = 0; k < 3; ++k) a.s[k] = sharp ? hbar * g.dinv[k] : hbar;
    a.mode = 1;
    k_adj_oneform<<<grid_n(g.N, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_adj_fold(const Grid& g, float* ubar, cudaStream_t s) {
    k_adj_fold<<<grid_n(g.NP, 256), 256, 0, s>>>(g, ubar);
    return cudaGetLastError();
}
cudaError_t launch_adj_restrict(const Grid& g, const float4* psi_in, float4* bar, const JetArgs& j, double* acc,
                                float wscale, cudaStream_t s) {
    k_adj_restrict<<<grid_n(g.N, 256), 256, 0, s>>>(g, psi_in, bar, j, acc, wscale);
    return cudaGetLastError();
}
cudaError_t launch_adj_advect(const Grid& g, const float* parts, float* lam, long long np, const float* vel,
                              float* ubar, cudaStream_t s) {
    if (np <= 0) return cudaSuccess;
    if (np > kMaxParticles) return cudaErrorInvalidValue;
    const unsigned b = grid_n(np, 256);
    const bool pow2 = g.d_pow2[0] && g.d_pow2[1] && g.d_pow2[2];
    if (g.norm_w) {
        if (pow2) k_adj_advect<true, true><<<b, 256, 0, s>>>(g, parts, lam, (int)np, vel, ubar);
        else k_adj_advect<false, true><<<b, 256, 0, s>>>(g, parts, lam, (int)np, vel, ubar);
    } else {
        if (pow2) k_adj_advect<true, false><<<b, 256, 0, s>>>(g, parts, lam, (int)np, vel, ubar);
        else k_adj_advect<false, false><<<b, 256, 0, s>>>(g, parts, lam, (int)np, vel, ubar);
    }
    return cudaGetLastError();
}
cudaError_t launch_loss(const float* x, const float* y, float* lam, long long np, double* loss, cudaStream_t s) {
    if (np <= 0) return cudaSuccess;
    k_loss<<<grid_n(np, 256), 256, 0, s>>>(x, y, lam, (int)np, loss);
    return cudaGetLastError();
}
cudaError_t launch_adj_from_aos(const Grid& g, const float* aos, float* ubar, cudaStream_t s) {
    k_adj_from_aos<<<grid_n(g.N, 256), 256, 0, s>>>(g, aos, ubar);
    return cudaGetLastError();
}
cudaError_t launch_adj_to_aos(const Grid& g, const float* ubar, float* aos, cudaStream_t s) {
    k_adj_to_aos<<<grid_n(g.N, 256), 256, 0, s>>>(g, ubar, aos);
    return cudaGetLastError();
}
cudaError_t launch_zero_slots(float* lam, long long nslots, long long start, long long count, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    k_zero_slots<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(lam, nslots, start % nslots, count);
    return cudaGetLastError();
}

}  // namespace isf
