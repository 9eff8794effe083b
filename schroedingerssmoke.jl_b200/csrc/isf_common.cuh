// Shared device helpers for the ISF sm_100a kernels.
//
// Layouts in HBM (identical to the reference's Julia arrays, 0-based):
//   cell index  c = x + nx*(y + ny*z)  (column-major, x fastest)
//   psi         float4 per cell = (re psi1, im psi1, re psi2, im psi2)
//               == NTuple{2,ComplexF32} of src/parallel.jl
//   velocity    one float4 (vx, vy, vz, 0) per cell of a padded
//               (nx+1) x (ny+1) x (nz+1) grid (internal to the handle), with
//               a periodic copy of the x = 0, y = 0 and z = 0 faces at x = nx,
//               y = ny, z = nz, so the +1 neighbour of any cell is a fixed
//               offset (+1, +pnx, +pnxy) and one 16-byte load gives all three
//               components of a cell
//   F           float2 per cell: the Poisson spectrum work array
//   particles   float3 per slot (AoS), dead slot = (-1,-1,-1)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace isf {

struct Grid {
    int n[3];          // grid_res
    long long N;       // nx*ny*nz
    float L[3];        // physical_size (integers in the reference, parallel.jl:12)
    float d[3];        // Float32(L/n)                      parallel.jl:46
    float inv_d2[3];   // inv.(d .^ 2f0)                    parallel.jl:150
    float dinv[3];     // inv.(d)                           benchmark.jl:62
    int d_pow2[3];     // d is a power of two: p * dinv == p / d exactly
    float feps[3];     // 4 ulp of n (a bound on 4 ulp of p / d for p <= L)
    float hbar, dt;
    const float2* tw[3];    // tw[a][j] = exp(-2 pi i j / n[a]) rounded from double
    const double2* mtab[3]; // per-axis Schroedinger phase factors exp(i th_a(k))
    const double* s2[3];    // (sin(pi k / n_a) / d_a)^2 in double
    double invN;            // 1 / N
    int pnx, pnxy;          // strides of the padded velocity grid: nx+1 (rounded up to the row alignment), pnx (ny+1)
    long long NP;           // cells of the padded velocity grid (float4 each)
    int norm_w;             // staggered interpolation weights divided by d (ISF_FLAG_NORMALIZED_WEIGHTS)
};

// floats per padded velocity cell: vx, vy, vz and one unused
constexpr int kVelComp = 4;

// index of cell (x, y, z), 0 <= x <= nx etc., in the padded velocity grid
__host__ __device__ __forceinline__ int pcell(const Grid& g, int x, int y, int z) {
    return x + g.pnx * y + g.pnxy * z;
}

// the periodic copies on the +faces of the padded velocity grid of the value
// at cell index pc (x == 0: cx, ...): seven predicated stores at the fixed
// offsets ox = nx, oy = ny pnx, oz = nz pnxy
__device__ __forceinline__ void pcopies(float4* __restrict__ vel, int pc, bool cx, bool cy, bool cz, int ox, int oy,
                                        int oz, float4 v) {
    if (cx) vel[pc + ox] = v;
    if (cy) vel[pc + oy] = v;
    if (cz) vel[pc + oz] = v;
    if (cx & cy) vel[pc + ox + oy] = v;
    if (cx & cz) vel[pc + ox + oz] = v;
    if (cy & cz) vel[pc + oy + oz] = v;
    if (cx & cy & cz) vel[pc + ox + oy + oz] = v;
}

// store the velocity v of cell (x, y, z) and its periodic copies on the
// +faces (only cells on a low face have copies)
__device__ __forceinline__ void pstore(const Grid& g, float4* __restrict__ vel, int x, int y, int z, float3 v) {
    const int pc = pcell(g, x, y, z);
    const float4 w = make_float4(v.x, v.y, v.z, 0.f);
    vel[pc] = w;
    const bool cx = x == 0, cy = y == 0, cz = z == 0;
    if (cx | cy | cz) pcopies(vel, pc, cx, cy, cz, g.n[0], g.n[1] * g.pnx, g.n[2] * g.pnxy, w);
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization (launch_pdl in isf_launch.h) may start while the kernel
// before it drains.  pdl_enter lets the next kernel's CTAs be scheduled and
// then waits until the previous kernel has finished and its writes are
// visible; every such kernel calls it before its first global memory access.
// Without the launch attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// The barrier of the threads that run one CTA's work: the whole CTA for a
// kernel launched on its own (CtaBar), or the named barrier of one virtual
// CTA, n threads of a larger block, in the persistent batch kernel
// (NamedBar; ids 1..15, n a multiple of 32).
// xsync() orders the exchanges between FFT stages (isf_fft.cuh); for
// these two it is the same barrier as sync().
struct CtaBar {
    static constexpr bool kLaunch = true;
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ void xsync() const { __syncthreads(); }
};
struct NamedBar {
    static constexpr bool kLaunch = false;
    int id, n;
    __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
    __device__ __forceinline__ void xsync() const { sync(); }
};

// The barriers of a pass whose every pencil is held by lanes of one warp
// (NT lanes per pencil with NT dividing 32, the C pencils of a group laid
// out lane after lane from a warp boundary).  An exchange between FFT stages
// writes and reads only its own pencil's slots of the shared tile, so it
// orders the warp (__syncwarp); sync() stays the barrier of the whole
// (virtual) CTA for the steps that share the tile across pencils.
template <class B>
struct WarpXBar {
    static constexpr bool kLaunch = B::kLaunch;
    B b;
    __device__ __forceinline__ void sync() const { b.sync(); }
    __device__ __forceinline__ void xsync() const { __syncwarp(); }
};
template <int NT, int C, class B>
__device__ __forceinline__ auto pencil_bar(const B& b) {
    if constexpr (NT <= 32 && 32 % NT == 0 && (NT * C) % 32 == 0) return WarpXBar<B>{b};
    else return b;
}

// Block coordinates and thread index of one (virtual) CTA: blockIdx /
// threadIdx for a kernel launched on its own, the work item's in the
// persistent batch kernel.
struct Blk {
    int x, y, z, tid;
};
__device__ __forceinline__ Blk launch_blk() {
    return Blk{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)threadIdx.x};
}

// A load of data that another pass writes: through the read-only path in a
// kernel launched on its own (the data is constant for its lifetime), a
// plain coherent load in the persistent batch kernel, where the writer ran
// earlier in the same launch.
template <class B, class T>
__device__ __forceinline__ T ldm(const T* p) {
    if constexpr (B::kLaunch) return __ldg(p);
    else return *p;
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float4 cadd(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 csub(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
__device__ __forceinline__ float4 cmul(float4 a, float2 w) {
    return make_float4(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x, a.z * w.x - a.w * w.y, a.z * w.y + a.w * w.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float4 cscale(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
// multiply by S*i (S = +1 or -1): (x + iy)(S i) = -S y + i S x
template <int S>
__device__ __forceinline__ float2 mul_si(float2 a) {
    return S < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
template <int S>
__device__ __forceinline__ float4 mul_si(float4 a) {
    return S < 0 ? make_float4(a.y, -a.x, a.w, -a.z) : make_float4(-a.y, a.x, -a.w, a.z);
}

__host__ __device__ __forceinline__ long long cell(const Grid& g, int x, int y, int z) {
    return (long long)x + (long long)g.n[0] * ((long long)y + (long long)g.n[1] * z);
}

// atan2(y, x) for the one-form angles: t = min(|x|,|y|) / max(|x|,|y|) in
// [0, 1], atan(t) = t P(t^2) with the degree-8 polynomial fitted by
// csrc/gen_atan_coeffs.py (Remez exchange, max error 1.1e-7 in float32), then
// the octant / quadrant fix-ups.  |error| <= 2.5e-7 rad for finite inputs;
// angle(0) = 0 as in Julia.
__device__ __forceinline__ float isf_atan2(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    const float t = (mx > 0.f) ? __fdividef(mn, mx) : 0.f;
    const float s = t * t;
    float p = 2.456725575e-03f;
    p = fmaf(p, s, -1.440136135e-02f);
    p = fmaf(p, s, 3.978123143e-02f);
    p = fmaf(p, s, -7.234857976e-02f);
    p = fmaf(p, s, 1.049894616e-01f);
    p = fmaf(p, s, -1.416122913e-01f);
    p = fmaf(p, s, 1.998590678e-01f);
    p = fmaf(p, s, -3.333259821e-01f);
    p = fmaf(p, s, 9.999998808e-01f);
    float a = t * p;
    if (ay > ax) a = 1.57079632679489662f - a;
    if (x < 0.f) a = 3.14159265358979324f - a;
    return copysignf(a, y);
}

// Julia `angle(conj(a1)*b1 + conj(a2)*b2)` for psi pairs a, b (parallel.jl:108-111)
__device__ __forceinline__ float pair_angle(float4 a, float4 b) {
    // conj(a1)*b1 = (a.x - i a.y)(b.x + i b.y)
    float re = a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    float im = a.x * b.y - a.y * b.x + a.z * b.w - a.w * b.z;
    return isf_atan2(im, re);
}

// particles.jl:6-10, evaluated in float with every operation rounded on its
// own (no fused multiply-add), as the reference's broadcast over Float32
// positions does.
__device__ __forceinline__ bool isjet_f32(float px, float py, float pz, const float* cen, float len, float rad) {
    float dx = fabsf(__fsub_rn(px, cen[0]));
    float h = __fdiv_rn(len, 2.0f);
    float dy = __fsub_rn(py, cen[1]);
    float dz = __fsub_rn(pz, cen[2]);
    float s = __fadd_rn(__fmul_rn(dy, dy), __fmul_rn(dz, dz));
    return (dx <= h) && (s <= __fmul_rn(rad, rad));
}

struct JetArgs {
    float kvec[3];
    float cen[3];
    float len, rad;
    float omgterm;
    int phase_mode;          // 0: reference tuple_dot = sum(k .+ x); 1: k . x
    const uint8_t* mask;     // optional precomputed isjet array (N bytes) or null
};

// restrict_kernel (particles.jl:12-20) for cell (x,y,z); returns true if
// the cell is a nozzle cell and v was replaced.
__device__ __forceinline__ bool restrict_cell(const Grid& g, const JetArgs& j, int x, int y, int z, long long c,
                                              float4& v) {
    const float px = __fmul_rn((float)x, g.d[0]);
    const float py = __fmul_rn((float)y, g.d[1]);
    const float pz = __fmul_rn((float)z, g.d[2]);
    bool jet = j.mask ? (j.mask[c] != 0) : isjet_f32(px, py, pz, j.cen, j.len, j.rad);
    if (!jet) return false;
    float ph;
    if (j.phase_mode == 0)
        ph = __fadd_rn(__fadd_rn(__fadd_rn(j.kvec[0], px), __fadd_rn(j.kvec[1], py)), __fadd_rn(j.kvec[2], pz));
    else
        ph = j.kvec[0] * px + j.kvec[1] * py + j.kvec[2] * pz;
    ph = ph - j.omgterm;
    float s, co;
    sincosf(ph, &s, &co);
    const float a1 = hypotf(v.x, v.y), a2 = hypotf(v.z, v.w);
    v = make_float4(a1 * co, a1 * s, a2 * co, a2 * s);
    return true;
}

// normalize_psi (parallel.jl:162-165): psi * (1 / |psi|) with the
// reciprocal square root rounded once, then four products (within 1.5 ulp of
// the four quotients psi / |psi|, at a quarter of their instructions)
__device__ __forceinline__ float4 normalize4(float4 v) {
    const float r = __frsqrt_rn(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w);
    return make_float4(v.x * r, v.y * r, v.z * r, v.w * r);
}

// gauge_transform (parallel.jl:125-129) with real q: psi * exp(-i q)
__device__ __forceinline__ float4 gauge4(float4 v, float q) {
    float s, c;
    sincosf(q, &s, &c);
    // (a + ib)(c - is) = (ac + bs) + i(bc - as)
    return make_float4(v.x * c + v.y * s, v.y * c - v.x * s, v.z * c + v.w * s, v.w * c - v.z * s);
}

}  // namespace isf
