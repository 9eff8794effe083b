/*
 * ORACLE -- test infrastructure only.  Nothing in the product library links,
 * includes or calls this file; only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it (through oracle/oracle.py).
 *
 * CPU restatement of the incompressible-Schroedinger-flow (ISF) time step of
 * SchroedingersSmoke.jl, operator by operator, templated on the real type:
 *   - double: the FP64 oracle every GPU parity test compares against;
 *   - float : the FP32 restatement timed as the CPU baseline (same unfused
 *             operator sequence as the reference's `ArrayType = Array` path).
 *
 * Followed reference code (paths inside the reference project):
 *   ISF constructor, mask / fac / d        src/parallel.jl:41-98
 *   velocity_one_form(!)                   src/parallel.jl:100-122
 *   gauge_transform                        src/parallel.jl:125-129
 *   div / div!                             src/parallel.jl:131-152
 *   pressure_project!                      src/parallel.jl:155-160
 *   normalize_psi                          src/parallel.jl:162-165
 *   poisson_solve                          src/parallel.jl:168-174
 *   schroedinger_flow!                     src/parallel.jl:176-187
 *   in_grid / staggered_advect(!)          src/parallel.jl:190-216, 248-261
 *   staggered_velocity                     src/parallel.jl:219-246
 *   isjet / restrict_kernel / tuple_dot    src/particles.jl:1-27
 *   add_particles! (CPU and GPU forms)     src/particles.jl:30-94
 *   staggered sharp (velocity .*= 1 ./ d)  examples/benchmark.jl:61-63
 *   time-step order (simloop body)         examples/benchmark.jl:46-65
 * Cross-spec: src/MatlabPort.jl:75-273 (restated independently in numpy in
 * oracle/matlabport.py and compared in tests/test_oracle_cpu.py).
 *
 * FFT: FFTW / CLFFT (third-party, unpinned, not in the reference tree) are
 * replaced by a self-written recursive mixed-radix (2,3,4,5,7) decimation-in-time
 * DFT with the AbstractFFTs conventions the reference relies on: forward
 * exp(-2 pi i jk/n) unnormalised, inverse exp(+2 pi i jk/n) scaled by 1/N.
 * It is checked against numpy.fft in FP64.
 *
 * Parity status: UNPINNED against the reference's own outputs.  Julia is not
 * installed and the reference ships no golden vectors (its only test,
 * test/runtests.jl, has no assertions).  The oracle is pinned instead by
 * numpy.fft, by the independent MatlabPort restatement, and by analytic
 * known answers (tests/test_oracle_cpu.py).
 *
 * Layouts (identical to the reference's Julia arrays, 0-based here):
 *   cell index  c = x + nx*(y + ny*z)            (column-major, x fastest)
 *   psi         4 reals per cell: re1, im1, re2, im2   (NTuple{2,ComplexF32})
 *   velocity    3 reals per cell (AoS)                 (NTuple{3,Float32})
 *   particles   3 reals per slot (AoS); dead slot = (-1,-1,-1)
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "philox.h"

namespace {

const double kPi = 3.14159265358979323846264338327950288;

// ---------------------------------------------------------------- 1D FFT
template <class R>
struct Plan1D {
    using C = std::complex<R>;
    int n = 0;
    std::vector<int> radix;   // factorisation, outermost first
    std::vector<C> tw;        // tw[j] = exp(-2 pi i j / n)

    void init(int n_) {
        n = n_;
        radix.clear();
        int m = n;
        while (m % 4 == 0) { radix.push_back(4); m /= 4; }
        while (m % 2 == 0) { radix.push_back(2); m /= 2; }
        while (m % 3 == 0) { radix.push_back(3); m /= 3; }
        while (m % 5 == 0) { radix.push_back(5); m /= 5; }
        while (m % 7 == 0) { radix.push_back(7); m /= 7; }
        tw.resize(n);
        for (int j = 0; j < n; ++j) {
            long double a = -2.0L * (long double)kPi * (long double)j / (long double)n;
            tw[j] = C((R)std::cos(a), (R)std::sin(a));
        }
    }
    bool ok() const {
        int m = 1;
        for (int r : radix) m *= r;
        return m == n;
    }
    inline C W(long j, int sign) const {
        C w = tw[(size_t)(j % n)];
        return sign < 0 ? w : std::conj(w);
    }
    // out[0..len) = DFT_len(in[0], in[is], ...), radices radix[stage..]
    void rec(const C* in, long is, C* out, int len, int stage, int sign) const {
        if (len == 1) { out[0] = in[0]; return; }
        const int r = radix[stage];
        const int m = len / r;
        for (int q = 0; q < r; ++q) rec(in + q * is, is * r, out + q * m, m, stage + 1, sign);
        const long step = n / len;  // W_len^j = tw[j * step]
        for (int k = 0; k < m; ++k) {
            C t[7];
            for (int q = 0; q < r; ++q) {
                C v = out[q * m + k];
                t[q] = (q == 0 || k == 0) ? v : v * W((long)q * k * step, sign);
            }
            if (r == 2) {
                out[k] = t[0] + t[1];
                out[k + m] = t[0] - t[1];
            } else if (r == 4) {
                // y_s = sum_q t_q w^{qs}, w = exp(sign*2 pi i/4) = sign*i
                C a = t[0] + t[2], b = t[0] - t[2], c = t[1] + t[3], d = t[1] - t[3];
                C e = (sign < 0) ? C(d.imag(), -d.real()) : C(-d.imag(), d.real());
                out[k] = a + c;
                out[k + m] = b + e;
                out[k + 2 * m] = a - c;
                out[k + 3 * m] = b - e;
            } else if (r == 5 || r == 7) {
                // y_s = sum_q t_q w^{qs}, w = exp(sign 2 pi i / r) = W(n / r) (direct DFT)
                const long wr = n / r;
                for (int s = 0; s < r; ++s) {
                    C acc = t[0];
                    for (int q = 1; q < r; ++q) acc += t[q] * W((long)((q * s) % r) * wr, sign);
                    out[k + s * m] = acc;
                }
            } else {  // r == 3
                const R h = (R)0.866025403784438646763723170752936183L;  // sin(pi/3)
                C s = t[1] + t[2], dd = t[1] - t[2];
                C u = (sign < 0) ? C(dd.imag() * h, -dd.real() * h) : C(-dd.imag() * h, dd.real() * h);
                C mid = t[0] - s * (R)0.5;
                out[k] = t[0] + s;
                out[k + m] = mid + u;
                out[k + 2 * m] = mid - u;
            }
        }
    }
    void run(const C* in, C* out, int sign) const { rec(in, 1, out, n, 0, sign); }
};

// ---------------------------------------------------------------- 3D FFT
template <class R>
struct FFT3 {
    using C = std::complex<R>;
    int n[3];
    Plan1D<R> p[3];
    void init(const int* dims) {
        for (int a = 0; a < 3; ++a) { n[a] = dims[a]; p[a].init(dims[a]); }
    }
    bool ok() const { return p[0].ok() && p[1].ok() && p[2].ok(); }
    // in-place 3D DFT; sign -1 forward (unnormalised), +1 inverse (scaled 1/N)
    void run(C* a, int sign) const {
        const long nx = n[0], ny = n[1], nz = n[2];
        const long N = nx * ny * nz;
        // x axis: contiguous rows
#pragma omp parallel
        {
            std::vector<C> buf(nx);
#pragma omp for schedule(static)
            for (long row = 0; row < ny * nz; ++row) {
                C* r = a + row * nx;
                p[0].run(r, buf.data(), sign);
                std::copy(buf.begin(), buf.end(), r);
            }
        }
        // y and z axes: gather blocks of up to 16 consecutive x pencils
        for (int ax = 1; ax < 3; ++ax) {
            const long len = n[ax];
            const long stride = (ax == 1) ? nx : nx * ny;
            const long other = (ax == 1) ? nz : ny;
            const long other_stride = (ax == 1) ? nx * ny : nx;
            const long XB = 16;
            const long nxb = (nx + XB - 1) / XB;
#pragma omp parallel
            {
                std::vector<C> blk(XB * len), buf(len);
#pragma omp for schedule(static)
                for (long job = 0; job < nxb * other; ++job) {
                    const long xb = job % nxb, o = job / nxb;
                    const long x0 = xb * XB, xw = std::min(XB, nx - x0);
                    C* base = a + o * other_stride + x0;
                    for (long j = 0; j < len; ++j)
                        for (long q = 0; q < xw; ++q) blk[q * len + j] = base[j * stride + q];
                    for (long q = 0; q < xw; ++q) {
                        p[ax].run(&blk[q * len], buf.data(), sign);
                        std::copy(buf.begin(), buf.end(), blk.begin() + q * len);
                    }
                    for (long j = 0; j < len; ++j)
                        for (long q = 0; q < xw; ++q) base[j * stride + q] = blk[q * len + j];
                }
            }
        }
        if (sign > 0) {
            const R s = (R)(1.0 / (double)N);
#pragma omp parallel for schedule(static)
            for (long i = 0; i < N; ++i) a[i] *= s;
        }
    }
};

// Julia's `mod(x, y)` for floats (result has the sign of y; r + y is rounded).
template <class R>
inline R jl_mod(R x, R y) {
    R r = std::fmod(x, y);
    if (r == 0) return std::copysign((R)0, y);
    if ((r > 0) != (y > 0)) r += y;
    return r;
}

template <class R>
struct Orc {
    using C = std::complex<R>;
    int n[3];
    int L[3];
    R d[3];
    R hbar, dt;
    long N;
    FFT3<R> fft;
    std::vector<C> mask, fac, fc;  // fac kept complex like the reference (parallel.jl:47)
    std::vector<R> f, vel;         // vel: AoS, 3 per cell
    std::vector<C> psi1, psi2;     // temporaries (parallel.jl:31-32)
    long clamp_events = 0;         // staggered_velocity index == n+1 events
    bool norm_w = false;           // weights divided by d (the normalized-weights flag; the reference does not)

    long idx(long x, long y, long z) const { return x + (long)n[0] * (y + (long)n[1] * z); }

    // parallel.jl:41-98
    void init(const int* dims, const int* size, float hbar_f, float dt_f) {
        for (int a = 0; a < 3; ++a) {
            n[a] = dims[a];
            L[a] = size[a];
            d[a] = (R)((double)L[a] / (double)n[a]);  // VF(physical_size ./ grid_res)
        }
        hbar = (R)hbar_f;
        dt = (R)dt_f;
        N = (long)n[0] * n[1] * n[2];
        fft.init(n);
        mask.assign(N, C(0, 0));
        fac.assign(N, C(0, 0));
        const double fm = -4.0 * kPi * kPi * (double)hbar_f;  // f = -4*pi^2*hbar
        const double dd[3] = {(double)d[0], (double)d[1], (double)d[2]};
        for (long z = 0; z < n[2]; ++z)
            for (long y = 0; y < n[1]; ++y)
                for (long x = 0; x < n[0]; ++x) {
                    const long xyz[3] = {x, y, z};
                    double denom = 0, ksq = 0;
                    for (int a = 0; a < 3; ++a) {
                        double s = std::sin(kPi * (double)xyz[a] / (double)n[a]) / dd[a];
                        denom += s * s;
                        double k = ((double)xyz[a] - (double)n[a] / 2.0) / (double)L[a];
                        ksq += k * k;
                    }
                    fac[idx(x, y, z)] = C((R)(-0.25 / denom), 0);
                    const double lam = fm * ksq;
                    const double th = lam * (double)dt_f / 2.0;
                    // fftshift (parallel.jl:62): value computed at index i lands at (i + n/2) mod n
                    const long sx = (x + n[0] / 2) % n[0], sy = (y + n[1] / 2) % n[1], sz = (z + n[2] / 2) % n[2];
                    mask[idx(sx, sy, sz)] = C((R)std::cos(th), (R)std::sin(th));
                }
        fac[0] = C(0, 0);  // parallel.jl:63
        f.assign(N, 0);
        fc.assign(N, C(0, 0));
        vel.assign(3 * N, 0);
        psi1.assign(N, C(0, 0));
        psi2.assign(N, C(0, 0));
    }

    // parallel.jl:176-187
    void schroedinger_flow(R* psi) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            psi1[i] = C(psi[4 * i + 0], psi[4 * i + 1]);
            psi2[i] = C(psi[4 * i + 2], psi[4 * i + 3]);
        }
        fft.run(psi1.data(), -1);
        fft.run(psi2.data(), -1);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            psi1[i] *= mask[i];
            psi2[i] *= mask[i];
        }
        fft.run(psi1.data(), +1);
        fft.run(psi2.data(), +1);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            psi[4 * i + 0] = psi1[i].real();
            psi[4 * i + 1] = psi1[i].imag();
            psi[4 * i + 2] = psi2[i].real();
            psi[4 * i + 3] = psi2[i].imag();
        }
    }

    // parallel.jl:162-165
    void normalize(R* psi) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            C a(psi[4 * i], psi[4 * i + 1]), b(psi[4 * i + 2], psi[4 * i + 3]);
            R nrm = std::hypot(std::abs(a), std::abs(b));
            a /= nrm;
            b /= nrm;
            psi[4 * i] = a.real();
            psi[4 * i + 1] = a.imag();
            psi[4 * i + 2] = b.real();
            psi[4 * i + 3] = b.imag();
        }
    }

    // parallel.jl:100-122 (i_shifted = +1 neighbour with periodic wrap)
    void velocity_one_form(const R* psi, R hb) {
#pragma omp parallel for schedule(static)
        for (long z = 0; z < n[2]; ++z)
            for (long y = 0; y < n[1]; ++y)
                for (long x = 0; x < n[0]; ++x) {
                    const long c = idx(x, y, z);
                    const long nb[3] = {idx((x + 1) % n[0], y, z), idx(x, (y + 1) % n[1], z),
                                        idx(x, y, (z + 1) % n[2])};
                    C a(psi[4 * c], psi[4 * c + 1]), b(psi[4 * c + 2], psi[4 * c + 3]);
                    for (int ax = 0; ax < 3; ++ax) {
                        const long o = nb[ax];
                        C an(psi[4 * o], psi[4 * o + 1]), bn(psi[4 * o + 2], psi[4 * o + 3]);
                        C s = std::conj(a) * an + std::conj(b) * bn;
                        vel[3 * c + ax] = std::arg(s) * hb;
                    }
                }
    }

    // parallel.jl:131-152 (i_shifted2 = -1 neighbour with periodic wrap)
    void div() {
        R ds[3];
        for (int a = 0; a < 3; ++a) ds[a] = (R)1 / (d[a] * d[a]);  // inv.(d .^ 2f0)
#pragma omp parallel for schedule(static)
        for (long z = 0; z < n[2]; ++z)
            for (long y = 0; y < n[1]; ++y)
                for (long x = 0; x < n[0]; ++x) {
                    const long c = idx(x, y, z);
                    const long mx = idx((x + n[0] - 1) % n[0], y, z);
                    const long my = idx(x, (y + n[1] - 1) % n[1], z);
                    const long mz = idx(x, y, (z + n[2] - 1) % n[2]);
                    R t0 = (vel[3 * c + 0] - vel[3 * mx + 0]) * ds[0];
                    R t1 = (vel[3 * c + 1] - vel[3 * my + 1]) * ds[1];
                    R t2 = (vel[3 * c + 2] - vel[3 * mz + 2]) * ds[2];
                    f[c] = t0 + t1 + t2;
                }
    }

    // parallel.jl:168-174 (result stays complex, as in the reference)
    void poisson_solve() {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) fc[i] = C(f[i], 0);
        fft.run(fc.data(), -1);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) fc[i] *= fac[i];
        fft.run(fc.data(), +1);
    }

    // parallel.jl:125-129: psi * exp(i * (-q)), complex q
    void gauge(R* psi) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            C x = C(0, 1) * (-fc[i]);
            C e = std::exp(x);
            C a(psi[4 * i], psi[4 * i + 1]), b(psi[4 * i + 2], psi[4 * i + 3]);
            a *= e;
            b *= e;
            psi[4 * i] = a.real();
            psi[4 * i + 1] = a.imag();
            psi[4 * i + 2] = b.real();
            psi[4 * i + 3] = b.imag();
        }
    }

    // parallel.jl:155-160 (hbar = 1 inside the projection)
    void pressure_project(R* psi) {
        velocity_one_form(psi, (R)1);
        div();
        poisson_solve();
        gauge(psi);
    }

    // examples/benchmark.jl:61-63
    void staggered_sharp() {
        R dinv[3];
        for (int a = 0; a < 3; ++a) dinv[a] = (R)1 / d[a];
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i)
            for (int a = 0; a < 3; ++a) vel[3 * i + a] *= dinv[a];
    }

    // particles.jl:6-10, evaluated in float like the reference's Float32
    // positions (parallel.jl:75-77) so that both precisions see the same mask.
    static bool isjet_f32(const float p[3], const float cen[3], float len, float rad) {
        float dx = std::fabs(p[0] - cen[0]);
        float h = len / 2.0f;
        float dy = p[1] - cen[1], dz = p[2] - cen[2];
        float s = dy * dy;
        float t = dz * dz;
        float r2 = rad * rad;
        return (dx <= h) && (s + t <= r2);
    }

    // particles.jl:12-27; phase_mode 0 = reference tuple_dot (sum of k .+ pos),
    // 1 = k . pos (MatlabPort driver, examples/matlabport/simple.jl:47,107).
    // kvec and omgterm arrive in double and are rounded to R: the FP32
    // restatement sees Float32 values as the reference does, the FP64 oracle
    // keeps them exact (finite differences in the jet velocity need that).
    void restrict_velocity(R* psi, const double kvec[3], const uint8_t* jetmask, const float cen[3], float len,
                           float rad, double omgterm, int phase_mode) {
#pragma omp parallel for schedule(static)
        for (long z = 0; z < n[2]; ++z)
            for (long y = 0; y < n[1]; ++y)
                for (long x = 0; x < n[0]; ++x) {
                    const long c = idx(x, y, z);
                    bool jet;
                    if (jetmask) {
                        jet = jetmask[c] != 0;
                    } else {
                        const float pf[3] = {(float)x * (float)d[0], (float)y * (float)d[1], (float)z * (float)d[2]};
                        jet = isjet_f32(pf, cen, len, rad);
                    }
                    if (!jet) continue;
                    const R pos[3] = {(R)x * d[0], (R)y * d[1], (R)z * d[2]};
                    R ph;
                    if (phase_mode == 0)
                        ph = ((R)kvec[0] + pos[0]) + ((R)kvec[1] + pos[1]) + ((R)kvec[2] + pos[2]);
                    else
                        ph = (R)kvec[0] * pos[0] + (R)kvec[1] * pos[1] + (R)kvec[2] * pos[2];
                    ph -= (R)omgterm;
                    C a(psi[4 * c], psi[4 * c + 1]), b(psi[4 * c + 2], psi[4 * c + 3]);
                    C e = std::exp(C(0, 1) * ph);
                    C ra = std::abs(a) * e, rb = std::abs(b) * e;
                    psi[4 * c] = ra.real();
                    psi[4 * c + 1] = ra.imag();
                    psi[4 * c + 2] = rb.real();
                    psi[4 * c + 3] = rb.imag();
                }
    }

    // parallel.jl:219-246
    void staggered_velocity(const R pt[3], R out[3], double* margin, long* clamps) const {
        R p[3];
        long i[3], ip[3];
        R w[3];
        for (int a = 0; a < 3; ++a) {
            const R La = (R)L[a];
            p[a] = jl_mod(pt[a], La);
            R q = p[a] / d[a];
            long ii = (long)std::floor(q);
            if (ii >= n[a]) { ii = n[a] - 1; ++*clamps; }
            if (ii < 0) ii = 0;
            i[a] = ii;
            ip[a] = (ii + 1) % n[a];
            w[a] = p[a] - (R)ii * d[a];
            if (norm_w) w[a] = w[a] / d[a];
            if (margin) {
                double fr = (double)q - std::floor((double)q);
                double mg = std::min(fr, 1.0 - fr);
                if (mg < *margin) *margin = mg;
            }
        }
        auto V = [&](long x, long y, long z, int c) { return vel[3 * idx(x, y, z) + c]; };
        const R v0[3] = {V(i[0], i[1], i[2], 0), V(i[0], i[1], i[2], 1), V(i[0], i[1], i[2], 2)};
        const R pxp[3] = {V(ip[0], i[1], i[2], 0), V(ip[0], i[1], i[2], 1), V(ip[0], i[1], i[2], 2)};
        const R pyp[3] = {V(i[0], ip[1], i[2], 0), V(i[0], ip[1], i[2], 1), V(i[0], ip[1], i[2], 2)};
        const R pzp[3] = {V(i[0], i[1], ip[2], 0), V(i[0], i[1], ip[2], 1), V(i[0], i[1], ip[2], 2)};
        const R vn[3] = {V(i[0], ip[1], ip[2], 0), V(ip[0], i[1], ip[2], 1), V(ip[0], ip[1], i[2], 2)};
        const R pp[3] = {pyp[0], pxp[1], pxp[2]};
        const R pp2[3] = {pzp[0], pzp[1], pyp[2]};
        const R w1[3] = {w[2], w[2], w[1]};
        const R w2[3] = {w[1], w[0], w[0]};
        for (int a = 0; a < 3; ++a)
            out[a] = ((R)1 - w1[a]) * (((R)1 - w2[a]) * v0[a] + w2[a] * pp[a]) +
                     w1[a] * (((R)1 - w2[a]) * pp2[a] + w2[a] * vn[a]);
    }

    bool in_grid(const R p[3]) const {
        for (int a = 0; a < 3; ++a)
            if (!(p[a] > (R)0 && p[a] < (R)L[a])) return false;
        return true;
    }

    // parallel.jl:197-216, 248-261.  margin (optional): per particle, the
    // smallest distance (in cell units) of any RK4 sample point to a cell face,
    // and of the start point to a box face; the parity tests use it to tell
    // FP32 floor() flips apart from real errors.
    void staggered_advect(R* parts, long np, double* margin) {
        long clamps = 0;
#pragma omp parallel for schedule(static) reduction(+ : clamps)
        for (long k = 0; k < np; ++k) {
            R p[3] = {parts[3 * k], parts[3 * k + 1], parts[3 * k + 2]};
            double mg = 1e30;
            double* mp = margin ? &mg : nullptr;
            if (margin) {
                for (int a = 0; a < 3; ++a) {
                    double q = (double)p[a] / (double)d[a];
                    mg = std::min(mg, std::min(std::fabs(q), std::fabs(q - (double)n[a])));
                }
            }
            if (in_grid(p)) {
                R k1[3], k2[3], k3[3], k4[3], q[3];
                long cl = 0;
                staggered_velocity(p, k1, mp, &cl);
                for (int a = 0; a < 3; ++a) q[a] = p[a] + k1[a] * dt * (R)0.5;
                staggered_velocity(q, k2, mp, &cl);
                for (int a = 0; a < 3; ++a) q[a] = p[a] + k2[a] * dt * (R)0.5;
                staggered_velocity(q, k3, mp, &cl);
                for (int a = 0; a < 3; ++a) q[a] = p[a] + k3[a] * dt;
                staggered_velocity(q, k4, mp, &cl);
                clamps += cl;
                const R s = dt / (R)6;
                for (int a = 0; a < 3; ++a)
                    parts[3 * k + a] = p[a] + s * (k1[a] + (R)2 * k2[a] + (R)2 * k3[a] + k4[a]);
            } else {
                parts[3 * k] = parts[3 * k + 1] = parts[3 * k + 2] = (R)-1;
            }
            if (margin) margin[k] = mg;
        }
        clamp_events += clamps;
    }
};

// Emission (particles.jl:30-94, restated with a seeded Philox stream).
// mode 0: reference ring (0.9 r at x - 0.1 with +-0.05 jitter, particles.jl:86-90)
// mode 1: uniform in the nozzle cross-section disc at x = cen.x (MatlabPort driver
//         spawns at the nozzle centre plane, examples/matlabport/simple.jl:115-118)
// mode 2: uniform in the nozzle cylinder volume
// mode 3: the MatlabPort driver's ring: 0.9 r in the plane x = cen.x, no jitter
//         (examples/matlabport/simple.jl:112-115)
// Stream: counter = (j, counter_lo, counter_hi, 0x15F0015F), key = (seed_lo, seed_hi).
template <class R>
void emit(R* parts, long nslots, long start, long count, const float cen[3], float len, float rad, uint64_t seed,
          uint64_t counter, int mode) {
    for (long j = 0; j < count; ++j) {
        orc_u32x4 c = {{(uint32_t)j, (uint32_t)counter, (uint32_t)(counter >> 32), 0x15F0015Fu}};
        orc_u32x4 r = orc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        const float u0 = orc_u01(r.v[0]), u1 = orc_u01(r.v[1]), u2 = orc_u01(r.v[2]), u3 = orc_u01(r.v[3]);
        R p[3];
        if (mode == 3) {
            const R rt = (R)u0 * (R)2 * (R)kPi;
            p[0] = (R)cen[0];
            p[1] = (R)cen[1] + (R)0.9f * (R)rad * std::cos(rt);
            p[2] = (R)cen[2] + (R)0.9f * (R)rad * std::sin(rt);
        } else if (mode == 0) {
            const R rt = (R)u0 * (R)2 * (R)kPi;
            const R o0 = (R)u1 * (R)0.1f - (R)0.05f, o1 = (R)u2 * (R)0.1f - (R)0.05f, o2 = (R)u3 * (R)0.1f - (R)0.05f;
            p[0] = ((R)cen[0] - (R)0.1f) + o0;
            p[1] = ((R)cen[1] + (R)0.9f * (R)rad * std::cos(rt)) + o1;
            p[2] = ((R)cen[2] + (R)0.9f * (R)rad * std::sin(rt)) + o2;
        } else {
            const R th = (R)u0 * (R)2 * (R)kPi;
            const R rho = (R)rad * std::sqrt((R)u1);
            p[0] = (mode == 1) ? (R)cen[0] : (R)cen[0] + ((R)u2 - (R)0.5) * (R)len;
            p[1] = (R)cen[1] + rho * std::cos(th);
            p[2] = (R)cen[2] + rho * std::sin(th);
        }
        const long s = (start + j) % nslots;
        parts[3 * s] = p[0];
        parts[3 * s + 1] = p[1];
        parts[3 * s + 2] = p[2];
    }
}

struct Handle {
    int prec;
    Orc<double>* d = nullptr;
    Orc<float>* f = nullptr;
};

}  // namespace

extern "C" {

// prec: 64 (FP64 oracle) or 32 (FP32 restatement / CPU baseline)
void* orc_create(int prec, const int* dims, const int* size, float hbar, float dt) {
    Handle* h = new Handle();
    h->prec = prec;
    if (prec == 64) {
        h->d = new Orc<double>();
        h->d->init(dims, size, hbar, dt);
        if (!h->d->fft.ok()) { delete h->d; delete h; return nullptr; }
    } else {
        h->f = new Orc<float>();
        h->f->init(dims, size, hbar, dt);
        if (!h->f->fft.ok()) { delete h->f; delete h; return nullptr; }
    }
    return h;
}

void orc_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    delete h->d;
    delete h->f;
    delete h;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

#define ORC_DISPATCH(h, ...)                   \
    do {                                       \
        Handle* hh = (Handle*)(h);             \
        if (hh->prec == 64) {                  \
            auto& o = *hh->d;                  \
            using R = double;                  \
            (void)sizeof(R);                   \
            __VA_ARGS__;                       \
        } else {                               \
            auto& o = *hh->f;                  \
            using R = float;                   \
            (void)sizeof(R);                   \
            __VA_ARGS__;                       \
        }                                      \
    } while (0)

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    orc_u32x4 c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    orc_u32x4 r = orc_philox4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

void orc_fft3(void* h, void* data, int sign) {
    ORC_DISPATCH(h, o.fft.run((std::complex<R>*)data, sign));
}
void orc_get_mask(void* h, void* out) {
    ORC_DISPATCH(h, std::memcpy(out, o.mask.data(), sizeof(std::complex<R>) * o.N));
}
void orc_get_fac(void* h, void* out) {
    ORC_DISPATCH(h, std::memcpy(out, o.fac.data(), sizeof(std::complex<R>) * o.N));
}
void orc_get_velocity(void* h, void* out) {
    ORC_DISPATCH(h, std::memcpy(out, o.vel.data(), sizeof(R) * 3 * o.N));
}
void orc_set_velocity(void* h, const void* in) {
    ORC_DISPATCH(h, std::memcpy(o.vel.data(), in, sizeof(R) * 3 * o.N));
}
void orc_get_f(void* h, void* out) { ORC_DISPATCH(h, std::memcpy(out, o.f.data(), sizeof(R) * o.N)); }
void orc_set_f(void* h, const void* in) { ORC_DISPATCH(h, std::memcpy(o.f.data(), in, sizeof(R) * o.N)); }
void orc_get_q(void* h, void* out) {
    ORC_DISPATCH(h, std::memcpy(out, o.fc.data(), sizeof(std::complex<R>) * o.N));
}
long orc_clamp_events(void* h) {
    long r = 0;
    ORC_DISPATCH(h, r = o.clamp_events);
    return r;
}

void orc_schroedinger_flow(void* h, void* psi) { ORC_DISPATCH(h, o.schroedinger_flow((R*)psi)); }
void orc_normalize(void* h, void* psi) { ORC_DISPATCH(h, o.normalize((R*)psi)); }
void orc_velocity_one_form(void* h, const void* psi, double hbar) {
    ORC_DISPATCH(h, o.velocity_one_form((const R*)psi, (R)hbar));
}
void orc_div(void* h) { ORC_DISPATCH(h, o.div()); }
// staggered_velocity with weights divided by d (on != 0) or as parallel.jl:238 (0)
void orc_set_normalized_weights(void* h, int on) { ORC_DISPATCH(h, o.norm_w = on != 0); }
void orc_poisson_solve(void* h) { ORC_DISPATCH(h, o.poisson_solve()); }
void orc_gauge(void* h, void* psi) { ORC_DISPATCH(h, o.gauge((R*)psi)); }
void orc_pressure_project(void* h, void* psi) { ORC_DISPATCH(h, o.pressure_project((R*)psi)); }
void orc_staggered_sharp(void* h) { ORC_DISPATCH(h, o.staggered_sharp()); }
void orc_restrict_velocity(void* h, void* psi, const double* kvec, const uint8_t* jetmask, const float* cen,
                           float len, float rad, double omgterm, int phase_mode) {
    ORC_DISPATCH(h, o.restrict_velocity((R*)psi, kvec, jetmask, cen, len, rad, omgterm, phase_mode));
}
void orc_isjet(void* h, uint8_t* out, const float* cen, float len, float rad) {
    ORC_DISPATCH(h, {
        for (long z = 0; z < o.n[2]; ++z)
            for (long y = 0; y < o.n[1]; ++y)
                for (long x = 0; x < o.n[0]; ++x) {
                    const float pf[3] = {(float)x * (float)o.d[0], (float)y * (float)o.d[1], (float)z * (float)o.d[2]};
                    out[o.idx(x, y, z)] = Orc<float>::isjet_f32(pf, cen, len, rad) ? 1 : 0;
                }
    });
}
void orc_add_particles(void* h, void* parts, long nslots, long start, long count, const float* cen, float len,
                       float rad, uint64_t seed, uint64_t counter, int mode) {
    ORC_DISPATCH(h, emit<R>((R*)parts, nslots, start, count, cen, len, rad, seed, counter, mode));
}
void orc_staggered_advect(void* h, void* parts, long np, double* margin) {
    ORC_DISPATCH(h, o.staggered_advect((R*)parts, np, margin));
}

// One time step in the order of examples/benchmark.jl:46-65.
// jet == 0: no nozzle (one projection per step).
void orc_step(void* h, void* psi, void* parts, long np, int jet, const double* kvec, double omega_t,
              const float* cen, float len, float rad, long emit_start, long emit_count, uint64_t seed,
              uint64_t counter, int emit_mode, int phase_mode, double* margin) {
    ORC_DISPATCH(h, {
        R* ps = (R*)psi;
        o.schroedinger_flow(ps);
        o.normalize(ps);
        o.pressure_project(ps);
        if (jet) {
            if (emit_count > 0 && np > 0)
                emit<R>((R*)parts, np, emit_start, emit_count, cen, len, rad, seed, counter, emit_mode);
            o.restrict_velocity(ps, kvec, nullptr, cen, len, rad, omega_t, phase_mode);
            o.pressure_project(ps);
        }
        o.velocity_one_form(ps, o.hbar);
        o.staggered_sharp();
        if (np > 0) o.staggered_advect((R*)parts, np, margin);
    });
}

}  // extern "C"
