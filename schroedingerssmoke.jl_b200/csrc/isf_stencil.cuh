// z-marching stencil of the velocity one-form: the body shared by the
// stencil kernels (k_stencil.cu) and the persistent batch kernel.
//
// One CTA (256 threads, two rows each) owns a 32 x 16 column block of the
// grid and walks up to 8 consecutive z planes.  The padded 34 x 18 psi tile of
// the current plane sits in shared memory, the tile of the next plane arrives
// in registers while the current one is worked on (prefetch), so psi is read
// from HBM about once and each angle of the one-form is evaluated about once
// per cell.
//
//   ST_DIV  f = div(velocity_one_form(psi, 1))       parallel.jl:100-122, 131-152
//           with psi optionally restricted in the nozzle on the fly
//           (restrict_kernel, particles.jl:12-20)
//   ST_VEL  padded velocity grid (vx, vy, vz, 0) = one_form(psi, hbar) [* 1/d]
//           (parallel.jl:115-122, staggered sharp examples/benchmark.jl:61-63)
#pragma once
#include "isf_launch.h"

namespace isf {

namespace st {

// z planes per CTA (both stencils: at 256x128x128 the div stencil ran 39.8
// us over 4 planes and 37.3 over 8; the one-form stencil 36.3 over 4 and
// 35.9 over 8)
#ifndef ISF_ST_SZ
#define ISF_ST_SZ 8
#endif
#ifndef ISF_ST_SZ_VEL
#define ISF_ST_SZ_VEL 8
#endif
#ifndef ISF_ST_RPT
#define ISF_ST_RPT 2
#endif
constexpr int BX = 32, TY = 8, RPT = ISF_ST_RPT, BY = TY * RPT;  // 256 threads
template <int OP>
constexpr int planes_per_cta() { return OP == ST_DIV ? ISF_ST_SZ : ISF_ST_SZ_VEL; }
constexpr int TW = BX + 2, TH = BY + 2, TILE = TW * TH;        // padded tile
constexpr int LPT = (TILE + BX * TY - 1) / (BX * TY);           // tile loads per thread

}  // namespace st

// shared memory of one stencil CTA: the psi tiles, and for the divergence
// the x / y one-form edges (the one-form stencil leaves them out, which
// leaves more of the SM's shared storage to L1)
template <int OP>
struct StencilSmem {
    float4 tile[2][st::TH][st::TW];
    float vxs[st::BY][st::BX + 1];  // v_x at x0-1+c (c = 0..W)
    float vys[st::BY + 1][st::BX];  // v_y at y0-1+r (r = 0..H)
};
template <>
struct StencilSmem<ST_VEL> {
    float4 tile[2][st::TH][st::TW];
};

// JET: psi is restricted in the nozzle on the fly (a.use_jet set).  A
// compile-time switch: left to a run-time test, the restriction's code shaped
// the plane loop of every launch (about 24 instructions per cell more, with
// use_jet 0).  SHARP (one-form stencil): the one-form is divided by the cell
// sizes (a.sharp set), also a compile-time switch.
template <int OP, bool JET, bool SHARP = false, class B = CtaBar>
__device__ __forceinline__ void stencil_body(const StencilArgs a, const Blk bk, StencilSmem<OP>& S,
                                             const B& bar = B()) {
    using namespace st;
    const Grid& g = a.g;
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int tid = bk.tid, tx = tid & (BX - 1), ty = tid / BX;
    // block z = simulation * (z chunks) + z chunk
    constexpr int SZ = planes_per_cta<OP>();
    const int zchunks = (nz + SZ - 1) / SZ;
    const int sim = bk.z / zchunks;
    const int x0 = bk.x * BX, y0 = bk.y * BY, z0 = (bk.z - sim * zchunks) * SZ;
    // partial tiles: the padded tile keeps its halo at column W+1 / row H+1
    const int W = min(BX, nx - x0), H = min(BY, ny - y0);
    const int zend = min(z0 + SZ, nz);
    const int x = x0 + tx;
    bool own[RPT];
#pragma unroll
    for (int m = 0; m < RPT; ++m) own[m] = (tx < W) && (ty + TY * m < H);

    auto& tile = S.tile;

    // Each thread loads the same LPT padded-tile elements in every plane:
    // padded column c <-> x0 + c - 1 and row r <-> y0 + r - 1 (periodic), so
    // column W+1 / row H+1 is the + halo even for a partial tile; columns and
    // rows past the halo repeat it and stay inside the grid.
    int toff[LPT], tx_[LPT], ty_[LPT], tsl[LPT];
#pragma unroll
    for (int k = 0; k < LPT; ++k) {
        const int e = tid + k * BX * TY;
        const int r = e / TW, c = e - r * TW;
        const int cc = min(c, W + 1), rr = min(r, H + 1);
        int xx = x0 + cc - 1, yy = y0 + rr - 1;
        xx = xx < 0 ? xx + nx : (xx >= nx ? xx - nx : xx);
        yy = yy < 0 ? yy + ny : (yy >= ny ? yy - ny : yy);
        tx_[k] = xx;
        ty_[k] = yy;
        toff[k] = xx + nx * yy;
        tsl[k] = (e < TILE) ? e : -1;
    }
    const int nxy = nx * ny;
    // kernel-parameter fields used in the plane loop, held in registers
    const float4* __restrict__ psi = a.psi + sim * a.bs_psi;
    float* __restrict__ out = a.out + sim * a.bs_out;
    JetArgs jet;
    if constexpr (JET) jet = a.jets ? a.jets[sim] : a.jet;
    const float id0 = g.inv_d2[0], id1 = g.inv_d2[1], id2 = g.inv_d2[2];
    const float hb = a.hbar;
    const float di0 = g.dinv[0], di1 = g.dinv[1], di2 = g.dinv[2];
    const int pnx = g.pnx, pnxy = g.pnxy;
    float4* __restrict__ out4 = reinterpret_cast<float4*>(out);
    const int ox = nx, oy = ny * pnx, oz = nz * pnxy;  // +face copy offsets
    auto tile_e = [&](int k, int z) -> float4 {
        const int cidx = toff[k] + nxy * z;
        float4 v = ldm<B>(&psi[cidx]);
        if constexpr (JET) restrict_cell(g, jet, tx_[k], ty_[k], z, cidx, v);
        return v;
    };
    float4* tflat0 = &tile[0][0][0];
    float4* tflat1 = &tile[1][0][0];

    float4 pre[LPT];
    int cur = 0;
    // prologue: plane z0 into the tile, plane z0+1 into registers
#pragma unroll
    for (int k = 0; k < LPT; ++k)
        if (tsl[k] >= 0) tflat0[tsl[k]] = tile_e(k, z0);
    const int z1 = (z0 + 1 == nz) ? 0 : z0 + 1;
#pragma unroll
    for (int k = 0; k < LPT; ++k)
        if (tsl[k] >= 0) pre[k] = tile_e(k, z1);
    float vz_prev[RPT];
#pragma unroll
    for (int m = 0; m < RPT; ++m) vz_prev[m] = 0.f;
    if constexpr (OP == ST_DIV) {
        // v_z(z0 - 1) needs psi of plane z0 - 1 at the block's own cells
        float4 pm[RPT];
        const int zm = (z0 == 0) ? nz - 1 : z0 - 1;
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            pm[m] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (own[m]) {
                const int y = y0 + ty + TY * m;
                const int cm = x + nx * y + nxy * zm;
                pm[m] = ldm<B>(&psi[cm]);
                if constexpr (JET) restrict_cell(g, jet, x, y, zm, cm, pm[m]);
            }
        }
        bar.sync();
#pragma unroll
        for (int m = 0; m < RPT; ++m)
            if (own[m]) vz_prev[m] = pair_angle(pm[m], tile[0][ty + TY * m + 1][tx + 1]);
    }

    for (int z = z0; z < zend; ++z) {
        bar.sync();  // tile[cur] complete; previous iteration's reads done
        const int nxt = cur ^ 1;
        float4* tn = nxt ? tflat1 : tflat0;
#pragma unroll
        for (int k = 0; k < LPT; ++k)
            if (tsl[k] >= 0) tn[tsl[k]] = pre[k];
        if (z + 1 < zend) {  // prefetch plane z+2
            const int z2 = (z + 2 >= nz) ? z + 2 - nz : z + 2;
#pragma unroll
            for (int k = 0; k < LPT; ++k)
                if (tsl[k] >= 0) pre[k] = tile_e(k, z2);
        }
        if constexpr (OP == ST_DIV) {
            auto& vxs = S.vxs;
            auto& vys = S.vys;
#pragma unroll
            for (int m = 0; m < RPT; ++m) {
                const int r = ty + TY * m;
                if (own[m]) {
                    const float4 c0 = tile[cur][r + 1][tx + 1];
                    vxs[r][tx + 1] = pair_angle(c0, tile[cur][r + 1][tx + 2]);
                    vys[r + 1][tx] = pair_angle(c0, tile[cur][r + 2][tx + 1]);
                }
            }
            // the tile's halo edges (x0-1 -> x0 per row, y0-1 -> y0 per column),
            // one per thread of the first two warps rather than one extra
            // predicated angle in every warp
            if (tid < BY) {
                if (tid < H) vxs[tid][0] = pair_angle(tile[cur][tid + 1][0], tile[cur][tid + 1][1]);
            } else if (tid >= 32 && tid < 32 + BX) {
                const int c = tid - 32;
                if (c < W) vys[0][c] = pair_angle(tile[cur][0][c + 1], tile[cur][1][c + 1]);
            }
            bar.sync();
#pragma unroll
            for (int m = 0; m < RPT; ++m) {
                const int r = ty + TY * m;
                if (own[m]) {
                    const float vz = pair_angle(tile[cur][r + 1][tx + 1], tile[nxt][r + 1][tx + 1]);
                    const float t0 = (vxs[r][tx + 1] - vxs[r][tx]) * id0;
                    const float t1 = (vys[r + 1][tx] - vys[r][tx]) * id1;
                    const float t2 = (vz - vz_prev[m]) * id2;
                    out[x + nx * (y0 + r) + nxy * z] = (t0 + t1) + t2;
                    vz_prev[m] = vz;
                }
            }
        } else {
            bar.sync();
#pragma unroll
            for (int m = 0; m < RPT; ++m) {
                const int r = ty + TY * m;
                if (own[m]) {
                    const float4 c0 = tile[cur][r + 1][tx + 1];
                    float ax = pair_angle(c0, tile[cur][r + 1][tx + 2]) * hb;
                    float ay = pair_angle(c0, tile[cur][r + 2][tx + 1]) * hb;
                    float az = pair_angle(c0, tile[nxt][r + 1][tx + 1]) * hb;
                    if constexpr (SHARP) {
                        ax = __fmul_rn(ax, di0);
                        ay = __fmul_rn(ay, di1);
                        az = __fmul_rn(az, di2);
                    }
                    const int y = y0 + r;
                    const int pc = x + pnx * y + pnxy * z;
                    const float4 v = make_float4(ax, ay, az, 0.f);
                    out4[pc] = v;
                    const bool cx = x == 0, cy = y == 0, cz = z == 0;
                    if (cx | cy | cz) pcopies(out4, pc, cx, cy, cz, ox, oy, oz, v);  // periodic copies on the +faces
                }
            }
        }
        cur = nxt;
    }
}

}  // namespace isf
