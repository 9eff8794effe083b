// The persistent batch kernel (see isf_persist.h): K ensemble steps in one
// launch, the pass bodies of the single-simulation kernels run as virtual
// CTAs of a 256-thread block, dependencies between passes as bounded waits.
#include <type_traits>

#include "isf_particles.cuh"
#include "isf_persist.h"
#include "isf_stencil.cuh"

namespace isf {

namespace {

// x pencil lengths and (y, z) plane sizes the kernel is instantiated for;
// every one gives virtual CTAs of whole warps (the named barriers count
// threads in warps)
template <class F>
__device__ __forceinline__ void with_xlen(int n, const F& f) {
    switch (n) {
        case 16: f(std::integral_constant<int, 16>()); break;
        case 32: f(std::integral_constant<int, 32>()); break;
        case 48: f(std::integral_constant<int, 48>()); break;
        case 64: f(std::integral_constant<int, 64>()); break;
        case 96: f(std::integral_constant<int, 96>()); break;
        case 128: f(std::integral_constant<int, 128>()); break;
        default: break;
    }
}
template <class F>
__device__ __forceinline__ void with_plane(int n, const F& f) {
    switch (n) {
        case 32: f(std::integral_constant<int, 32>()); break;
        case 48: f(std::integral_constant<int, 48>()); break;
        case 64: f(std::integral_constant<int, 64>()); break;
        case 96: f(std::integral_constant<int, 96>()); break;
        default: break;
    }
}

template <int N>
using PShape = PlaneShape<N, kPersistThreads>;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Poll *p (acquire: what the counted items wrote is visible after it) until
// it reaches need, at most limit times; false if the limit ran out or
// another block reported an error.
__device__ bool bounded_wait(const unsigned* p, unsigned need, long long limit, const int* status) {
    for (long long k = 0;; ++k) {
        if (ld_acquire(p) >= need) return true;
        if (ld_relaxed(status) != 0 || k >= limit) return false;
        __nanosleep(k < 64 ? 32 : 256);
    }
}

__device__ void report(const PPlan& P, int slot, int step) {
    if (atomicCAS(&P.status[0], 0, ISF_ERR_TIMEOUT) == 0) {
        P.status[1] = slot;
        P.status[2] = step;
    }
    __threadfence();
}

// Wait until phase q of step `step` has finished the tiles that an item in
// completion groups [g0, g1] of a phase with nsg groups depends on: the same
// simulations when both count per simulation, else all of q.
__device__ bool wait_groups(const PPlan& P, const PPhase& q, int step, int nsg, int g0, int g1) {
    const unsigned* dn = P.done + (size_t)step * P.dstride + q.doff;
    if (q.nsg != nsg) {
        g0 = 0;
        g1 = q.nsg - 1;
    }
    for (int g = g0; g <= g1; ++g)
        if (!bounded_wait(&dn[g], (unsigned)q.tps, P.spin_limit, P.status)) return false;
    return true;
}

// one tile (virtual CTA) of a phase; the persistent grids have whole tiles
// only (nx and ny = nz multiples of 8), so the passes take their
// whole-tile variants
__device__ __forceinline__ void run_tile(const PPlan& P, const PPhase& ph, int tile, int step, int vt,
                                         unsigned char* sm, const NamedBar& bar) {
    Blk bk;
    bk.x = tile % ph.gx;
    bk.y = (tile / ph.gx) % ph.gy;
    bk.z = tile / (ph.gx * ph.gy);
    bk.tid = vt;
    switch (ph.kind) {
        case PK_PROLOGUE: {
            // the step-graph prologue of isf_batch.cu for this class's simulations
            const long long it = *P.step + step + 1;
            for (int s = vt; s < ph.nsim; s += ph.vblk) {
                const int i = ph.first + s;
                const SimRT r = P.rt[i];
                P.jets[i].omgterm = __fmul_rn(r.omega, __fmul_rn((float)it, r.dt));
                P.emits[i].e.counter = (uint64_t)it;
                P.emits[i].start = r.nslots > 0 ? ((it - 1) * r.count) % r.nslots : 0;
            }
            break;
        }
        case PK_X_FWD:
            with_xlen(ph.len, [&](auto n) { xpass_body<decltype(n)::value, X_PSI_FWD, 1, true>(ph.x, bk, sm, bar); });
            break;
        case PK_X_INV_NORM:
            with_xlen(ph.len, [&](auto n) { xpass_body<decltype(n)::value, X_PSI_INV_NORM, 1, true>(ph.x, bk, sm, bar); });
            break;
        case PK_Y_FWD:
            with_plane(ph.len, [&](auto n) { yzpass_body<decltype(n)::value, float4, YZ_FWD, 1, true>(ph.yz, bk, sm, bar); });
            break;
        case PK_Z_MASK:
            with_plane(ph.len, [&](auto n) { yzpass_body<decltype(n)::value, float4, YZ_MASK, 1, true>(ph.yz, bk, sm, bar); });
            break;
        case PK_Y_INV:
            with_plane(ph.len, [&](auto n) { yzpass_body<decltype(n)::value, float4, YZ_INV, 1, true>(ph.yz, bk, sm, bar); });
            break;
        case PK_XR_FWD:
            with_xlen(ph.len, [&](auto n) { xreal_body<decltype(n)::value, XR_FWD, 1, true>(ph.x, bk, sm, bar); });
            break;
        case PK_XR_INV_GAUGE:
            with_xlen(ph.len,
                      [&](auto n) {
                          if (ph.x.use_jet)
                              xreal_body<decltype(n)::value, XR_INV_GAUGE_JET, 1, true>(ph.x, bk, sm, bar);
                          else
                              xreal_body<decltype(n)::value, XR_INV_GAUGE, 1, true>(ph.x, bk, sm, bar);
                      });
            break;
        case PK_PLANE:
            with_plane(ph.len, [&](auto n) {
                constexpr int N = decltype(n)::value;
                plane_body<N, PShape<N>>(ph.pl, bk, sm, bar);
            });
            break;
        case PK_DIV:
            if (ph.st.use_jet)
                stencil_body<ST_DIV, true>(ph.st, bk, *reinterpret_cast<StencilSmem<ST_DIV>*>(sm), bar);
            else
                stencil_body<ST_DIV, false>(ph.st, bk, *reinterpret_cast<StencilSmem<ST_DIV>*>(sm), bar);
            break;
        case PK_VEL:  // the one-form is never restricted (isf_batch.cu builds it with use_jet 0)
            if (ph.st.sharp)
                stencil_body<ST_VEL, false, true>(ph.st, bk, *reinterpret_cast<StencilSmem<ST_VEL>*>(sm), bar);
            else
                stencil_body<ST_VEL, false>(ph.st, bk, *reinterpret_cast<StencilSmem<ST_VEL>*>(sm), bar);
            break;
        case PK_EMIT: {
            const long long j = (long long)bk.x * ph.vblk + vt;
            if (j < ph.count) {
                const EmitState& st = P.emits[ph.first + bk.y];
                const float3 p = emit_point(j, st.e);
                const long long s = (st.start + j) % ph.nslots;
                float* parts = ph.parts + bk.y * 3 * ph.nslots;
                parts[3 * s + 0] = p.x;
                parts[3 * s + 1] = p.y;
                parts[3 * s + 2] = p.z;
            }
            break;
        }
        case PK_ADVECT: {
            // kAdvectSlots slots per thread: slot bk.x * vblk * kAdvectSlots + j vblk + vt
            unsigned clamps = 0, live = 0;
            const AdvConst kc = adv_const(ph.g, ph.vel + bk.y * ph.bs_vel);
            const float dt = ph.g.dt, s6 = ph.g.dt / 6.0f;
            float* parts = ph.parts + bk.y * 3 * ph.nslots;
            for (int j = 0; j < kAdvectSlots; ++j) {
                const long long k = ((long long)bk.x * kAdvectSlots + j) * ph.vblk + vt;
                if (k >= ph.nslots) break;
                if (ph.normw) {
                    if (ph.pow2)
                        advect_slot<true, true, NamedBar>(kc, parts, (int)k, dt, s6, clamps, live, nullptr);
                    else
                        advect_slot<false, true, NamedBar>(kc, parts, (int)k, dt, s6, clamps, live, nullptr);
                } else {
                    if (ph.pow2)
                        advect_slot<true, false, NamedBar>(kc, parts, (int)k, dt, s6, clamps, live, nullptr);
                    else
                        advect_slot<false, false, NamedBar>(kc, parts, (int)k, dt, s6, clamps, live, nullptr);
                }
            }
            // warp-aggregated counters (a virtual CTA is whole warps)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                clamps += __shfl_down_sync(0xffffffffu, clamps, o);
                live += __shfl_down_sync(0xffffffffu, live, o);
            }
            if ((vt & 31) == 0) {
                unsigned long long* c = P.counters + (size_t)(ph.first + bk.y) * kCounterStride;
                if (clamps) atomicAdd(&c[0], (unsigned long long)clamps);
                if (live) atomicAdd(&c[1], (unsigned long long)live);
            }
            break;
        }
        default:
            break;
    }
}

}  // namespace

// resident blocks per SM the kernel is compiled for (caps its registers at
// 65536 / (256 x ISF_PERSIST_MINB)): at 3 (80 registers, the larger bodies
// spill) the 64-jet ensemble step takes 1.27 ms against 1.39 ms at 2 (128
// registers) and 1.40 ms at 4 (64 registers)
#ifndef ISF_PERSIST_MINB
#define ISF_PERSIST_MINB 3
#endif
__global__ void __launch_bounds__(kPersistThreads, ISF_PERSIST_MINB) k_persist(PPlan P) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int s_item, s_go;
    __shared__ int s_start[kPersistMaxSlots + 1];  // the slot table, searched per item
    for (int i = threadIdx.x; i <= P.nslot; i += blockDim.x) s_start[i] = P.slot_start[i];
    const int total = P.items_per_step * P.nsteps;
    // thread 0 claims the block's next item while the block works on the
    // current one (the lowest unfinished item always belongs to a block
    // that runs it or starts it next, so the waits still resolve)
    int next = threadIdx.x == 0 ? (int)atomicAdd(&P.ctl[0], 1u) : 0;
    for (;;) {
        if (threadIdx.x == 0) {
            int it = next;
            if (it >= total || ld_relaxed(&P.status[0]) != 0) it = -1;
            if (it >= 0) next = (int)atomicAdd(&P.ctl[0], 1u);
            s_item = it;
        }
        __syncthreads();
        const int it = s_item;
        if (it < 0) break;
        const int step = it / P.items_per_step, r = it - step * P.items_per_step;
        int lo = 0, hi = P.nslot - 1;  // the slot with s_start[slot] <= r < s_start[slot + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_start[mid] <= r) lo = mid;
            else hi = mid - 1;
        }
        const int slot = lo;
        const PPhase& ph = P.ph[slot];
        // the item's tiles [t0, t1) and the completion groups (simulations) they lie in
        const int t0 = (r - s_start[slot]) * ph.reps * ph.vper;
        const int t1 = min(ph.tiles, t0 + ph.reps * ph.vper);
        const int g0 = t0 / ph.tps, g1 = (t1 - 1) / ph.tps;
        if (threadIdx.x == 0) {
            bool ok = true;
            if (ph.dep >= 0) ok = wait_groups(P, P.ph[ph.dep], step, ph.nsg, g0, g1);
            if (ok && step > 0 && ph.dep_prev >= 0) ok = wait_groups(P, P.ph[ph.dep_prev], step - 1, ph.nsg, g0, g1);
            // the stall switch: an item with a dependency also waits for
            // status[3], which nothing writes, so the wait runs out
            if (ok && P.stall && (ph.dep >= 0 || (step > 0 && ph.dep_prev >= 0)))
                ok = bounded_wait(reinterpret_cast<const unsigned*>(&P.status[3]), 1u, P.spin_limit, P.status);
            if (!ok) report(P, slot, step);
            s_go = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_go) break;
        // the item: reps rounds of vper virtual CTAs, one tile each per round
        const int v = threadIdx.x / ph.vblk;
        if (v < ph.vper) {
            const NamedBar bar{1 + v, ph.vblk};
            for (int rr = 0; rr < ph.reps; ++rr) {
                const int tile = ((r - s_start[slot]) * ph.reps + rr) * ph.vper + v;
                if (tile >= ph.tiles) break;
                if (rr > 0) bar.sync();  // the previous tile's last reads of the shared tile are done
                run_tile(P, ph, tile, step, threadIdx.x - v * ph.vblk, smraw + v * ph.smem_v, bar);
            }
        }
        __syncthreads();  // every virtual CTA of the item is done
        if (threadIdx.x == 0) {
            __threadfence();  // release: the item's writes before its counts
            unsigned* dn = P.done + (size_t)step * P.dstride + ph.doff;
            for (int g = g0; g <= g1; ++g)
                atomicAdd(&dn[g], (unsigned)(min(t1, (g + 1) * ph.tps) - max(t0, g * ph.tps)));
            // the item that completes the launch's last step advances the
            // ensemble's step counter (every prologue has read it by then)
            if (step == P.nsteps - 1 &&
                atomicAdd(&P.ctl[1], (unsigned)(t1 - t0)) + (unsigned)(t1 - t0) == (unsigned)P.tiles_per_step)
                *P.step += P.nsteps;
        }
    }
}

bool persist_len_ok(int n) {
    switch (n) {
        case 16: case 32: case 48: case 64: case 96: case 128: return true;
        default: return false;
    }
}

bool persist_plane_ok(int n) { return n == 32 || n == 48 || n == 64 || n == 96; }

namespace {
template <class F>
int host_xlen(int n, const F& f) {
    switch (n) {
        case 16: return f(std::integral_constant<int, 16>());
        case 32: return f(std::integral_constant<int, 32>());
        case 48: return f(std::integral_constant<int, 48>());
        case 64: return f(std::integral_constant<int, 64>());
        case 96: return f(std::integral_constant<int, 96>());
        case 128: return f(std::integral_constant<int, 128>());
        default: return 0;
    }
}
template <class F>
int host_plane(int n, const F& f) {
    switch (n) {
        case 32: return f(std::integral_constant<int, 32>());
        case 48: return f(std::integral_constant<int, 48>());
        case 64: return f(std::integral_constant<int, 64>());
        case 96: return f(std::integral_constant<int, 96>());
        default: return 0;
    }
}
}  // namespace

int persist_vblk(int kind, int len) {
    switch (kind) {
        case PK_X_FWD: case PK_X_INV_NORM:
            return host_xlen(len, [](auto n) { return XShape<decltype(n)::value, X_PSI_FWD, 1>::BLK; });
        case PK_Y_FWD: case PK_Z_MASK: case PK_Y_INV:
            return host_plane(len, [](auto n) { return YZShape<decltype(n)::value, float4, YZ_FWD, 1>::BLK; });
        case PK_XR_FWD: case PK_XR_INV_GAUGE:
            return host_xlen(len, [](auto n) { return XRShape<decltype(n)::value, 1, true>::BLK; });
        case PK_PLANE:
            return host_plane(len, [](auto n) { return PlaneShape<decltype(n)::value, kPersistThreads>::BLK; });
        default:
            return kPersistThreads;
    }
}

int persist_smem(int kind, int len) {
    switch (kind) {
        case PK_X_FWD: case PK_X_INV_NORM:
            return host_xlen(len, [](auto n) { return (int)XShape<decltype(n)::value, X_PSI_FWD, 1>::SMEM; });
        case PK_Y_FWD: case PK_Z_MASK: case PK_Y_INV:
            return host_plane(len, [](auto n) { return (int)YZShape<decltype(n)::value, float4, YZ_FWD, 1>::SMEM; });
        case PK_XR_FWD: case PK_XR_INV_GAUGE:
            return host_xlen(len, [](auto n) { return (int)XRShape<decltype(n)::value, 1, true>::SMEM; });
        case PK_PLANE:
            return host_plane(len, [](auto n) { return (int)PlaneShape<decltype(n)::value, kPersistThreads>::SMEM; });
        case PK_DIV:
            return (int)sizeof(StencilSmem<ST_DIV>);
        case PK_VEL:
            return (int)sizeof(StencilSmem<ST_VEL>);
        default:
            return 0;
    }
}

cudaError_t persist_setup(int smem_bytes, int* blocks_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(k_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_persist, kPersistThreads, smem_bytes);
}

cudaError_t launch_persist(const PPlan& p, int grid, int smem_bytes, cudaStream_t s) {
    k_persist<<<grid, kPersistThreads, smem_bytes, s>>>(p);
    return cudaGetLastError();
}

}  // namespace isf
