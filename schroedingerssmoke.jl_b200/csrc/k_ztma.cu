// The Schroedinger z pass (forward FFT along z, * mask(k) / N, inverse) with
// its pencils staged by the tensor memory accelerator.
//
// The register-staged pass (k_yzpass<N, float4, YZ_MASK>) needs 128
// registers per thread, so only 16 warps fit an SM and a CTA's loads wait
// while the SM's other CTAs compute.  Here each CTA walks its tiles (8
// consecutive x of one y row, all nz planes: N x 128 bytes) in a loop and
// keeps the next tile's copy in flight while it transforms the current one:
// tile k+1 arrives in the second of two shared buffers (cp.async.bulk.tensor,
// 2D, completion counted on an mbarrier) while tile k goes through the
// same register-staged Stockham stages as the launched pass, using its own
// buffer as the stage-exchange tile.  The arithmetic of a pencil is the
// same, so the results are bitwise those of k_yzpass.
//
// The tensor map covers this GPU's own psi only; there is no cluster
// multicast.  Every mbarrier wait is bounded: a wait that runs out adds one
// to the error counter, drains (again bounded) the copy still in flight,
// and the CTA returns.  A test switch (stall) makes the first wait run out
// on purpose after its copy has arrived.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "isf_launch.h"
#include "isf_passes.cuh"

namespace isf {

namespace {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// test the phase of the given parity (non-blocking) at most `limit` times,
// backing off between tests
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
    for (long long k = 0; k < limit; ++k) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (k >= 32) __nanosleep(128);
    }
    return false;
}

// poll a flag in global memory until it is non-zero, at most `limit` times
__device__ __forceinline__ bool flag_wait(const unsigned long long* flag, long long limit) {
    for (long long k = 0; k < limit; ++k) {
        unsigned long long v;
        asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(flag) : "memory");
        if (v != 0) return true;
        __nanosleep(128);
    }
    return false;
}

// 2D tile copy global -> shared, completion counted on bar (x innermost, in elements)
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

template <int N>
struct ZT {
    static constexpr int C = 8;                     // float4 pencils per tile (128 bytes of x)
    static constexpr int NT = Plan<N>::NT;
    static constexpr int BLK = C * NT;
    static constexpr int MINB = (512 / BLK) > 1 ? 512 / BLK : 1;  // the register budget of the launched pass
    static constexpr int TILE = N * C;              // float4 per tile
    static constexpr size_t SMEM = 2 * (size_t)TILE * sizeof(float4) + 128;
};

template <int N>
__global__ void __launch_bounds__(ZT<N>::BLK, ZT<N>::MINB)
    k_zmask_tma(const __grid_constant__ CUtensorMap map, YZArgs a, int ntiles, long long limit,
                unsigned long long* __restrict__ err, const unsigned long long* stall) {
    using Z = ZT<N>;
    constexpr int C = Z::C, TILE = Z::TILE;
    extern __shared__ unsigned char smraw[];
    // the copies' destination: 128-byte aligned
    float4* buf = reinterpret_cast<float4*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) unsigned long long bars[2];
    const int tid = threadIdx.x, q = tid % C, t = tid / C;
    const int rl = a.row, ny = a.g.n[1];
    const int xt = rl / C;  // x tiles per row
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    pdl_enter();  // psi comes from the previous pass
    auto issue = [&](int k) {
        const int tt = blockIdx.x + k * gridDim.x;
        if (tt >= ntiles) return;
        const int b = k & 1;
        const int x0 = (tt % xt) * C, o = tt / xt;
        mbar_expect_tx(&bars[b], TILE * (unsigned)sizeof(float4));
        tma_load_2d(buf + b * TILE, &map, (o * rl + x0) * 4, 0, &bars[b]);
    };
    if (tid == 0) {
        issue(0);
        issue(1);
    }
    float4* __restrict__ data = reinterpret_cast<float4*>(a.data);
    const long long stride = (long long)rl * ny;
    const float2* tw = a.g.tw[2];
    const double2* __restrict__ mt = a.g.mtab[2];
    const double msign = a.conj_mask ? -1.0 : 1.0;
    float4 x[Plan<N>::EMAX];
    for (int k = 0;; ++k) {
        const int tt = blockIdx.x + k * gridDim.x;
        if (tt >= ntiles) break;
        const int b = k & 1;
        bool ok = mbar_wait(&bars[b], (unsigned)((k >> 1) & 1), limit);
        // the timeout test: the first tile has arrived, then a flag that
        // nothing sets is awaited (briefly), so the error path runs
        if (stall != nullptr && k == 0 && tid == 0) ok = ok && flag_wait(stall, 256);
        if (__syncthreads_or(ok ? 0 : 1)) {
            // a copy that did not arrive: count it, wait (bounded) for the
            // other buffer's copy if one is in flight, and return
            if (tid == 0) {
                atomicAdd(err, 1ull);
                if (blockIdx.x + (k + 1) * gridDim.x < ntiles) mbar_wait(&bars[b ^ 1], (unsigned)(((k + 1) >> 1) & 1), limit);
            }
            return;
        }
        float4* sm = buf + b * TILE;
        const int x0 = (tt % xt) * C, o = tt / xt;
        const int kx = x0 + q;
        const long long base = x0 + (long long)o * rl;
        // the z-mask multiply of k_yzpass (axis 2): exp(i (th_x + th_y + th_z)) / N
        double2 cxo = zmul(a.g.mtab[0][kx], a.g.mtab[1][o]);
        cxo.x *= a.g.invN;
        cxo.y *= a.g.invN;
        auto src = [&](int j) -> float4 { return sm[j * C + q]; };
        auto mmul = [&](int j, const float4& v) -> float4 {
            double2 m = zmul(cxo, __ldg(&mt[j]));
            m.y *= msign;
            return cmul(v, make_float2((float)m.x, (float)m.y));
        };
        auto dst = [&](int j, const float4& v) { data[base + j * stride + q] = v; };
        // the buffer is the stage-exchange tile too: a barrier after the first gather
        Plan<N>::template run_spectral<C, true>(x, t, q, sm, tw, src, mmul, dst);
        // the buffer's generic accesses are done before the copy engine refills it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) issue(k + 2);
    }
}

template <int N>
cudaError_t launch_zt(const CUtensorMap& map, const YZArgs& a, long long limit, unsigned long long* err,
                      const unsigned long long* stall, cudaStream_t s) {
    using Z = ZT<N>;
    static int grid_cap = 0;  // CTAs resident on the device
    static std::once_flag once;
    static cudaError_t setup = cudaSuccess;
    std::call_once(once, [&] {
        setup = cudaFuncSetAttribute(k_zmask_tma<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::SMEM);
        int dev = 0, sms = 0, per = 0;
        if (setup == cudaSuccess) setup = cudaGetDevice(&dev);
        if (setup == cudaSuccess) setup = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (setup == cudaSuccess)
            setup = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_zmask_tma<N>, Z::BLK, Z::SMEM);
        grid_cap = sms * (per > 0 ? per : 1);
    });
    if (setup != cudaSuccess) return setup;
    const int ntiles = (a.row / Z::C) * a.g.n[1];
    const int grid = ntiles < grid_cap ? ntiles : grid_cap;
    return launch_pdl(k_zmask_tma<N>, dim3(grid), dim3(Z::BLK), Z::SMEM, s, map, a, ntiles, limit, err, stall);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace

bool zmask_tma_len(int n) { return n == 64 || n == 96 || n == 128 || n == 192 || n == 256; }

// psi (nx ny nz float4, 16-byte aligned) as a 2D array of floats: planes of
// nx ny * 4 floats, nz of them; a box is one tile (8 float4 x nz planes)
bool encode_psi_zmap(CUtensorMapStorage* out, const float* psi, const Grid& g) {
    static_assert(sizeof(CUtensorMapStorage) == sizeof(CUtensorMap), "tensor map storage");
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || !zmask_tma_len(g.n[2]) || g.n[0] % 8 != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)g.n[0] * g.n[1] * 4, (cuuint64_t)g.n[2]};
    const cuuint64_t strides[1] = {(cuuint64_t)g.n[0] * g.n[1] * 4 * sizeof(float)};
    const cuuint32_t box[2] = {8 * 4, (cuuint32_t)g.n[2]};
    const cuuint32_t estr[2] = {1, 1};
    CUtensorMap* m = reinterpret_cast<CUtensorMap*>(out);
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(psi), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_zmask_tma(const CUtensorMapStorage& map, const YZArgs& a, long long limit, unsigned long long* err,
                             const unsigned long long* stall, cudaStream_t s) {
    const CUtensorMap& m = reinterpret_cast<const CUtensorMap&>(map);
    switch (a.g.n[2]) {
        case 64: return launch_zt<64>(m, a, limit, err, stall, s);
        case 96: return launch_zt<96>(m, a, limit, err, stall, s);
        case 128: return launch_zt<128>(m, a, limit, err, stall, s);
        case 192: return launch_zt<192>(m, a, limit, err, stall, s);
        case 256: return launch_zt<256>(m, a, limit, err, stall, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace isf
