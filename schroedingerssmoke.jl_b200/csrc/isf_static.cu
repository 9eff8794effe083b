// Poisson solve that allocates no device memory (isf_poisson_solve_static).
//
// Some callers cannot let a library call cudaMalloc: a host runtime whose
// own pool manages all device memory (the way CUDA.jl / GPUArrays arrays
// are handed to a ccall), a process running under a hard memory cap, or a
// loop that must not allocate after its set-up.  They cannot create an
// isf_handle (isf_create allocates the tables and workspaces), so this entry
// point keeps its workspace in file-scope device arrays instead:
//
//   g_spectrum  ISF_STATIC_MAX_SPECTRUM complex64 values (2 MiB): the padded
//               half spectrum, (round_up(nx/2 + 1, 16)) * ny * nz values
//   g_tables    the per-axis tables (twiddles, Laplacian symbols)
//
// Every GPU that loads libisf holds both arrays until the process exits.
// All calls share them: a call leaves its values there for the next one,
// and nothing in them needs to start at zero (every value a call reads was
// written by that call).  Calls whose work overlaps on the GPU (different
// streams, or different host threads on one stream without ordering) race
// on the shared arrays; serialise them.  The first call on a device looks up
// the arrays' device addresses (cudaGetSymbolAddress, once per device, with
// that device current); make that first call before any stream capture.
//
// The tables depend only on the grid parameters (grid_res, physical_size,
// hbar, dt).  A call uploads them from host memory when they differ from the
// last upload on that device and skips the upload otherwise.  An upload is a
// copy from a host buffer that lives only during the call, so a call that
// needs one while its stream is being captured is refused (ISF_ERR_INVALID)
// before anything is queued.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "isf_launch.h"
#include "isf_passes.cuh"

using namespace isf;

namespace {

constexpr long long ISF_STATIC_MAX_SPECTRUM = 262144;  // complex values (2 MiB)
constexpr size_t ISF_STATIC_TABLE_BYTES = 3 * 512 * (sizeof(double2) + sizeof(double) + sizeof(float2));

__device__ __align__(256) float2 g_spectrum[ISF_STATIC_MAX_SPECTRUM];
__device__ __align__(256) unsigned char g_tables[ISF_STATIC_TABLE_BYTES];

struct StaticAddrs {
    float2* spectrum = nullptr;
    char* tables = nullptr;
    bool ready = false;
    // grid parameters of the tables last uploaded to this device
    bool have_key = false;
    int key_n[3] = {0, 0, 0}, key_L[3] = {0, 0, 0};
    float key_hbar = 0.f, key_dt = 0.f;
};
constexpr int kMaxDevices = 64;
StaticAddrs g_addrs[kMaxDevices];
std::mutex g_addrs_mutex;

thread_local std::string g_static_error;

int static_fail(int code, const std::string& msg) {
    g_static_error = msg;
    return code;
}

// device addresses of the file-scope arrays on the current device (host code
// cannot use the arrays' names as device pointers)
cudaError_t static_addrs(int dev, StaticAddrs& out) {
    std::lock_guard<std::mutex> lock(g_addrs_mutex);
    StaticAddrs& a = g_addrs[dev];
    if (!a.ready) {
        void* sp = nullptr;
        void* tp = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&sp, g_spectrum);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(&tp, g_tables);
        if (e != cudaSuccess) return e;
        a.spectrum = static_cast<float2*>(sp);
        a.tables = static_cast<char*>(tp);
        a.ready = true;
    }
    out = a;
    return cudaSuccess;
}

bool same_key(const StaticAddrs& a, const isf_params* p) {
    if (!a.have_key) return false;
    for (int k = 0; k < 3; ++k)
        if (a.key_n[k] != p->grid_res[k] || a.key_L[k] != p->physical_size[k]) return false;
    return std::memcmp(&a.key_hbar, &p->hbar, sizeof(float)) == 0 && std::memcmp(&a.key_dt, &p->dt, sizeof(float)) == 0;
}

void set_key(int dev, const isf_params* p) {
    std::lock_guard<std::mutex> lock(g_addrs_mutex);
    StaticAddrs& a = g_addrs[dev];
    for (int k = 0; k < 3; ++k) {
        a.key_n[k] = p->grid_res[k];
        a.key_L[k] = p->physical_size[k];
    }
    a.key_hbar = p->hbar;
    a.key_dt = p->dt;
    a.have_key = true;
}

}  // namespace

extern "C" {

const char* isf_static_last_error(void) { return g_static_error.c_str(); }

int isf_poisson_solve_static(const isf_params* p, const float* f, float* q) {
    std::string why;
    if (!check_params(p, why)) return static_fail(ISF_ERR_INVALID, "isf_poisson_solve_static: " + why);
    if (!f || !q) return static_fail(ISF_ERR_INVALID, "isf_poisson_solve_static: null argument");
    const int wp = half_spectrum_row(p->grid_res[0]);
    const long long need = (long long)wp * p->grid_res[1] * p->grid_res[2];
    if (need > ISF_STATIC_MAX_SPECTRUM)
        return static_fail(ISF_ERR_INVALID, "isf_poisson_solve_static: the grid needs " + std::to_string(need) +
                                                 " spectrum values, the static workspace holds " +
                                                 std::to_string(ISF_STATIC_MAX_SPECTRUM) +
                                                 " (round_up(nx/2 + 1, 16) * ny * nz must not exceed it)");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return static_fail(ISF_ERR_CUDA, std::string("isf_poisson_solve_static: ") + cudaGetErrorString(e));
    if (p->device < 0 || p->device >= ndev || p->device >= kMaxDevices)
        return static_fail(ISF_ERR_INVALID, "isf_poisson_solve_static: bad device ordinal");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device && (e = cudaSetDevice(p->device)) != cudaSuccess)
        return static_fail(ISF_ERR_CUDA, std::string("isf_poisson_solve_static: cudaSetDevice: ") + cudaGetErrorString(e));
    auto finish = [&](int code, const std::string& msg) {
        if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
        return code == ISF_OK ? ISF_OK : static_fail(code, msg);
    };
    StaticAddrs addrs;
    if ((e = static_addrs(p->device, addrs)) != cudaSuccess)
        return finish(ISF_ERR_CUDA, std::string("isf_poisson_solve_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));

    Grid g;
    std::vector<char> host;
    fill_grid(p->grid_res, p->physical_size, p->hbar, p->dt, g, host);
    cudaStream_t s = (cudaStream_t)p->stream;
    if (!same_key(addrs, p)) {
        // a new upload: refused under stream capture, which would record a
        // copy from this call's host buffer (freed when the call returns)
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        e = cudaStreamIsCapturing(s, &cap);
        if (e != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
            if (e != cudaSuccess) cudaGetLastError();
            return finish(ISF_ERR_INVALID,
                          "isf_poisson_solve_static: new grid parameters need a table upload, which cannot be made "
                          "while the stream is being captured; make one call with these parameters first");
        }
        // pageable source: the copy is staged before cudaMemcpyAsync returns
        if ((e = cudaMemcpyAsync(addrs.tables, host.data(), host.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return finish(ISF_ERR_CUDA, std::string("isf_poisson_solve_static: table upload: ") + cudaGetErrorString(e));
        set_key(p->device, p);
    }
    bind_tables(g, addrs.tables);

    XArgs xa;
    std::memset(&xa, 0, sizeof(xa));
    xa.g = g;
    xa.F = addrs.spectrum;
    xa.wp = wp;
    xa.rin = f;
    xa.rout = q;
    YZArgs ya;
    std::memset(&ya, 0, sizeof(ya));
    ya.g = g;
    ya.data = addrs.spectrum;
    ya.row = wp;
    ya.kx_valid = g.n[0] / 2 + 1;
    const char* where = "";
    if ((e = launch_xreal(XR_FWD, xa, s)) != cudaSuccess) where = "x fwd";
    if (e == cudaSuccess) {
        ya.axis = 1;
        if ((e = launch_yzpass_c(YZ_FWD, ya, s)) != cudaSuccess) where = "y fwd";
    }
    if (e == cudaSuccess) {
        ya.axis = 2;
        if ((e = launch_yzpass_c(YZ_FAC, ya, s)) != cudaSuccess) where = "z fac";
    }
    if (e == cudaSuccess) {
        ya.axis = 1;
        if ((e = launch_yzpass_c(YZ_INV, ya, s)) != cudaSuccess) where = "y inv";
    }
    if (e == cudaSuccess && (e = launch_xreal(XR_INV_REAL, xa, s)) != cudaSuccess) where = "x inv";
    if (e != cudaSuccess)
        return finish(ISF_ERR_CUDA, std::string("isf_poisson_solve_static: ") + where + ": " + cudaGetErrorString(e));
    return finish(ISF_OK, "");
}

}  // extern "C"
