// C ABI of libisf (declared in include/isf.h): the ISF handle, its device
// tables and temporaries, and the kernel sequences behind each reference
// operator.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/isf.h"
#include "isf_handle.h"

// row pitch (cells) of the padded velocity grid is a multiple of this
#ifndef ISF_VEL_ROW_ALIGN
#define ISF_VEL_ROW_ALIGN 1
#endif

namespace isf {

// tests of one mbarrier wait of the TMA-staged pass before it gives up (a
// tile arrives within microseconds; this is about half a second)
constexpr long long kTmaWaitLimit = 1LL << 22;

int half_spectrum_row(int nx) { return ((nx / 2 + 1 + 15) / 16) * 16; }

size_t table_bytes(const int n[3]) {
    size_t b = 0;
    for (int a = 0; a < 3; ++a) b += (sizeof(double2) + sizeof(double) + sizeof(float2)) * (size_t)n[a];
    return b;
}

// Grid scalars and the host image of the device tables (ISF constructor,
// parallel.jl:41-63): per-axis Schroedinger phase factors exp(i th_a(k)) with
// th_a = (-4 pi^2 hbar) (k'/L_a)^2 dt / 2, k' the fftshift'ed frequency;
// Laplacian symbols (sin(pi k / n_a) / d_a)^2; twiddles exp(-2 pi i k / n_a).
// Table layout: mtab (double2) | s2 (double) | tw (float2), each axis after axis.
void fill_grid(const int n[3], const int L[3], float hbar, float dt, Grid& g, std::vector<char>& host) {
    const double kPi = 3.14159265358979323846264338327950288;
    std::memset(&g, 0, sizeof(g));
    for (int a = 0; a < 3; ++a) {
        g.n[a] = n[a];
        g.L[a] = (float)L[a];
        g.d[a] = (float)((double)L[a] / (double)n[a]);  // parallel.jl:46
        g.inv_d2[a] = 1.0f / (g.d[a] * g.d[a]);          // parallel.jl:150
        g.dinv[a] = 1.0f / g.d[a];                        // benchmark.jl:62
        int ex = 0;
        g.d_pow2[a] = (std::frexp(g.d[a], &ex) == 0.5f) ? 1 : 0;
        g.feps[a] = 4.0f * (std::nextafter((float)n[a], 1e30f) - (float)n[a]);
    }
    g.N = (long long)n[0] * n[1] * n[2];
    g.pnx = ((n[0] + 1 + ISF_VEL_ROW_ALIGN - 1) / ISF_VEL_ROW_ALIGN) * ISF_VEL_ROW_ALIGN;
    g.pnxy = g.pnx * (n[1] + 1);
    g.NP = (long long)g.pnxy * (n[2] + 1);
    g.hbar = hbar;
    g.dt = dt;
    g.invN = 1.0 / (double)g.N;

    size_t mt_bytes = 0, s2_bytes = 0;
    for (int a = 0; a < 3; ++a) {
        mt_bytes += sizeof(double2) * n[a];
        s2_bytes += sizeof(double) * n[a];
    }
    host.assign(table_bytes(n), 0);
    double2* mt = reinterpret_cast<double2*>(host.data());
    double* s2 = reinterpret_cast<double*>(host.data() + mt_bytes);
    float2* tw = reinterpret_cast<float2*>(host.data() + mt_bytes + s2_bytes);
    const double fm = -4.0 * kPi * kPi * (double)hbar;  // f = -4 pi^2 hbar (parallel.jl:49)
    size_t off = 0;
    for (int a = 0; a < 3; ++a) {
        const int na = n[a];
        for (int k = 0; k < na; ++k) {
            // fftshift'ed frequency (parallel.jl:58, 62): k' = k for k < n/2, k - n otherwise
            const double ks = (k < na / 2) ? (double)k : (double)(k - na);
            const double kk = ks / (double)L[a];
            const double th = fm * kk * kk * (double)dt / 2.0;
            mt[off + k] = make_double2(std::cos(th), std::sin(th));
            const double sn = std::sin(kPi * (double)k / (double)na) / (double)g.d[a];  // parallel.jl:53
            s2[off + k] = sn * sn;
            const long double ang = -2.0L * (long double)kPi * (long double)k / (long double)na;
            tw[off + k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        off += na;
    }
}

void bind_tables(Grid& g, const char* dev) {
    size_t mt_bytes = 0, s2_bytes = 0;
    for (int a = 0; a < 3; ++a) {
        mt_bytes += sizeof(double2) * g.n[a];
        s2_bytes += sizeof(double) * g.n[a];
    }
    size_t off = 0;
    for (int a = 0; a < 3; ++a) {
        g.mtab[a] = reinterpret_cast<const double2*>(dev) + off;
        g.s2[a] = reinterpret_cast<const double*>(dev + mt_bytes) + off;
        g.tw[a] = reinterpret_cast<const float2*>(dev + mt_bytes + s2_bytes) + off;
        off += g.n[a];
    }
}

bool valid_grid(const int n[3], std::string& why) {
    for (int a = 0; a < 3; ++a) {
        if (!supported_len(n[a])) {
            why = "grid_res[" + std::to_string(a) + "] = " + std::to_string(n[a]) +
                  " is not one of 8,12,16,20,24,32,40,48,50,56,64,80,96,100,112,128,160,192,200,256,384,512";
            return false;
        }
    }
    return true;
}

bool check_params(const isf_params* p, std::string& why) {
    if (!p) {
        why = "null parameters";
        return false;
    }
    if (!valid_grid(p->grid_res, why)) return false;
    for (int a = 0; a < 3; ++a)
        if (p->physical_size[a] <= 0) {
            why = "physical_size must be > 0";
            return false;
        }
    if (!(p->dt > 0.f) || !std::isfinite(p->hbar) || !std::isfinite(p->dt)) {
        why = "hbar and dt must be finite, dt > 0";
        return false;
    }
    if (p->flags & ~(ISF_FLAG_NORMALIZED_WEIGHTS | ISF_FLAG_CHECK_NAN | ISF_FLAG_TMA_Z_PASS | ISF_FLAG_TMA_Z_STALL)) {
        why = "unknown flags";
        return false;
    }
    return true;
}

}  // namespace isf

using namespace isf;

namespace isf_int {

thread_local std::string g_create_error;

int fail(isf_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

int cuda_fail(isf_handle* h, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorName(e) + ": " + cudaGetErrorString(e);
    return fail(h, ISF_ERR_CUDA, m);
}


int prof_site(isf_handle* h, const char* name) {
    for (size_t i = 0; i < h->site_names.size(); ++i)
        if (h->site_names[i] == name) return (int)i;
    h->site_names.push_back(name);
    h->site_ms.push_back(0.0);
    h->site_count.push_back(0);
    return (int)h->site_names.size() - 1;
}

cudaEvent_t prof_event(isf_handle* h) {
    if (h->ev_used == h->ev_pool.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        h->ev_pool.push_back(e);
    }
    return h->ev_pool[h->ev_used++];
}

// Records an event pair around one launch when profiling is on.
int prof_begin(isf_handle* h, const char* site, cudaStream_t st) {
    if (!h->prof_on) return -1;
    isf_handle::Rec r;
    r.site = prof_site(h, site);
    r.a = prof_event(h);
    r.b = prof_event(h);
    if (!r.a || !r.b) return -1;
    cudaEventRecord(r.a, st ? st : h->stream);
    h->recs.push_back(r);
    return (int)h->recs.size() - 1;
}

void prof_end(isf_handle* h, int slot, cudaStream_t st) {
    if (slot >= 0) cudaEventRecord(h->recs[slot].b, st ? st : h->stream);
}

int join(isf_handle* h) {
    if (!h->side_pending) return ISF_OK;
    ISF_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_side, 0), "join the particle stream");
    h->side_pending = false;
    return ISF_OK;
}

void destroy_side(isf_handle* h) {
    for (cudaEvent_t e : {h->ev_vel, h->ev_side, h->ev_read[0], h->ev_read[1]})
        if (e) cudaEventDestroy(e);
    if (h->side) cudaStreamDestroy(h->side);
    h->side = nullptr;
}

XArgs xargs(isf_handle* h) {
    XArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = h->g;
    a.F = h->F;
    a.wp = h->wp;
    a.kmajor = h->kmajor;
    return a;
}

YZArgs yzargs(isf_handle* h, void* data, int axis) {
    YZArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = h->g;
    a.data = data;
    a.axis = axis;
    a.row = h->g.n[0];
    a.kx_valid = h->g.n[0];
    return a;
}

// y / z passes over the half spectrum of the Poisson solve
YZArgs yzhalf(isf_handle* h, int axis) {
    YZArgs a = yzargs(h, h->F, axis);
    a.row = h->wp;
    a.kx_valid = h->g.n[0] / 2 + 1;
    return a;
}

// schroedinger_flow! (+ normalize fused into the last pass when norm != 0)
int run_schroedinger(isf_handle* h, float* psi, bool norm) {
    XArgs xa = xargs(h);
    xa.psi = reinterpret_cast<float4*>(psi);
    ISF_LAUNCH(h, launch_xpass(X_PSI_FWD, xa, h->stream), "schroedinger x fwd");
    ISF_LAUNCH(h, launch_yzpass_psi(YZ_FWD, yzargs(h, psi, 1), h->stream), "schroedinger y fwd");
    // the z pass with TMA-staged pencils, when asked for and built for the length
    bool tma = (h->flags & ISF_FLAG_TMA_Z_PASS) && zmask_tma_len(h->g.n[2]) && h->g.n[0] % 8 == 0;
    if (tma && h->zmap_psi != psi) {
        h->zmap_ok = encode_psi_zmap(&h->zmap, psi, h->g);
        h->zmap_psi = psi;
    }
    tma = tma && h->zmap_ok;
    if (tma)
        ISF_LAUNCH(h, launch_zmask_tma(h->zmap, yzargs(h, psi, 2), kTmaWaitLimit, h->counters + 14,
                                       (h->flags & ISF_FLAG_TMA_Z_STALL) ? h->counters + 13 : nullptr, h->stream),
                   "schroedinger z mask");
    else
        ISF_LAUNCH(h, launch_yzpass_psi(YZ_MASK, yzargs(h, psi, 2), h->stream), "schroedinger z mask");
    ISF_LAUNCH(h, launch_yzpass_psi(YZ_INV, yzargs(h, psi, 1), h->stream), "schroedinger y inv");
    ISF_LAUNCH(h, launch_xpass(norm ? X_PSI_INV_NORM : X_PSI_INV, xa, h->stream), "schroedinger x inv");
    return ISF_OK;
}

StencilArgs stargs(isf_handle* h, const float* psi, float* out) {
    StencilArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = h->g;
    a.psi = reinterpret_cast<const float4*>(psi);
    a.out = out;
    return a;
}

// velocity_one_form!(isf, psi, hbar) [+ staggered sharp] into the handle's
// velocity: the grid no in-flight advection reads, which becomes current
int run_one_form(isf_handle* h, const float* psi, float hbar, int sharp, const char* site) {
    const int nb = h->vcur ^ 1;
    if (h->side) ISF_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_read[nb], 0), "velocity buffer reuse");
    h->vcur = nb;
    h->vel = h->vel_buf[nb];
    StencilArgs sa = stargs(h, psi, h->vel);
    sa.hbar = hbar;
    sa.sharp = sharp;
    ISF_LAUNCH(h, launch_stencil(ST_VEL, sa, h->stream), site);
    return ISF_OK;
}

// pressure_project! with the optional nozzle restriction fused in front:
// f = div(one-form) -> Poisson solve -> gauge
int run_projection(isf_handle* h, float* psi, const JetArgs* jet) {
    StencilArgs sa = stargs(h, psi, h->f);
    XArgs xa = xargs(h);
    xa.psi = reinterpret_cast<float4*>(psi);
    xa.rin = h->f;
    if (jet) {
        sa.jet = *jet;
        sa.use_jet = 1;
        xa.jet = *jet;
        xa.use_jet = 1;
    }
    ISF_LAUNCH(h, launch_stencil(ST_DIV, sa, h->stream), "projection div");
    ISF_LAUNCH(h, launch_xreal(XR_FWD, xa, h->stream), "projection x fwd");
    if (int rc = run_poisson_spectral(h, "projection")) return rc;
    ISF_LAUNCH(h, launch_xreal(jet ? XR_INV_GAUGE_JET : XR_INV_GAUGE, xa, h->stream), "projection x inv + gauge");
    return ISF_OK;
}

// y / z transforms with fac/N between them, on the handle's half spectrum:
// one plane kernel for a k-major spectrum, three y / z passes otherwise
int run_poisson_spectral(isf_handle* h, const char* site) {
    if (h->kmajor) {
        ISF_LAUNCH(h, launch_poisson_plane(h->g, h->F, 0, 1, h->stream), (std::string(site) + " yz planes").c_str());
        return ISF_OK;
    }
    ISF_LAUNCH(h, launch_yzpass_c(YZ_FWD, yzhalf(h, 1), h->stream), (std::string(site) + " y fwd").c_str());
    ISF_LAUNCH(h, launch_yzpass_c(YZ_FAC, yzhalf(h, 2), h->stream), (std::string(site) + " z fac").c_str());
    ISF_LAUNCH(h, launch_yzpass_c(YZ_INV, yzhalf(h, 1), h->stream), (std::string(site) + " y inv").c_str());
    return ISF_OK;
}

void free_order(isf_handle* h) {
    cudaFree(h->ord.hist);
    cudaFree(h->ord.rank);
    cudaFree(h->ord.sums);
    cudaFree(h->ord.total);
    cudaFree(h->ord.order);
    h->ord = OrderBufs{};
    h->ord_cap = 0;
    h->order_n = 0;
}

// buffers of the cell order for np slots (allocated on first use, grown as needed)
int ensure_order(isf_handle* h, long long np) {
    if (h->ord.hist && h->ord_cap >= np) return ISF_OK;
    free_order(h);
    const long long cap = np > 0 ? np : 1;
    if (cudaMalloc(&h->ord.hist, sizeof(unsigned) * order_keys(h->g)) != cudaSuccess ||
        cudaMalloc(&h->ord.sums, sizeof(unsigned) * order_sums(h->g)) != cudaSuccess ||
        cudaMalloc(&h->ord.total, sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&h->ord.rank, sizeof(unsigned) * cap) != cudaSuccess ||
        cudaMalloc(&h->ord.order, sizeof(int) * cap) != cudaSuccess) {
        cudaGetLastError();
        free_order(h);
        return fail(h, ISF_ERR_NOMEM, "particle order: device allocation failed");
    }
    h->ord_cap = cap;
    return ISF_OK;
}

int run_order(isf_handle* h, const float* parts, long long np, cudaStream_t st, const char* site) {
    const std::string s(site);
    ISF_LAUNCH_ON(h, st, launch_order_count(h->g, parts, np, h->ord, st), (s + " order count").c_str());
    ISF_LAUNCH_ON(h, st, launch_order_scan(h->g, h->ord, st), (s + " order scan").c_str());
    h->launches += 2;  // the scan is three kernels
    ISF_LAUNCH_ON(h, st, launch_order_scatter(h->g, parts, np, h->ord, st), (s + " order scatter").c_str());
    h->order_n = np;
    h->order_parts = parts;
    h->order_age = 0;
    return ISF_OK;
}

JetArgs make_jet(const float kvec[3], const uint8_t* mask, const float cen[3], float len, float rad, float omgterm,
                 int mode) {
    JetArgs j;
    for (int a = 0; a < 3; ++a) {
        j.kvec[a] = kvec[a];
        j.cen[a] = cen[a];
    }
    j.len = len;
    j.rad = rad;
    j.omgterm = omgterm;
    j.phase_mode = mode;
    j.mask = mask;
    return j;
}

}  // namespace isf_int

using namespace isf_int;

extern "C" {

int isf_create(const isf_params* p, isf_handle** out) {
    if (!p || !out) return fail(nullptr, ISF_ERR_INVALID, "isf_create: null argument");
    *out = nullptr;
    std::string why;
    if (!check_params(p, why)) return fail(nullptr, ISF_ERR_INVALID, "isf_create: " + why);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "isf_create: cudaGetDeviceCount");
    if (p->device < 0 || p->device >= ndev) return fail(nullptr, ISF_ERR_INVALID, "isf_create: bad device ordinal");

    isf_handle* h = new isf_handle();
    h->device = p->device;
    DeviceGuard guard(h->device);
    if (guard.err != cudaSuccess) {
        delete h;
        return cuda_fail(nullptr, guard.err, "isf_create: cudaSetDevice");
    }
    Grid& g = h->g;
    std::vector<char> host;
    fill_grid(p->grid_res, p->physical_size, p->hbar, p->dt, g, host);
    h->wp = half_spectrum_row(g.n[0]);
    h->kmajor = plane_supported(g.n) ? 1 : 0;
    h->flags = p->flags;
    g.norm_w = (p->flags & ISF_FLAG_NORMALIZED_WEIGHTS) ? 1 : 0;
    const size_t total = host.size();
    auto cleanup = [&](int code, const std::string& msg) {
        if (h->F) cudaFree(h->F);
        if (h->f) cudaFree(h->f);
        for (float* v : h->vel_buf)
            if (v) cudaFree(v);
        if (h->tables) cudaFree(h->tables);
        if (h->counters) cudaFree(h->counters);
        destroy_side(h);
        if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return fail(nullptr, code, msg);
    };
    if (p->stream) {
        h->stream = (cudaStream_t)p->stream;
    } else {
        e = cudaStreamCreateWithFlags(&h->stream, cudaStreamDefault);  // orders with the legacy default stream
        if (e != cudaSuccess) return cleanup(ISF_ERR_CUDA, std::string("isf_create: stream: ") + cudaGetErrorString(e));
        h->own_stream = true;
        // the particle stream of isf_step (blocking as well, so work on the
        // legacy default stream is ordered after its advection)
        e = cudaStreamCreateWithFlags(&h->side, cudaStreamDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_vel, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_side, cudaEventDisableTiming);
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&h->ev_read[i], cudaEventDisableTiming);
        if (e != cudaSuccess) return cleanup(ISF_ERR_CUDA, std::string("isf_create: particle stream: ") + cudaGetErrorString(e));
    }
    if (cudaMalloc(&h->F, sizeof(float2) * g.N) != cudaSuccess || cudaMalloc(&h->f, sizeof(float) * g.N) != cudaSuccess ||
        cudaMalloc(&h->vel_buf[0], sizeof(float) * kVelComp * g.NP) != cudaSuccess ||
        cudaMalloc(&h->vel_buf[1], sizeof(float) * kVelComp * g.NP) != cudaSuccess ||
        cudaMalloc(&h->tables, total) != cudaSuccess ||
        cudaMalloc(&h->counters, 16 * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return cleanup(ISF_ERR_NOMEM, "isf_create: device allocation failed");
    }
    e = cudaMemcpy(h->tables, host.data(), total, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->counters, 0, 16 * sizeof(unsigned long long));
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMemset(h->vel_buf[i], 0, sizeof(float) * kVelComp * g.NP);
    h->vel = h->vel_buf[0];
    if (e == cudaSuccess) e = cudaMemset(h->F, 0, sizeof(float2) * g.N);
    if (e != cudaSuccess) return cleanup(ISF_ERR_CUDA, std::string("isf_create: upload: ") + cudaGetErrorString(e));
    bind_tables(g, reinterpret_cast<const char*>(h->tables));
    *out = h;
    return ISF_OK;
}

int isf_destroy(isf_handle* h) {
    if (!h) return ISF_OK;
    {
        DeviceGuard guard(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        if (h->side) cudaStreamSynchronize(h->side);
        cudaFree(h->F);
        cudaFree(h->f);
        cudaFree(h->vel_buf[0]);
        cudaFree(h->vel_buf[1]);
        cudaFree(h->tables);
        cudaFree(h->counters);
        cudaFree(h->keep_counts);
        free_order(h);
        adj_free(h);
        destroy_side(h);
        if (h->own_stream) cudaStreamDestroy(h->stream);
        for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    }
    delete h;
    return ISF_OK;
}

const char* isf_last_error(const isf_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int isf_sync(isf_handle* h) {
    ISF_ENTER(h);
    ISF_CUDA(h, cudaStreamSynchronize(h->stream), "isf_sync");
    return ISF_OK;
}

int isf_join(isf_handle* h) {
    ISF_ENTER(h);
    return ISF_OK;
}

int isf_malloc(isf_handle* h, void** dptr, size_t bytes) {
    ISF_ENTER(h);
    if (!dptr) return fail(h, ISF_ERR_INVALID, "isf_malloc: null out pointer");
    if (cudaMalloc(dptr, bytes) != cudaSuccess) {
        cudaGetLastError();
        *dptr = nullptr;
        return fail(h, ISF_ERR_NOMEM, "isf_malloc: cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    return ISF_OK;
}

int isf_free(isf_handle* h, void* dptr) {
    ISF_ENTER(h);
    ISF_CUDA(h, cudaStreamSynchronize(h->stream), "isf_free: sync");
    ISF_CUDA(h, cudaFree(dptr), "isf_free");
    return ISF_OK;
}

int isf_memcpy_h2d(isf_handle* h, void* dst, const void* src, size_t bytes) {
    ISF_ENTER(h);
    if (bytes == 0) return ISF_OK;
    if (!dst || !src) return fail(h, ISF_ERR_INVALID, "isf_memcpy_h2d: null pointer");
    ISF_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream), "isf_memcpy_h2d");
    return ISF_OK;
}

int isf_memcpy_d2h(isf_handle* h, void* dst, const void* src, size_t bytes) {
    ISF_ENTER(h);
    if (bytes == 0) return ISF_OK;
    if (!dst || !src) return fail(h, ISF_ERR_INVALID, "isf_memcpy_d2h: null pointer");
    ISF_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream), "isf_memcpy_d2h");
    return ISF_OK;
}

int isf_get_stream(const isf_handle* h, void** stream) {
    if (!h || !stream) return fail(nullptr, ISF_ERR_INVALID, "isf_get_stream: null argument");
    *stream = (void*)h->stream;
    return ISF_OK;
}

int isf_grid_info(const isf_handle* h, int32_t n_out[3], float d_out[3]) {
    if (!h) return fail(nullptr, ISF_ERR_INVALID, "null isf handle");
    for (int a = 0; a < 3; ++a) {
        if (n_out) n_out[a] = h->g.n[a];
        if (d_out) d_out[a] = h->g.d[a];
    }
    return ISF_OK;
}

int isf_schroedinger_flow(isf_handle* h, float* psi) {
    ISF_ENTER(h);
    if (!psi) return fail(h, ISF_ERR_INVALID, "isf_schroedinger_flow: null psi");
    ISF_ALIGNED(h, psi, 16, "psi");
    return run_schroedinger(h, psi, false);
}

int isf_normalize_psi(isf_handle* h, float* psi) {
    ISF_ENTER(h);
    if (!psi) return fail(h, ISF_ERR_INVALID, "isf_normalize_psi: null psi");
    ISF_ALIGNED(h, psi, 16, "psi");
    ISF_LAUNCH(h, launch_normalize(h->g, reinterpret_cast<float4*>(psi), h->stream), "normalize");
    return ISF_OK;
}

int isf_pressure_project(isf_handle* h, float* psi) {
    ISF_ENTER(h);
    if (!psi) return fail(h, ISF_ERR_INVALID, "isf_pressure_project: null psi");
    ISF_ALIGNED(h, psi, 16, "psi");
    return run_projection(h, psi, nullptr);
}

int isf_velocity_one_form(isf_handle* h, const float* psi, float hbar) {
    ISF_ENTER(h);
    if (!psi) return fail(h, ISF_ERR_INVALID, "isf_velocity_one_form: null psi");
    ISF_ALIGNED(h, psi, 16, "psi");
    return run_one_form(h, psi, hbar, 0, "one_form");
}

int isf_staggered_sharp(isf_handle* h) {
    ISF_ENTER(h);
    ISF_LAUNCH(h, launch_sharp(h->g, h->vel, h->stream), "staggered_sharp");
    return ISF_OK;
}

int isf_get_velocity(isf_handle* h, float* aos) {
    ISF_ENTER(h);
    if (!aos) return fail(h, ISF_ERR_INVALID, "isf_get_velocity: null buffer");
    ISF_LAUNCH(h, launch_vel_to_aos(h->g, h->vel, aos, h->stream), "get_velocity");
    return ISF_OK;
}

int isf_set_velocity(isf_handle* h, const float* aos) {
    ISF_ENTER(h);
    if (!aos) return fail(h, ISF_ERR_INVALID, "isf_set_velocity: null buffer");
    ISF_LAUNCH(h, launch_vel_from_aos(h->g, aos, h->vel, h->stream), "set_velocity");
    return ISF_OK;
}

int isf_isjet(isf_handle* h, uint8_t* mask, const float cen[3], float len, float rad) {
    ISF_ENTER(h);
    if (!mask || !cen) return fail(h, ISF_ERR_INVALID, "isf_isjet: null argument");
    ISF_LAUNCH(h, launch_isjet(h->g, mask, cen, len, rad, h->stream), "isjet");
    return ISF_OK;
}

int isf_restrict_velocity(isf_handle* h, float* psi, const float kvec[3], const uint8_t* mask, const float cen[3],
                          float len, float rad, float omgterm, int32_t phase_mode) {
    ISF_ENTER(h);
    if (!psi || !kvec || (!mask && !cen)) return fail(h, ISF_ERR_INVALID, "isf_restrict_velocity: null argument");
    ISF_ALIGNED(h, psi, 16, "psi");
    if (phase_mode != ISF_PHASE_REFERENCE_SUM && phase_mode != ISF_PHASE_DOT)
        return fail(h, ISF_ERR_INVALID, "isf_restrict_velocity: bad phase_mode");
    const float zero[3] = {0.f, 0.f, 0.f};
    JetArgs j = make_jet(kvec, mask, cen ? cen : zero, len, rad, omgterm, phase_mode);
    ISF_LAUNCH(h, launch_restrict(h->g, reinterpret_cast<float4*>(psi), j, h->stream), "restrict_velocity");
    return ISF_OK;
}

int isf_init_jet(isf_handle* h, float* psi, int32_t iters, const float kvec[3], const uint8_t* mask, const float cen[3],
                 float len, float rad, int32_t phase_mode) {
    ISF_ENTER(h);
    if (!psi || !kvec || (!mask && !cen) || iters < 0) return fail(h, ISF_ERR_INVALID, "isf_init_jet: bad argument");
    ISF_ALIGNED(h, psi, 16, "psi");
    if (phase_mode != ISF_PHASE_REFERENCE_SUM && phase_mode != ISF_PHASE_DOT)
        return fail(h, ISF_ERR_INVALID, "isf_init_jet: bad phase_mode");
    const float zero[3] = {0.f, 0.f, 0.f};
    // restrict_velocity!(isf, psi, kvec, isjet, 0) + pressure_project!, the
    // restriction fused into the projection's stencil and gauge pass as in isf_step
    JetArgs j = make_jet(kvec, mask, cen ? cen : zero, len, rad, 0.f, phase_mode);
    for (int it = 0; it < iters; ++it)
        if (int rc = run_projection(h, psi, &j)) return rc;
    return ISF_OK;
}

int isf_add_particles(isf_handle* h, float* parts, int64_t nslots, int64_t start, int64_t count, const float cen[3],
                      float len, float rad, uint64_t seed, uint64_t counter, int32_t mode) {
    ISF_ENTER(h);
    if (!parts || !cen) return fail(h, ISF_ERR_INVALID, "isf_add_particles: null argument");
    if (nslots <= 0 || count < 0 || start < 0) return fail(h, ISF_ERR_INVALID, "isf_add_particles: bad slot range");
    if (count > nslots) return fail(h, ISF_ERR_INVALID, "isf_add_particles: count exceeds the number of slots");
    if (mode < ISF_EMIT_RING || mode > ISF_EMIT_RING_PLANE) return fail(h, ISF_ERR_INVALID, "isf_add_particles: bad mode");
    EmitArgs e;
    for (int a = 0; a < 3; ++a) e.cen[a] = cen[a];
    e.len = len;
    e.rad = rad;
    e.seed = seed;
    e.counter = counter;
    e.mode = mode;
    ISF_LAUNCH(h, launch_emit(parts, nslots, start % nslots, count, e, h->stream), "add_particles");
    return ISF_OK;
}

int isf_staggered_advect(isf_handle* h, float* parts, int64_t np) {
    ISF_ENTER(h);
    if (np < 0 || (np > 0 && !parts)) return fail(h, ISF_ERR_INVALID, "isf_staggered_advect: bad particles");
    if (np > kMaxParticles) return fail(h, ISF_ERR_INVALID, "isf_staggered_advect: more than 715827882 particles");
    ISF_LAUNCH(h, launch_advect(h->g, parts, np, h->vel, h->counters, h->stream), "staggered_advect");
    return ISF_OK;
}

int isf_set_particle_order(isf_handle* h, int32_t every) {
    ISF_ENTER(h);
    if (every < 0) return fail(h, ISF_ERR_INVALID, "isf_set_particle_order: every must be >= 0");
    h->order_every = every;
    if (every == 0) h->order_n = 0;
    return ISF_OK;
}

int isf_sort_particles(isf_handle* h, const float* parts, int64_t np) {
    ISF_ENTER(h);
    if (np <= 0 || !parts) return fail(h, ISF_ERR_INVALID, "isf_sort_particles: bad particles");
    if (np > kMaxParticles) return fail(h, ISF_ERR_INVALID, "isf_sort_particles: more than 715827882 particles");
    if (int rc = ensure_order(h, np)) return rc;
    return run_order(h, parts, np, h->stream, "sort");
}

int isf_get_particle_order(isf_handle* h, int32_t* order, int64_t cap, int64_t* n) {
    ISF_ENTER(h);
    if (!n) return fail(h, ISF_ERR_INVALID, "isf_get_particle_order: null count");
    *n = h->order_n;
    if (h->order_n == 0 || !order) return ISF_OK;  // no permutation, or only its length asked for
    if (cap < h->order_n) return fail(h, ISF_ERR_INVALID, "isf_get_particle_order: buffer too small");
    ISF_CUDA(h, cudaMemcpyAsync(order, h->ord.order, sizeof(int) * h->order_n, cudaMemcpyDeviceToDevice, h->stream),
             "isf_get_particle_order");
    return ISF_OK;
}

int isf_step(isf_handle* h, float* psi, float* parts, int64_t np, const isf_step_args* a) {
    ISF_ENTER_NOJOIN(h);
    if (!psi || !a) return fail(h, ISF_ERR_INVALID, "isf_step: null argument");
    ISF_ALIGNED(h, psi, 16, "psi");
    if (np < 0 || (np > 0 && !parts)) return fail(h, ISF_ERR_INVALID, "isf_step: bad particles");
    if (np > kMaxParticles) return fail(h, ISF_ERR_INVALID, "isf_step: more than 715827882 particles");
    if (a->jet) {
        if (a->phase_mode != ISF_PHASE_REFERENCE_SUM && a->phase_mode != ISF_PHASE_DOT)
            return fail(h, ISF_ERR_INVALID, "isf_step: bad phase_mode");
        if (a->emit_count < 0 || a->emit_start < 0 || (a->emit_count > 0 && (np <= 0 || a->emit_count > np)))
            return fail(h, ISF_ERR_INVALID, "isf_step: bad emission range");
        if (a->emit_count > 0 && (a->emit_mode < ISF_EMIT_RING || a->emit_mode > ISF_EMIT_RING_PLANE))
            return fail(h, ISF_ERR_INVALID, "isf_step: bad emit_mode");
    }
    // the cell order of the slots: re-sorted every order_every steps, and
    // whenever the slot array or its length changes
    const bool resort = h->order_every > 0 && np > 0 &&
                        (h->order_n != np || h->order_parts != parts || h->order_age >= h->order_every);
    if (resort)
        if (int rc = ensure_order(h, np)) return rc;
    int rc = run_schroedinger(h, psi, true);  // schroedinger_flow! + normalize_psi
    if (rc) return rc;
    rc = run_projection(h, psi, nullptr);     // pressure_project!
    if (rc) return rc;
    if (a->jet) {
        JetArgs j = make_jet(a->kvec, a->jetmask, a->nozzle_cen, a->nozzle_len, a->nozzle_rad, a->omega_t,
                             a->phase_mode);
        rc = run_projection(h, psi, &j);  // restrict_velocity! + pressure_project!
        if (rc) return rc;
    }
    // velocity_one_form!(isf, psi, isf.hbar) + staggered sharp
    rc = run_one_form(h, psi, h->g.hbar, 1, "step one_form");
    if (rc) return rc;
    // add_particles! (before the projections in the reference; the particles
    // are independent of psi) and staggered_advect!.  With a particle stream
    // they run there, after this step's velocity, while the caller queues the
    // next step's psi passes; the velocity grid they read is not written
    // again until they are done (run_one_form alternates between two).
    cudaStream_t ps = h->side ? h->side : h->stream;
    const bool emit = a->jet && a->emit_count > 0;
    if (h->side && (emit || np > 0)) {
        ISF_CUDA(h, cudaEventRecord(h->ev_vel, h->stream), "step velocity event");
        ISF_CUDA(h, cudaStreamWaitEvent(h->side, h->ev_vel, 0), "step velocity event");
    }
    if (emit) {
        EmitArgs e;
        for (int k = 0; k < 3; ++k) e.cen[k] = a->nozzle_cen[k];
        e.len = a->nozzle_len;
        e.rad = a->nozzle_rad;
        e.seed = a->seed;
        e.counter = a->counter;
        e.mode = a->emit_mode;
        ISF_LAUNCH_ON(h, ps, launch_emit(parts, np, a->emit_start % np, a->emit_count, e, ps), "step emit");
    }
    const int* order = nullptr;
    if (h->order_every > 0 && np > 0) {
        if (resort)
            if (int rc_o = run_order(h, parts, np, ps, "step")) return rc_o;
        ++h->order_age;
        order = h->ord.order;
    }
    if (np > 0)
        ISF_LAUNCH_ON(h, ps, launch_advect(h->g, parts, np, h->vel, h->counters, ps, 1, 0, order), "step advect");
    if (h->side && (emit || np > 0)) {
        ISF_CUDA(h, cudaEventRecord(h->ev_read[h->vcur], h->side), "step particle event");
        ISF_CUDA(h, cudaEventRecord(h->ev_side, h->side), "step particle event");
        h->side_pending = true;
    }
    if (h->flags & ISF_FLAG_CHECK_NAN) {
        if (int rc_j = join(h)) return rc_j;  // after any counter reset queued on the particle stream
        // counters[15]: non-finite psi cells after this step
        ISF_CUDA(h, cudaMemsetAsync(h->counters + 15, 0, sizeof(unsigned long long), h->stream), "nan check");
        ISF_LAUNCH(h, launch_count_nonfinite(h->g, reinterpret_cast<const float4*>(psi), h->counters + 15, h->stream),
                   "step nan check");
        unsigned long long bad = 0;
        ISF_CUDA(h, cudaMemcpyAsync(&bad, h->counters + 15, sizeof(bad), cudaMemcpyDeviceToHost, h->stream), "nan check");
        ISF_CUDA(h, cudaStreamSynchronize(h->stream), "nan check");
        if (bad) return fail(h, ISF_ERR_NAN, "isf_step: " + std::to_string(bad) + " psi cells are not finite");
    }
    return ISF_OK;
}

int isf_div(isf_handle* h, float* f) {
    ISF_ENTER(h);
    if (!f) return fail(h, ISF_ERR_INVALID, "isf_div: null output");
    ISF_LAUNCH(h, launch_div(h->g, h->vel, f, h->stream), "div");
    return ISF_OK;
}

int isf_poisson_solve(isf_handle* h, const float* f, float* q) {
    ISF_ENTER(h);
    if (!f || !q) return fail(h, ISF_ERR_INVALID, "isf_poisson_solve: null argument");
    XArgs xa = xargs(h);
    xa.rin = f;
    xa.rout = q;
    ISF_LAUNCH(h, launch_xreal(XR_FWD, xa, h->stream), "poisson x fwd");
    if (int rc = run_poisson_spectral(h, "poisson")) return rc;
    ISF_LAUNCH(h, launch_xreal(XR_INV_REAL, xa, h->stream), "poisson x inv");
    return ISF_OK;
}

int isf_fft3(isf_handle* h, float* data, int32_t sign) {
    ISF_ENTER(h);
    if (!data || (sign != -1 && sign != 1)) return fail(h, ISF_ERR_INVALID, "isf_fft3: bad argument");
    ISF_ALIGNED(h, data, 8, "data");
    XArgs xa = xargs(h);
    xa.F = reinterpret_cast<float2*>(data);
    if (sign < 0) {
        ISF_LAUNCH(h, launch_xpass(X_C_FWD, xa, h->stream), "fft3 x");
        ISF_LAUNCH(h, launch_yzpass_c(YZ_FWD, yzargs(h, data, 1), h->stream), "fft3 y");
        ISF_LAUNCH(h, launch_yzpass_c(YZ_FWD, yzargs(h, data, 2), h->stream), "fft3 z");
    } else {
        ISF_LAUNCH(h, launch_yzpass_c(YZ_INV, yzargs(h, data, 2), h->stream), "ifft3 z");
        ISF_LAUNCH(h, launch_yzpass_c(YZ_INV, yzargs(h, data, 1), h->stream), "ifft3 y");
        ISF_LAUNCH(h, launch_xpass(X_C_INV, xa, h->stream), "ifft3 x");
        ISF_LAUNCH(h, launch_scale_c(h->g, reinterpret_cast<float2*>(data), (float)h->g.invN, h->stream), "ifft3 scale");
    }
    return ISF_OK;
}

int isf_profile_start(isf_handle* h) {
    ISF_ENTER(h);
    h->prof_on = true;
    h->ev_used = 0;
    h->recs.clear();
    for (size_t i = 0; i < h->site_ms.size(); ++i) {
        h->site_ms[i] = 0.0;
        h->site_count[i] = 0;
    }
    return ISF_OK;
}

int isf_profile_stop(isf_handle* h) {
    ISF_ENTER(h);
    h->prof_on = false;
    ISF_CUDA(h, cudaStreamSynchronize(h->stream), "isf_profile_stop: sync");
    for (const auto& r : h->recs) {
        float ms = 0.f;
        ISF_CUDA(h, cudaEventElapsedTime(&ms, r.a, r.b), "isf_profile_stop: elapsed");
        h->site_ms[r.site] += ms;
        h->site_count[r.site] += 1;
    }
    h->recs.clear();
    h->ev_used = 0;
    return ISF_OK;
}

int isf_profile_sites(const isf_handle* h, int32_t* n) {
    if (!h || !n) return fail(nullptr, ISF_ERR_INVALID, "isf_profile_sites: null argument");
    *n = (int32_t)h->site_names.size();
    return ISF_OK;
}

int isf_profile_get(const isf_handle* h, int32_t i, char* name, size_t cap, double* total_ms, int64_t* launches) {
    if (!h || i < 0 || (size_t)i >= h->site_names.size())
        return fail(nullptr, ISF_ERR_INVALID, "isf_profile_get: bad index");
    if (name && cap) {
        std::strncpy(name, h->site_names[i].c_str(), cap - 1);
        name[cap - 1] = '\0';
    }
    if (total_ms) *total_ms = h->site_ms[i];
    if (launches) *launches = h->site_count[i];
    return ISF_OK;
}

int isf_launch_count(const isf_handle* h, uint64_t* out) {
    if (!h || !out) return fail(nullptr, ISF_ERR_INVALID, "isf_launch_count: null argument");
    *out = h->launches;
    return ISF_OK;
}

int isf_counters(isf_handle* h, uint64_t* out, int32_t n, int32_t reset) {
    ISF_ENTER(h);
    if (n < 0 || n > 16 || (n > 0 && !out)) return fail(h, ISF_ERR_INVALID, "isf_counters: n must be 0..16");
    unsigned long long tmp[16] = {0};
    ISF_CUDA(h, cudaMemcpyAsync(tmp, h->counters, sizeof(tmp), cudaMemcpyDeviceToHost, h->stream), "counters");
    ISF_CUDA(h, cudaStreamSynchronize(h->stream), "counters sync");
    for (int i = 0; i < n; ++i) out[i] = tmp[i];
    if (reset) ISF_CUDA(h, cudaMemsetAsync(h->counters, 0, sizeof(tmp), h->stream), "counters reset");
    return ISF_OK;
}

int isf_counters_async(isf_handle* h, uint64_t* host_out, int32_t n, int32_t reset) {
    ISF_ENTER_NOJOIN(h);
    if (n < 1 || n > 16 || !host_out) return fail(h, ISF_ERR_INVALID, "isf_counters_async: n must be 1..16");
    // behind the last step's advection on the particle stream, so the read
    // does not hold the handle's stream back; everything else that touched
    // the counters is ordered before that advection
    cudaStream_t st = h->side_pending ? h->side : h->stream;
    ISF_CUDA(h, cudaMemcpyAsync(host_out, h->counters, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, st),
             "counters");
    if (reset) ISF_CUDA(h, cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * 16, st), "counters reset");
    if (h->side_pending) ISF_CUDA(h, cudaEventRecord(h->ev_side, h->side), "counters event");
    return ISF_OK;
}

}  // extern "C"
