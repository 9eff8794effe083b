// C ABI of the FP64 structure-of-arrays front-end (src/MatlabPort.jl): layout
// conversions, the standalone gauge transform and the Particles type (x, y, z
// vectors with a list of active slots) on the handle's kernels.
#include <string>

#include "../../include/isf.h"
#include "isf_handle.h"

using namespace isf;
using namespace isf_int;

namespace {

// slot lists index 32-bit positions in the keep-inside scan
constexpr long long kMaxList = (1LL << 31) - 1;

int check_xyz(isf_handle* h, const void* x, const void* y, const void* z, long long n, const char* where) {
    if (n < 0 || n > kMaxList) return fail(h, ISF_ERR_INVALID, std::string(where) + ": bad count");
    if (n > 0 && (!x || !y || !z)) return fail(h, ISF_ERR_INVALID, std::string(where) + ": null x, y or z");
    return ISF_OK;
}

}  // namespace

extern "C" {

int isf_psi_from_f64(isf_handle* h, const double* psi1, const double* psi2, float* psi) {
    ISF_ENTER(h);
    if (!psi1 || !psi2 || !psi) return fail(h, ISF_ERR_INVALID, "isf_psi_from_f64: null argument");
    ISF_ALIGNED(h, psi1, 16, "psi1");
    ISF_ALIGNED(h, psi2, 16, "psi2");
    ISF_ALIGNED(h, psi, 16, "psi");
    ISF_LAUNCH(h, launch_psi_from_f64(psi1, psi2, psi, h->g.N, h->stream), "psi from f64");
    return ISF_OK;
}

int isf_psi_to_f64(isf_handle* h, const float* psi, double* psi1, double* psi2) {
    ISF_ENTER(h);
    if (!psi1 || !psi2 || !psi) return fail(h, ISF_ERR_INVALID, "isf_psi_to_f64: null argument");
    ISF_ALIGNED(h, psi1, 16, "psi1");
    ISF_ALIGNED(h, psi2, 16, "psi2");
    ISF_ALIGNED(h, psi, 16, "psi");
    ISF_LAUNCH(h, launch_psi_to_f64(psi, psi1, psi2, h->g.N, h->stream), "psi to f64");
    return ISF_OK;
}

int isf_velocity_from_f64(isf_handle* h, const double* vx, const double* vy, const double* vz) {
    ISF_ENTER(h);
    if (!vx || !vy || !vz) return fail(h, ISF_ERR_INVALID, "isf_velocity_from_f64: null argument");
    ISF_LAUNCH(h, launch_vel_from_f64(h->g, vx, vy, vz, h->vel, h->stream), "velocity from f64");
    return ISF_OK;
}

int isf_velocity_to_f64(isf_handle* h, double* vx, double* vy, double* vz) {
    ISF_ENTER(h);
    if (!vx || !vy || !vz) return fail(h, ISF_ERR_INVALID, "isf_velocity_to_f64: null argument");
    ISF_LAUNCH(h, launch_vel_to_f64(h->g, h->vel, vx, vy, vz, h->stream), "velocity to f64");
    return ISF_OK;
}

int isf_real_from_f64(isf_handle* h, const double* src, int64_t stride, double scale, float* dst, int64_t n) {
    ISF_ENTER(h);
    if (n < 0 || stride < 1 || (n > 0 && (!src || !dst)))
        return fail(h, ISF_ERR_INVALID, "isf_real_from_f64: bad argument");
    ISF_LAUNCH(h, launch_real_from_f64(src, stride, scale, dst, n, h->stream), "real from f64");
    return ISF_OK;
}

int isf_real_to_f64(isf_handle* h, const float* src, double* dst, int64_t n) {
    ISF_ENTER(h);
    if (n < 0 || (n > 0 && (!src || !dst))) return fail(h, ISF_ERR_INVALID, "isf_real_to_f64: bad argument");
    ISF_LAUNCH(h, launch_real_to_f64(src, dst, n, h->stream), "real to f64");
    return ISF_OK;
}

int isf_complex_to_f64(isf_handle* h, const float* re, const float* im, double* dst, int64_t n) {
    ISF_ENTER(h);
    if (n < 0 || (n > 0 && (!re || !dst))) return fail(h, ISF_ERR_INVALID, "isf_complex_to_f64: bad argument");
    ISF_ALIGNED(h, dst, 16, "dst");
    ISF_LAUNCH(h, launch_complex_to_f64(re, im, dst, n, h->stream), "complex to f64");
    return ISF_OK;
}

int isf_gauge_transform(isf_handle* h, float* psi, const float* q_re, const float* q_im) {
    ISF_ENTER(h);
    if (!psi || !q_re) return fail(h, ISF_ERR_INVALID, "isf_gauge_transform: null argument");
    ISF_ALIGNED(h, psi, 16, "psi");
    ISF_LAUNCH(h, launch_gauge_complex(psi, q_re, q_im, h->g.N, h->stream), "gauge_transform");
    return ISF_OK;
}

int isf_add_particles_soa(isf_handle* h, float* x, float* y, float* z, int64_t nslots, int64_t start, int64_t count,
                          const float cen[3], float len, float rad, uint64_t seed, uint64_t counter, int32_t mode) {
    ISF_ENTER(h);
    if (int rc = check_xyz(h, x, y, z, nslots, "isf_add_particles_soa")) return rc;
    if (!cen || count < 0 || start < 0 || (count > 0 && (nslots <= 0 || count > nslots)))
        return fail(h, ISF_ERR_INVALID, "isf_add_particles_soa: bad range");
    if (mode < ISF_EMIT_RING || mode > ISF_EMIT_RING_PLANE)
        return fail(h, ISF_ERR_INVALID, "isf_add_particles_soa: bad mode");
    if (count == 0) return ISF_OK;
    EmitArgs e;
    for (int k = 0; k < 3; ++k) e.cen[k] = cen[k];
    e.len = len;
    e.rad = rad;
    e.seed = seed;
    e.counter = counter;
    e.mode = mode;
    ISF_LAUNCH(h, launch_emit_soa(x, y, z, nslots, start % nslots, count, e, h->stream), "add_particles soa");
    return ISF_OK;
}

int isf_staggered_velocity(isf_handle* h, const float* x, const float* y, const float* z, int64_t n, float* ux,
                           float* uy, float* uz) {
    ISF_ENTER(h);
    if (int rc = check_xyz(h, x, y, z, n, "isf_staggered_velocity")) return rc;
    if (n > 0 && (!ux || !uy || !uz)) return fail(h, ISF_ERR_INVALID, "isf_staggered_velocity: null output");
    ISF_LAUNCH(h, launch_sample_velocity(h->g, x, y, z, n, h->vel, ux, uy, uz, h->counters, h->stream),
               "staggered_velocity");
    return ISF_OK;
}

int isf_advect_active(isf_handle* h, float* x, float* y, float* z, int64_t nslots, const int64_t* active, int64_t n,
                      float dt) {
    ISF_ENTER(h);
    if (int rc = check_xyz(h, x, y, z, nslots, "isf_advect_active")) return rc;
    if (n < 0 || n > kMaxList || (!active && n > nslots))
        return fail(h, ISF_ERR_INVALID, "isf_advect_active: bad active count");
    if (!(dt == dt)) return fail(h, ISF_ERR_INVALID, "isf_advect_active: dt is NaN");
    ISF_LAUNCH(h,
               launch_advect_active(h->g, x, y, z, nslots, reinterpret_cast<const long long*>(active), n, dt, h->vel,
                                    h->counters, h->stream),
               "advect active");
    return ISF_OK;
}

int isf_keep_inside(isf_handle* h, const float* x, const float* y, const float* z, int64_t nslots,
                    const int64_t* active, int64_t n, int64_t* out_active, int64_t* out_n) {
    ISF_ENTER(h);
    if (int rc = check_xyz(h, x, y, z, nslots, "isf_keep_inside")) return rc;
    if (n < 0 || n > kMaxList || (!active && n > nslots) || !out_n || (n > 0 && !out_active))
        return fail(h, ISF_ERR_INVALID, "isf_keep_inside: bad argument");
    if (active && n > 0 && out_active < active + n && active < out_active + n)
        return fail(h, ISF_ERR_INVALID, "isf_keep_inside: out_active overlaps active");
    const long long nb = keep_blocks(n);
    if (nb > h->keep_cap) {
        if (h->keep_counts) {
            ISF_CUDA(h, cudaStreamSynchronize(h->stream), "isf_keep_inside: sync");
            cudaFree(h->keep_counts);
            h->keep_counts = nullptr;
            h->keep_cap = 0;
        }
        if (cudaMalloc(&h->keep_counts, sizeof(unsigned) * nb) != cudaSuccess) {
            cudaGetLastError();
            h->keep_counts = nullptr;
            return fail(h, ISF_ERR_NOMEM, "isf_keep_inside: scratch allocation failed");
        }
        h->keep_cap = nb;
    }
    ISF_LAUNCH(h,
               launch_keep_inside(h->g, x, y, z, nslots, reinterpret_cast<const long long*>(active), n, h->keep_counts,
                                  reinterpret_cast<long long*>(out_active), reinterpret_cast<long long*>(out_n),
                                  h->stream),
               "keep inside");
    return ISF_OK;
}

int isf_gather_particles(isf_handle* h, const float* x, const float* y, const float* z, int64_t nslots,
                         const int64_t* ind, int64_t n, float* ox, float* oy, float* oz) {
    ISF_ENTER(h);
    if (int rc = check_xyz(h, x, y, z, nslots, "isf_gather_particles")) return rc;
    if (n < 0 || n > kMaxList || (n > 0 && (!ind || !ox || !oy || !oz)))
        return fail(h, ISF_ERR_INVALID, "isf_gather_particles: bad argument");
    ISF_LAUNCH(h,
               launch_gather3(x, y, z, nslots, reinterpret_cast<const long long*>(ind), n, ox, oy, oz, h->counters,
                              h->stream),
               "gather particles");
    return ISF_OK;
}

}  // extern "C"
