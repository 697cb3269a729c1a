// Host evaluation of the device physics kinds (fv_physics_exact.cuh, the
// reference's exact arithmetic).  A caller that holds user physics functions
// (the fvhyper C++ shim: calc_flux, limiter_func, boundaries::bounds) compares
// them with these on probe states to pick the device kind, and refuses what
// matches none.  Built with -ffp-contract=off, so the results are the
// reference's bits.
#include <stdint.h>
#include <string.h>

#include "fv_physics_exact.cuh"
#include "fvgpu.h"

extern "C" {

int fv_kind_flux(int32_t flux, double gamma, const double* qi, const double* qj, const double* n, double* f) {
    if (!qi || !qj || !n || !f) return FV_ERR_ARG;
    switch (flux) {
        case FV_FLUX_ROE_FS: fvgpu::exact::roe<true>(gamma, f, qi, qj, n[0], n[1]); return FV_OK;
        case FV_FLUX_ROE_ST: fvgpu::exact::roe<false>(gamma, f, qi, qj, n[0], n[1]); return FV_OK;
        case FV_FLUX_BURGERS: fvgpu::exact::burgers(f, qi, qj, n[0], n[1]); return FV_OK;
        default: return FV_ERR_UNSUPPORTED;
    }
}

int fv_kind_flux_grad(const fv_physics* ph, const double* qi, const double* qj, const double* gx,
                      const double* gy, const double* n, double* f) {
    if (!ph || !qi || !qj || !gx || !gy || !n || !f) return FV_ERR_ARG;
    if (ph->flux == FV_FLUX_DIFFUSION) {
        fvgpu::exact::diffusion(f, gx, gy, n[0], n[1]);
        return FV_OK;
    }
    if (ph->flux == FV_FLUX_BURGERS_DIFF) {
        fvgpu::exact::burgers_diffusion(f, qi, qj, gx, gy, n[0], n[1]);
        return FV_OK;
    }
    if (ph->flux == FV_FLUX_NS) {
        fvgpu::Params P;
        memset(&P, 0, sizeof(P));
        P.gamma = ph->gamma; P.mu = ph->mu; P.pr = ph->pr; P.cp = ph->cp; P.r = ph->r;
        fvgpu::exact::roe<false>(P.gamma, f, qi, qj, n[0], n[1]);
        fvgpu::exact::ns_viscous(P, f, qi, qj, gx, gy, n[0], n[1]);
        return FV_OK;
    }
    return fv_kind_flux(ph->flux, ph->gamma, qi, qj, n, f);
}

int fv_kind_face_gradient(int32_t V, const double* gxi, const double* gyi, const double* gxj, const double* gyj,
                          const double* qi, const double* qj, const double* ci, const double* cj, double* gxf,
                          double* gyf) {
    if (!gxi || !gyi || !gxj || !gyj || !qi || !qj || !ci || !cj || !gxf || !gyf) return FV_ERR_ARG;
    switch (V) {
        case 1: fvgpu::exact::face_gradient<1>(gxf, gyf, gxi, gyi, gxj, gyj, qi, qj, ci[0], ci[1], cj[0], cj[1]); break;
        case 2: fvgpu::exact::face_gradient<2>(gxf, gyf, gxi, gyi, gxj, gyj, qi, qj, ci[0], ci[1], cj[0], cj[1]); break;
        case 4: fvgpu::exact::face_gradient<4>(gxf, gyf, gxi, gyi, gxj, gyj, qi, qj, ci[0], ci[1], cj[0], cj[1]); break;
        default: return FV_ERR_ARG;
    }
    return FV_OK;
}

int fv_kind_output(int32_t kind, double gamma, const double* q, double* out) {
    if (!q || !out) return FV_ERR_ARG;
    const int nc = fvgpu::exact::output_field(kind, gamma, q, out);
    return nc > 0 ? nc : FV_ERR_UNSUPPORTED;
}

int fv_kind_limiter(int32_t kind, double y, double* out) {
    if (!out) return FV_ERR_ARG;
    if (kind < FV_LIM_ZERO || kind > FV_LIM_MINMOD) return FV_ERR_UNSUPPORTED;
    *out = fvgpu::exact::limiter_func(kind, y);
    return FV_OK;
}

int fv_kind_bc(int32_t kind, int32_t V, double gamma, const double* bv, const double* q, const double* n,
               double* b) {
    if (!q || !n || !b || (V != 1 && V != 2 && V != 4)) return FV_ERR_ARG;
    if (kind < FV_BC_COPY || kind > FV_BC_TANGENT) return FV_ERR_UNSUPPORTED;
    if ((kind == FV_BC_INLET_OUTLET || kind == FV_BC_FARFIELD || kind == FV_BC_FARFIELD_B0) && !bv)
        return FV_ERR_ARG;
    fvgpu::Params P;
    memset(&P, 0, sizeof(P));
    P.V = V;
    P.gamma = gamma;
    P.n_groups = 1;
    P.group_bc[0] = kind;
    if (bv) memcpy(P.group_bv, bv, 4 * sizeof(double));
    if (V == 4) fvgpu::exact::bc<4>(P, 0, 0, b, q, n[0], n[1]);
    else if (V == 2) fvgpu::exact::bc<2>(P, 0, 0, b, q, n[0], n[1]);
    else fvgpu::exact::bc<1>(P, 0, 0, b, q, n[0], n[1]);
    return FV_OK;
}

}  // extern "C"
