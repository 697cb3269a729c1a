// Device physics kinds in the reference's exact evaluation order.
//
// Compiled with -fmad=false (device) and -ffp-contract=off (host): every
// expression below is evaluated with the same operations, operand order,
// IEEE divisions and square roots as the reference example code it cites, so
// the FP64 results are bit-identical to the reference CPU solver.  The same
// functions run on the host (fv_kinds.cu), where the fvhyper shim uses them to
// match a user's physics functions to a device kind.
#pragma once
#include <math.h>
#include "fv_internal.h"

#ifndef FV_HD
#define FV_HD __host__ __device__ __forceinline__
#endif

namespace fvgpu {
namespace exact {

FV_HD double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
FV_HD double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

// Roe flux with the "cures" eigenvalue modification.
// FS_ASSOC: examples/forwardStep/main.cpp:72-135 (central flux as one sum);
// otherwise examples/shockTube/main.cpp:68-135 = examples/naca/main.cpp:71-137.
// T: double, or a forward-mode dual number (the adjoint's element Jacobians).
template <bool FS_ASSOC, class T>
FV_HD void roe(double gamma, T* f, const T* qi, const T* qj, double n0, double n1) {
    const T pi = (gamma - 1) * (qi[3] - 0.5 / qi[0] * (qi[1] * qi[1] + qi[2] * qi[2]));
    const T pj = (gamma - 1) * (qj[3] - 0.5 / qj[0] * (qj[1] * qj[1] + qj[2] * qj[2]));
    const T Vi = (qi[1] * n0 + qi[2] * n1) / qi[0];
    const T Vj = (qj[1] * n0 + qj[2] * n1) / qj[0];
    if (FS_ASSOC) {
        f[0] = (qi[0] * Vi + qj[0] * Vj) * 0.5;
        f[1] = (qi[1] * Vi + pi * n0 + qj[1] * Vj + pj * n0) * 0.5;
        f[2] = (qi[2] * Vi + pi * n1 + qj[2] * Vj + pj * n1) * 0.5;
        f[3] = ((qi[3] + pi) * Vi + (qj[3] + pj) * Vj) * 0.5;
    } else {
        f[0] = qi[0] * Vi;
        f[1] = qi[1] * Vi + pi * n0;
        f[2] = qi[2] * Vi + pi * n1;
        f[3] = (qi[3] + pi) * Vi;
        f[0] += qj[0] * Vj;
        f[1] += qj[1] * Vj + pj * n0;
        f[2] += qj[2] * Vj + pj * n1;
        f[3] += (qj[3] + pj) * Vj;
#pragma unroll
        for (int i = 0; i < 4; ++i) f[i] *= 0.5;
    }
    const T pL = pi, pR = pj;
    const T uL = qi[1] / qi[0], vL = qi[2] / qi[0];
    const T uR = qj[1] / qj[0], vR = qj[2] / qj[0];
    const T srhoL = sqrt(qi[0]), srhoR = sqrt(qj[0]);
    const T rho = srhoR * srhoL;
    const T u = (uL * srhoL + uR * srhoR) / (srhoL + srhoR);
    const T v = (vL * srhoL + vR * srhoR) / (srhoL + srhoR);
    const T h = ((qi[3] + pL) / qi[0] * srhoL + (qj[3] + pR) / qj[0] * srhoR) / (srhoL + srhoR);
    const T q2 = u * u + v * v;
    const T c = sqrt((gamma - 1.) * (h - 0.5 * q2));
    const T V = u * n0 + v * n1;
    const T VR = uR * n0 + vR * n1;
    const T VL = uL * n0 + vL * n1;
    const T lambda_cm = fabs(dmin(V - c, VL - c));
    const T lambda_c = fabs(V);
    const T lambda_cp = fabs(dmax(V + c, VR + c));
    const T kF1 = lambda_cm * ((pR - pL) - rho * c * (VR - VL)) / (2. * c * c);
    const T kF234_0 = lambda_c * ((qj[0] - qi[0]) - (pR - pL) / (c * c));
    const T kF234_1 = lambda_c * rho;
    const T kF5 = lambda_cp * ((pR - pL) + rho * c * (VR - VL)) / (2. * c * c);
    f[0] -= 0.5 * (kF1 + kF234_0 + kF5);
    f[1] -= 0.5 * (kF1 * (u - c * n0) + kF234_0 * u + kF234_1 * (uR - uL - (VR - VL) * n0) + kF5 * (u + c * n0));
    f[2] -= 0.5 * (kF1 * (v - c * n1) + kF234_0 * v + kF234_1 * (vR - vL - (VR - VL) * n1) + kF5 * (v + c * n1));
    f[3] -= 0.5 * (kF1 * (h - c * V) + kF234_0 * q2 * 0.5 + kF234_1 * (u * (uR - uL) + v * (vR - vL) - V * (VR - VL)) + kF5 * (h + c * V));
}

// Upwind advection flux, examples/burgers/main.cpp:68-96.
FV_HD void burgers(double* f, const double* qi, const double* qj, double n0, double n1) {
    const double Vi = qi[0] * n0 + qi[1] * n1;
    const double Vj = qj[0] * n0 + qj[1] * n1;
    const double fi0 = Vi * qi[0], fi1 = Vi * qi[1];
    const double fj0 = Vj * qj[0], fj1 = Vj * qj[1];
    const double V = dmax(fabs(Vi), fabs(Vj));
    f[0] = 0.5 * (fi0 + fj0) - 0.5 * V * (qj[0] - qi[0]);
    f[1] = 0.5 * (fi1 + fj1) - 0.5 * V * (qj[1] - qi[1]);
}

template <int FLUX>
FV_HD void flux(double gamma, double* f, const double* qi, const double* qj,
                                     double n0, double n1) {
    if (FLUX == 3) burgers(f, qi, qj, n0, n1);
    else roe<FLUX == 1>(gamma, f, qi, qj, n0, n1);
}

// Face gradient of the diffusive fluxes (gradient_for_diffusion,
// explicit.cpp:70-109): the mean of the two cell gradients, with its
// component along the centroid line ci - cj replaced by the difference
// quotient of the two cell states.
template <int V>
FV_HD void face_gradient(double* gxf, double* gyf, const double* gxi, const double* gyi, const double* gxj,
                         const double* gyj, const double* qi, const double* qj, double cix, double ciy, double cjx,
                         double cjy) {
    double t0 = cix - cjx, t1 = ciy - cjy;
    const double lij = sqrt(t0 * t0 + t1 * t1);
    t0 = t0 / lij;
    t1 = t1 / lij;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const double dir = (qi[k] - qj[k]) / lij;
        const double bx = (gxi[k] + gxj[k]) * 0.5, by = (gyi[k] + gyj[k]) * 0.5;
        const double dot = bx * t0 + by * t1;
        gxf[k] = bx - (dot - dir) * t0;
        gyf[k] = by - (dot - dir) * t1;
    }
}

// Diffusion flux F = -grad(u) . n of the face gradient
// (examples/heatTransfer/main.cpp:63-73, V = 1).
FV_HD void diffusion(double* f, const double* gxf, const double* gyf, double n0, double n1) {
    f[0] = -(gxf[0] * n0 + gyf[0] * n1);
}

// Viscous part of the Navier-Stokes flux (examples/flatPlate/main.cpp:193-224
// with calc_p, calc_grad_p, calc_grad_t, calc_grad_u, calc_grad_v of
// :38-92): stresses and heat flux at the mean of the face states qi, qj from
// the face gradient (gx, gy), subtracted from f (the roe<false> flux).
FV_HD void ns_viscous(const Params& P, double* f, const double* qi, const double* qj, const double* gx,
                      const double* gy, double n0, double n1) {
    const double gamma = P.gamma, mu = P.mu;
    double q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = 0.5 * (qi[i] + qj[i]);
    const double p = (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
    double gp0 = 2. * gx[3];
    gp0 -= gx[1] * q[1] / q[0] + q[1] * (gx[1] * q[0] - gx[0] * q[1]) / (q[0] * q[0]);
    gp0 -= gx[2] * q[2] / q[0] + q[2] * (gx[2] * q[0] - gx[0] * q[2]) / (q[0] * q[0]);
    gp0 *= 0.5 * (gamma - 1);
    double gp1 = 2. * gy[3];
    gp1 -= gy[1] * q[1] / q[0] + q[1] * (gy[1] * q[0] - gy[0] * q[1]) / (q[0] * q[0]);
    gp1 -= gy[2] * q[2] / q[0] + q[2] * (gy[2] * q[0] - gy[0] * q[2]) / (q[0] * q[0]);
    gp1 *= 0.5 * (gamma - 1);
    const double gt0 = (1. / P.r) * ((gp0 * q[0] - gx[0] * p) / (q[0] * q[0]));
    const double gt1 = (1. / P.r) * ((gp1 * q[0] - gy[0] * p) / (q[0] * q[0]));
    const double gu0 = (q[0] * gx[1] - q[1] * gx[0]) / (q[0] * q[0]);
    const double gu1 = (q[0] * gy[1] - q[1] * gy[0]) / (q[0] * q[0]);
    const double gv0 = (q[0] * gx[2] - q[2] * gx[0]) / (q[0] * q[0]);
    const double gv1 = (q[0] * gy[2] - q[2] * gy[0]) / (q[0] * q[0]);
    const double div_v = gu0 + gv1;
    const double tau_xx = 2. * mu * (gu0 - div_v / 3.);
    const double tau_yy = 2. * mu * (gv1 - div_v / 3.);
    const double tau_xy = mu * (gu1 + gv0);
    const double k = P.cp * mu / P.pr;
    const double phi0 = q[1] / q[0] * tau_xx + q[2] / q[0] * tau_xy + k * gt0;
    const double phi1 = q[1] / q[0] * tau_xy + q[2] / q[0] * tau_yy + k * gt1;
    f[1] -= n0 * tau_xx + n1 * tau_xy;
    f[2] -= n0 * tau_xy + n1 * tau_yy;
    f[3] -= n0 * phi0 + n1 * phi1;
}

// Regression-test physics (tests/tests.cpp:94-116): the upwind advection flux
// plus -(grad q . n) of the face gradient per variable.
FV_HD void burgers_diffusion(double* f, const double* qi, const double* qj, const double* gx, const double* gy,
                             double n0, double n1) {
    burgers(f, qi, qj, n0, n1);
    f[0] += -(gx[0] * n0 + gy[0] * n1);
    f[1] += -(gx[1] * n0 + gy[1] * n1);
}

// Viscous eigenvalue of the viscous time steps, max(4/(3 rho), gamma/rho) *
// (mu/pr) * le^2 / A (flatPlate/main.cpp:264-267).
FV_HD double visc_eig(const Params& P, double rho, double le, double A) {
    return dmax(4. / (3. * rho), P.gamma / rho) * (P.mu / P.pr) * le * le / A;
}

// Extra output fields of the examples' post:: callbacks (post.h:24-30), in
// their evaluation order: 1 pressure (examples/forwardStep/main.cpp:37-39,
// 289-292; shockTube/main.cpp:181-184), 2 Mach number (forwardStep/main.cpp:
// 293-299), 3 velocity (forwardStep/main.cpp:283-287), 4 the first two state
// components (burgers/main.cpp:133-137).  Returns the number of components.
FV_HD int output_field(int kind, double gamma, const double* q, double* out) {
    if (kind == 1) {
        out[0] = (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
        return 1;
    }
    if (kind == 2) {
        const double p = (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
        const double c = sqrt(gamma * p / q[0]);
        const double unorm = sqrt(q[1] * q[1] + q[2] * q[2]) / q[0];
        out[0] = unorm / c;
        return 1;
    }
    if (kind == 3) {
        out[0] = q[1] / q[0];
        out[1] = q[2] / q[0];
        return 2;
    }
    if (kind == 4) {
        out[0] = q[0];
        out[1] = q[1];
        return 2;
    }
    return 0;
}

// Limiter functions phi (limiter_func).  ZERO: shockTube/main.cpp:60-62.
// MICHALAK (y_t = 2): forwardStep/main.cpp:57-66.  MINMOD: burgers/main.cpp:
// 51-53.  VENKAT: (y^2 + 2y)/(y^2 + y + 2), Venkatakrishnan (1995).
FV_HD double limiter_func(int kind, double y) {
    if (kind == 1) {
        const double yt = 2.0;
        if (y >= yt) return 1.0;
        const double a = 1.0 / (yt * yt) - 2.0 / (yt * yt * yt);
        const double b = -3.0 / 2.0 * a * yt - 0.5 / yt;
        return a * y * y * y + b * y * y + y;
    }
    if (kind == 2) return (y * y + 2.0 * y) / (y * y + y + 2.0);
    if (kind == 3) return dmax(0., dmin(1., y));
    return 0.;
}

// Boundary conditions (boundaries::bounds entries).  COPY: shockTube/main.cpp:
// 158-163.  WALL: forwardStep/main.cpp:262-269.  INLET_OUTLET: forwardStep/
// main.cpp:194-261.  FARFIELD: naca/main.cpp:192-259.  Subsonic outlets keep
// the reference's b[2] = b[1]*(...).  NOSLIP: flatPlate/main.cpp:361-366.
// FARFIELD_B0: flatPlate/main.cpp:286-352, FARFIELD with b[2] = b[0]*(...).
// TANGENT (V = 2): tests/tests.cpp:132-135.
template <int V, class T>
FV_HD void bc_state(int kind, double gamma, const T* bv, T* b, const T* q, double n0, double n1) {
    if (kind == 6 && V == 2) {  // TANGENT, tests/tests.cpp:132-135
        b[0] = -n1;
        b[1] = n0;
        return;
    }
    if (kind == 0 || V != 4) {
#pragma unroll
        for (int k = 0; k < V; ++k) b[k] = q[k];
        return;
    }
    if (kind == 1) {
        b[0] = q[0];
        b[1] = q[1] - 2.0 * n0 * (n0 * q[1] + n1 * q[2]);
        b[2] = q[2] - 2.0 * n1 * (n0 * q[1] + n1 * q[2]);
        b[3] = q[3];
        return;
    }
    if (kind == 4) {
        b[0] = q[0]; b[1] = -q[1]; b[2] = -q[2]; b[3] = q[3];
        return;
    }
    const bool b0 = kind == 5;  // FARFIELD_B0: the tangential momentum's factor is b[0], not b[1]
    const T U0 = q[1] / q[0], U1 = q[2] / q[0];
    const T u_norm = sqrt(U0 * U0 + U1 * U1);
    const T u_dot_n = U0 * n0 + U1 * n1;
    const T p = (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
    const T c = sqrt(gamma * p / q[0]);
    const T mach = u_norm / c;
    if (mach > 1) {
        if (u_dot_n < 0) {
            b[0] = bv[0]; b[1] = bv[1]; b[2] = bv[2]; b[3] = bv[3];
        } else {
            b[0] = q[0]; b[1] = q[1]; b[2] = q[2]; b[3] = q[3];
        }
        return;
    }
    const T pa = (gamma - 1) * (bv[3] - 0.5 / bv[0] * (bv[1] * bv[1] + bv[2] * bv[2]));
    const T rhoa = bv[0], ua = bv[1] / bv[0], va = bv[2] / bv[0];
    const T pd = p, rhod = q[0], ud = q[1] / q[0], vd = q[2] / q[0];
    const T rho0 = q[0], c0 = c;
    if (u_dot_n < 0) {
        if (kind == 2) {
            const T pb = pd;
            b[0] = bv[0]; b[1] = bv[1]; b[2] = bv[2];
            b[3] = pb / (gamma - 1.) + 0.5 / b[0] * (b[1] * b[1] + b[2] * b[2]);
        } else {
            const T pb = 0.5 * (pa + pd - rho0 * c0 * (n0 * (ua - ud) + n1 * (va - vd)));
            b[0] = rhoa + (pb - pa) / (c0 * c0);
            b[1] = b[0] * (ua - n0 * (pa - pb) / (rho0 * c0));
            b[2] = (b0 ? b[0] : b[1]) * (va - n1 * (pa - pb) / (rho0 * c0));
            b[3] = pb / (gamma - 1) + 0.5 / b[0] * (b[1] * b[1] + b[2] * b[2]);
        }
    } else {
        const T pb = pa;
        b[0] = rhod + (pb - pd) / (c0 * c0);
        b[1] = b[0] * (ud + n0 * (pd - pb) / (rho0 * c0));
        b[2] = (b0 ? b[0] : b[1]) * (va + n1 * (pd - pb) / (rho0 * c0));
        b[3] = pb / (gamma - 1.) + 0.5 / b[0] * (b[1] * b[1] + b[2] * b[2]);
    }
}

// Ghost gb of boundary group `group`: the group's boundary kind, with the
// ghost's own boundary state when a per-ghost inflow is set (P.ghost_bv).
template <int V>
FV_HD void bc(const Params& P, int group, int gb, double* b, const double* q, double n0, double n1) {
    const double* bv = P.ghost_bv ? P.ghost_bv + 4 * (size_t)gb : P.group_bv + 4 * group;
    bc_state<V>(P.group_bc[group], P.gamma, bv, b, q, n0, n1);
}

// Pressure, forwardStep/main.cpp:37-39.
FV_HD double pres(double gamma, const double* q) {
    return (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
}

}  // namespace exact
}  // namespace fvgpu
