// Device physics kinds for the FP64 and FP32-bulk modes.
//
// Same mathematics as the reference example code (cited per function) with
// the algebra rearranged for throughput: 1/rho, 1/(sqrt(rho_L)+sqrt(rho_R))
// and 1/c^2 are computed once and reused, products fuse into FMAs.  Results
// differ from the reference at rounding level only.
#pragma once
#include "fv_internal.h"

namespace fvgpu {
namespace fast {

template <class T> __device__ __forceinline__ T rcp(T x);
template <> __device__ __forceinline__ double rcp<double>(double x) { return 1.0 / x; }
// FP32: single MUFU approximations (<= 1 ulp rcp, <= 2 ulp sqrt; ftz)
template <> __device__ __forceinline__ float rcp<float>(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <class T> __device__ __forceinline__ T sqrt_(T x);
template <> __device__ __forceinline__ double sqrt_<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float sqrt_<float>(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <class T> __device__ __forceinline__ T div_(T a, T b);
template <> __device__ __forceinline__ double div_<double>(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float div_<float>(float a, float b) { return a * rcp<float>(b); }
template <class T> __device__ __forceinline__ T tmin(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T tmax(T a, T b) { return (a < b) ? b : a; }

// Roe flux with the "cures" eigenvalues (examples/forwardStep/main.cpp:72-135).
template <class T>
__device__ __forceinline__ void roe(T gamma, T* f, const T* qi, const T* qj, T n0, T n1) {
    const T gm1 = gamma - T(1);
    const T ri = rcp(qi[0]), rj = rcp(qj[0]);
    const T uL = qi[1] * ri, vL = qi[2] * ri, uR = qj[1] * rj, vR = qj[2] * rj;
    const T pL = gm1 * (qi[3] - T(0.5) * (qi[1] * uL + qi[2] * vL));
    const T pR = gm1 * (qj[3] - T(0.5) * (qj[1] * uR + qj[2] * vR));
    const T VL = uL * n0 + vL * n1, VR = uR * n0 + vR * n1;
    f[0] = T(0.5) * (qi[0] * VL + qj[0] * VR);
    f[1] = T(0.5) * (qi[1] * VL + qj[1] * VR + (pL + pR) * n0);
    f[2] = T(0.5) * (qi[2] * VL + qj[2] * VR + (pL + pR) * n1);
    f[3] = T(0.5) * ((qi[3] + pL) * VL + (qj[3] + pR) * VR);
    const T srL = sqrt_(qi[0]), srR = sqrt_(qj[0]);
    const T rho = srL * srR;
    const T w = rcp(srL + srR);
    const T u = (uL * srL + uR * srR) * w;
    const T v = (vL * srL + vR * srR) * w;
    const T h = ((qi[3] + pL) * ri * srL + (qj[3] + pR) * rj * srR) * w;
    const T q2 = u * u + v * v;
    const T c2 = gm1 * (h - T(0.5) * q2);
    const T c = sqrt_(c2);
    const T rc2 = rcp(c2);
    const T V = u * n0 + v * n1;
    const T l1 = fabs(tmin(V - c, VL - c));
    const T l2 = fabs(V);
    const T l5 = fabs(tmax(V + c, VR + c));
    const T dp = pR - pL, dV = VR - VL, rcdV = rho * c * dV;
    const T kF1 = l1 * (dp - rcdV) * (T(0.5) * rc2);
    const T kF0 = l2 * ((qj[0] - qi[0]) - dp * rc2);
    const T kFr = l2 * rho;
    const T kF5 = l5 * (dp + rcdV) * (T(0.5) * rc2);
    f[0] -= T(0.5) * (kF1 + kF0 + kF5);
    f[1] -= T(0.5) * (kF1 * (u - c * n0) + kF0 * u + kFr * (uR - uL - dV * n0) + kF5 * (u + c * n0));
    f[2] -= T(0.5) * (kF1 * (v - c * n1) + kF0 * v + kFr * (vR - vL - dV * n1) + kF5 * (v + c * n1));
    f[3] -= T(0.5) * (kF1 * (h - c * V) + kF0 * q2 * T(0.5) + kFr * (u * (uR - uL) + v * (vR - vL) - V * dV) +
                      kF5 * (h + c * V));
}

// Upwind advection flux (examples/burgers/main.cpp:68-96).
template <class T>
__device__ __forceinline__ void burgers(T* f, const T* qi, const T* qj, T n0, T n1) {
    const T Vi = qi[0] * n0 + qi[1] * n1, Vj = qj[0] * n0 + qj[1] * n1;
    const T V = tmax(fabs(Vi), fabs(Vj));
    f[0] = T(0.5) * (Vi * qi[0] + Vj * qj[0]) - T(0.5) * V * (qj[0] - qi[0]);
    f[1] = T(0.5) * (Vi * qi[1] + Vj * qj[1]) - T(0.5) * V * (qj[1] - qi[1]);
}

template <int FLUX, class T>
__device__ __forceinline__ void flux(T gamma, T* f, const T* qi, const T* qj, T n0, T n1) {
    if (FLUX == 3) burgers(f, qi, qj, n0, n1);
    else roe(gamma, f, qi, qj, n0, n1);
}

// Diffusion flux -grad(u) . n with the corrected face gradient (see
// fv_physics_exact.cuh): one reciprocal of |ci - cj|, and the normal
// component of the correction taken once, (t . n).
template <int V, class T>
__device__ __forceinline__ void diffusion(T* f, const T* gxi, const T* gyi, const T* gxj, const T* gyj, const T* qi,
                                          const T* qj, T t0, T t1, T n0, T n1) {
    const T rl = rcp(sqrt_(t0 * t0 + t1 * t1));
    t0 *= rl;
    t1 *= rl;
    const T tn = t0 * n0 + t1 * n1;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const T bx = T(0.5) * (gxi[k] + gxj[k]), by = T(0.5) * (gyi[k] + gyj[k]);
        const T corr = bx * t0 + by * t1 - (qi[k] - qj[k]) * rl;
        f[k] = -(bx * n0 + by * n1 - corr * tn);
    }
}

// Viscous part of the Navier-Stokes flux (see fv_physics_exact.cuh): the
// gradients of u, v and T at the mean face state from the face gradient,
// with 1/rho taken once.
template <class T>
__device__ __forceinline__ void ns_viscous(const Params& P, T* f, const T* qi, const T* qj, const T* gx,
                                           const T* gy, T n0, T n1) {
    const T gm1 = (T)P.gamma - T(1), mu = (T)P.mu;
    T q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = T(0.5) * (qi[i] + qj[i]);
    const T ri = rcp(q[0]);
    const T u = q[1] * ri, v = q[2] * ri, E = q[3] * ri;
    // d(u), d(v), d(E) = (d(rho x) - x d(rho)) / rho; T = (gamma-1)/r * (E - (u^2+v^2)/2)
    const T gu0 = (gx[1] - u * gx[0]) * ri, gu1 = (gy[1] - u * gy[0]) * ri;
    const T gv0 = (gx[2] - v * gx[0]) * ri, gv1 = (gy[2] - v * gy[0]) * ri;
    const T cT = gm1 * (T)(1.0 / P.r);
    const T gt0 = cT * ((gx[3] - E * gx[0]) * ri - (u * gu0 + v * gv0));
    const T gt1 = cT * ((gy[3] - E * gy[0]) * ri - (u * gu1 + v * gv1));
    const T div3 = (gu0 + gv1) * T(1.0 / 3.0);
    const T tau_xx = T(2) * mu * (gu0 - div3);
    const T tau_yy = T(2) * mu * (gv1 - div3);
    const T tau_xy = mu * (gu1 + gv0);
    const T k = (T)(P.cp * P.mu / P.pr);
    const T phi0 = u * tau_xx + v * tau_xy + k * gt0;
    const T phi1 = u * tau_xy + v * tau_yy + k * gt1;
    f[1] -= n0 * tau_xx + n1 * tau_xy;
    f[2] -= n0 * tau_xy + n1 * tau_yy;
    f[3] -= n0 * phi0 + n1 * phi1;
}

// limiter_func kinds (see fv_physics_exact.cuh for the references).
template <class T>
__device__ __forceinline__ T limiter_func(int kind, T y) {
    if (kind == 1) {  // Michalak, y_t = 2: a = 0, b = -1/4
        return (y >= T(2)) ? T(1) : y - T(0.25) * y * y;
    }
    if (kind == 2) return div_(y * y + T(2) * y, y * y + y + T(2));
    if (kind == 3) return tmax(T(0), tmin(T(1), y));
    return T(0);
}
// phi(num / den) for den != 0.  Venkatakrishnan's phi is a ratio of
// quadratics in y = num / den: multiplied through by den^2 it needs one
// reciprocal, (num^2 + 2 num den) / (num^2 + num den + 2 den^2).
template <class T>
__device__ __forceinline__ T limiter_ratio(int kind, T num, T den) {
    if (kind == 2) return num * (num + T(2) * den) * rcp(num * (num + den) + T(2) * den * den);
    return limiter_func(kind, div_(num, den));
}

// Boundary conditions (see fv_physics_exact.cuh for the references).
template <int V, class T>
__device__ __forceinline__ void bc(const Params& P, int group, int gb, T* b, const T* q, T n0, T n1) {
    const int kind = P.group_bc[group];
    if (kind == 6 && V == 2) {  // TANGENT
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
        const T dn = T(2) * (n0 * q[1] + n1 * q[2]);
        b[0] = q[0]; b[1] = q[1] - n0 * dn; b[2] = q[2] - n1 * dn; b[3] = q[3];
        return;
    }
    if (kind == 4) {
        b[0] = q[0]; b[1] = -q[1]; b[2] = -q[2]; b[3] = q[3];
        return;
    }
    const bool b0 = kind == 5;  // FARFIELD_B0: the tangential momentum's factor is b[0], not b[1]
    const T gamma = (T)P.gamma, gm1 = gamma - T(1);
    const double* bvd = P.ghost_bv ? P.ghost_bv + 4 * (size_t)gb : P.group_bv + 4 * group;
    const T bv[4] = {(T)bvd[0], (T)bvd[1], (T)bvd[2], (T)bvd[3]};
    const T r = rcp(q[0]);
    const T U0 = q[1] * r, U1 = q[2] * r;
    const T u2 = U0 * U0 + U1 * U1;
    const T u_dot_n = U0 * n0 + U1 * n1;
    const T p = gm1 * (q[3] - T(0.5) * q[0] * u2);
    const T c2 = gamma * p * r;
    if (c2 >= T(0) && u2 > c2) {  // |u| / c > 1 (a non-physical state takes the subsonic branch, as in the reference)
        if (u_dot_n < T(0)) { b[0] = bv[0]; b[1] = bv[1]; b[2] = bv[2]; b[3] = bv[3]; }
        else { b[0] = q[0]; b[1] = q[1]; b[2] = q[2]; b[3] = q[3]; }
        return;
    }
    const T c0 = sqrt_(c2);
    const T rbv = rcp(bv[0]);
    const T pa = gm1 * (bv[3] - T(0.5) * rbv * (bv[1] * bv[1] + bv[2] * bv[2]));
    const T ua = bv[1] * rbv, va = bv[2] * rbv;
    const T pd = p, ud = U0, vd = U1, rho0 = q[0];
    // 1/c0^2 from c0 (not c2): a state with p < 0 gives NaN in every
    // component, as the reference's (pb - pd)/(c0*c0) does
    const T rrc = rcp(rho0 * c0), rc2 = rcp(c0 * c0);
    const T rgm1 = rcp(gm1);
    if (u_dot_n < T(0)) {
        if (kind == 2) {
            b[0] = bv[0]; b[1] = bv[1]; b[2] = bv[2];
            b[3] = pd * rgm1 + T(0.5) * rcp(b[0]) * (b[1] * b[1] + b[2] * b[2]);
        } else {
            const T pb = T(0.5) * (pa + pd - rho0 * c0 * (n0 * (ua - ud) + n1 * (va - vd)));
            b[0] = bv[0] + (pb - pa) * rc2;
            b[1] = b[0] * (ua - n0 * (pa - pb) * rrc);
            b[2] = (b0 ? b[0] : b[1]) * (va - n1 * (pa - pb) * rrc);
            b[3] = pb * rgm1 + T(0.5) * rcp(b[0]) * (b[1] * b[1] + b[2] * b[2]);
        }
    } else {
        const T pb = pa;
        b[0] = q[0] + (pb - pd) * rc2;
        b[1] = b[0] * (ud + n0 * (pd - pb) * rrc);
        b[2] = (b0 ? b[0] : b[1]) * (va + n1 * (pd - pb) * rrc);  // b[1] (b[0] for FARFIELD_B0) as in the reference
        b[3] = pb * rgm1 + T(0.5) * rcp(b[0]) * (b[1] * b[1] + b[2] * b[2]);
    }
}

}  // namespace fast
}  // namespace fvgpu
