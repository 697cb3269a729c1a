// Discrete adjoint kernels of the explicit step (FP64, Euler, V = 4).
//
// Each kernel owns the cells it writes (one thread per real cell, which also
// owns its boundary ghosts; the gradient kernel one thread per real cell and
// variable) and gathers what flows into them, so results do not depend on
// scheduling.  Element Jacobians come from the primal element functions of
// fv_physics_exact.cuh evaluated on dual numbers (fv_dual.cuh): Dual<4>
// seeded on one stencil cell's 4 conserved variables for the flux, boundary
// and time-step functions, a scalar dual seeded on one variable for the
// gradient + limiter, which is block-diagonal over the variables; the linear parts
// (MUSCL reconstruction, RK update, Green-Gauss sums) are differentiated by
// hand.  Reference arithmetic followed: gradients explicit.cpp:112-171,
// limiters 174-258, MUSCL + flux 261-364, update 368-378, ghost fill
// 380-417, min_dt 555-564; Roe flux examples/forwardStep/main.cpp:72-135;
// CFL time step forwardStep/main.cpp:140-185.
#include <algorithm>

#include "fv_adjoint.h"
#include "fv_dual.cuh"
#include "fv_physics_exact.cuh"

namespace fvgpu {
namespace {

using D4 = Dual<4>;
using D1 = Dual<1>;
constexpr int kAB = 128;  // threads per block
constexpr int kFaces = 4;
constexpr uint32_t kNone = 0xFFFFFFFFu;

__device__ __forceinline__ void ld4(const double* __restrict__ a, int c, double* v) {
    const double2* p = reinterpret_cast<const double2*>(a + 4 * (size_t)c);
    const double2 x = p[0], y = p[1];
    v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
__device__ __forceinline__ void st4(double* a, int c, const double* v) {
    double2* p = reinterpret_cast<double2*>(a + 4 * (size_t)c);
    p[0] = make_double2(v[0], v[1]);
    p[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void add4(double* a, int c, const double* v) {
    double w[4];
    ld4(a, c, w);
    for (int k = 0; k < 4; ++k) w[k] += v[k];
    st4(a, c, w);
}
__device__ __forceinline__ void seed(D4* x, const double* v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) { x[k] = D4(v[k]); x[k].d[k] = 1.0; }
}
__device__ __forceinline__ void constant(D4* x, const double* v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = D4(v[k]);
}
// out[m] = sum_k lam[k] * y[k].d[m]  (J^T lam)
__device__ __forceinline__ void jt(const D4* y, const double* lam, double* out) {
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) s += lam[k] * y[k].d[m];
        out[m] = s;
    }
}

// MUSCL face state q + (g . d) lim with the positivity guard (returns true
// when the guard replaced it by the cell value)
__device__ __forceinline__ bool recon(const Params& P, const double* q, const double* gx, const double* gy,
                                      const double* lim, double dx, double dy, double* out) {
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = q[k] + (gx[k] * dx + gy[k] * dy) * lim[k];
    if (!P.positivity_guard) return false;
    const double p = (P.gamma - 1.0) * (out[3] - 0.5 / out[0] * (out[1] * out[1] + out[2] * out[2]));
    if (!(out[0] > 0.0) || !(p > 0.0)) {
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = q[k];
        return true;
    }
    return false;
}

__device__ __forceinline__ void flux_d(const Params& P, D4* f, const D4* a, const D4* b, double n0, double n1) {
    if (P.flux == 1) exact::roe<true>(P.gamma, f, a, b, n0, n1);
    else exact::roe<false>(P.gamma, f, a, b, n0, n1);
}

template <class T>
__device__ __forceinline__ T limiter_t(int kind, const T& y) {
    if (kind == 1) {  // Michalak, y_t = 2
        const double yt = 2.0;
        if (y >= yt) return T(1.0);
        const double a = 1.0 / (yt * yt) - 2.0 / (yt * yt * yt);
        const double b = -3.0 / 2.0 * a * yt - 0.5 / yt;
        return a * y * y * y + b * y * y + y;
    }
    if (kind == 2) return (y * y + 2.0 * y) / (y * y + y + 2.0);
    if (kind == 3) return dmax(T(0.), dmin(T(1.), y));
    return T(0.);
}

// Gradient + limiter of variable k of real cell c: the operator is
// block-diagonal over the conserved variables (variable k's Green-Gauss
// gradient, min/max and limiter read only variable k of the stencil), so one
// scalar dual seeded on variable k of one stencil cell gives the nonzero
// entries of the cell's Jacobian block (calc_gradients + calc_limiters,
// explicit.cpp:112-258).
__device__ void gradlim_d1(const Params& P, const AdjFaces& F, const double* __restrict__ qs, int c, int seed_slot,
                           int k, D1& gx, D1& gy, D1& lim) {
    const int N = P.n_real;
    D1 q(qs[4 * (size_t)c + k]);
    if (seed_slot < 0) q.d[0] = 1.0;
    gx = D1(0.0); gy = D1(0.0);
    D1 qmn = q, qmx = q;
    for (int f = 0; f < kFaces; ++f) {
        const size_t s = (size_t)f * N + c;
        const uint32_t w = F.nbr[s];
        if (w == kNone) continue;
        const int j = (int)(w & 0x7FFFFFFFu), side = (int)(w >> 31);
        const double nx = F.nx[s], ny = F.ny[s], le = F.le[s], g = F.g[s];
        D1 qn(qs[4 * (size_t)j + k]);
        if (f == seed_slot) qn.d[0] = 1.0;
        if (!side) {
            const D1 fl = (q * (1.0 - g) + qn * g) * le;
            gx += fl * nx; gy += fl * ny;
        } else {
            const D1 fl = (qn * (1.0 - g) + q * g) * le;
            gx -= fl * nx; gy -= fl * ny;
        }
        qmn = dmin(qmn, qn); qmx = dmax(qmx, qn);
    }
    const double A = F.area[c];
    const double invA = 1. / A;
    gx *= invA; gy *= invA; lim = D1(1.0);
    const double Ka = P.K * sqrt(A);
    const double K3a = Ka * Ka * Ka;
    const double tol = 1e-15;
    for (int f = 0; f < kFaces; ++f) {
        const size_t s = (size_t)f * N + c;
        if (F.nbr[s] == kNone) continue;
        const double dx = F.dsx[s], dy = F.dsy[s];
        const D1 dqg = gx * dx + gy * dy;
        const D1 delta_max = qmx - q;
        const D1 delta_min = qmn - q;
        const D1 d2 = (delta_max - delta_min) * (delta_max - delta_min);
        D1 sig;
        if (d2 <= K3a) sig = D1(1.);
        else if (d2 <= 2 * K3a) {
            const D1 y = (d2 / K3a - 1.0);
            sig = 2.0 * y * y * y - 3.0 * y * y + 1.0;
        } else sig = D1(0.);
        D1 lv(1.0);
        if (sig < 1.0) {
            if (dqg > tol) lv = limiter_t(P.limiter, delta_max / dqg);
            else if (dqg < -tol) lv = limiter_t(P.limiter, delta_min / dqg);
        }
        lv = sig + (1.0 - sig) * lv;
        lim = dmin(lim, lv);
    }
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAB) k_adj_ghosts(Params P, AdjFaces F, AdjStage S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.n_real;
    if (i >= N) return;
    const bool rec = P.order2 && !S.zero_grad;
    double qi[4], gxi[4] = {0, 0, 0, 0}, gyi[4] = {0, 0, 0, 0}, limi[4] = {0, 0, 0, 0};
    ld4(S.qs1, i, qi);
    if (rec) { ld4(S.gx, i, gxi); ld4(S.gy, i, gyi); ld4(S.lim, i, limi); }
    double aq[4] = {0, 0, 0, 0}, agx[4] = {0, 0, 0, 0}, agy[4] = {0, 0, 0, 0}, alim[4] = {0, 0, 0, 0};
    bool any = false;
    for (int f = 0; f < kFaces; ++f) {
        const uint32_t w = F.nbr[(size_t)f * N + i];
        if (w == kNone) continue;
        const int j = (int)(w & 0x7FFFFFFFu);
        if (j < N) continue;
        any = true;
        const int gb = j - N;
        double lb[4];
        ld4(S.lam_next, j, lb);
        const double dx = P.g_dx[gb], dy = P.g_dy[gb], n0 = P.g_nx[gb], n1 = P.g_ny[gb];
        double x[4];
        bool guarded = false;
        if (rec) guarded = recon(P, qi, gxi, gyi, limi, dx, dy, x);
        else for (int k = 0; k < 4; ++k) x[k] = qi[k];
        const int group = P.ghost_group[gb];
        const int kind = P.group_bc[group];
        const double* bv = P.ghost_bv ? P.ghost_bv + 4 * (size_t)gb : P.group_bv + 4 * group;
        D4 xd[4], bvd[4], bd[4];
        seed(xd, x);
        constant(bvd, bv);
        exact::bc_state<4>(kind, P.gamma, bvd, bd, xd, n0, n1);
        double lx[4];
        jt(bd, lb, lx);
        if (kind == 2 || kind == 3 || kind == 5) {  // boundary state of an inflow / far-field ghost
            constant(xd, x);
            seed(bvd, bv);
            exact::bc_state<4>(kind, P.gamma, bvd, bd, xd, n0, n1);
            double lbv[4];
            jt(bd, lb, lbv);
            add4(S.lam_bv, gb, lbv);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            aq[m] += lx[m];
            if (rec && !guarded) {
                agx[m] += lx[m] * dx * limi[m];
                agy[m] += lx[m] * dy * limi[m];
                alim[m] += lx[m] * (gxi[m] * dx + gyi[m] * dy);
            }
        }
    }
    if (any) add4(S.lam_next, i, aq);
    if (S.lam_gx) { st4(S.lam_gx, i, agx); st4(S.lam_gy, i, agy); st4(S.lam_lim, i, alim); }
}

__global__ void __launch_bounds__(kAB) k_adj_residual(Params P, AdjFaces F, AdjStage S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.n_real;
    double dsum = 0.0;
    if (i < N) {
        const bool o2 = P.order2 != 0;
        double qi[4], gxi[4] = {0, 0, 0, 0}, gyi[4] = {0, 0, 0, 0}, limi[4] = {0, 0, 0, 0};
        ld4(S.qs, i, qi);
        if (o2) { ld4(S.gx, i, gxi); ld4(S.gy, i, gyi); ld4(S.lim, i, limi); }
        double ln[4], lqt[4];
        ld4(S.lam_next, i, ln);
        const double ad = S.alpha * S.dt;
#pragma unroll
        for (int k = 0; k < 4; ++k) lqt[k] = ad * ln[k];
        const double Ai = F.area[i];
        double oq[4] = {0, 0, 0, 0}, ogx[4] = {0, 0, 0, 0}, ogy[4] = {0, 0, 0, 0}, olim[4] = {0, 0, 0, 0};
        double qt[4] = {0, 0, 0, 0};
        for (int f = 0; f < kFaces; ++f) {
            const size_t s = (size_t)f * N + i;
            const uint32_t w = F.nbr[s];
            if (w == kNone) continue;
            const int j = (int)(w & 0x7FFFFFFFu), side = (int)(w >> 31);
            const double n0 = F.nx[s], n1 = F.ny[s], le = F.le[s];
            double qj[4], xi[4], xj[4];
            ld4(S.qs, j, qj);
            bool gi = false;
            if (o2) {
                gi = recon(P, qi, gxi, gyi, limi, F.dsx[s], F.dsy[s], xi);
                if (j < N) {
                    double gxj[4], gyj[4], limj[4];
                    ld4(S.gx, j, gxj); ld4(S.gy, j, gyj); ld4(S.lim, j, limj);
                    recon(P, qj, gxj, gyj, limj, F.dnx[s], F.dny[s], xj);
                } else {
                    for (int k = 0; k < 4; ++k) xj[k] = qj[k];  // ghosts: zero gradient
                }
            } else {
                for (int k = 0; k < 4; ++k) { xi[k] = qi[k]; xj[k] = qj[k]; }
            }
            // dL/dF: qt_left -= F le / A_left, qt_right += F le / A_right
            const double si = side ? 1.0 : -1.0;
            double lF[4];
            if (j < N) {
                double lnj[4];
                ld4(S.lam_next, j, lnj);
                const double Aj = F.area[j];
#pragma unroll
                for (int k = 0; k < 4; ++k) lF[k] = le * (si * lqt[k] / Ai - si * ad * lnj[k] / Aj);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) lF[k] = le * (si * lqt[k] / Ai);
            }
            D4 a[4], b[4], fd[4];
            if (!side) { seed(a, xi); constant(b, xj); } else { constant(a, xj); seed(b, xi); }
            flux_d(P, fd, a, b, n0, n1);
#pragma unroll
            for (int k = 0; k < 4; ++k) qt[k] += si * fd[k].v * le / Ai;
            double lx[4];
            jt(fd, lF, lx);
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                oq[m] += lx[m];
                if (o2 && !gi) {
                    ogx[m] += lx[m] * F.dsx[s] * limi[m];
                    ogy[m] += lx[m] * F.dsy[s] * limi[m];
                    olim[m] += lx[m] * (gxi[m] * F.dsx[s] + gyi[m] * F.dsy[s]);
                }
            }
            if (j >= N) {  // the ghost's own adjoint (this cell owns it)
                if (!side) { constant(a, xi); seed(b, xj); } else { seed(a, xj); constant(b, xi); }
                flux_d(P, fd, a, b, n0, n1);
                double lg[4];
                jt(fd, lF, lg);
                st4(S.lam_cur, j, lg);
            }
        }
        st4(S.lam_cur, i, oq);
        if (o2) { add4(S.lam_gx, i, ogx); add4(S.lam_gy, i, ogy); add4(S.lam_lim, i, olim); }
        add4(S.lam_qn, i, ln);
#pragma unroll
        for (int k = 0; k < 4; ++k) dsum += S.alpha * ln[k] * qt[k];
    }
    if (S.dt_partials) {
        __shared__ double red[kAB];
        red[threadIdx.x] = dsum;
        __syncthreads();
        for (int w = kAB / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) S.dt_partials[blockIdx.x] = red[0];
    }
}

// lam_cur += (d g_k / d qs_k)^T lam_g, one thread per (real cell, variable):
// variable k of cell m gathers from its own gradient and limiter and from
// those of its face neighbours (scalar duals, gradlim_d1).
__global__ void __launch_bounds__(kAB) k_adj_gradlim1(Params P, AdjFaces F, AdjStage S) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.n_real;
    const int m = t >> 2, k = t & 3;
    if (m >= N) return;
    D1 gx, gy, lim;
    auto contribute = [&](int c, int seed_slot) {
        gradlim_d1(P, F, S.qs, c, seed_slot, k, gx, gy, lim);
        const size_t i = 4 * (size_t)c + k;
        return S.lam_gx[i] * gx.d[0] + S.lam_gy[i] * gy.d[0] + S.lam_lim[i] * lim.d[0];
    };
    double acc = contribute(m, -1);
    for (int f = 0; f < kFaces; ++f) {
        const uint32_t w = F.nbr[(size_t)f * N + m];
        if (w == kNone) continue;
        const int c = (int)(w & 0x7FFFFFFFu);
        if (c < N) {
            // m in the stencil of its neighbour c: find m's slot among c's faces
            for (int h = 0; h < kFaces; ++h) {
                const uint32_t wc = F.nbr[(size_t)h * N + c];
                if (wc != kNone && (int)(wc & 0x7FFFFFFFu) == m) { acc += contribute(c, h); break; }
            }
        } else {
            // ghost neighbour: only this cell's gradients and limiter use it
            S.lam_cur[4 * (size_t)c + k] += contribute(m, f);
        }
    }
    S.lam_cur[4 * (size_t)m + k] += acc;
}

__global__ void k_add(double* y, const double* x, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] += x[i];
}

// out = sum of p[0..n) in a fixed order: each of the block's threads sums a
// contiguous run, then a fixed tree over the threads.
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_sum(const double* p, int n, double* out) {
    __shared__ double red[kSumThreads];
    const int per = (n + kSumThreads - 1) / kSumThreads;
    const int a = threadIdx.x * per, b = min(n, a + per);
    double s = 0.0;
    for (int i = a; i < b; ++i) s += p[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

__device__ __forceinline__ double key_inv(unsigned long long k) {
    if (k == ~0ull) return __longlong_as_double(0x7ff8000000000000ll);
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__global__ void k_dt_finalize(const unsigned long long* keys, const double* dt_cells, int cell0, double* dt_fill,
                              int n, double* dt_out) {
    unsigned long long key = ~0ull;
    for (int i = 0; i < 64; ++i) key = keys[i] < key ? keys[i] : key;
    const double d0 = dt_cells[cell0];
    const double mn = (d0 != d0) ? d0 : key_inv(key);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dt_fill[i] = mn;
    if (blockIdx.x == 0 && threadIdx.x == 0) *dt_out = mn;
}

__global__ void k_argmin(const double* dt_cells, int n, const double* dt_n, int* argmin) {
    const double v = *dt_n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (dt_cells[i] == v) atomicMin(argmin, i);
}

// CFL time step of cell a (forwardStep calc_dt kind) with one stencil cell seeded
__device__ D4 dt_cell_d(const Params& P, const AdjFaces& F, const double* q, int a, int seed_cell) {
    const int N = P.n_real;
    const double gamma = P.gamma, gm1 = gamma - 1, cfl = P.cfl;
    auto load = [&](int c, D4* x) {
        double v[4];
        ld4(q, c, v);
        if (c == seed_cell) seed(x, v); else constant(x, v);
    };
    auto sound = [&](const D4* x) {
        return sqrt((gm1 * (x[3] - 0.5 / x[0] * (x[1] * x[1] + x[2] * x[2]))) * gamma / x[0]);
    };
    if (a >= N) {  // ghost: its one face to the interior cell
        const int gb = a - N, i = P.ghost_cell[gb];
        D4 qs[4], qn[4];
        load(i, qs); load(a, qn);
        const double n0 = P.g_nx[gb], n1 = P.g_ny[gb], le = P.g_le[gb];
        const D4 es = sound(qs) + fabs(qs[1] / qs[0] * n0 + qs[2] / qs[0] * n1);
        const D4 en = sound(qn) + fabs(qn[1] / qn[0] * n0 + qn[2] / qn[0] * n1);
        const D4 center = dmax(es, en);
        return cfl * F.area[a] / (center * le);
    }
    D4 qs[4];
    load(a, qs);
    const D4 cs = sound(qs);
    D4 acc(0.0);
    for (int f = 0; f < kFaces; ++f) {
        const size_t s = (size_t)f * N + a;
        const uint32_t w = F.nbr[s];
        if (w == kNone) continue;
        const int j = (int)(w & 0x7FFFFFFFu), side = (int)(w >> 31);
        const double n0 = F.nx[s], n1 = F.ny[s], le = F.le[s];
        D4 qn[4];
        load(j, qn);
        const D4 es = cs + fabs(qs[1] / qs[0] * n0 + qs[2] / qs[0] * n1);
        const D4 en = sound(qn) + fabs(qn[1] / qn[0] * n0 + qn[2] / qn[0] * n1);
        const D4 center = side ? dmax(en, es) : dmax(es, en);
        acc += center * le;
    }
    return cfl * F.area[a] / acc;
}

__global__ void k_adj_dt(Params P, AdjFaces F, const double* q, const double* lam_dt, const int* argmin,
                         double* lam_q) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int a = *argmin;
    const int N = P.n_real;
    if (a < 0 || a >= P.n_total) return;
    const double ld = *lam_dt;
    auto push = [&](int c) {
        const D4 d = dt_cell_d(P, F, q, a, c);
        double g[4];
        for (int k = 0; k < 4; ++k) g[k] = ld * d.d[k];
        add4(lam_q, c, g);
    };
    if (a >= N) {
        push(P.ghost_cell[a - N]);
        push(a);
        return;
    }
    push(a);
    for (int f = 0; f < kFaces; ++f) {
        const uint32_t w = F.nbr[(size_t)f * N + a];
        if (w != kNone) push((int)(w & 0x7FFFFFFFu));
    }
}

__device__ __forceinline__ double pres(double gamma, const double* q) {
    return (gamma - 1) * (q[3] - 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2]));
}

__global__ void k_loss(Params P, const double* q, const double* dt_n, const int32_t* ghosts, int n, double* loss) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int t = 0; t < n; ++t) {
        const int gb = ghosts[t];
        double v[4];
        ld4(q, P.ghost_cell[gb], v);
        s += pres(P.gamma, v) * P.g_le[gb];
    }
    *loss += s * *dt_n;
}

__global__ void k_loss_adjoint(Params P, const double* q, const double* dt_n, const int32_t* ghosts, int n, double w,
                               double* lam_q, double* lam_dt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double gm1 = P.gamma - 1.0, dt = *dt_n;
    double s = 0.0;
    for (int t = 0; t < n; ++t) {
        const int gb = ghosts[t], c = P.ghost_cell[gb];
        double v[4];
        ld4(q, c, v);
        const double le = P.g_le[gb];
        s += pres(P.gamma, v) * le;
        const double u = v[1] / v[0], vv = v[2] / v[0];
        const double dp[4] = {gm1 * 0.5 * (u * u + vv * vv), -gm1 * u, -gm1 * vv, gm1};
        double g[4];
        for (int k = 0; k < 4; ++k) g[k] = w * dt * le * dp[k];
        add4(lam_q, c, g);
    }
    *lam_dt += w * s;
}

int blocks_for(int n) { return (n + kAB - 1) / kAB; }

}  // namespace

int adj_residual_blocks(const Params& P) { return blocks_for(P.n_real); }

void adj_launch_ghosts(const Params& P, const AdjFaces& F, const AdjStage& S, cudaStream_t st) {
    k_adj_ghosts<<<blocks_for(P.n_real), kAB, 0, st>>>(P, F, S);
}
void adj_launch_residual(const Params& P, const AdjFaces& F, const AdjStage& S, cudaStream_t st) {
    k_adj_residual<<<blocks_for(P.n_real), kAB, 0, st>>>(P, F, S);
}
void adj_launch_gradlim(const Params& P, const AdjFaces& F, const AdjStage& S, cudaStream_t st) {
    k_adj_gradlim1<<<blocks_for(4 * P.n_real), kAB, 0, st>>>(P, F, S);
}
void adj_launch_add(double* y, const double* x, size_t n, cudaStream_t st) {
    const int b = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_add<<<b > 0 ? b : 1, 256, 0, st>>>(y, x, n);
}
void adj_launch_sum(const double* partials, int n, double* out, cudaStream_t st) {
    k_sum<<<1, kSumThreads, 0, st>>>(partials, n, out);
}
void adj_launch_dt_finalize(const unsigned long long* keys, const double* dt_cells, int cell0, double* dt_fill, int n,
                            double* dt_out, cudaStream_t st) {
    const int b = std::min((n + 255) / 256, 148 * 8);
    k_dt_finalize<<<b > 0 ? b : 1, 256, 0, st>>>(keys, dt_cells, cell0, dt_fill, n, dt_out);
}
void adj_launch_dt(const Params& P, const AdjFaces& F, const double* q, const double* dt_cells, const double* dt_n,
                   const double* lam_dt, double* lam_qn, int* argmin, cudaStream_t st) {
    cudaMemsetAsync(argmin, 0x7F, sizeof(int), st);
    const int b = std::min((P.n_total + 255) / 256, 148 * 8);
    k_argmin<<<b > 0 ? b : 1, 256, 0, st>>>(dt_cells, P.n_total, dt_n, argmin);
    k_adj_dt<<<1, 32, 0, st>>>(P, F, q, lam_dt, argmin, lam_qn);
}
void adj_launch_loss(const Params& P, const double* q, const double* dt_n, const int32_t* ghosts, int n_ghosts,
                     double* loss, cudaStream_t st) {
    k_loss<<<1, 32, 0, st>>>(P, q, dt_n, ghosts, n_ghosts, loss);
}
void adj_launch_loss_adjoint(const Params& P, const double* q, const double* dt_n, const int32_t* ghosts,
                             int n_ghosts, double w, double* lam_q, double* lam_dt, cudaStream_t st) {
    k_loss_adjoint<<<1, 32, 0, st>>>(P, q, dt_n, ghosts, n_ghosts, w, lam_q, lam_dt);
}

}  // namespace fvgpu
