// FP64 kernels of the explicit FV step in the reference's exact evaluation
// order (compile with -fmad=false).  One thread per real cell; each cell
// gathers its faces in increasing reference edge order, so every per-cell
// sum is accumulated in the same order as the reference's edge-scatter loops
// and the results are bit-identical -- with no atomics anywhere.
#include <cuda_runtime.h>

#include "fv_launch.h"
#include "fv_physics_exact.cuh"

namespace fvgpu {

__device__ __forceinline__ unsigned long long dkey(double x) {
    if (x != x) return ~0ull;  // NaN never wins the minimum
    const long long b = __double_as_longlong(x);
    return b < 0 ? ~(unsigned long long)b : ((unsigned long long)b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
    if (k == ~0ull) return __longlong_as_double(0x7ff8000000000000ll);
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}
__device__ __forceinline__ bool inactive(const Ctrl* c) {
    return c != nullptr && *(volatile const int*)&c->active == 0;
}
// min_dt (explicit.cpp:555-564): min over all cells; a NaN in dt[0] wins.
__device__ __forceinline__ double global_dt_value(const Params& P, const double* dt, unsigned long long key) {
    const double d0 = dt[P.cell0];
    return (d0 != d0) ? d0 : dkey_inv(key);
}

template <int V>
__device__ __forceinline__ void load_cell(const double* __restrict__ a, int c, double* v) {
    if (V == 4) {
        const double2* p = reinterpret_cast<const double2*>(a + 4 * (size_t)c);
        double2 x = p[0], y = p[1];
        v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = a[(size_t)V * c + k];
    }
}
template <int V>
__device__ __forceinline__ void store_cell(double* __restrict__ a, int c, const double* v) {
    if (V == 4) {
        double2* p = reinterpret_cast<double2*>(a + 4 * (size_t)c);
        p[0] = make_double2(v[0], v[1]);
        p[1] = make_double2(v[2], v[3]);
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) a[(size_t)V * c + k] = v[k];
    }
}

// ------------------------------------------------------------ step control --
__global__ void k_step_begin(Ctrl* c, const RunLimits* L, int V) {
    if (threadIdx.x != 0) return;
    double Rmax;
    if (c->step > 0) {
        Rmax = 0.0;
        for (int k = 0; k < V; ++k) Rmax = exact::dmax(c->R[k], Rmax);
    } else {
        Rmax = 1.0;
    }
    const int stop = (c->step >= L->max_step) | (c->time >= L->max_time) | (Rmax < L->tolerance);
    c->active = !stop;
    c->need_R = !stop && (c->step == 0 || (c->step % L->print_interval) == 0 || (L->tolerance > 1.01e-16));
    c->dtmin_key = ~0ull;
}

// Residual norms, step/time bookkeeping and print records
// (explicit.cpp:752-800).  Partial sums are reduced in a fixed order.
__global__ void k_step_end(Params P, Ctrl* c, const RunLimits* L, const double* partials, int nblocks,
                           const double* dt, PrintRec* hist, int hist_cap) {
    if (!c->active) return;
    __shared__ double red[kBlock][kMaxV];
    const int V = P.V;
    if (c->need_R) {
        double s[kMaxV] = {0, 0, 0, 0};
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
            for (int k = 0; k < V; ++k) s[k] += partials[(size_t)b * V + k];
        for (int k = 0; k < V; ++k) red[threadIdx.x][k] = s[k];
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w)
                for (int k = 0; k < V; ++k) red[threadIdx.x][k] += red[threadIdx.x + w][k];
            __syncthreads();
        }
    }
    if (threadIdx.x != 0) return;
    if (c->need_R) {
        for (int k = 0; k < V; ++k) c->Rraw[k] = sqrt(red[0][k]);
        if (c->step == 0) {
            for (int k = 0; k < V; ++k) { c->R0[k] = c->Rraw[k]; c->R[k] = c->Rraw[k]; }
        } else {
            for (int k = 0; k < V; ++k) c->R[k] = c->Rraw[k] / c->R0[k];
        }
    }
    const bool print = (c->step == 0) || (c->step % L->print_interval) == 0;
    if (print && c->n_hist < hist_cap) {
        PrintRec& r = hist[c->n_hist++];
        r.step = c->step;
        r.time = c->time;
        for (int k = 0; k < V; ++k) r.R[k] = (c->step == 0) ? 1.0 : c->R[k];
    }
    const double dt0 = P.global_dt ? global_dt_value(P, dt, c->dtmin_key) : dt[P.cell0];
    c->step += 1;
    c->time += dt0;
}

void launch_step_begin(Ctrl* c, const RunLimits* lim, int V, cudaStream_t st) {
    k_step_begin<<<1, 32, 0, st>>>(c, lim, V);
}
void launch_step_end(const Params& P, Ctrl* c, const RunLimits* lim, const double* partials, int nblocks,
                     const double* dt, PrintRec* hist, int hist_cap, cudaStream_t st) {
    k_step_end<<<1, kBlock, 0, st>>>(P, c, lim, partials, nblocks, dt, hist, hist_cap);
}

namespace exact {

// ---------------------------------------------------------------- time step --
// calc_dt kinds (forwardStep/main.cpp:140-185, naca/main.cpp:142-183,
// shockTube/main.cpp:140-147).  Each real cell also computes the dt of its
// boundary ghosts (their only edge is the cell's boundary face).  With a
// global dt the block minimum goes to *dtmin_key (ordered-key atomicMin,
// exact since min is order independent).
template <int V>
__global__ void __launch_bounds__(kBlock) k_dt(Params P, const double* __restrict__ q, double* __restrict__ dt,
                                               unsigned long long* dtmin_key, const Ctrl* ctrl) {
    if (inactive(ctrl)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long kmin = ~0ull;
    if (i < P.n_real) {
        const double gamma = P.gamma, gm1 = gamma - 1, cfl = P.cfl;
        const int N = P.n_real;
        if (P.dt_kind == 0) {
            dt[i] = P.dt_const;
            kmin = dkey(P.dt_const);
            for (int f = 0; f < kMaxFaces; ++f) {
                const uint32_t w = P.face_nbr[f * N + i];
                if (w == kNoFace) break;
                const int nb = (int)(w & 0x7fffffffu);
                if (nb >= N) dt[nb] = P.dt_const;
            }
        } else if (V == 4) {
            double qs[4];
            load_cell<4>(q, i, qs);
            const double cs = sqrt(((gm1) * (qs[3] - 0.5 / qs[0] * (qs[1] * qs[1] + qs[2] * qs[2]))) * gamma / qs[0]);
            const bool sum = P.dt_kind == 1;
            const double Ai = P.area[i];
            double acc = sum ? 0. : 1.0;
            for (int f = 0; f < kMaxFaces; ++f) {
                const uint32_t w = P.face_nbr[f * N + i];
                if (w == kNoFace) break;
                const int nb = (int)(w & 0x7fffffffu);
                const bool side1 = (w >> 31) != 0;
                const double n0 = P.f_nx[f * N + i], n1 = P.f_ny[f * N + i], le = P.f_le[f * N + i];
                double qn[4];
                load_cell<4>(q, nb, qn);
                const double cn = sqrt(((gm1) * (qn[3] - 0.5 / qn[0] * (qn[1] * qn[1] + qn[2] * qn[2]))) * gamma / qn[0]);
                if (sum) {
                    const double es = cs + fabs(qs[1] / qs[0] * n0 + qs[2] / qs[0] * n1);
                    const double en = cn + fabs(qn[1] / qn[0] * n0 + qn[2] / qn[0] * n1);
                    const double center = side1 ? dmax(en, es) : dmax(es, en);
                    acc += center * le;
                    if (nb >= N) {
                        double d = 0.;
                        d += center * le;
                        const double dg = cfl * P.area[nb] / d;
                        dt[nb] = dg;
                        const unsigned long long kg = dkey(dg);
                        kmin = kg < kmin ? kg : kmin;
                    }
                } else {
                    const double es = (cs + fabs(qs[1] / qs[0])) * n0 + (cs + fabs(qs[2] / qs[0])) * n1;
                    const double dti = cfl * (Ai / le) / fabs(es);
                    acc = dmin(acc, dti);
                    if (nb >= N) {
                        const double en = (cn + fabs(qn[1] / qn[0])) * n0 + (cn + fabs(qn[2] / qn[0])) * n1;
                        const double dg = dmin(1.0, cfl * (P.area[nb] / le) / fabs(en));
                        dt[nb] = dg;
                        const unsigned long long kg = dkey(dg);
                        kmin = kg < kmin ? kg : kmin;
                    }
                }
            }
            const double di = sum ? cfl * Ai / acc : acc;
            dt[i] = di;
            const unsigned long long ki = dkey(di);
            kmin = ki < kmin ? ki : kmin;
        }
    }
    if (P.global_dt && dtmin_key != nullptr) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, kmin, o);
            kmin = other < kmin ? other : kmin;
        }
        if ((threadIdx.x & 31) == 0 && kmin != ~0ull) atomicMin(dtmin_key, kmin);
    }
}

// ------------------------------------------------ gradients + limiters (K1) --
// Green-Gauss gradients (explicit.cpp:112-171) and the min/max smooth-switch
// limiter (explicit.cpp:174-258) fused per cell.  Ghost cells keep gx=gy=0,
// lim=1, as the reference leaves them.
template <int V>
__global__ void __launch_bounds__(kBlock) k_grad_lim(Params P, StageIO io) {
    if (inactive(io.ctrl)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.n_real;
    if (i >= N) return;
    double qs[V], gx[V], gy[V], qmn[V], qmx[V];
    load_cell<V>(io.q_stage, i, qs);
#pragma unroll
    for (int k = 0; k < V; ++k) { gx[k] = 0.; gy[k] = 0.; qmn[k] = qs[k]; qmx[k] = qs[k]; }
    for (int f = 0; f < kMaxFaces; ++f) {
        const uint32_t w = P.face_nbr[f * N + i];
        if (w == kNoFace) break;
        const int nb = (int)(w & 0x7fffffffu);
        const bool side1 = (w >> 31) != 0;
        const double nx = P.f_nx[f * N + i], ny = P.f_ny[f * N + i], le = P.f_le[f * N + i];
        const double g = P.f_g[f * N + i];
        double qn[V];
        load_cell<V>(io.q_stage, nb, qn);
#pragma unroll
        for (int k = 0; k < V; ++k) {
            if (!side1) {
                const double fl = (qs[k] * (1.0 - g) + qn[k] * g) * le;
                gx[k] += fl * nx;
                gy[k] += fl * ny;
            } else {
                const double fl = (qn[k] * (1.0 - g) + qs[k] * g) * le;
                gx[k] -= fl * nx;
                gy[k] -= fl * ny;
            }
            qmn[k] = dmin(qmn[k], qn[k]);
            qmx[k] = dmax(qmx[k], qn[k]);
        }
    }
    const double A = P.area[i];
    const double invA = 1. / A;
#pragma unroll
    for (int k = 0; k < V; ++k) { gx[k] *= invA; gy[k] *= invA; }
    double lim[V];
#pragma unroll
    for (int k = 0; k < V; ++k) lim[k] = 1.;
    const double sqrt_area = sqrt(A);
    const double tol = 1e-15;
    for (int f = 0; f < kMaxFaces; ++f) {
        const uint32_t w = P.face_nbr[f * N + i];
        if (w == kNoFace) break;
        const double dx = P.f_dsx[f * N + i], dy = P.f_dsy[f * N + i];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const double dqg = gx[k] * dx + gy[k] * dy;
            const double delta_max = qmx[k] - qs[k];
            const double delta_min = qmn[k] - qs[k];
            const double Ka = P.K * sqrt_area;
            const double K3a = Ka * Ka * Ka;
            const double d2 = (delta_max - delta_min) * (delta_max - delta_min);
            double sig;
            if (d2 <= K3a) {
                sig = 1.;
            } else if (d2 <= 2 * K3a) {
                const double y = (d2 / K3a - 1.0);
                sig = 2.0 * y * y * y - 3.0 * y * y + 1.0;
            } else {
                sig = 0.;
            }
            double l = 1.0;
            if (sig < 1.0) {
                if (dqg > tol) l = limiter_func(P.limiter, delta_max / dqg);
                else if (dqg < -tol) l = limiter_func(P.limiter, delta_min / dqg);
                else l = 1.0;
            }
            l = sig + (1.0 - sig) * l;
            lim[k] = dmin(lim[k], l);
        }
    }
    store_cell<V>(io.gx, i, gx);
    store_cell<V>(io.gy, i, gy);
    store_cell<V>(io.lim, i, lim);
}

// --------------------------------------- flux + RK update + ghost fill (K2) --
// calc_time_derivatives (explicit.cpp:261-364), update_cells (368-378) and
// update_bounds (380-417) fused per cell.  The ghost fill uses the updated
// interior state with this stage's (stale) gradients and limiters, exactly
// as the reference does.  Optionally writes per-block sums of qt^2 * A.
template <int V, bool ORDER2, int FLUX>
__global__ void __launch_bounds__(kBlock) k_stage(Params P, StageIO io) {
    if (inactive(io.ctrl)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = P.n_real;
    double res[V];
#pragma unroll
    for (int k = 0; k < V; ++k) res[k] = 0.;
    if (i < N) {
        double qs[V], gxs[V], gys[V], lms[V];
        load_cell<V>(io.q_stage, i, qs);
        if (ORDER2) {
            load_cell<V>(io.gx, i, gxs);
            load_cell<V>(io.gy, i, gys);
            load_cell<V>(io.lim, i, lms);
        }
        const double A = P.area[i];
        double qt[V];
#pragma unroll
        for (int k = 0; k < V; ++k) qt[k] = 0.;
        for (int f = 0; f < kMaxFaces; ++f) {
            const uint32_t w = P.face_nbr[f * N + i];
            if (w == kNoFace) break;
            const int nb = (int)(w & 0x7fffffffu);
            const bool side1 = (w >> 31) != 0;
            const double nx = P.f_nx[f * N + i], ny = P.f_ny[f * N + i], le = P.f_le[f * N + i];
            double qn[V], qsf[V], qnf[V];
            load_cell<V>(io.q_stage, nb, qn);
            if (ORDER2) {
                double gxn[V], gyn[V], lmn[V];
                load_cell<V>(io.gx, nb, gxn);
                load_cell<V>(io.gy, nb, gyn);
                load_cell<V>(io.lim, nb, lmn);
                const double dsx = P.f_dsx[f * N + i], dsy = P.f_dsy[f * N + i];
                const double dnx = P.f_dnx[f * N + i], dny = P.f_dny[f * N + i];
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    qsf[k] = qs[k] + (gxs[k] * dsx + gys[k] * dsy) * lms[k];
                    qnf[k] = qn[k] + (gxn[k] * dnx + gyn[k] * dny) * lmn[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k) { qsf[k] = qs[k]; qnf[k] = qn[k]; }
            }
            double fl[V];
            if (!side1) {
                flux<FLUX>(P.gamma, fl, qsf, qnf, nx, ny);
#pragma unroll
                for (int k = 0; k < V; ++k) qt[k] -= fl[k] * le / A;
            } else {
                flux<FLUX>(P.gamma, fl, qnf, qsf, nx, ny);
#pragma unroll
                for (int k = 0; k < V; ++k) qt[k] += fl[k] * le / A;
            }
        }
        double dtc;
        if (io.ctrl != nullptr && P.global_dt) dtc = global_dt_value(P, io.dt, io.ctrl->dtmin_key);
        else dtc = io.dt[i];
        double qb[V], qnew[V];
        load_cell<V>(io.q_base, i, qb);
#pragma unroll
        for (int k = 0; k < V; ++k) qnew[k] = qb[k] + qt[k] * dtc * io.alpha;
        store_cell<V>(io.q_out, i, qnew);
        // boundary ghosts of this cell
        for (int f = 0; f < kMaxFaces; ++f) {
            const uint32_t w = P.face_nbr[f * N + i];
            if (w == kNoFace) break;
            const int nb = (int)(w & 0x7fffffffu);
            if (nb < N) continue;
            const double nx = P.f_nx[f * N + i], ny = P.f_ny[f * N + i];
            double qint[V], b[V];
            if (ORDER2) {
                const double d0 = P.f_dsx[f * N + i], d1 = P.f_dsy[f * N + i];
#pragma unroll
                for (int k = 0; k < V; ++k) qint[k] = qnew[k] + (gxs[k] * d0 + gys[k] * d1) * lms[k];
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k) qint[k] = qnew[k];
            }
            bc<V>(P, P.ghost_group[nb - N], b, qint, nx, ny);
            store_cell<V>(io.q_out, nb, b);
        }
        if (io.partials != nullptr) {
#pragma unroll
            for (int k = 0; k < V; ++k) res[k] = qt[k] * qt[k] * A;
        }
    }
    if (io.partials != nullptr) {
        __shared__ double red[kBlock / 32][V];
#pragma unroll
        for (int k = 0; k < V; ++k)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) res[k] += __shfl_xor_sync(0xffffffffu, res[k], o);
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int k = 0; k < V; ++k) red[threadIdx.x >> 5][k] = res[k];
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < V; ++k) {
                double s = 0.;
                for (int w = 0; w < kBlock / 32; ++w) s += red[w][k];
                io.partials[(size_t)blockIdx.x * V + k] = s;
            }
        }
    }
}

// Standalone ghost fill (update_bounds, explicit.cpp:380-417), one thread
// per ghost.  zero_grad: the initial fill run() does before the loop with
// freshly zeroed gx, gy, limiters (explicit.cpp:712).
template <int V>
__global__ void k_bounds(Params P, double* __restrict__ q, const double* __restrict__ gx,
                         const double* __restrict__ gy, const double* __restrict__ lim, int zero_grad) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= P.n_bound) return;
    const int N = P.n_real;
    const int c = P.ghost_cell[b], f = P.ghost_slot[b];
    const double nx = P.f_nx[f * N + c], ny = P.f_ny[f * N + c];
    double qc[V], qint[V], out[V];
    load_cell<V>(q, c, qc);
    if (P.order2) {
        const double d0 = P.f_dsx[f * N + c], d1 = P.f_dsy[f * N + c];
        double gxc[V], gyc[V], lc[V];
        if (zero_grad) {
#pragma unroll
            for (int k = 0; k < V; ++k) { gxc[k] = 0.; gyc[k] = 0.; lc[k] = 0.; }
        } else {
            load_cell<V>(gx, c, gxc); load_cell<V>(gy, c, gyc); load_cell<V>(lim, c, lc);
        }
#pragma unroll
        for (int k = 0; k < V; ++k) qint[k] = qc[k] + (gxc[k] * d0 + gyc[k] * d1) * lc[k];
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) qint[k] = qc[k];
    }
    bc<V>(P, P.ghost_group[b], out, qint, nx, ny);
    store_cell<V>(q, N + b, out);
}

// ----------------------------------------------------------------- launchers --
void launch_dt(const Params& P, const double* q, double* dt, unsigned long long* key, const Ctrl* c,
               cudaStream_t st) {
    const int g = grid_for(P.n_real);
    if (P.V == 4) k_dt<4><<<g, kBlock, 0, st>>>(P, q, dt, key, c);
    else k_dt<2><<<g, kBlock, 0, st>>>(P, q, dt, key, c);
}

void launch_grad_lim(const Params& P, const StageIO& io, cudaStream_t st) {
    const int g = grid_for(P.n_real);
    if (P.V == 4) k_grad_lim<4><<<g, kBlock, 0, st>>>(P, io);
    else k_grad_lim<2><<<g, kBlock, 0, st>>>(P, io);
}

void launch_stage(const Params& P, const StageIO& io, cudaStream_t st) {
    const int g = grid_for(P.n_real);
    if (P.flux == 3) {
        if (P.order2) k_stage<2, true, 3><<<g, kBlock, 0, st>>>(P, io);
        else k_stage<2, false, 3><<<g, kBlock, 0, st>>>(P, io);
    } else if (P.flux == 1) {
        if (P.order2) k_stage<4, true, 1><<<g, kBlock, 0, st>>>(P, io);
        else k_stage<4, false, 1><<<g, kBlock, 0, st>>>(P, io);
    } else {
        if (P.order2) k_stage<4, true, 2><<<g, kBlock, 0, st>>>(P, io);
        else k_stage<4, false, 2><<<g, kBlock, 0, st>>>(P, io);
    }
}

}  // namespace exact

namespace exact {
void launch_bounds(const Params& P, double* q, const double* gx, const double* gy, const double* lim,
                   int zero_grad, cudaStream_t st) {
    if (P.n_bound == 0) return;
    const int g = grid_for(P.n_bound);
    if (P.V == 4) k_bounds<4><<<g, kBlock, 0, st>>>(P, q, gx, gy, lim, zero_grad);
    else k_bounds<2><<<g, kBlock, 0, st>>>(P, q, gx, gy, lim, zero_grad);
}
}  // namespace exact

// ----------------------------------------------------------------- utilities --
__global__ void k_permute_to_device(const double* __restrict__ qr, double* __restrict__ qd,
                                    const int32_t* __restrict__ new2ref, int n, int V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = new2ref[i];
    for (int k = 0; k < V; ++k) qd[(size_t)V * i + k] = qr[(size_t)V * r + k];
}
__global__ void k_permute_to_ref(const double* __restrict__ qd, double* __restrict__ qr,
                                 const int32_t* __restrict__ new2ref, int n, int V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = new2ref[i];
    for (int k = 0; k < V; ++k) qr[(size_t)V * r + k] = qd[(size_t)V * i + k];
}
void launch_permute_to_device(const double* q_ref, double* q_dev, const int32_t* new2ref, int n, int V,
                              cudaStream_t st) {
    k_permute_to_device<<<grid_for(n), kBlock, 0, st>>>(q_ref, q_dev, new2ref, n, V);
}
void launch_permute_to_ref(const double* q_dev, double* q_ref, const int32_t* new2ref, int n, int V,
                           cudaStream_t st) {
    k_permute_to_ref<<<grid_for(n), kBlock, 0, st>>>(q_dev, q_ref, new2ref, n, V);
}

__global__ void k_fill_ghost_grad(double* gx, double* gy, double* lim, int n_real, int n_total, int V) {
    const int i = n_real + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total) return;
    for (int k = 0; k < V; ++k) {
        gx[(size_t)V * i + k] = 0.;
        gy[(size_t)V * i + k] = 0.;
        lim[(size_t)V * i + k] = 1.;
    }
}
void launch_fill_ghost_grad(double* gx, double* gy, double* lim, int n_real, int n_total, int V, cudaStream_t st) {
    if (n_total > n_real) k_fill_ghost_grad<<<grid_for(n_total - n_real), kBlock, 0, st>>>(gx, gy, lim, n_real, n_total, V);
}

__global__ void k_check_state(Params P, const double* __restrict__ q, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_real) return;
    bool bad = false;
    const int V = P.V;
    for (int k = 0; k < V; ++k) {
        const double v = q[(size_t)V * i + k];
        bad |= !(v == v) || fabs(v) > 1.7e308;
    }
    if (V == 4 && !bad) {
        double s[4];
        for (int k = 0; k < 4; ++k) s[k] = q[(size_t)4 * i + k];
        bad = !(s[0] > 0.) || !(exact::pres(P.gamma, s) > 0.);
    }
    if (bad) atomicExch(flag, 1);
}
void launch_check_state(const Params& P, const double* q, int* flag, cudaStream_t st) {
    k_check_state<<<grid_for(P.n_real), kBlock, 0, st>>>(P, q, flag);
}

// Pressure force over one boundary group; one block, fixed summation order.
__global__ void k_force(Params P, const double* __restrict__ q, int group, double* out) {
    __shared__ double sx[kBlock], sy[kBlock];
    double ax = 0., ay = 0.;
    const int N = P.n_real;
    for (int b = threadIdx.x; b < P.n_bound; b += blockDim.x) {
        if (P.ghost_group[b] != group) continue;
        const int c = P.ghost_cell[b], f = P.ghost_slot[b];
        double s[4];
        load_cell<4>(q, c, s);
        const double p = exact::pres(P.gamma, s);
        const double le = P.f_le[f * N + c];
        ax += p * P.f_nx[f * N + c] * le;
        ay += p * P.f_ny[f * N + c] * le;
    }
    sx[threadIdx.x] = ax; sy[threadIdx.x] = ay;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) { sx[threadIdx.x] += sx[threadIdx.x + w]; sy[threadIdx.x] += sy[threadIdx.x + w]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = sx[0]; out[1] = sy[0]; }
}
void launch_force(const Params& P, const double* q, int group, double* out2, cudaStream_t st) {
    k_force<<<1, kBlock, 0, st>>>(P, q, group, out2);
}

}  // namespace fvgpu
