// Discrete adjoint of the explicit step (FP64): device arrays and launchers.
//
// The adjoint reverses one RK stage at a time.  The forward stage is
//   qs_{k+1}[real]  = q_n + alpha_k dt_n qt(qs_k, g_k)            (update_cells)
//   qs_{k+1}[ghost] = bc(qs_{k+1}[interior] + (g_k . d) lim_k)    (update_bounds,
//                     with the gradients g_k of the stage's input, explicit.cpp:380-417)
//   g_k = (gx, gy, lim)(qs_k)                                     (gradients + limiters)
// and dt_n = min over cells of the CFL time step of q_n (min_dt).
// All arrays use the device cell numbering; per-face data are the
// cell-centric face lists ([4][n_real], slot-major) in increasing reference
// edge order.  Every kernel gathers into the cells it owns, so the adjoint
// is deterministic (no floating-point atomics).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "fv_internal.h"

namespace fvgpu {

struct AdjFaces {
    const uint32_t* nbr;   // [4][n_real] neighbour | side << 31, 0xFFFFFFFF = none
    const double *nx, *ny, *le, *g;      // face normal (reference orientation), length, Green-Gauss weight
    const double *dsx, *dsy, *dnx, *dny; // x_f - x_self, x_f - x_neighbour
    const double* area;                  // [n_total]
};

struct AdjStage {
    // primal
    const double* qs;      // stage input qs_k [n_total][4]
    const double* qs1;     // stage output qs_{k+1} [n_total][4]
    const double* gx;      // g_k [n_total][4] (ghosts: 0, 0, 1)
    const double* gy;
    const double* lim;
    double dt;             // dt_n
    double alpha;          // alpha_k
    int zero_grad;         // the initial ghost fill of run(): no reconstruction
    // adjoint
    double* lam_next;      // in: dL/d qs_{k+1}; its real part gains the ghost-fill terms
    double* lam_cur;       // out: dL/d qs_k (written for every cell)
    double* lam_gx;        // dL/d g_k [n_real][4]
    double* lam_gy;
    double* lam_lim;
    double* lam_qn;        // += dL/d q_n through the update's base state (real cells)
    double* lam_bv;        // [n_bound][4] += dL/d (ghost boundary state)
    double* dt_partials;   // [blocks] alpha_k sum(lam_next . qt) per block, or nullptr
};

// ghost fill of qs_{k+1}: lam_next[interior] += ..., lam_g = contributions, lam_bv += ...
void adj_launch_ghosts(const Params& P, const AdjFaces& F, const AdjStage& S, cudaStream_t st);
// flux residual + RK update: lam_cur = ..., lam_g += ..., lam_qn += lam_next[real], dt partials
void adj_launch_residual(const Params& P, const AdjFaces& F, const AdjStage& S, cudaStream_t st);
// gradients + limiters: lam_cur += (d g_k / d qs_k)^T lam_g
void adj_launch_gradlim(const Params& P, const AdjFaces& F, const AdjStage& S, cudaStream_t st);
int adj_residual_blocks(const Params& P);

// y[i] += x[i], i < n
void adj_launch_add(double* y, const double* x, size_t n, cudaStream_t st);
// out = sum(partials[0..n)) in a fixed order (one thread)
void adj_launch_sum(const double* partials, int n, double* out, cudaStream_t st);

// time step: dt_cells [n_total] per-cell CFL time steps of q_n, keys the
// ordered-key minimum.  Finalise writes dt_n (min_dt, a NaN in dt[0] wins)
// to *dt_out and to every entry of dt_fill.
void adj_launch_dt_finalize(const unsigned long long* keys, const double* dt_cells, int cell0, double* dt_fill,
                            int n, double* dt_out, cudaStream_t st);
// lam_qn += lam_dt * d dt_n / d q_n (the arg-min cell's CFL time step,
// forwardStep calc_dt kind with the global minimum)
void adj_launch_dt(const Params& P, const AdjFaces& F, const double* q, const double* dt_cells, const double* dt_n,
                   const double* lam_dt, double* lam_qn, int* argmin, cudaStream_t st);

// boundary pressure functional: loss += dt_n sum_b p(q[interior(b)]) le_b
// over the listed ghosts (device ghost indices, fixed order)
void adj_launch_loss(const Params& P, const double* q, const double* dt_n, const int32_t* ghosts, int n_ghosts,
                     double* loss, cudaStream_t st);
// its adjoint: lam_q[interior] += w dt_n le dp/dq, lam_dt += w sum p le
void adj_launch_loss_adjoint(const Params& P, const double* q, const double* dt_n, const int32_t* ghosts,
                             int n_ghosts, double w, double* lam_q, double* lam_dt, cudaStream_t st);

}  // namespace fvgpu
