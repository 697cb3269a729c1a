// Kernel launchers (host side).  Every launcher enqueues on `st` and does
// not synchronise.
#pragma once
#include <cuda_runtime.h>

#include "fv_internal.h"

namespace fvgpu {

inline int grid_for(int n) { return (n + kBlock - 1) / kBlock; }

// step control
// run control without copies (dst of launch_ctrl_copy may be mapped host memory)
void launch_ctrl_reset(Ctrl* c, cudaStream_t st);
void launch_ctrl_copy(const Ctrl* src, Ctrl* dst, cudaStream_t st);
void launch_set_limits(RunLimits* d, const RunLimits& v, cudaStream_t st);
// keys: the dt minimum's ordered-key slots ([n_cases][64]), reset every step
void launch_step_begin(Ctrl* c, const RunLimits* lim, int V, unsigned long long* keys, int nkeys, cudaStream_t st);
void launch_step_end(const Params& P, Ctrl* c, const RunLimits* lim, const double* partials,
                     int nblocks, const double* dt, unsigned long long* keys, int nkeys, PrintRec* hist, int hist_cap,
                     cudaStream_t st, bool pdl = false);

// initial / standalone ghost fill (update_bounds) in FP64 (fv_kernels_exact.cu)
namespace exact {
void launch_bounds(const Params& P, double* q, const double* gx, const double* gy,
                   const double* lim, int zero_grad, cudaStream_t st);
}  // namespace exact

// One Jacobi sweep of residual smoothing (explicit.cpp:32-66) over the real
// cells: out = (qt0 - s) / (1 + ne eps), s = -eps * sum of the neighbours'
// qt_in in face (reference edge) order.  nbr: [4][n_real] neighbour device
// index | side << 31, 0xFFFFFFFF = no face; ghosts hold qt = 0.
void launch_smooth(const Params& P, const uint32_t* nbr, const double* qt_in, const double* qt0, double* qt_out,
                   cudaStream_t st);

// utilities (fv_kernels_exact.cu)
void launch_permute_to_device(const double* q_ref, double* q_dev, const int32_t* new2ref,
                              int n_total, int V, cudaStream_t st);
// extra output fields (exact::output_field) of the real cells, reference order
struct OutputPlan {
    int n;
    int kind[8];
    int64_t off[8];
};
void launch_output_fields(const double* q, int V, const int32_t* new2ref, int n_real, double gamma,
                          const OutputPlan& plan, double* out, cudaStream_t st);
void launch_permute_to_ref(const double* q_dev, double* q_ref, const int32_t* new2ref,
                           int n_total, int V, cudaStream_t st);
void launch_fill_ghost_grad(void* gx, void* gy, void* lim, int n_real, int n_total, int V, bool f32,
                            cudaStream_t st);
void launch_to_float(const double* a, float* b, size_t n, cudaStream_t st);
void launch_to_double(const float* a, double* b, size_t n, cudaStream_t st);
void launch_check_state(const Params& P, const double* q, int* flag, cudaStream_t st);
void launch_force(const Params& P, const double* q, int group, double* out2, cudaStream_t st);

}  // namespace fvgpu
