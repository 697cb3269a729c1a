/*
 * fvhyper/explicit.h — explicit solver API of fvhyper, B200 build.
 *
 * Same user-facing declarations as the reference (fvhyper/explicit.h:31-181):
 * the user program defines vars, var_names, the solver:: flags,
 * limiter_func, generate_initial_solution, calc_flux, calc_dt and
 * boundaries::bounds; the library defines solver::limiter_k_value,
 * solverOptions and run().  An unchanged example main() compiles against this
 * header and libfvhyper_gpu.a + libfvgpu.so, and run() advances it on the GPU.
 *
 * run() identifies the user's physics callbacks with a device physics kind
 * by evaluating them on probe states and comparing bit for bit with the host
 * copy of each kind (fv_kind_*, include/fvgpu.h):
 *  - fluxes: Roe with the cures eigenvalues in either of the reference's two
 *    operand orders, upwind advection, and with diffusive_gradients the heat
 *    diffusion flux (vars = 1), the Navier-Stokes flux (vars = 4, constants
 *    from fvhyper::consts) and the Burgers + diffusion flux (vars = 2);
 *  - limiter functions: Michalak, Venkatakrishnan, minmod, zero;
 *  - boundaries: copy, reflecting wall, inlet-outlet, far field (both of the
 *    reference's forms), no-slip wall, tangential state;
 *  - time steps: constant, edge-sum and edge-min CFL, and the two viscous
 *    CFL forms.
 * Residual smoothing (solverOptions::smooth_residuals) runs with the Burgers
 * + diffusion kind.  Callbacks that match no kind, and residual smoothing
 * with any other kind, are refused with std::invalid_argument: there is no
 * CPU fallback.
 */
#pragma once

#include <math.h>
#include <sys/types.h>

#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include <fvhyper/mesh.h>
#include <fvhyper/parallel.h>

namespace fvhyper {

extern const int vars;
extern const std::vector<std::string> var_names;

namespace solver {
extern const bool do_calc_gradients;
extern const bool do_calc_limiters;
extern const bool linear_interpolate;
extern const bool diffusive_gradients;
extern const bool global_dt;
extern const bool smooth_residuals;
extern const double limiter_k_value;  // 7.5, as fvhyper/src/explicit.cpp:26-28
}  // namespace solver

// ---- user-defined physics (called by run() on the host to identify them)
double limiter_func(const double& r);

void gradient_for_diffusion(double* gradx, double* grady, const double* gxi, const double* gyi,
                            const double* gxj, const double* gyj, const double* qi, const double* qj,
                            const double* di, const double* dj);

void generate_initial_solution(std::vector<double>& v, const mesh& m);

void calc_flux(double* f, const double* qi, const double* qj, const double* gx, const double* gy,
               const double* n);

void calc_dt(std::vector<double>& dt, const std::vector<double>& q, mesh& m);

// ---- library
struct solverOptions {
    double max_time = 1e10;
    uint max_step = 1e8;
    uint print_interval = 1;
    bool verbose = true;
    double tolerance = 1e-16;
    bool save_time_series = false;
    double time_series_interval = 0.2;
    // B200 build: arithmetic of the device step.  -1 = the FVGPU_PRECISION
    // environment variable ("fp64_exact", "fp64", "fp32") or, unset,
    // fp64_exact (bit-identical to the reference CPU solver).
    int precision = -1;
    // B200 build: CUDA device.  -1 = FVGPU_DEVICE, else 0.
    int device = -1;
};

// The explicit time loop (fvhyper/src/explicit.cpp:657-817) on the GPU: q is
// resized to vars * (real + ghost cells), filled by generate_initial_solution,
// advanced with the 5-stage scheme until max_step / max_time / tolerance, and
// returned.  Prints the reference's log lines; writes times/<name>_<k>.vtu
// snapshots when save_time_series is set.
void run(const std::string name, std::vector<double>& q, mpi_wrapper& pool, mesh& m, solverOptions& opt);

}  // namespace fvhyper
