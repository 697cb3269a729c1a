/*
 * fvoracle — CPU restatement of fvhyper's explicit finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke()
 * and bench.py's cpu_baseline leg compare the CUDA path against; the product
 * never links it.  It is written operation-for-operation after the reference
 * (same evaluation order, same divisions, no FMA contraction: build with
 * -ffp-contract=off) so that it reproduces the reference bit for bit; the
 * CPU tests pin it against the reference compiled from its own sources
 * (oracle/_ref) and against committed golden fixtures.
 *
 * Layout follows the reference: AoS state q[V*cell + k] over n_total = real
 * cells + boundary ghost cells, reference cell/edge numbering.
 */
#ifndef FVORACLE_H
#define FVORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t n_nodes, n_real, n_total, n_edges, n_bound;
    uint32_t* edge_cells; /* [E][2]: cell 0 created the edge, cell 1 the other side */
    uint32_t* edge_nodes; /* [E][2] */
    double *enx, *eny, *elen, *ecx, *ecy; /* [E] */
    double *area, *ccx, *ccy;             /* [n_total] */
    uint32_t* bound_edges;                /* [n_bound] edge of ghost cell n_real+b */
    int32_t* bound_group;                 /* [n_bound] boundary group of ghost b */
} fvo_mesh;

/* DIFFUSION: the heat-equation flux F = -(grad T . n) of examples/heatTransfer
   (V = 1), with the face gradient of gradient_for_diffusion.  NS: the
   compressible Navier-Stokes flux of examples/flatPlate and
   examples/nacaTransient (the shockTube Roe flux plus viscous stresses and
   heat conduction from the face gradient). */
/* BURGERS_DIFF: the upwind advection flux plus -(grad q . n) per variable
   from the face gradient (tests/tests.cpp:76-117, V = 2). */
enum { FVO_FLUX_ROE_FS = 1, FVO_FLUX_ROE_ST = 2, FVO_FLUX_BURGERS = 3, FVO_FLUX_DIFFUSION = 4,
       FVO_FLUX_NS = 5, FVO_FLUX_BURGERS_DIFF = 6 };
enum { FVO_LIM_ZERO = 0, FVO_LIM_MICHALAK = 1, FVO_LIM_VENKAT = 2, FVO_LIM_MINMOD = 3 };
/* VISC_MIN: examples/flatPlate/main.cpp:230-277; VISC_SUM:
   examples/nacaTransient/main.cpp:234-288 (convective + viscous eigenvalues). */
enum { FVO_DT_CONST = 0, FVO_DT_CFL_SUM = 1, FVO_DT_CFL_MIN_SIGNED = 2, FVO_DT_VISC_MIN = 3,
       FVO_DT_VISC_SUM = 4 };
/* NOSLIP: the viscous wall of examples/flatPlate/main.cpp:361-366.
   FARFIELD_B0: the far field of examples/flatPlate/main.cpp:284-352, whose
   tangential momentum is b[0]*(...) where examples/naca has b[1]*(...). */
/* TANGENT: b = (-n_y, n_x), the fixed tangential state of tests/tests.cpp:132-135 (V = 2). */
enum { FVO_BC_COPY = 0, FVO_BC_WALL = 1, FVO_BC_INLET_OUTLET = 2, FVO_BC_FARFIELD = 3,
       FVO_BC_NOSLIP = 4, FVO_BC_FARFIELD_B0 = 5, FVO_BC_TANGENT = 6 };

typedef struct {
    int V;
    int flux;
    double gamma;
    int order2; /* do_calc_gradients && do_calc_limiters && linear_interpolate */
    int limiter;
    double K;
    int dt_kind;
    double cfl, dt_const;
    int global_dt;
    int n_groups;
    const int32_t* group_bc;  /* [n_groups] */
    const double* group_bv;   /* [n_groups][4] far-field / inflow state */
    int positivity_guard;     /* 1: a MUSCL face state with rho <= 0 or p <= 0 falls back
                                 to the cell value (not in the reference; 0 = reference) */
    const double* ghost_bv;   /* [n_bound][4] per-ghost far-field / inflow state overriding
                                 group_bv (a spatially varying inflow; NULL = group_bv) */
    int diffusive;            /* solver::diffusive_gradients (with order2 = 0: gradients are
                                 computed, no limiter, no interpolation) */
    double mu, pr, cp, r;     /* viscosity, Prandtl number, heat capacity, gas constant
                                 (consts:: of the Navier-Stokes examples) */
    int smooth;               /* solver::smooth_residuals (explicit.cpp:32-66, 743) */
} fvo_physics;

int fvo_mesh_build(int64_t n_nodes, const double* nodes_x, const double* nodes_y,
                   int64_t n_cells, const int32_t* cells4, int64_t n_bnd,
                   const int32_t* bnd_nodes, const int32_t* bnd_group, fvo_mesh* out);
void fvo_mesh_free(fvo_mesh* m);

void fvo_flux(const fvo_physics* ph, double* f, const double* qi, const double* qj, const double* n);
void fvo_flux_grad(const fvo_physics* ph, double* f, const double* qi, const double* qj, const double* gx,
                   const double* gy, const double* n);
void fvo_bc(const fvo_physics* ph, int group, double* b, const double* q, const double* n);
double fvo_limiter_func(const fvo_physics* ph, double y);

void fvo_calc_dt(const fvo_mesh* m, const fvo_physics* ph, const double* q, double* dt);
void fvo_min_dt(const fvo_mesh* m, double* dt);
void fvo_calc_gradients(const fvo_mesh* m, const fvo_physics* ph, const double* q, double* gx, double* gy);
void fvo_calc_limiters(const fvo_mesh* m, const fvo_physics* ph, const double* q, const double* gx,
                       const double* gy, double* lim);
void fvo_calc_time_derivatives(const fvo_mesh* m, const fvo_physics* ph, const double* q,
                               const double* gx, const double* gy, const double* lim, double* qt);
void fvo_update_bounds(const fvo_mesh* m, const fvo_physics* ph, double* q, const double* gx,
                       const double* gy, const double* lim);
void fvo_calc_residuals(const fvo_mesh* m, const fvo_physics* ph, const double* qt, double* R);
/* Implicit residual smoothing, explicit.cpp:32-66 (2 Jacobi sweeps, epsilon 0.6), in place on qt. */
void fvo_smooth_residuals(const fvo_mesh* m, const fvo_physics* ph, double* qt);

int fvo_run_loop(const fvo_mesh* m, const fvo_physics* ph, double* q_io, const double* alpha,
                 int n_alpha, uint64_t max_step, double max_time, double tolerance,
                 uint64_t print_interval, uint64_t* out_step, double* out_time, double* out_R,
                 double* out_qt);

/* Pressure force on the faces of boundary group `group`:
   F = sum_b p(q_int_b) * n_b * le_b with p from the interior state (FP64). */
void fvo_boundary_force(const fvo_mesh* m, const fvo_physics* ph, const double* q, int group,
                        double* fx, double* fy);

#ifdef __cplusplus
}
#endif
#endif
