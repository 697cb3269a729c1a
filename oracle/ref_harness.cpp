/*
 * ref_harness.cpp — C entry points into the UNMODIFIED reference library
 * (fvhyper/src/{explicit,mesh,parallel,post}.cpp) plus one reference example
 * translation unit (examples/<name>/main.cpp), compiled together into
 * oracle/_ref/libref_<variant>.so by oracle/Makefile.
 *
 * Test infrastructure only: the tests use these symbols to pin the C
 * restatement (oracle/fvoracle.c) and to make golden fixtures.  Nothing in
 * the product links or loads this code.
 *
 * Build-time switches (set by oracle/Makefile):
 *   FVREF_EX_<NAME>    which example TU is linked (decides which of the
 *                      example's `consts::` globals exist).
 *   FVREF_OVERRIDE     when 1 the example TU was compiled with its solver
 *                      flags and limiter_func renamed (fvref_ex_*), and this
 *                      file defines them instead from FVREF_ORDER2,
 *                      FVREF_GLOBAL_DT and FVREF_LIMITER (0 = the example's
 *                      own limiter_func, 1 = Venkatakrishnan's phi).
 */
#include <fvhyper/explicit.h>
#include <fvhyper/mesh.h>
#include <fvhyper/parallel.h>
#include <cstring>
#include <cstdint>
#include <string>
#include <vector>

namespace fvhyper {

// The reference header (explicit.h:88-103) declares calc_gradients and
// calc_limiters with signatures that differ from their definitions
// (explicit.cpp:112-117, 174-182); declare the definitions' signatures.
void calc_gradients(std::vector<double>& gx, std::vector<double>& gy,
                    const std::vector<double>& q, mesh& m);
void calc_limiters(std::vector<double>& limiters, std::vector<double>& qmin,
                   std::vector<double>& qmax, const std::vector<double>& q,
                   const std::vector<double>& gx, const std::vector<double>& gy,
                   mesh& m);

namespace consts {
#if defined(FVREF_EX_FORWARDSTEP)
extern double gamma; extern double cfl; extern double mach;
#elif defined(FVREF_EX_NACA)
extern double gamma; extern double cfl;
#elif defined(FVREF_EX_SHOCKTUBE)
extern double gamma;
#elif defined(FVREF_EX_FLATPLATE)
extern double gamma; extern double cfl;
#elif defined(FVREF_EX_NACATRANSIENT)
extern double gamma; extern double cfl; extern double mach;
#endif  // heatTransfer, burgers and the regression-test physics have no consts:: globals
}

#if FVREF_OVERRIDE
double fvref_ex_limiter_func(const double& y);
namespace solver {
const bool do_calc_gradients = FVREF_ORDER2;
const bool do_calc_limiters = FVREF_ORDER2;
const bool linear_interpolate = FVREF_ORDER2;
const bool global_dt = FVREF_GLOBAL_DT;
}
double limiter_func(const double& y) {
#if FVREF_LIMITER == 1
    // Venkatakrishnan (1995) limiter function phi(y) = (y^2 + 2y)/(y^2 + y + 2)
    return (y * y + 2.0 * y) / (y * y + y + 2.0);
#else
    return fvref_ex_limiter_func(y);
#endif
}
#endif

}  // namespace fvhyper

using fvhyper::mesh;

namespace {
fvhyper::mpi_wrapper& pool() {
    static fvhyper::mpi_wrapper p;
    return p;
}
mesh* g_mesh = nullptr;
std::vector<double> vec(const double* p, size_t n) { return std::vector<double>(p, p + n); }
void put(double* dst, const std::vector<double>& v) { std::memcpy(dst, v.data(), v.size() * sizeof(double)); }
size_t nq() { return (size_t)fvhyper::vars * g_mesh->cellsAreas.size(); }
}  // namespace

int fvref_example_main();  // the example main(), renamed by oracle/Makefile

extern "C" {

int ref_vars() { return fvhyper::vars; }

int ref_flags(int* out6) {
    out6[0] = fvhyper::solver::do_calc_gradients;
    out6[1] = fvhyper::solver::do_calc_limiters;
    out6[2] = fvhyper::solver::linear_interpolate;
    out6[3] = fvhyper::solver::diffusive_gradients;
    out6[4] = fvhyper::solver::global_dt;
    out6[5] = fvhyper::solver::smooth_residuals;
    return 0;
}

double ref_limiter_k() { return fvhyper::solver::limiter_k_value; }
double ref_limiter_func(double y) { return fvhyper::limiter_func(y); }

/* Set the example's tunable globals; a negative value leaves it unchanged. */
void ref_set_consts(double gamma, double cfl, double mach) {
#if defined(FVREF_EX_FORWARDSTEP) || defined(FVREF_EX_NACA) || defined(FVREF_EX_SHOCKTUBE) || \
    defined(FVREF_EX_FLATPLATE) || defined(FVREF_EX_NACATRANSIENT)
    if (gamma > 0) fvhyper::consts::gamma = gamma;
#endif
#if defined(FVREF_EX_FORWARDSTEP) || defined(FVREF_EX_NACA) || defined(FVREF_EX_FLATPLATE) || \
    defined(FVREF_EX_NACATRANSIENT)
    if (cfl > 0) fvhyper::consts::cfl = cfl;
#endif
#if defined(FVREF_EX_FORWARDSTEP) || defined(FVREF_EX_NACATRANSIENT)
    if (mach > 0) fvhyper::consts::mach = mach;
#endif
    (void)gamma; (void)cfl; (void)mach;
}

typedef void (*bc_fn)(double*, double*, double*);

void* ref_bc_get(const char* name) {
    auto it = fvhyper::boundaries::bounds.find(name);
    return it == fvhyper::boundaries::bounds.end() ? nullptr : (void*)it->second;
}

void ref_bc_set(const char* name, void* fn) { fvhyper::boundaries::bounds[name] = (bc_fn)fn; }

void ref_flux(double* f, const double* qi, const double* qj, const double* n) {
    std::vector<double> z(fvhyper::vars, 0.0);
    fvhyper::calc_flux(f, qi, qj, z.data(), z.data(), n);
}

/* calc_flux with face gradients (the diffusive fluxes read them). */
void ref_flux_grad(double* f, const double* qi, const double* qj, const double* gx, const double* gy,
                   const double* n) {
    fvhyper::calc_flux(f, qi, qj, gx, gy, n);
}

/* Read <basename>.msh with the reference reader (mesh.cpp:803-855). */
int ref_read_mesh(const char* basename) {
    delete g_mesh;
    g_mesh = new mesh();
    try {
        g_mesh->read_file(basename, pool());
    } catch (const std::exception& e) {
        delete g_mesh;
        g_mesh = nullptr;
        return -1;
    }
    return 0;
}

void ref_mesh_sizes(int64_t* out) {
    mesh& m = *g_mesh;
    out[0] = m.nodesX.size();
    out[1] = m.nRealCells;
    out[2] = m.cellsAreas.size();
    out[3] = m.edgesLengths.size();
    out[4] = m.boundaryEdges.size();
}

void ref_mesh_get(uint32_t* edge_cells, uint32_t* edge_nodes, double* enx, double* eny,
                  double* elen, double* ecx, double* ecy, double* area, double* ccx,
                  double* ccy, uint32_t* bound_edges, uint32_t* bound_tag) {
    mesh& m = *g_mesh;
    const size_t E = m.edgesLengths.size();
    for (size_t e = 0; e < E; ++e) {
        edge_cells[2 * e] = m.edgesCells(e, 0);
        edge_cells[2 * e + 1] = m.edgesCells(e, 1);
        edge_nodes[2 * e] = m.edgesNodes(e, 0);
        edge_nodes[2 * e + 1] = m.edgesNodes(e, 1);
    }
    put(enx, m.edgesNormalsX); put(eny, m.edgesNormalsY); put(elen, m.edgesLengths);
    put(ecx, m.edgesCentersX); put(ecy, m.edgesCentersY);
    put(area, m.cellsAreas); put(ccx, m.cellsCentersX); put(ccy, m.cellsCentersY);
    for (size_t b = 0; b < m.boundaryEdges.size(); ++b) {
        bound_edges[b] = m.boundaryEdges[b];
        bound_tag[b] = m.boundaryEdgesIntTag[b];
    }
}

void ref_initial_state(double* q) {
    std::vector<double> v(nq());
    fvhyper::generate_initial_solution(v, *g_mesh);
    put(q, v);
}

void ref_calc_dt(const double* q, double* dt, int apply_global_min) {
    std::vector<double> qv = vec(q, nq()), d(nq());
    fvhyper::calc_dt(d, qv, *g_mesh);
    if (apply_global_min) fvhyper::min_dt(d, *g_mesh);
    put(dt, d);
}

void ref_calc_gradients(const double* q, double* gx, double* gy) {
    std::vector<double> qv = vec(q, nq()), a(nq()), b(nq());
    fvhyper::calc_gradients(a, b, qv, *g_mesh);
    put(gx, a); put(gy, b);
}

void ref_calc_limiters(const double* q, const double* gx, const double* gy, double* lim) {
    std::vector<double> qv = vec(q, nq()), a = vec(gx, nq()), b = vec(gy, nq());
    std::vector<double> l(nq()), mn(nq()), mx(nq());
    fvhyper::calc_limiters(l, mn, mx, qv, a, b, *g_mesh);
    put(lim, l);
}

void ref_calc_time_derivatives(const double* q, const double* gx, const double* gy,
                               const double* lim, double* qt) {
    std::vector<double> qv = vec(q, nq()), a = vec(gx, nq()), b = vec(gy, nq());
    std::vector<double> l = vec(lim, nq()), t(nq());
    fvhyper::calc_time_derivatives(t, qv, a, b, l, *g_mesh);
    put(qt, t);
}

/* Residual smoothing (explicit.cpp:32-66) of qt, in place. */
void ref_smooth_residuals(double* qt) {
    std::vector<double> t = vec(qt, nq()), s0(nq()), s1(nq());
    fvhyper::smooth_residuals(t, s0, s1, *g_mesh);
    put(qt, t);
}

void ref_update_bounds(double* q, const double* gx, const double* gy, const double* lim) {
    std::vector<double> qv = vec(q, nq()), a = vec(gx, nq()), b = vec(gy, nq()), l = vec(lim, nq());
    fvhyper::update_bounds(qv, a, b, l, *g_mesh);
    put(q, qv);
}

/*
 * The body of fvhyper::run (explicit.cpp:665-801) driven through the
 * reference's own stage functions, with the RK coefficients as an argument
 * (run() hard-codes the 5-stage set at explicit.cpp:681-687; RK1 needs {1}).
 * q_io holds the initial state on entry (ghost cells are filled here by the
 * initial update_bounds, explicit.cpp:712) and the final state on exit.
 * out_R receives R (normalised as run() leaves it), out_qt the last qt.
 */
int ref_run_loop(double* q_io, const double* alpha, int n_alpha, uint64_t max_step,
                 double max_time, double tolerance, uint64_t print_interval,
                 uint64_t* out_step, double* out_time, double* out_R, double* out_qt) {
    mesh& m = *g_mesh;
    const int V = fvhyper::vars;
    std::vector<double> q = vec(q_io, nq());
    std::vector<double> qk(q.size()), qt(q.size()), gx(q.size()), gy(q.size()),
        limiters(q.size()), qmin(q.size()), qmax(q.size()), dt(q.size()),
        q_smooth0(q.size()), q_smooth1(q.size());
    std::vector<double> R0(V), R(V, 1.0);
    uint64_t step = 0;
    double time = 0;
    fvhyper::update_bounds(q, gx, gy, limiters, m);
    while (true) {
        double Rmax = 0.0;
        if (step > 0) {
            for (int i = 0; i < V; ++i) Rmax = std::max(R[i], Rmax);
        } else {
            Rmax = 1.0;
        }
        if ((step >= max_step) | (time >= max_time) | (Rmax < tolerance)) break;
        fvhyper::calc_dt(dt, q, m);
        if (fvhyper::solver::global_dt) fvhyper::min_dt(dt, m);
        for (size_t i = 0; i < q.size(); ++i) qk[i] = q[i];
        for (int s = 0; s < n_alpha; ++s) {
            fvhyper::complete_calc_qt(qt, qk, gx, gy, qmin, qmax, limiters, m, pool());
            if (fvhyper::solver::smooth_residuals) fvhyper::smooth_residuals(qt, q_smooth0, q_smooth1, m);
            fvhyper::update_cells(qk, q, qt, dt, alpha[s]);
            fvhyper::update_bounds(qk, gx, gy, limiters, m);
        }
        for (size_t i = 0; i < q.size(); ++i) q[i] = qk[i];
        if (step == 0) {
            fvhyper::calc_residuals(R0.data(), qt, m, pool());
            for (int i = 0; i < V; ++i) R[i] = R0[i];
        } else if ((step % print_interval == 0) | (tolerance > 1.01e-16)) {
            fvhyper::calc_residuals(R.data(), qt, m, pool());
            for (int i = 0; i < V; ++i) R[i] = R[i] / R0[i];
        }
        step += 1;
        time += dt[0];
    }
    put(q_io, q);
    if (out_step) *out_step = step;
    if (out_time) *out_time = time;
    if (out_R) std::memcpy(out_R, R.data(), V * sizeof(double));
    if (out_qt) put(out_qt, qt);
    return 0;
}

/* fvhyper::run itself (explicit.cpp:657-817): the example's own initial
 * condition and the hard-coded 5-stage scheme.  q_out gets the final state. */
int ref_run(double* q_out, uint64_t max_step, double max_time, double tolerance,
            uint64_t print_interval, int verbose) {
    fvhyper::solverOptions opt;
    opt.max_step = (uint)max_step;
    opt.max_time = max_time;
    opt.tolerance = tolerance;
    opt.print_interval = (uint)print_interval;
    opt.verbose = verbose != 0;
    std::vector<double> q;
    fvhyper::run("ref_run", q, pool(), *g_mesh, opt);
    put(q_out, q);
    return 0;
}

/* The example program's own main() (renamed at compile time), run as is in
 * the caller's working directory: reads its mesh file, prints its log,
 * writes its output files. */
int ref_example_main(void) { return fvref_example_main(); }

}  // extern "C"
