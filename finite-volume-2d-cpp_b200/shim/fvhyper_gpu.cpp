// fvhyper C++ API on the B200 device path (libfvhyper_gpu.a).
//
// Implements the library side of fvhyper's user-facing API with the
// reference's signatures, on top of the C ABI in include/fvgpu.h:
//   mpi_wrapper               fvhyper/parallel.h:24-33 (one process, no MPI)
//   mesh::read_file           fvhyper/mesh.h:193, src/mesh.cpp:800-855
//   run                       fvhyper/explicit.h:175-181, src/explicit.cpp:657-817
//   writeVtk                  fvhyper/post.h:35-42, src/post.cpp:21-200
//   solver::limiter_k_value   src/explicit.cpp:26-28
//
// The user's physics callbacks are ordinary host functions; run() matches
// each one to a device physics kind by evaluating both on probe states and
// requiring identical bits (see identify_* below), then runs the whole time
// loop on the GPU.  Nothing of the step runs on the host.
#include <fvhyper/explicit.h>
#include <fvhyper/post.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>

#include "fvgpu.h"

namespace fvhyper {

namespace solver {
const double limiter_k_value = 7.5;
}

// The Navier-Stokes programs keep their constants in fvhyper::consts
// (examples/flatPlate/main.cpp:30-37, nacaTransient/main.cpp:32-40).  Weak
// references: they bind to the program's definitions and are null in
// programs that define none; the kind they parameterise is still confirmed
// bit for bit on probe states before it is used.
namespace consts {
extern double mu __attribute__((weak));
extern double pr __attribute__((weak));
extern double cp __attribute__((weak));
extern double r __attribute__((weak));
}  // namespace consts

mpi_wrapper::mpi_wrapper() : rank(0), size(1) {}
int mpi_wrapper::exit() { return 0; }

namespace {

[[noreturn]] void fail_rc(int rc, const std::string& what) {
    const std::string msg = what + ": " + fv_last_error();
    if (rc == FV_ERR_MESH || rc == FV_ERR_UNSUPPORTED || rc == FV_ERR_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}
void check(int rc, const char* what) {
    if (rc != FV_OK) fail_rc(rc, what);
}

bool same_bits(double a, double b) { return std::memcmp(&a, &b, sizeof(double)) == 0; }

}  // namespace

// ------------------------------------------------------------------ mesh --

void mesh::attach(::fv_mesh* dm, bool bind_bounds) {
    dev_.reset(dm, [](::fv_mesh* p) { fv_mesh_destroy(p); });
    int64_t sz[5];
    check(fv_mesh_sizes(dm, sz), "fv_mesh_sizes");
    const size_t n_nodes = (size_t)sz[0], n_real = (size_t)sz[1], n_total = (size_t)sz[2];
    const size_t n_edges = (size_t)sz[3], n_bound = (size_t)sz[4];

    nodesX.assign(n_nodes, 0.0);
    nodesY.assign(n_nodes, 0.0);
    std::vector<int32_t> cells4(n_real * 4);
    check(fv_mesh_elements(dm, nodesX.data(), nodesY.data(), cells4.data()), "fv_mesh_elements");

    std::vector<uint32_t> ec(2 * n_edges), en(2 * n_edges), be(n_bound);
    std::vector<int32_t> bg(n_bound);
    edgesNormalsX.assign(n_edges, 0.0);
    edgesNormalsY.assign(n_edges, 0.0);
    edgesLengths.assign(n_edges, 0.0);
    edgesCentersX.assign(n_edges, 0.0);
    edgesCentersY.assign(n_edges, 0.0);
    cellsAreas.assign(n_total, 0.0);
    cellsCentersX.assign(n_total, 0.0);
    cellsCentersY.assign(n_total, 0.0);
    check(fv_mesh_geometry(dm, ec.data(), en.data(), edgesNormalsX.data(), edgesNormalsY.data(),
                           edgesLengths.data(), edgesCentersX.data(), edgesCentersY.data(), cellsAreas.data(),
                           cellsCentersX.data(), cellsCentersY.data(), be.data(), bg.data()),
          "fv_mesh_geometry");
    edgesCells.data().assign(ec.begin(), ec.end());
    edgesNodes.data().assign(en.begin(), en.end());

    // real cells, then one two-node row per ghost (mesh.cpp:645-650)
    std::vector<uint>& cn = cellsNodes.data();
    cn.assign(4 * n_total, 0u);
    cellsIsTriangle.assign(n_total, true);
    for (size_t i = 0; i < n_real; ++i) {
        for (int k = 0; k < 4; ++k) cn[4 * i + k] = cells4[4 * i + k] < 0 ? 0u : (uint)cells4[4 * i + k];
        cellsIsTriangle[i] = cells4[4 * i + 3] < 0;
    }
    for (size_t b = 0; b < n_bound; ++b) {
        const uint n0 = en[2 * be[b]], n1 = en[2 * be[b] + 1];
        cn[4 * (n_real + b)] = std::min(n0, n1);
        cn[4 * (n_real + b) + 1] = std::max(n0, n1);
    }
    cellsIsGhost.assign(n_real, false);
    nRealCells = (uint)n_real;

    physicalNames.clear();
    const int ng = fv_mesh_group_count(dm);
    for (int g = 0; g < ng; ++g) {
        char buf[256];
        check(fv_mesh_group_name(dm, g, buf, (int32_t)sizeof(buf)), "fv_mesh_group_name");
        physicalNames[(uint)g] = buf;
    }
    boundaryEdges.assign(be.begin(), be.end());
    boundaryEdgesIntTag.assign(bg.begin(), bg.end());
    boundaryFuncs.clear();
    if (bind_bounds) {
        for (size_t b = 0; b < n_bound; ++b) {
            const std::string& nm = physicalNames[(uint)bg[b]];
            if (boundaries::bounds.find(nm) == boundaries::bounds.end())
                throw std::invalid_argument("Physical name " + nm + " of tag " + std::to_string(bg[b]) +
                                            " not in mesh");
            boundaryFuncs.push_back(boundaries::bounds.at(nm));
        }
    }
}

void mesh::read_file(std::string name, mpi_wrapper& pool) {
    filename = (pool.size > 1) ? (name + "_" + std::to_string(pool.rank + 1) + ".msh") : name + ".msh";
    ::fv_mesh* dm = nullptr;
    int rc;
    // B200 build: without <name>.msh, an SU2 mesh <name>.su2 is read instead
    // (marker tags are the boundary names)
    const std::string su2 = name + ".su2";
    if (!std::ifstream(filename).good() && std::ifstream(su2).good()) {
        filename = su2;
        rc = fv_mesh_read_su2(filename.c_str(), &dm);
    } else {
        rc = fv_mesh_read_msh(filename.c_str(), &dm);
    }
    if (rc != FV_OK) fail_rc(rc, "mesh::read_file(" + filename + ")");
    attach(dm, true);
}

std::vector<std::string> cut_str(const std::string s, const char c) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        if (ch == c) {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur.push_back(ch);
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

std::vector<uint> str_to_ints(std::string s) {
    std::vector<uint> out;
    for (const std::string& w : cut_str(s, ' ')) out.push_back((uint)std::stoul(w));
    return out;
}

// ------------------------------------------------- physics identification --
namespace {

struct Probe {
    std::mt19937_64 rng{0x5eedf00dull};
    double uni(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }
    // an Euler state with rho, p > 0 for any gamma in (1, 2]
    void euler(double* q, double gamma, double mach_max = 1.8) {
        const double rho = uni(0.2, 2.0), p = uni(0.2, 2.0);
        const double c = std::sqrt(gamma * p / rho);
        const double m = uni(0.0, mach_max), th = uni(0.0, 6.283185307179586);
        const double u = m * c * std::cos(th), v = m * c * std::sin(th);
        q[0] = rho; q[1] = rho * u; q[2] = rho * v;
        q[3] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v);
    }
    void normal(double* n) {
        const double th = uni(0.0, 6.283185307179586);
        n[0] = std::cos(th); n[1] = std::sin(th);
    }
};

const char* flux_name(int k) {
    return k == FV_FLUX_ROE_FS ? "roe (forwardStep operand order)"
           : k == FV_FLUX_ROE_ST ? "roe (shockTube/naca operand order)"
           : k == FV_FLUX_DIFFUSION ? "diffusion"
           : k == FV_FLUX_NS ? "navier-stokes" : "upwind advection";
}

// gamma of an Euler-type calc_flux from a fluid at rest: f[1] = p = gamma-1
// for q = (1, 0, 0, 1), n = (1, 0), zero face gradients.
double rest_state_gamma() {
    double zg[4] = {0, 0, 0, 0}, q0[4] = {1.0, 0.0, 0.0, 1.0}, n0[2] = {1.0, 0.0}, f0[4] = {0, 0, 0, 0};
    calc_flux(f0, q0, q0, zg, zg, n0);
    const double g = f0[1] + 1.0;
    if (!(g > 1.0 && g <= 3.0))
        throw std::invalid_argument("fvhyper GPU: calc_flux is not an Euler flux (rest-state pressure test)");
    return g;
}

// A calc_flux that reads the face gradient (diffusive_gradients) -> the
// diffusion kind (vars = 1) or the Navier-Stokes kind (vars = 4, constants
// from fvhyper::consts); 256 random states and face gradients must agree
// bit for bit with the kind's host copy.
void identify_diffusive_flux(int V, fv_physics* ph) {
    if (V == 1) {
        ph->flux = FV_FLUX_DIFFUSION;
        ph->gamma = 1.4;
    } else if (V == 2) {
        ph->flux = FV_FLUX_BURGERS_DIFF;
        ph->gamma = 1.4;
    } else if (V == 4) {
        if (!&consts::mu || !&consts::pr || !&consts::cp || !&consts::r)
            throw std::invalid_argument("fvhyper GPU: a vars = 4 calc_flux with diffusive_gradients runs as the "
                                        "Navier-Stokes kind, whose constants are read from fvhyper::consts::mu, "
                                        "pr, cp and r; the program defines no such constants");
        ph->flux = FV_FLUX_NS;
        ph->gamma = rest_state_gamma();
        ph->mu = consts::mu; ph->pr = consts::pr; ph->cp = consts::cp; ph->r = consts::r;
    } else {
        throw std::invalid_argument("fvhyper GPU: diffusive_gradients with vars = " + std::to_string(V) +
                                    " matches no device kind (vars = 1 diffusion, vars = 2 Burgers-diffusion, "
                                    "vars = 4 Navier-Stokes)");
    }
    Probe pr;
    for (int t = 0; t < 256; ++t) {
        double qi[4] = {0, 0, 0, 0}, qj[4] = {0, 0, 0, 0}, gx[4], gy[4], n[2];
        if (V == 4) { pr.euler(qi, ph->gamma); pr.euler(qj, ph->gamma); }
        else for (int k = 0; k < V; ++k) { qi[k] = pr.uni(-2, 2); qj[k] = pr.uni(-2, 2); }
        for (int k = 0; k < 4; ++k) { gx[k] = pr.uni(-5, 5); gy[k] = pr.uni(-5, 5); }
        pr.normal(n);
        double fu[4] = {0, 0, 0, 0}, fk[4] = {0, 0, 0, 0};
        calc_flux(fu, qi, qj, gx, gy, n);
        fv_kind_flux_grad(ph, qi, qj, gx, gy, n, fk);
        for (int c = 0; c < V; ++c)
            if (!same_bits(fu[c], fk[c]))
                throw std::invalid_argument(std::string("fvhyper GPU: calc_flux (diffusive_gradients) is not the ") +
                                            (V == 1   ? "diffusion flux -grad(u).n of examples/heatTransfer"
                                             : V == 2 ? "Burgers-diffusion flux of tests/tests.cpp"
                                                      : "Navier-Stokes flux of examples/flatPlate") +
                                            "; no device kind matches it");
    }
}

// calc_flux -> (kind, gamma).  gamma from the rest state, then 256 random
// state pairs must agree bit for bit.
void identify_flux(int V, int32_t* kind, double* gamma) {
    double zg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    Probe pr;
    if (V == 1)
        throw std::invalid_argument("fvhyper GPU: vars = 1 runs the diffusion kind only (diffusive_gradients)");
    if (V == 2) {
        for (int t = 0; t < 256; ++t) {
            double qi[2] = {pr.uni(-2, 2), pr.uni(-2, 2)}, qj[2] = {pr.uni(-2, 2), pr.uni(-2, 2)}, n[2];
            pr.normal(n);
            double fu[2] = {0, 0}, fk[2] = {0, 0};
            calc_flux(fu, qi, qj, zg, zg, n);
            fv_kind_flux(FV_FLUX_BURGERS, 0.0, qi, qj, n, fk);
            if (!same_bits(fu[0], fk[0]) || !same_bits(fu[1], fk[1]))
                throw std::invalid_argument("fvhyper GPU: calc_flux (vars = 2) is not the upwind advection flux "
                                            "of examples/burgers; no device kind matches it");
        }
        *kind = FV_FLUX_BURGERS;
        *gamma = 1.4;
        return;
    }
    if (V != 4) throw std::invalid_argument("fvhyper GPU: vars must be 1, 2 or 4");
    const double g = rest_state_gamma();
    for (int k : {FV_FLUX_ROE_FS, FV_FLUX_ROE_ST}) {
        Probe p2;
        bool ok = true;
        for (int t = 0; t < 256 && ok; ++t) {
            double qi[4], qj[4], n[2];
            p2.euler(qi, g);
            p2.euler(qj, g);
            p2.normal(n);
            double fu[4] = {0, 0, 0, 0}, fk[4] = {0, 0, 0, 0};
            calc_flux(fu, qi, qj, zg, zg, n);
            fv_kind_flux(k, g, qi, qj, n, fk);
            for (int c = 0; c < 4; ++c) ok = ok && same_bits(fu[c], fk[c]);
        }
        if (ok) {
            *kind = k;
            *gamma = g;
            return;
        }
    }
    throw std::invalid_argument("fvhyper GPU: calc_flux matches no device flux kind (Roe with the cures "
                                "eigenvalues, examples/forwardStep or examples/shockTube form)");
}

int32_t identify_limiter() {
    std::vector<double> ys = {-3.0, -1.0, -0.25, 0.0, 1e-3, 0.3, 0.5, 0.99, 1.0, 1.5, 1.999, 2.0, 2.5, 7.0};
    Probe pr;
    for (int t = 0; t < 128; ++t) ys.push_back(pr.uni(-4.0, 6.0));
    for (int k : {FV_LIM_MICHALAK, FV_LIM_VENKAT, FV_LIM_MINMOD, FV_LIM_ZERO}) {
        bool ok = true;
        for (double y : ys) {
            double want = 0.0;
            fv_kind_limiter(k, y, &want);
            ok = ok && same_bits(limiter_func(y), want);
        }
        if (ok) return k;
    }
    throw std::invalid_argument("fvhyper GPU: limiter_func matches no device limiter kind (Michalak y_t = 2, "
                                "Venkatakrishnan, minmod, zero)");
}

// boundaries::bounds entry -> (kind, bv).  bv is read back from a supersonic
// inflow state (b = boundary state), then random sub/supersonic in/outflow
// states must agree bit for bit.
void identify_bc(const std::string& name, void (*fn)(double*, double*, double*), int V, double gamma,
                 int32_t* kind, double* bv) {
    std::vector<int> kinds = {FV_BC_COPY};
    if (V == 2) kinds.push_back(FV_BC_TANGENT);
    if (V == 4) {
        kinds.push_back(FV_BC_WALL);
        kinds.push_back(FV_BC_NOSLIP);
        double q[4], n[2] = {0.6, 0.8};
        const double u = -3.0;
        q[0] = 1.0; q[1] = u * n[0]; q[2] = u * n[1];
        q[3] = 1.0 / (gamma - 1.0) + 0.5 * (q[1] * q[1] + q[2] * q[2]);
        double b[4] = {0, 0, 0, 0};
        fn(b, q, n);
        for (int k = 0; k < 4; ++k) bv[k] = b[k];
        if (b[0] > 0.0) {
            kinds.push_back(FV_BC_INLET_OUTLET);
            kinds.push_back(FV_BC_FARFIELD);
            kinds.push_back(FV_BC_FARFIELD_B0);
        }
    } else {
        for (int k = 0; k < 4; ++k) bv[k] = 0.0;
    }
    for (int k : kinds) {
        Probe pr;
        bool ok = true;
        for (int t = 0; t < 256 && ok; ++t) {
            double q[4] = {0, 0, 0, 0}, n[2];
            if (V == 4) pr.euler(q, gamma, 2.5);
            else for (int c = 0; c < V; ++c) q[c] = pr.uni(-2, 2);
            pr.normal(n);
            double bu[4] = {0, 0, 0, 0}, bk[4] = {0, 0, 0, 0};
            double qc[4] = {q[0], q[1], q[2], q[3]}, nc[2] = {n[0], n[1]};
            fn(bu, qc, nc);
            fv_kind_bc(k, V, gamma, bv, q, n, bk);
            for (int c = 0; c < V; ++c) ok = ok && same_bits(bu[c], bk[c]);
        }
        if (ok) {
            *kind = k;
            if (k == FV_BC_COPY || k == FV_BC_WALL || k == FV_BC_NOSLIP)
                for (int c = 0; c < 4; ++c) bv[c] = 0.0;
            return;
        }
    }
    throw std::invalid_argument("fvhyper GPU: boundary function \"" + name +
                                "\" matches no device boundary kind (copy, wall, no-slip wall, inlet_outlet, "
                                "farfield, farfield with b[0] tangential momentum, tangent)");
}

// A small jittered triangle mesh for probing calc_dt (the user function only
// reads the mesh arrays).
::fv_mesh* probe_mesh() {
    const int nx = 7, ny = 5;
    Probe pr;
    std::vector<double> x, y;
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            const bool edge = i == 0 || j == 0 || i == nx || j == ny;
            x.push_back(i + (edge ? 0.0 : pr.uni(-0.2, 0.2)));
            y.push_back(0.8 * j + (edge ? 0.0 : pr.uni(-0.15, 0.15)));
        }
    auto id = [&](int i, int j) { return (int32_t)(j * (nx + 1) + i); };
    std::vector<int32_t> cells;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            if ((i + j) % 3 == 0) {  // a few quads among the triangles
                cells.insert(cells.end(), {id(i, j), id(i + 1, j), id(i + 1, j + 1), id(i, j + 1)});
            } else {
                cells.insert(cells.end(), {id(i, j), id(i + 1, j), id(i + 1, j + 1), -1});
                cells.insert(cells.end(), {id(i, j), id(i + 1, j + 1), id(i, j + 1), -1});
            }
        }
    std::vector<int32_t> bn, bgp;
    for (int i = 0; i < nx; ++i) { bn.insert(bn.end(), {id(i, 0), id(i + 1, 0)}); bn.insert(bn.end(), {id(i + 1, ny), id(i, ny)}); }
    for (int j = 0; j < ny; ++j) { bn.insert(bn.end(), {id(nx, j), id(nx, j + 1)}); bn.insert(bn.end(), {id(0, j + 1), id(0, j)}); }
    bgp.assign(bn.size() / 2, 0);
    ::fv_mesh* m = nullptr;
    check(fv_mesh_create((int64_t)x.size(), x.data(), y.data(), (int64_t)cells.size() / 4, cells.data(),
                         (int64_t)bgp.size(), bn.data(), bgp.data(), 1, &m),
          "probe mesh");
    return m;
}

int choose_precision(int requested) {
    if (requested >= 0) return requested;
    const char* e = std::getenv("FVGPU_PRECISION");
    if (!e || !*e) return FV_PREC_FP64_EXACT;
    const std::string s(e);
    if (s == "fp64_exact") return FV_PREC_FP64_EXACT;
    if (s == "fp64") return FV_PREC_FP64;
    if (s == "fp32") return FV_PREC_FP32;
    throw std::invalid_argument("FVGPU_PRECISION must be fp64_exact, fp64 or fp32 (got " + s + ")");
}

int choose_device(int requested) {
    if (requested >= 0) return requested;
    const char* e = std::getenv("FVGPU_DEVICE");
    return (e && *e) ? std::atoi(e) : 0;
}

struct SolverHandle {
    ::fv_solver* s = nullptr;
    ~SolverHandle() { if (s) fv_solver_destroy(s); }
};

// The last run()'s solver and the device output kinds of the post::
// callbacks.  writeVtk evaluates a callback whose results match a device
// output kind bit for bit on probe states with fv_output_fields, on the
// device; a callback that matches none runs on the host.  The solver is kept
// until the next run() (and, deliberately, not destroyed at process exit,
// when the CUDA runtime may already be gone).
struct OutputState {
    ::fv_solver* solver = nullptr;
    int V = 0;
    int64_t n_real = 0, n_total = 0;
    std::map<std::string, int> kinds;  // "s:" / "v:" + callback name -> FV_OUT_* or 0
};
OutputState& out_state() {
    static OutputState* o = new OutputState();
    return *o;
}

int identify_output(void (*fn)(double*, double*), bool vector, int V, double gamma) {
    const int cands[2] = {vector ? FV_OUT_VELOCITY : FV_OUT_PRESSURE, vector ? FV_OUT_STATE01 : FV_OUT_MACH};
    for (int k : cands) {
        if ((k == FV_OUT_STATE01 && V < 2) || (k != FV_OUT_STATE01 && V != 4)) continue;
        Probe pr;
        bool ok = true;
        for (int t = 0; t < 64 && ok; ++t) {
            double q[4] = {0., 0., 0., 0.};
            if (V == 4) pr.euler(q, gamma);
            else for (int i = 0; i < V && i < 4; ++i) q[i] = pr.uni(-2.0, 2.0);
            double a[2] = {0., 0.}, b[2] = {0., 0.};
            fn(a, q);
            const int nc = fv_kind_output(k, gamma, q, b);
            ok = nc > 0 && std::memcmp(a, b, sizeof(double) * (size_t)nc) == 0;
        }
        if (ok) return k;
    }
    return 0;
}

// calc_dt -> (dt_kind, cfl, dt_const) on the probe mesh: the user's dt over
// random states against the device's fv_stage_dt (FP64_EXACT), bit for bit.
// cfl is recovered from the ratio to a cfl = 1 run, rounded to 12 significant
// digits, and confirmed by a second device run.
void identify_dt(fv_physics ph, int device, int32_t* dt_kind, double* cfl, double* dt_const) {
    mesh pm;
    pm.attach(probe_mesh(), false);
    const int V = ph.V;
    const size_t nt = pm.cellsAreas.size();
    std::vector<double> q(V * nt), dtu(V * nt, 0.0);
    Probe pr;
    for (size_t i = 0; i < nt; ++i) {
        if (V == 4) pr.euler(&q[4 * i], ph.gamma);
        else for (int k = 0; k < V; ++k) q[V * i + k] = pr.uni(-2, 2);
    }
    calc_dt(dtu, q, pm);
    for (size_t i = 0; i < nt; ++i)
        for (int k = 1; k < V; ++k)
            if (!same_bits(dtu[V * i + k], dtu[V * i]))
                throw std::invalid_argument("fvhyper GPU: calc_dt gives different time steps to the variables "
                                            "of one cell; the device keeps one dt per cell");
    std::vector<double> du(nt);
    for (size_t i = 0; i < nt; ++i) du[i] = dtu[V * i];
    bool all_same = true;
    for (size_t i = 1; i < nt; ++i) all_same = all_same && same_bits(du[i], du[0]);
    if (all_same) {
        *dt_kind = FV_DT_CONST;
        *cfl = 0.0;
        *dt_const = du[0];
        return;
    }
    if (V != 4)
        throw std::invalid_argument("fvhyper GPU: calc_dt (vars = " + std::to_string(V) +
                                    ") must be a constant time step");
    const int32_t group_bc[1] = {FV_BC_COPY};
    const double group_bv[4] = {0, 0, 0, 0};
    ph.n_groups = 1;
    ph.group_bc = group_bc;
    ph.group_bv = group_bv;
    ph.order2 = 0;
    auto device_dt = [&](int32_t kind, double c, std::vector<double>& out) {
        ph.dt_kind = kind;
        ph.cfl = c;
        SolverHandle h;
        check(fv_solver_create(pm.device_mesh(), &ph, FV_PREC_FP64_EXACT, device, &h.s), "probe solver");
        out.assign(nt, 0.0);
        std::vector<double> qq(q);
        check(fv_stage_dt(h.s, qq.data(), out.data(), 0), "fv_stage_dt (probe)");
    };
    std::vector<int32_t> kinds = {FV_DT_CFL_SUM, FV_DT_CFL_MIN_SIGNED};
    if (ph.flux == FV_FLUX_NS) kinds = {FV_DT_VISC_MIN, FV_DT_VISC_SUM, FV_DT_CFL_SUM, FV_DT_CFL_MIN_SIGNED};
    for (int32_t kind : kinds) {
        std::vector<double> d1;
        device_dt(kind, 1.0, d1);
        double ratio = 0.0;
        for (size_t i = 0; i < nt && ratio == 0.0; ++i)
            if (d1[i] > 0.0 && d1[i] < 1.0 && std::isfinite(du[i])) ratio = du[i] / d1[i];
        if (!(ratio > 0.0) || !std::isfinite(ratio)) continue;
        char buf[64];
        std::snprintf(buf, sizeof(buf), "%.12g", ratio);
        const double c = std::strtod(buf, nullptr);
        std::vector<double> dc;
        device_dt(kind, c, dc);
        bool ok = true;
        for (size_t i = 0; i < nt && ok; ++i) ok = same_bits(dc[i], du[i]);
        if (ok) {
            *dt_kind = kind;
            *cfl = c;
            *dt_const = 0.0;
            return;
        }
    }
    throw std::invalid_argument("fvhyper GPU: calc_dt matches no device time-step kind (constant, CFL over the "
                                "edge sum as examples/forwardStep, CFL edge minimum as examples/naca, viscous "
                                "minimum as examples/flatPlate, viscous sum as examples/nacaTransient)");
}

struct PrintCtx {
    std::chrono::steady_clock::time_point begin;
    bool verbose;
    int V;
};

double seconds_since(std::chrono::steady_clock::time_point b) {
    const auto us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - b).count();
    return ((double)(int)us) / 1e6;
}

// log line of explicit.cpp:765-785 (step 0 prints "1.0" for every R)
void on_print(void* user, uint64_t step, double time, const double* R, int32_t V) {
    const PrintCtx* c = static_cast<const PrintCtx*>(user);
    if (!c->verbose) return;
    std::cout << (uint)step << ", " << time << ", " << seconds_since(c->begin) << ", ";
    for (int i = 0; i < V; ++i) {
        if (step == 0) std::cout << "1.0";
        else std::cout << R[i];
        if (i < V - 1) std::cout << ", ";
    }
    std::cout << std::endl;
}

}  // namespace

// ------------------------------------------------------------------- run --

void run(const std::string name, std::vector<double>& q, mpi_wrapper& pool, mesh& m, solverOptions& opt) {
    if (!m.device_mesh()) throw std::invalid_argument("fvhyper GPU: run() needs a mesh from mesh::read_file");
    const int V = vars;
    q.resize((size_t)V * m.cellsAreas.size());
    generate_initial_solution(q, m);

    const bool D = solver::diffusive_gradients;
    const bool o2 = solver::do_calc_gradients && solver::do_calc_limiters && solver::linear_interpolate;
    const bool o1 = !solver::do_calc_gradients && !solver::do_calc_limiters && !solver::linear_interpolate && !D;
    // gradients for the viscous face gradient only, cell values as face states
    const bool dg = solver::do_calc_gradients && !solver::do_calc_limiters && !solver::linear_interpolate && D;
    if (!o1 && !o2 && !dg)
        throw std::invalid_argument("fvhyper GPU: the device runs first order (no gradients, limiters or "
                                    "interpolation), second order (all three) or gradients for the diffusive "
                                    "fluxes alone (with diffusive_gradients); this flag mix is none of them");

    const int precision = choose_precision(opt.precision);
    const int device = choose_device(opt.device);

    fv_physics ph;
    std::memset(&ph, 0, sizeof(ph));
    ph.V = V;
    if (D) identify_diffusive_flux(V, &ph);
    else identify_flux(V, &ph.flux, &ph.gamma);
    ph.order2 = o2 ? 1 : 0;
    ph.diffusive = D ? 1 : 0;
    if (solver::smooth_residuals && ph.flux != FV_FLUX_BURGERS_DIFF)
        throw std::invalid_argument("fvhyper GPU: smooth_residuals runs on the device with the Burgers-diffusion "
                                    "kind only (the physics of tests/tests.cpp)");
    ph.smooth_residuals = solver::smooth_residuals ? 1 : 0;
    ph.limiter = o2 ? identify_limiter() : FV_LIM_ZERO;
    ph.K = solver::limiter_k_value;
    ph.global_dt = solver::global_dt ? 1 : 0;
    identify_dt(ph, device, &ph.dt_kind, &ph.cfl, &ph.dt_const);

    const int ng = (int)m.physicalNames.size();
    std::vector<int32_t> group_bc(std::max(ng, 1), FV_BC_COPY);
    std::vector<double> group_bv(4 * std::max(ng, 1), 0.0);
    for (int g = 0; g < ng; ++g) {
        const std::string& nm = m.physicalNames[(uint)g];
        auto it = boundaries::bounds.find(nm);
        if (it == boundaries::bounds.end())
            throw std::invalid_argument("Physical name " + nm + " of tag " + std::to_string(g) + " not in mesh");
        identify_bc(nm, it->second, V, ph.gamma, &group_bc[g], &group_bv[4 * g]);
    }
    ph.n_groups = ng;
    ph.group_bc = group_bc.data();
    ph.group_bv = group_bv.data();
    ph.positivity_guard = 0;

    OutputState& os = out_state();
    if (os.solver) { fv_solver_destroy(os.solver); os.solver = nullptr; }
    os.V = V;
    os.n_real = m.nRealCells;
    os.n_total = (int64_t)m.cellsAreas.size();
    os.kinds.clear();
    for (auto& kv : post::extra_scalars) os.kinds["s:" + kv.first] = identify_output(kv.second, false, V, ph.gamma);
    for (auto& kv : post::extra_vectors) os.kinds["v:" + kv.first] = identify_output(kv.second, true, V, ph.gamma);
    check(fv_solver_create(m.device_mesh(), &ph, precision, device, &os.solver), "fv_solver_create");
    ::fv_solver* const hs = os.solver;
    check(fv_set_state(hs, q.data()), "fv_set_state");

    // RK5 stage coefficients (explicit.cpp:681-687)
    const double alpha[5] = {0.0695, 0.1602, 0.2898, 0.506, 1.};
    const bool verbose = opt.verbose && pool.rank == 0;
    if (verbose) {
        std::cout << "Step, Time, RealTime, ";
        for (int i = 0; i < V; ++i) {
            std::cout << "R(q[" << i << "])";
            if (i < V - 1) std::cout << ", ";
        }
        std::cout << std::endl;
    }
    PrintCtx pc{std::chrono::steady_clock::now(), verbose, V};

    fv_run_options ro;
    std::memset(&ro, 0, sizeof(ro));
    ro.max_step = opt.max_step;
    ro.tolerance = opt.tolerance;
    ro.print_interval = opt.print_interval;
    ro.n_alpha = 5;
    ro.alpha = alpha;
    ro.on_print = on_print;
    ro.user = &pc;
    fv_run_info info;
    std::memset(&info, 0, sizeof(info));

    double save_time = opt.time_series_interval;
    uint time_step = 0;
    ro.restart = 1;
    for (;;) {
        // Run until a stop criterion, or until the first step that starts
        // with time > save_time (explicit.cpp:789-797): that step is taken
        // alone and the state after it is saved.
        ro.max_step = opt.max_step;
        ro.max_time = opt.max_time;
        if (opt.save_time_series) ro.max_time = std::min(opt.max_time, std::nextafter(save_time, INFINITY));
        check(fv_run(hs, &ro, &info), "fv_run");
        ro.restart = 0;
        if (!opt.save_time_series) break;
        ro.max_time = opt.max_time;
        ro.max_step = std::min<uint64_t>(opt.max_step, info.step + 1);
        if (ro.max_step <= info.step) break;
        const uint64_t before = info.step;
        check(fv_run(hs, &ro, &info), "fv_run");
        if (info.step == before) break;
        check(fv_get_state(hs, q.data()), "fv_get_state");
        writeVtk(name, q, m, pool.rank, pool.size, std::to_string(time_step));
        save_time += opt.time_series_interval;
        time_step += 1;
    }
    check(fv_get_state(hs, q.data()), "fv_get_state");

    if (verbose) {
        std::cout << (uint)info.step << ", " << info.time << ", " << seconds_since(pc.begin) << ", ";
        for (int i = 0; i < V; ++i) {
            std::cout << info.R[i];
            if (i < V - 1) std::cout << ", ";
        }
        std::cout << std::endl;
    }
}

// -------------------------------------------------------------- writeVtk --
namespace {

// The post:: extra fields of the real cells, in the callbacks' map order:
// scalars (N values), then vectors (N pairs).  Callbacks identified with a
// device output kind are evaluated on the device by the last run's solver
// (FVGPU_POST=host evaluates every callback on the host instead).
struct Extras {
    std::vector<std::vector<double>> scalars, vectors;
};
Extras extra_fields(std::vector<double>& q, mesh& m) {
    const size_t nv = var_names.size();
    const uint N = m.nRealCells;
    Extras ex;
    const OutputState& os = out_state();
    const char* pe = std::getenv("FVGPU_POST");
    const bool host_only = pe && std::string(pe) == "host";
    const int64_t nq = nv ? (int64_t)(q.size() / nv) : 0;
    const bool device = !host_only && os.solver && os.V == (int)nv && os.n_real == (int64_t)N &&
                        (nq == os.n_real || nq == os.n_total);
    auto kind_of = [&](const std::string& key) {
        auto it = os.kinds.find(key);
        return (device && it != os.kinds.end()) ? it->second : 0;
    };
    std::vector<int32_t> kinds;
    for (auto& kv : post::extra_scalars) if (int k = kind_of("s:" + kv.first)) kinds.push_back(k);
    for (auto& kv : post::extra_vectors) if (int k = kind_of("v:" + kv.first)) kinds.push_back(k);
    std::vector<double> dev;
    if (!kinds.empty()) {
        size_t total = 0;
        for (int k : kinds) total += (k == FV_OUT_VELOCITY || k == FV_OUT_STATE01 ? 2 : 1) * (size_t)N;
        dev.resize(total);
        check(fv_output_fields(os.solver, q.data(), nq, (int32_t)kinds.size(), kinds.data(), dev.data()),
              "fv_output_fields");
    }
    size_t off = 0;
    for (auto& kv : post::extra_scalars) {
        std::vector<double> col(N);
        if (kind_of("s:" + kv.first)) {
            std::copy(dev.begin() + (long)off, dev.begin() + (long)(off + N), col.begin());
            off += N;
        } else {
            for (uint c = 0; c < N; ++c) {
                double v[1];
                kv.second(v, &q[nv * c]);
                col[c] = v[0];
            }
        }
        ex.scalars.push_back(std::move(col));
    }
    for (auto& kv : post::extra_vectors) {
        std::vector<double> vec(2 * (size_t)N);
        if (kind_of("v:" + kv.first)) {
            std::copy(dev.begin() + (long)off, dev.begin() + (long)(off + 2 * (size_t)N), vec.begin());
            off += 2 * (size_t)N;
        } else {
            for (uint c = 0; c < N; ++c) {
                double v[2];
                kv.second(v, &q[nv * c]);
                vec[2 * c] = v[0]; vec[2 * c + 1] = v[1];
            }
        }
        ex.vectors.push_back(std::move(vec));
    }
    return ex;
}

// the reference's ASCII layout, byte for byte (fvhyper/src/post.cpp:21-200)
std::string vtu_ascii(std::vector<double>& q, mesh& m, int rank, const Extras& ex) {
    const size_t nv = var_names.size();
    const uint N = m.nRealCells;
    std::string s;
    s.reserve((size_t)N * 64 * (4 + nv));
    s += "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"BigEndian\">\n";
    s += "  <UnstructuredGrid>\n";
    s += "    <Piece NumberOfPoints=\"" + std::to_string(m.nodesX.size()) + "\" NumberOfCells=\"" +
         std::to_string(N) + "\">\n";
    s += "      <Points>\n";
    s += "        <DataArray type=\"Float32\" NumberOfComponents=\"3\" Format=\"ascii\">\n";
    for (size_t i = 0; i < m.nodesX.size(); ++i)
        s += "          " + std::to_string(m.nodesX[i]) + " " + std::to_string(m.nodesY[i]) + " 0.0\n";
    s += "        </DataArray>\n";
    s += "      </Points>\n";
    s += "      <Cells>\n";
    s += "        <DataArray type=\"Int32\" Name=\"connectivity\" Format=\"ascii\">\n";
    s += "          ";
    for (uint c = 0; c < N; ++c) {
        const int nn = m.cellsIsTriangle[c] ? 3 : 4;
        for (int k = 0; k < nn; ++k) s += std::to_string(m.cellsNodes(c, k)) + "  ";
        s += "\n          ";
    }
    s += "        </DataArray>\n";
    s += "        <DataArray type=\"Int32\" Name=\"offsets\" Format=\"ascii\">\n";
    s += "          ";
    uint off = 0;
    for (uint c = 0; c < N; ++c) {
        off += m.cellsIsTriangle[c] ? 3 : 4;
        s += std::to_string(off) + "  ";
    }
    s += "\n";
    s += "        </DataArray>\n";
    s += "        <DataArray type=\"Int32\" Name=\"types\" Format=\"ascii\">\n";
    s += "          ";
    for (uint c = 0; c < N; ++c) s += m.cellsIsTriangle[c] ? "5  " : "9  ";
    s += "\n";
    s += "        </DataArray>\n";
    s += "      </Cells>\n";
    s += "      <CellData Scalars=\"scalars\">\n";
    s += "        <DataArray type=\"Float32\" Name=\"rank\" Format=\"ascii\">\n";
    const std::string rank_line = "          " + std::to_string(rank) + "\n";
    for (uint c = 0; c < N; ++c) s += rank_line;
    s += "        </DataArray>\n";
    for (size_t i = 0; i < nv; ++i) {
        s += "        <DataArray type=\"Float32\" Name=\"" + var_names[i] + "\" Format=\"ascii\">\n";
        for (uint c = 0; c < N; ++c) s += "          " + std::to_string(q[nv * c + i]) + "\n";
        s += "        </DataArray>\n";
    }
    size_t f = 0;
    for (auto& kv : post::extra_scalars) {
        s += "        <DataArray type=\"Float32\" Name=\"" + kv.first + "\" Format=\"ascii\">\n";
        const std::vector<double>& col = ex.scalars[f++];
        for (uint c = 0; c < N; ++c) s += "          " + std::to_string(col[c]) + "\n";
        s += "        </DataArray>\n";
    }
    f = 0;
    for (auto& kv : post::extra_vectors) {
        s += "        <DataArray type=\"Float32\" Name=\"" + kv.first +
             "\" NumberOfComponents=\"3\" Format=\"ascii\">\n";
        const std::vector<double>& vec = ex.vectors[f++];
        for (uint c = 0; c < N; ++c) {
            s += "          " + std::to_string(vec[2 * c]) + " ";
            s += std::to_string(vec[2 * c + 1]) + " 0.0\n";
        }
        s += "        </DataArray>\n";
    }
    s += "      </CellData>\n";
    s += "    </Piece>\n";
    s += "  </UnstructuredGrid>\n";
    s += "</VTKFile>";
    return s;
}

// VTK XML, raw appended data: each block is a UInt64 byte count + the bytes.
struct Appended {
    std::string xml, data;
    template <class T>
    void array(const std::string& attrs, const std::vector<T>& v, const std::string& indent) {
        xml += indent + "<DataArray " + attrs + " format=\"appended\" offset=\"" + std::to_string(data.size()) +
               "\"/>\n";
        const uint64_t nb = (uint64_t)v.size() * sizeof(T);
        data.append(reinterpret_cast<const char*>(&nb), sizeof(nb));
        data.append(reinterpret_cast<const char*>(v.data()), (size_t)nb);
    }
};

std::string vtu_binary(std::vector<double>& q, mesh& m, int rank, const Extras& ex) {
    const size_t nv = var_names.size();
    const uint N = m.nRealCells;
    Appended a;
    a.xml += "<?xml version=\"1.0\"?>\n";
    a.xml += "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    a.xml += "  <UnstructuredGrid>\n";
    a.xml += "    <Piece NumberOfPoints=\"" + std::to_string(m.nodesX.size()) + "\" NumberOfCells=\"" +
             std::to_string(N) + "\">\n";
    a.xml += "      <Points>\n";
    {
        std::vector<double> p(3 * m.nodesX.size());
        for (size_t i = 0; i < m.nodesX.size(); ++i) { p[3 * i] = m.nodesX[i]; p[3 * i + 1] = m.nodesY[i]; p[3 * i + 2] = 0.0; }
        a.array("type=\"Float64\" NumberOfComponents=\"3\"", p, "        ");
    }
    a.xml += "      </Points>\n";
    a.xml += "      <Cells>\n";
    {
        std::vector<int32_t> conn, offs;
        std::vector<uint8_t> types;
        conn.reserve((size_t)N * 3);
        offs.reserve(N);
        types.reserve(N);
        for (uint c = 0; c < N; ++c) {
            const int nn = m.cellsIsTriangle[c] ? 3 : 4;
            for (int k = 0; k < nn; ++k) conn.push_back((int32_t)m.cellsNodes(c, k));
            offs.push_back((int32_t)conn.size());
            types.push_back(nn == 3 ? 5 : 9);
        }
        a.array("type=\"Int32\" Name=\"connectivity\"", conn, "        ");
        a.array("type=\"Int32\" Name=\"offsets\"", offs, "        ");
        a.array("type=\"UInt8\" Name=\"types\"", types, "        ");
    }
    a.xml += "      </Cells>\n";
    a.xml += "      <CellData Scalars=\"scalars\">\n";
    a.array("type=\"Float32\" Name=\"rank\"", std::vector<float>(N, (float)rank), "        ");
    std::vector<double> col(N);
    for (size_t i = 0; i < nv; ++i) {
        for (uint c = 0; c < N; ++c) col[c] = q[nv * c + i];
        a.array("type=\"Float64\" Name=\"" + var_names[i] + "\"", col, "        ");
    }
    size_t f = 0;
    for (auto& kv : post::extra_scalars)
        a.array("type=\"Float64\" Name=\"" + kv.first + "\"", ex.scalars[f++], "        ");
    f = 0;
    for (auto& kv : post::extra_vectors) {
        const std::vector<double>& v2 = ex.vectors[f++];
        std::vector<double> vec(3 * (size_t)N);
        for (uint c = 0; c < N; ++c) { vec[3 * c] = v2[2 * c]; vec[3 * c + 1] = v2[2 * c + 1]; vec[3 * c + 2] = 0.0; }
        a.array("type=\"Float64\" Name=\"" + kv.first + "\" NumberOfComponents=\"3\"", vec, "        ");
    }
    a.xml += "      </CellData>\n";
    a.xml += "    </Piece>\n";
    a.xml += "  </UnstructuredGrid>\n";
    a.xml += "  <AppendedData encoding=\"raw\">\n   _";
    std::string out = std::move(a.xml);
    out += a.data;
    out += "\n  </AppendedData>\n</VTKFile>\n";
    return out;
}

std::string pvtu(const std::string& name, const std::string& dash_time, int world_size, bool ascii) {
    const std::string ft = ascii ? "Float32" : "Float64";
    std::string c;
    c += ascii ? "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"BigEndian\">\n"
               : "<VTKFile type=\"PUnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    c += "<PUnstructuredGrid GhostLevel=\"1\">\n";
    c += "  <PPoints>\n";
    c += "    <PDataArray type=\"" + std::string(ascii ? "Float32" : "Float64") + "\" NumberOfComponents=\"3\"/>\n";
    c += "  </PPoints>\n";
    c += "  <PCells>\n";
    c += "    <PDataArray type=\"Int32\" Name=\"connectivity\"/>\n";
    c += "    <PDataArray type=\"Int32\" Name=\"offsets\"/>\n";
    c += std::string("    <PDataArray type=\"") + (ascii ? "Int32" : "UInt8") + "\" Name=\"types\"/>\n";
    c += "  </PCells>\n";
    c += "  <PCellData Scalars=\"scalars\">\n";
    c += "    <PDataArray type=\"Float32\" Name=\"rank\"/>\n";
    for (auto& vn : var_names) c += "    <PDataArray type=\"" + ft + "\" Name=\"" + vn + "\"/>\n";
    for (auto& kv : post::extra_scalars) c += "    <PDataArray type=\"" + ft + "\" Name=\"" + kv.first + "\"/>\n";
    for (auto& kv : post::extra_vectors)
        c += "    <PDataArray type=\"" + ft + "\" Name=\"" + kv.first + "\" NumberOfComponents=\"3\"/>\n";
    c += "  </PCellData>\n";
    for (int i = 0; i < world_size; ++i)
        c += "  <Piece Source=\"" + name + "_" + std::to_string(i) + dash_time + ".vtu\"/>\n";
    c += "</PUnstructuredGrid>\n";
    c += "</VTKFile>";
    return c;
}

}  // namespace

void writeVtk(const std::string name, std::vector<double>& q, mesh& m, int rank, int world_size,
              const std::string time) {
    const char* fe = std::getenv("FVGPU_VTK_FORMAT");
    const bool ascii = fe && std::string(fe) == "ascii";
    const std::string dash_time = time.empty() ? "" : "_" + time;
    std::string filename =
        (world_size > 1) ? name + "_" + std::to_string(rank) + dash_time + ".vtu" : name + dash_time + ".vtu";
    if (!time.empty()) filename = "times/" + filename;
    if (rank == 0 && world_size > 1) {
        std::string core = name + "_parallel" + dash_time + ".pvtu";
        if (!time.empty()) core = "times/" + core;
        std::ofstream out(core, std::ios::binary);
        out << pvtu(name, dash_time, world_size, ascii);
    }
    // as the reference: a missing times/ folder means no file, not an error
    std::ofstream out(filename, std::ios::binary);
    const Extras ex = extra_fields(q, m);
    const std::string body = ascii ? vtu_ascii(q, m, rank, ex) : vtu_binary(q, m, rank, ex);
    out.write(body.data(), (std::streamsize)body.size());
}

}  // namespace fvhyper
