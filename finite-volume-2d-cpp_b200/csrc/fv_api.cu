// C ABI of the B200 explicit finite-volume step (include/fvgpu.h).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fvgpu.h"
#include "fv_launch.h"
#include "fv_mesh.h"

using namespace fvgpu;

namespace {
thread_local std::string g_err;
int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? FV_ERR_NOMEM : FV_ERR_CUDA,         \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& v) {
    size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)dst, bytes);
    if (e != cudaSuccess) return e;
    if (!v.empty()) e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}
}  // namespace

struct fv_mesh {
    HostMesh m;
};

struct GraphEntry {
    std::vector<double> alpha;
    int chunk = 0;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
};

struct fv_solver {
    int device = 0;
    int precision = FV_PREC_FP64_EXACT;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int V = 4;
    int64_t n_real = 0, n_total = 0, n_bound = 0;
    std::vector<int32_t> new2ref_h;
    Params P{};
    // device buffers
    std::vector<void*> allocs;
    double *qA = nullptr, *qB = nullptr, *qC = nullptr;
    double *gx = nullptr, *gy = nullptr, *lim = nullptr, *dt = nullptr;
    double *stage_buf = nullptr;  // [n_total*V] staging for host transfers / stage tests
    double *partials = nullptr;
    double *scratch2 = nullptr;
    int *flag = nullptr;
    int32_t* new2ref = nullptr;
    Ctrl* ctrl = nullptr;
    RunLimits* limits = nullptr;
    PrintRec* hist = nullptr;
    int hist_cap = 0;
    int chunk = 16;
    std::vector<GraphEntry> graphs;
    double last_ms = 0.0;
    int64_t last_launches = 0;

    template <class T>
    cudaError_t alloc(T** p, size_t n) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) allocs.push_back(*p);
        return e;
    }
    ~fv_solver() {
        cudaSetDevice(device);
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        for (void* p : allocs) cudaFree(p);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

const char* fv_last_error(void) { return g_err.c_str(); }
int fv_version(void) { return 1; }

// ---------------------------------------------------------------- mesh ----
static int finish_mesh(fv_mesh* fm, fv_mesh** out) {
    std::string err = build_geometry(fm->m);
    if (!err.empty()) {
        delete fm;
        return fail(FV_ERR_MESH, err);
    }
    build_device_numbering(fm->m);
    *out = fm;
    return FV_OK;
}

int fv_mesh_create(int64_t n_nodes, const double* x, const double* y, int64_t n_cells, const int32_t* cells4,
                   int64_t n_bnd, const int32_t* bnd_nodes, const int32_t* bnd_group, int32_t n_groups,
                   fv_mesh** out) {
    if (!out || n_nodes <= 0 || n_cells <= 0 || !x || !y || !cells4 || n_bnd < 0 || (n_bnd > 0 && (!bnd_nodes || !bnd_group)))
        return fail(FV_ERR_ARG, "fv_mesh_create: invalid arguments");
    if (n_cells + n_bnd >= (int64_t)0x7fffffff) return fail(FV_ERR_ARG, "mesh too large for 31-bit cell indices");
    auto* fm = new fv_mesh();
    HostMesh& m = fm->m;
    m.nodes_x.assign(x, x + n_nodes);
    m.nodes_y.assign(y, y + n_nodes);
    m.cells4.assign(cells4, cells4 + 4 * n_cells);
    m.bnd_nodes.assign(bnd_nodes, bnd_nodes + 2 * n_bnd);
    m.bnd_group.assign(bnd_group, bnd_group + n_bnd);
    for (int64_t b = 0; b < n_bnd; ++b)
        if (bnd_group[b] < 0 || bnd_group[b] >= n_groups) {
            delete fm;
            return fail(FV_ERR_ARG, "boundary group index out of range");
        }
    for (int32_t g = 0; g < n_groups; ++g) m.group_names.push_back("group" + std::to_string(g));
    return finish_mesh(fm, out);
}

int fv_mesh_read_msh(const char* path, fv_mesh** out) {
    if (!path || !out) return fail(FV_ERR_ARG, "fv_mesh_read_msh: invalid arguments");
    auto* fm = new fv_mesh();
    std::string err = read_msh41(path, fm->m);
    if (!err.empty()) {
        delete fm;
        return fail(err.rfind("cannot open", 0) == 0 ? FV_ERR_IO : FV_ERR_MESH, err);
    }
    return finish_mesh(fm, out);
}

void fv_mesh_destroy(fv_mesh* m) { delete m; }

int fv_mesh_sizes(const fv_mesh* fm, int64_t* out) {
    if (!fm || !out) return fail(FV_ERR_ARG, "fv_mesh_sizes: null");
    const HostMesh& m = fm->m;
    out[0] = (int64_t)m.nodes_x.size(); out[1] = m.n_real; out[2] = m.n_total;
    out[3] = m.n_edges; out[4] = m.n_bound;
    return FV_OK;
}

int fv_mesh_group_count(const fv_mesh* fm) { return fm ? (int)fm->m.group_names.size() : 0; }

int fv_mesh_group_name(const fv_mesh* fm, int32_t i, char* buf, int32_t cap) {
    if (!fm || !buf || cap <= 0 || i < 0 || i >= (int32_t)fm->m.group_names.size())
        return fail(FV_ERR_ARG, "fv_mesh_group_name: invalid arguments");
    std::snprintf(buf, (size_t)cap, "%s", fm->m.group_names[i].c_str());
    return FV_OK;
}

int fv_mesh_geometry(const fv_mesh* fm, uint32_t* edge_cells, uint32_t* edge_nodes, double* enx, double* eny,
                     double* elen, double* ecx, double* ecy, double* area, double* ccx, double* ccy,
                     uint32_t* bound_edges, int32_t* bound_group) {
    if (!fm) return fail(FV_ERR_ARG, "fv_mesh_geometry: null mesh");
    const HostMesh& m = fm->m;
    auto cp = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(edge_cells, m.edge_cells); cp(edge_nodes, m.edge_nodes);
    cp(enx, m.enx); cp(eny, m.eny); cp(elen, m.elen); cp(ecx, m.ecx); cp(ecy, m.ecy);
    cp(area, m.area); cp(ccx, m.ccx); cp(ccy, m.ccy); cp(bound_edges, m.bound_edges);
    cp(bound_group, m.bnd_group);
    return FV_OK;
}

int fv_mesh_elements(const fv_mesh* fm, double* nodes_x, double* nodes_y, int32_t* cells4) {
    if (!fm) return fail(FV_ERR_ARG, "fv_mesh_elements: null mesh");
    const HostMesh& m = fm->m;
    if (nodes_x) std::memcpy(nodes_x, m.nodes_x.data(), m.nodes_x.size() * 8);
    if (nodes_y) std::memcpy(nodes_y, m.nodes_y.data(), m.nodes_y.size() * 8);
    if (cells4) std::memcpy(cells4, m.cells4.data(), m.cells4.size() * 4);
    return FV_OK;
}

int fv_mesh_device_order(const fv_mesh* fm, int32_t* new2ref) {
    if (!fm || !new2ref) return fail(FV_ERR_ARG, "fv_mesh_device_order: null");
    std::memcpy(new2ref, fm->m.new2ref.data(), fm->m.new2ref.size() * 4);
    return FV_OK;
}

// -------------------------------------------------------------- solver ----
static int validate_physics(const fv_physics* ph, int n_groups_mesh) {
    if (!ph) return fail(FV_ERR_ARG, "physics is null");
    if (ph->flux == FV_FLUX_BURGERS) {
        if (ph->V != 2) return fail(FV_ERR_UNSUPPORTED, "the Burgers flux kind has V = 2");
        if (ph->dt_kind != FV_DT_CONST) return fail(FV_ERR_UNSUPPORTED, "the Burgers kind supports a constant dt only");
    } else if (ph->flux == FV_FLUX_ROE_FS || ph->flux == FV_FLUX_ROE_ST) {
        if (ph->V != 4) return fail(FV_ERR_UNSUPPORTED, "the Roe flux kinds have V = 4");
    } else {
        return fail(FV_ERR_UNSUPPORTED, "unknown flux kind " + std::to_string(ph->flux));
    }
    if (ph->limiter < 0 || ph->limiter > 3) return fail(FV_ERR_UNSUPPORTED, "unknown limiter kind");
    if (ph->dt_kind < 0 || ph->dt_kind > 2) return fail(FV_ERR_UNSUPPORTED, "unknown dt kind");
    if (ph->n_groups < n_groups_mesh) return fail(FV_ERR_ARG, "physics has fewer boundary groups than the mesh");
    if (ph->n_groups > kMaxGroups) return fail(FV_ERR_UNSUPPORTED, "more than 16 boundary groups");
    for (int g = 0; g < ph->n_groups; ++g) {
        const int k = ph->group_bc[g];
        if (k < 0 || k > 3) return fail(FV_ERR_UNSUPPORTED, "unknown boundary condition kind");
        if (ph->V != 4 && k != FV_BC_COPY) return fail(FV_ERR_UNSUPPORTED, "V = 2 supports the copy boundary only");
    }
    return FV_OK;
}

int fv_solver_create(const fv_mesh* fm, const fv_physics* ph, int32_t precision, int32_t device, fv_solver** out) {
    if (!fm || !out) return fail(FV_ERR_ARG, "fv_solver_create: null");
    const HostMesh& m = fm->m;
    int rc = validate_physics(ph, (int)m.group_names.size());
    if (rc) return rc;
    if (precision != FV_PREC_FP64_EXACT) return fail(FV_ERR_UNSUPPORTED, "precision mode not built yet");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(FV_ERR_ARG, "no such CUDA device");
    CK(cudaSetDevice(device));
    std::unique_ptr<fv_solver> s(new fv_solver());
    s->device = device;
    s->precision = precision;
    s->V = ph->V;
    s->n_real = m.n_real; s->n_total = m.n_total; s->n_bound = m.n_bound;
    s->new2ref_h = m.new2ref;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
    FaceArrays fa;
    build_face_arrays(m, fa);
    Params& P = s->P;
    P.n_real = (int)m.n_real; P.n_total = (int)m.n_total; P.n_bound = (int)m.n_bound; P.V = ph->V;
    P.cell0 = fa.cell0;
    uint32_t* d_nbr; double *d_nx, *d_ny, *d_le, *d_g, *d_dsx, *d_dsy, *d_dnx, *d_dny, *d_area;
    int32_t *d_gg, *d_gc; uint8_t* d_gs; int32_t* d_n2r;
    CK(upload(&d_nbr, fa.nbr)); s->allocs.push_back(d_nbr);
    CK(upload(&d_nx, fa.nx)); s->allocs.push_back(d_nx);
    CK(upload(&d_ny, fa.ny)); s->allocs.push_back(d_ny);
    CK(upload(&d_le, fa.le)); s->allocs.push_back(d_le);
    CK(upload(&d_g, fa.g)); s->allocs.push_back(d_g);
    CK(upload(&d_dsx, fa.dsx)); s->allocs.push_back(d_dsx);
    CK(upload(&d_dsy, fa.dsy)); s->allocs.push_back(d_dsy);
    CK(upload(&d_dnx, fa.dnx)); s->allocs.push_back(d_dnx);
    CK(upload(&d_dny, fa.dny)); s->allocs.push_back(d_dny);
    CK(upload(&d_area, fa.area)); s->allocs.push_back(d_area);
    CK(upload(&d_gg, fa.ghost_group)); s->allocs.push_back(d_gg);
    CK(upload(&d_gc, fa.ghost_cell)); s->allocs.push_back(d_gc);
    CK(upload(&d_gs, fa.ghost_slot)); s->allocs.push_back(d_gs);
    CK(upload(&d_n2r, m.new2ref)); s->allocs.push_back(d_n2r);
    s->new2ref = d_n2r;
    P.face_nbr = d_nbr; P.f_nx = d_nx; P.f_ny = d_ny; P.f_le = d_le; P.f_g = d_g;
    P.f_dsx = d_dsx; P.f_dsy = d_dsy; P.f_dnx = d_dnx; P.f_dny = d_dny; P.area = d_area;
    P.ghost_group = d_gg; P.ghost_cell = d_gc; P.ghost_slot = d_gs;
    P.flux = ph->flux; P.order2 = ph->order2 ? 1 : 0; P.limiter = ph->limiter; P.dt_kind = ph->dt_kind;
    P.global_dt = ph->global_dt ? 1 : 0;
    P.gamma = ph->gamma; P.K = ph->K; P.cfl = ph->cfl; P.dt_const = ph->dt_const;
    P.n_groups = ph->n_groups;
    for (int g = 0; g < ph->n_groups; ++g) {
        P.group_bc[g] = ph->group_bc[g];
        for (int k = 0; k < 4; ++k) P.group_bv[4 * g + k] = ph->group_bv ? ph->group_bv[4 * g + k] : 0.0;
    }
    const size_t nq = (size_t)m.n_total * ph->V;
    CK(s->alloc(&s->qA, nq)); CK(s->alloc(&s->qB, nq)); CK(s->alloc(&s->qC, nq));
    CK(s->alloc(&s->gx, nq)); CK(s->alloc(&s->gy, nq)); CK(s->alloc(&s->lim, nq));
    CK(s->alloc(&s->stage_buf, nq));
    CK(s->alloc(&s->dt, (size_t)m.n_total));
    CK(s->alloc(&s->partials, (size_t)grid_for((int)m.n_real) * ph->V));
    CK(s->alloc(&s->scratch2, 8));
    CK(s->alloc(&s->flag, 4));
    CK(s->alloc(&s->ctrl, 1));
    CK(s->alloc(&s->limits, 1));
    s->hist_cap = 4096;
    CK(s->alloc(&s->hist, (size_t)s->hist_cap));
    CK(cudaMemsetAsync(s->qA, 0, nq * 8, s->stream));
    CK(cudaMemsetAsync(s->gx, 0, nq * 8, s->stream));
    CK(cudaMemsetAsync(s->gy, 0, nq * 8, s->stream));
    CK(cudaMemsetAsync(s->lim, 0, nq * 8, s->stream));
    CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), s->stream));
    launch_fill_ghost_grad(s->gx, s->gy, s->lim, (int)m.n_real, (int)m.n_total, ph->V, s->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    *out = s.release();
    return FV_OK;
}

int fv_solver_destroy(fv_solver* s) {
    delete s;
    return FV_OK;
}

int fv_solver_set_stream(fv_solver* s, void* stream) {
    if (!s) return fail(FV_ERR_ARG, "null solver");
    CK(cudaSetDevice(s->device));
    if (s->own_stream && s->stream) {
        CK(cudaStreamSynchronize(s->stream));
        CK(cudaStreamDestroy(s->stream));
    }
    if (stream) {
        s->stream = (cudaStream_t)stream;
        s->own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    return FV_OK;
}

int fv_solver_sync(fv_solver* s) {
    if (!s) return fail(FV_ERR_ARG, "null solver");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_solver_set_chunk(fv_solver* s, int32_t steps) {
    if (!s || steps < 1 || steps > 4096) return fail(FV_ERR_ARG, "chunk must be in [1, 4096]");
    s->chunk = steps;
    return FV_OK;
}

static int set_state_common(fv_solver* s, const double* q, cudaMemcpyKind kind) {
    if (!s || !q) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    const size_t nq = (size_t)s->n_total * s->V;
    CK(cudaMemcpyAsync(s->stage_buf, q, nq * 8, kind, s->stream));
    launch_permute_to_device(s->stage_buf, s->qA, s->new2ref, (int)s->n_total, s->V, s->stream);
    CK(cudaGetLastError());
    return FV_OK;
}
static int get_state_common(fv_solver* s, double* q, cudaMemcpyKind kind) {
    if (!s || !q) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    const size_t nq = (size_t)s->n_total * s->V;
    launch_permute_to_ref(s->qA, s->stage_buf, s->new2ref, (int)s->n_total, s->V, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q, s->stage_buf, nq * 8, kind, s->stream));
    if (kind == cudaMemcpyDeviceToHost) CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}
int fv_set_state(fv_solver* s, const double* q) {
    int rc = set_state_common(s, q, cudaMemcpyHostToDevice);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}
int fv_get_state(fv_solver* s, double* q) { return get_state_common(s, q, cudaMemcpyDeviceToHost); }
int fv_set_state_device(fv_solver* s, const double* q) { return set_state_common(s, q, cudaMemcpyDeviceToDevice); }
int fv_get_state_device(fv_solver* s, double* q) { return get_state_common(s, q, cudaMemcpyDeviceToDevice); }

// ---------------------------------------------------------------- run ----
// Kernel kinds for per-kernel timing.
enum { KK_BEGIN = 0, KK_DT = 1, KK_GRADLIM = 2, KK_STAGE = 3, KK_END = 4, KK_N = 5 };

struct EventLog {
    std::vector<cudaEvent_t> ev;  // ev[0] before the first kernel, ev[k+1] after kernel k
    std::vector<int> kind;
    cudaStream_t st;
    void mark(int k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev.push_back(e);
        kind.push_back(k);
    }
};

// Enqueues one time step (explicit.cpp:715-801) reading/writing the base
// state in `base`.  Returns the number of kernels launched.
static int enqueue_step(fv_solver* s, const std::vector<double>& alpha, double* base, double* other,
                        EventLog* log = nullptr) {
    const Params& P = s->P;
    cudaStream_t st = s->stream;
    int n = 0;
    auto mark = [&](int k) { if (log) log->mark(k); };
    launch_step_begin(s->ctrl, s->limits, s->V, st); ++n; mark(KK_BEGIN);
    exact::launch_dt(P, base, s->dt, &s->ctrl->dtmin_key, s->ctrl, st); ++n; mark(KK_DT);
    const int ns = (int)alpha.size();
    const double* in = base;
    for (int k = 0; k < ns; ++k) {
        double* out;
        if (ns == 1) out = other;
        else if (k == ns - 1) out = base;
        else out = (k % 2 == 0) ? s->qB : s->qC;
        StageIO io{};
        io.q_stage = in; io.q_base = base; io.q_out = out;
        io.gx = s->gx; io.gy = s->gy; io.lim = s->lim; io.dt = s->dt; io.alpha = alpha[k];
        io.ctrl = s->ctrl;
        io.partials = (k == ns - 1) ? s->partials : nullptr;
        if (P.order2) { exact::launch_grad_lim(P, io, st); ++n; mark(KK_GRADLIM); }
        exact::launch_stage(P, io, st); ++n; mark(KK_STAGE);
        in = out;
    }
    launch_step_end(P, s->ctrl, s->limits, s->partials, grid_for((int)s->n_real), s->dt, s->hist, s->hist_cap, st);
    ++n; mark(KK_END);
    return n;
}

static int get_graph(fv_solver* s, const std::vector<double>& alpha, GraphEntry** out) {
    const int chunk = (alpha.size() == 1 && s->chunk % 2) ? s->chunk + 1 : s->chunk;
    for (auto& g : s->graphs)
        if (g.alpha == alpha && g.chunk == chunk) { *out = &g; return FV_OK; }
    GraphEntry g;
    g.alpha = alpha;
    g.chunk = chunk;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    for (int k = 0; k < chunk; ++k) {
        double* base = (alpha.size() == 1 && (k % 2)) ? s->qB : s->qA;
        double* other = (alpha.size() == 1 && (k % 2)) ? s->qA : s->qB;
        launches += enqueue_step(s, alpha, base, other);
    }
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (e != cudaSuccess) return fail(FV_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(FV_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    g.launches = launches;
    s->graphs.push_back(g);
    *out = &s->graphs.back();
    return FV_OK;
}

int fv_run(fv_solver* s, const fv_run_options* o, fv_run_info* info) {
    if (!s || !o) return fail(FV_ERR_ARG, "fv_run: null argument");
    if (o->n_alpha < 1 || o->n_alpha > 16 || !o->alpha) return fail(FV_ERR_ARG, "fv_run: need 1..16 RK stages");
    if (o->print_interval == 0) return fail(FV_ERR_ARG, "fv_run: print_interval must be > 0");
    CK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    std::vector<double> alpha(o->alpha, o->alpha + o->n_alpha);
    RunLimits L{o->max_step, o->max_time, o->tolerance, o->print_interval};
    CK(cudaMemcpyAsync(s->limits, &L, sizeof(L), cudaMemcpyHostToDevice, st));
    Ctrl hc;
    if (o->restart) {
        std::memset(&hc, 0, sizeof(hc));
        for (int k = 0; k < kMaxV; ++k) hc.R[k] = 1.0;
        hc.active = 1;
        CK(cudaMemcpyAsync(s->ctrl, &hc, sizeof(hc), cudaMemcpyHostToDevice, st));
        // run(): initial ghost fill with zeroed gx, gy, limiters (explicit.cpp:712)
        exact::launch_bounds(s->P, s->qA, s->gx, s->gy, s->lim, 1, st);
        CK(cudaGetLastError());
    }
    if (!o->restart) CK(cudaMemcpyAsync(&hc, s->ctrl, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const unsigned long long start_step = o->restart ? 0ull : hc.step;
    GraphEntry* g = nullptr;
    int rc = get_graph(s, alpha, &g);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
    std::vector<PrintRec> recs(s->hist_cap);
    double total_ms = 0.0;
    int64_t launches = 0;
    for (;;) {
        CK(cudaMemsetAsync(&s->ctrl->n_hist, 0, sizeof(int), st));
        CK(cudaEventRecord(e0, st));
        CK(cudaGraphLaunch(g->exec, st));
        CK(cudaEventRecord(e1, st));
        launches += g->launches;
        CK(cudaMemcpyAsync(&hc, s->ctrl, sizeof(hc), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        total_ms += ms;
        if (o->on_print && hc.n_hist > 0) {
            CK(cudaMemcpy(recs.data(), s->hist, sizeof(PrintRec) * hc.n_hist, cudaMemcpyDeviceToHost));
            for (int k = 0; k < hc.n_hist; ++k) o->on_print(o->user, recs[k].step, recs[k].time, recs[k].R, s->V);
        }
        double Rmax = 1.0;
        if (hc.step > 0) {
            Rmax = 0.0;
            for (int k = 0; k < s->V; ++k) Rmax = (Rmax < hc.R[k]) ? hc.R[k] : Rmax;
        }
        const bool done = !hc.active || hc.step >= o->max_step || hc.time >= o->max_time || Rmax < o->tolerance;
        if (done) break;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    // RK1 alternates the base buffer; an odd number of steps leaves it in qB.
    if (alpha.size() == 1) {
        // every graph replay starts from qA and full chunks are even, so the
        // base ends in qB exactly when this run took an odd number of steps
        if ((hc.step - start_step) % 2) {
            CK(cudaMemcpyAsync(s->qA, s->qB, (size_t)s->n_total * s->V * 8, cudaMemcpyDeviceToDevice, st));
        }
    }
    CK(cudaStreamSynchronize(st));
    s->last_ms = total_ms;
    s->last_launches = launches;
    if (info) {
        info->step = hc.step;
        info->time = hc.time;
        for (int k = 0; k < kMaxV; ++k) { info->R[k] = hc.R[k]; info->R0[k] = hc.R0[k]; }
        for (int k = kMaxV; k < 8; ++k) { info->R[k] = 0; info->R0[k] = 0; }
    }
    return FV_OK;
}

int fv_profile_kernels(fv_solver* s, const double* alpha, int32_t n_alpha, int32_t n_steps, double* out_ms,
                       int64_t* out_count) {
    if (!s || !alpha || n_alpha < 1 || n_steps < 1 || !out_ms || !out_count)
        return fail(FV_ERR_ARG, "fv_profile_kernels: invalid arguments");
    CK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    std::vector<double> a(alpha, alpha + n_alpha);
    Ctrl hc;
    CK(cudaMemcpyAsync(&hc, s->ctrl, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    RunLimits L{hc.step + (unsigned long long)n_steps, 1e300, -1.0, 1ull << 62};
    CK(cudaMemcpyAsync(s->limits, &L, sizeof(L), cudaMemcpyHostToDevice, st));
    EventLog log;
    log.st = st;
    cudaEvent_t e0;
    CK(cudaEventCreate(&e0));
    CK(cudaEventRecord(e0, st));
    log.ev.push_back(e0);
    log.kind.push_back(-1);
    for (int k = 0; k < n_steps; ++k) {
        const bool odd = a.size() == 1 && (k % 2);
        enqueue_step(s, a, odd ? s->qB : s->qA, odd ? s->qA : s->qB, &log);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k < KK_N; ++k) { out_ms[k] = 0.0; out_count[k] = 0; }
    for (size_t i = 1; i < log.ev.size(); ++i) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, log.ev[i - 1], log.ev[i]));
        out_ms[log.kind[i]] += ms;
        out_count[log.kind[i]] += 1;
    }
    for (auto e : log.ev) cudaEventDestroy(e);
    if (a.size() == 1 && (n_steps % 2))
        CK(cudaMemcpyAsync(s->qA, s->qB, (size_t)s->n_total * s->V * 8, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    return FV_OK;
}

int fv_last_run_stats(fv_solver* s, double* device_ms, int64_t* kernel_launches) {
    if (!s) return fail(FV_ERR_ARG, "null solver");
    if (device_ms) *device_ms = s->last_ms;
    if (kernel_launches) *kernel_launches = s->last_launches;
    return FV_OK;
}

int fv_residuals(fv_solver* s, double* R) {
    if (!s || !R) return fail(FV_ERR_ARG, "null argument");
    Ctrl hc;
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(&hc, s->ctrl, sizeof(hc), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < s->V; ++k) R[k] = hc.Rraw[k];
    return FV_OK;
}

int fv_check_state(fv_solver* s) {
    if (!s) return fail(FV_ERR_ARG, "null solver");
    CK(cudaSetDevice(s->device));
    int h = 0;
    CK(cudaMemsetAsync(s->flag, 0, 4, s->stream));
    launch_check_state(s->P, s->qA, s->flag, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h, s->flag, 4, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (h) return fail(FV_ERR_NONFINITE, "non-finite or non-physical state (rho <= 0 or p <= 0)");
    return FV_OK;
}

int fv_boundary_force(fv_solver* s, int32_t group, double* fx, double* fy) {
    if (!s || !fx || !fy || s->V != 4) return fail(FV_ERR_ARG, "fv_boundary_force: invalid arguments");
    CK(cudaSetDevice(s->device));
    launch_force(s->P, s->qA, group, s->scratch2, s->stream);
    CK(cudaGetLastError());
    double h[2];
    CK(cudaMemcpyAsync(h, s->scratch2, 16, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *fx = h[0]; *fy = h[1];
    return FV_OK;
}

// ------------------------------------------------------- stage entry points --
static int to_device(fv_solver* s, const double* h, double* d, int V) {
    CK(cudaMemcpyAsync(s->stage_buf, h, (size_t)s->n_total * V * 8, cudaMemcpyHostToDevice, s->stream));
    launch_permute_to_device(s->stage_buf, d, s->new2ref, (int)s->n_total, V, s->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}
static int to_host(fv_solver* s, const double* d, double* h, int V) {
    launch_permute_to_ref(d, s->stage_buf, s->new2ref, (int)s->n_total, V, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h, s->stage_buf, (size_t)s->n_total * V * 8, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_stage_dt(fv_solver* s, const double* q, double* dt, int32_t global_min) {
    if (!s || !q || !dt) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    int rc = to_device(s, q, s->qB, s->V);
    if (rc) return rc;
    unsigned long long init = ~0ull;
    CK(cudaMemcpyAsync(s->scratch2, &init, 8, cudaMemcpyHostToDevice, s->stream));
    Params P = s->P;
    P.global_dt = global_min ? 1 : 0;
    exact::launch_dt(P, s->qB, s->dt, (unsigned long long*)s->scratch2, nullptr, s->stream);
    CK(cudaGetLastError());
    std::vector<double> dd(s->n_total);
    rc = to_host(s, s->dt, dd.data(), 1);
    if (rc) return rc;
    if (global_min) {
        unsigned long long key;
        CK(cudaMemcpy(&key, s->scratch2, 8, cudaMemcpyDeviceToHost));
        double mn;
        if (key == ~0ull) {
            mn = std::nan("");
        } else {
            unsigned long long b = (key & 0x8000000000000000ull) ? (key & 0x7fffffffffffffffull) : ~key;
            std::memcpy(&mn, &b, 8);
        }
        if (dd[0] != dd[0]) mn = dd[0];
        for (auto& v : dd) v = mn;
    }
    std::memcpy(dt, dd.data(), dd.size() * 8);
    return FV_OK;
}

int fv_stage_gradients_limiters(fv_solver* s, const double* q, double* gx, double* gy, double* lim) {
    if (!s || !q || !gx || !gy || !lim) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    int rc = to_device(s, q, s->qB, s->V);
    if (rc) return rc;
    StageIO io{};
    io.q_stage = s->qB; io.gx = s->gx; io.gy = s->gy; io.lim = s->lim;
    exact::launch_grad_lim(s->P, io, s->stream);
    CK(cudaGetLastError());
    if ((rc = to_host(s, s->gx, gx, s->V))) return rc;
    if ((rc = to_host(s, s->gy, gy, s->V))) return rc;
    return to_host(s, s->lim, lim, s->V);
}

int fv_stage_update(fv_solver* s, const double* q_base, const double* q_stage, const double* gx, const double* gy,
                    const double* lim, const double* dt, double alpha, double* q_out) {
    if (!s || !q_base || !q_stage || !gx || !gy || !lim || !dt || !q_out) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    int rc;
    if ((rc = to_device(s, q_base, s->qA, s->V))) return rc;
    if ((rc = to_device(s, q_stage, s->qB, s->V))) return rc;
    if ((rc = to_device(s, gx, s->gx, s->V))) return rc;
    if ((rc = to_device(s, gy, s->gy, s->V))) return rc;
    if ((rc = to_device(s, lim, s->lim, s->V))) return rc;
    if ((rc = to_device(s, dt, s->dt, 1))) return rc;
    // the output buffer starts as the stage state so untouched ghosts match
    CK(cudaMemcpyAsync(s->qC, s->qB, (size_t)s->n_total * s->V * 8, cudaMemcpyDeviceToDevice, s->stream));
    StageIO io{};
    io.q_stage = s->qB; io.q_base = s->qA; io.q_out = s->qC;
    io.gx = s->gx; io.gy = s->gy; io.lim = s->lim; io.dt = s->dt; io.alpha = alpha;
    exact::launch_stage(s->P, io, s->stream);
    CK(cudaGetLastError());
    rc = to_host(s, s->qC, q_out, s->V);
    // restore the invariant ghost gradient/limiter values
    launch_fill_ghost_grad(s->gx, s->gy, s->lim, (int)s->n_real, (int)s->n_total, s->V, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    return rc;
}

int fv_stage_bounds(fv_solver* s, double* q, const double* gx, const double* gy, const double* lim) {
    if (!s || !q || !gx || !gy || !lim) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    int rc;
    if ((rc = to_device(s, q, s->qB, s->V))) return rc;
    if ((rc = to_device(s, gx, s->gx, s->V))) return rc;
    if ((rc = to_device(s, gy, s->gy, s->V))) return rc;
    if ((rc = to_device(s, lim, s->lim, s->V))) return rc;
    exact::launch_bounds(s->P, s->qB, s->gx, s->gy, s->lim, 0, s->stream);
    CK(cudaGetLastError());
    rc = to_host(s, s->qB, q, s->V);
    launch_fill_ghost_grad(s->gx, s->gy, s->lim, (int)s->n_real, (int)s->n_total, s->V, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    return rc;
}

}  // extern "C"
