// C ABI of the B200 explicit finite-volume step (include/fvgpu.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fvgpu.h"
#include "fv_launch.h"
#include "fv_mesh.h"
#include "fv_tile.cuh"
#include "fv_fused.cuh"
#include "fv_adjoint.h"
#include "fv_solver.h"
#include <cmath>

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

// Drops the captured step graphs (their kernels change with s->fused).
static void clear_graphs(fv_solver* s) {
    for (auto& g : s->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    s->graphs.clear();
}

namespace {
// host vector<double> -> device array of the stage precision
int upload_s(fv_solver* s, const std::vector<double>& v, const void** out) {
    void* d = nullptr;
    CK(s->alloc(&d, v.size(), s->ssz));
    if (s->f32) {
        std::vector<float> f(v.begin(), v.end());
        CK(cudaMemcpy(d, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
    } else {
        CK(cudaMemcpy(d, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
    }
    *out = d;
    return FV_OK;
}
template <class T>
int upload_v(fv_solver* s, const std::vector<T>& v, const T** out) {
    T* d = nullptr;
    CK(s->alloc(&d, v.size()));
    if (!v.empty()) CK(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    *out = d;
    return FV_OK;
}
}  // namespace

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

int fv_mesh_create_batch(int32_t n_cases, const fv_mesh* const* cases, fv_mesh** out) {
    if (!out || !cases || n_cases < 1) return fail(FV_ERR_ARG, "fv_mesh_create_batch: invalid arguments");
    auto* fm = new fv_mesh();
    HostMesh& u = fm->m;
    u.case_real_off.push_back(0);
    u.case_bound_off.push_back(0);
    int64_t total_cells = 0, total_bnd = 0;
    for (int32_t k = 0; k < n_cases; ++k) {
        if (!cases[k]) {
            delete fm;
            return fail(FV_ERR_ARG, "fv_mesh_create_batch: null case mesh");
        }
        const HostMesh& c = cases[k]->m;
        const int32_t node0 = (int32_t)u.nodes_x.size();
        u.nodes_x.insert(u.nodes_x.end(), c.nodes_x.begin(), c.nodes_x.end());
        u.nodes_y.insert(u.nodes_y.end(), c.nodes_y.begin(), c.nodes_y.end());
        for (int32_t v : c.cells4) u.cells4.push_back(v < 0 ? v : v + node0);
        for (int32_t v : c.bnd_nodes) u.bnd_nodes.push_back(v + node0);
        // boundary groups are merged by name, in order of first use
        for (int32_t g : c.bnd_group) {
            const std::string& name = c.group_names[(size_t)g];
            auto it = std::find(u.group_names.begin(), u.group_names.end(), name);
            if (it == u.group_names.end()) {
                u.group_names.push_back(name);
                it = u.group_names.end() - 1;
            }
            u.bnd_group.push_back((int32_t)(it - u.group_names.begin()));
        }
        total_cells += (int64_t)c.cells4.size() / 4;
        total_bnd += (int64_t)c.bnd_group.size();
        u.case_real_off.push_back(total_cells);
        u.case_bound_off.push_back(total_bnd);
    }
    if (total_cells + total_bnd >= (int64_t)0x7fffffff) {
        delete fm;
        return fail(FV_ERR_ARG, "batch too large for 31-bit cell indices");
    }
    if (n_cases == 1) { u.case_real_off.clear(); u.case_bound_off.clear(); }
    return finish_mesh(fm, out);
}

int fv_mesh_case_count(const fv_mesh* fm) {
    if (!fm) return 0;
    return fm->m.case_real_off.size() > 2 ? (int)fm->m.case_real_off.size() - 1 : 1;
}

int fv_mesh_case_offsets(const fv_mesh* fm, int64_t* real_off, int64_t* bound_off) {
    if (!fm || !real_off || !bound_off) return fail(FV_ERR_ARG, "fv_mesh_case_offsets: null argument");
    const HostMesh& m = fm->m;
    if (m.case_real_off.size() > 2) {
        std::copy(m.case_real_off.begin(), m.case_real_off.end(), real_off);
        std::copy(m.case_bound_off.begin(), m.case_bound_off.end(), bound_off);
    } else {
        real_off[0] = 0; real_off[1] = m.n_real;
        bound_off[0] = 0; bound_off[1] = m.n_bound;
    }
    return FV_OK;
}

int fv_mesh_read_su2(const char* path, fv_mesh** out) {
    if (!path || !out) return fail(FV_ERR_ARG, "fv_mesh_read_su2: invalid arguments");
    auto* fm = new fv_mesh();
    std::string err = read_su2(path, fm->m);
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

int fv_mesh_tile_layout(const fv_mesh* fm, int32_t tile_cells, int64_t* sizes, int32_t* info, int32_t* halo,
                        uint32_t* edge_ij, uint16_t* face) {
    if (!fm || !sizes) return fail(FV_ERR_ARG, "fv_mesh_tile_layout: null");
    if (tile_cells != 64 && tile_cells != 128 && tile_cells != 256)
        return fail(FV_ERR_ARG, "tile_cells must be 64, 128 or 256");
    FaceArrays fa;
    build_face_arrays(fm->m, fa);
    TileArrays ta;
    build_tiles(fm->m, fa, tile_cells, ta);
    // the layouts a solver refuses (16-bit tile-local indices) are refused here too
    if (ta.max_halo + tile_cells > 65535 || ta.max_edges > kFaceEdgeMask)
        return fail(FV_ERR_MESH, "tile halo too large for 16-bit local indices");
    sizes[0] = ta.n_tiles; sizes[1] = ta.max_halo; sizes[2] = ta.max_edges;
    sizes[3] = (int64_t)ta.halo.size(); sizes[4] = (int64_t)ta.edge_ij.size();
    if (info) std::memcpy(info, ta.info.data(), ta.info.size() * sizeof(int32_t));
    if (halo) std::memcpy(halo, ta.halo.data(), ta.halo.size() * sizeof(int32_t));
    if (edge_ij) std::memcpy(edge_ij, ta.edge_ij.data(), ta.edge_ij.size() * sizeof(uint32_t));
    if (face) std::memcpy(face, ta.face.data(), ta.face.size() * sizeof(uint16_t));
    return FV_OK;
}

int fv_mesh_tile2_layout(const fv_mesh* fm, int32_t tile_cells, int64_t* sizes, int32_t* info, int32_t* halo,
                         uint32_t* edge_ij, uint16_t* face) {
    if (!fm || !sizes) return fail(FV_ERR_ARG, "fv_mesh_tile2_layout: null");
    if (tile_cells != 64 && tile_cells != 128 && tile_cells != 256)
        return fail(FV_ERR_ARG, "tile_cells must be 64, 128 or 256");
    FaceArrays fa;
    build_face_arrays(fm->m, fa);
    Tile2Arrays ta;
    build_tiles2(fm->m, fa, tile_cells, ta);
    if (ta.max_slots > 65535 || ta.max_edges > kFaceEdgeMask)
        return fail(FV_ERR_MESH, "two-ring tiles too large for 16-bit local indices");
    sizes[0] = ta.n_tiles; sizes[1] = ta.max_slots; sizes[2] = ta.max_grad; sizes[3] = ta.max_edges;
    sizes[4] = ta.max_flux; sizes[5] = (int64_t)ta.halo.size(); sizes[6] = (int64_t)ta.edge_ij.size();
    sizes[7] = (int64_t)ta.face.size() / 4;
    if (info) std::memcpy(info, ta.info.data(), ta.info.size() * sizeof(int32_t));
    if (halo) std::memcpy(halo, ta.halo.data(), ta.halo.size() * sizeof(int32_t));
    if (edge_ij) std::memcpy(edge_ij, ta.edge_ij.data(), ta.edge_ij.size() * sizeof(uint32_t));
    if (face) std::memcpy(face, ta.face.data(), ta.face.size() * sizeof(uint16_t));
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
    } else if (ph->flux == FV_FLUX_BURGERS_DIFF) {
        if (ph->V != 2) return fail(FV_ERR_UNSUPPORTED, "the Burgers-diffusion flux kind has V = 2");
        if (!ph->diffusive) return fail(FV_ERR_UNSUPPORTED, "the Burgers-diffusion flux kind needs diffusive = 1");
        if (ph->dt_kind != FV_DT_CONST)
            return fail(FV_ERR_UNSUPPORTED, "the Burgers-diffusion kind supports a constant dt only");
    } else if (ph->flux == FV_FLUX_NS) {
        if (ph->V != 4) return fail(FV_ERR_UNSUPPORTED, "the Navier-Stokes flux kind has V = 4");
        if (!ph->diffusive) return fail(FV_ERR_UNSUPPORTED, "the Navier-Stokes flux kind needs diffusive = 1");
    } else if (ph->flux == FV_FLUX_DIFFUSION) {
        if (ph->V != 1) return fail(FV_ERR_UNSUPPORTED, "the diffusion flux kind has V = 1");
        if (!ph->diffusive) return fail(FV_ERR_UNSUPPORTED, "the diffusion flux kind needs diffusive = 1");
        if (ph->order2)
            return fail(FV_ERR_UNSUPPORTED, "the diffusion flux kind runs without MUSCL face states (order2 = 0)");
        if (ph->dt_kind != FV_DT_CONST) return fail(FV_ERR_UNSUPPORTED, "the diffusion kind supports a constant dt only");
    } else {
        return fail(FV_ERR_UNSUPPORTED, "unknown flux kind " + std::to_string(ph->flux));
    }
    if (ph->diffusive && ph->flux != FV_FLUX_DIFFUSION && ph->flux != FV_FLUX_NS && ph->flux != FV_FLUX_BURGERS_DIFF)
        return fail(FV_ERR_UNSUPPORTED, "diffusive gradients are used by the diffusive flux kinds only");
    if (ph->smooth_residuals && ph->flux != FV_FLUX_BURGERS_DIFF)
        return fail(FV_ERR_UNSUPPORTED, "residual smoothing runs with the Burgers-diffusion kind only");
    if (ph->limiter < 0 || ph->limiter > 3) return fail(FV_ERR_UNSUPPORTED, "unknown limiter kind");
    if (ph->dt_kind < 0 || ph->dt_kind > 4) return fail(FV_ERR_UNSUPPORTED, "unknown dt kind");
    if (ph->dt_kind >= FV_DT_VISC_MIN && ph->V != 4) return fail(FV_ERR_UNSUPPORTED, "the viscous dt kinds have V = 4");
    if (ph->flux == FV_FLUX_NS || ph->dt_kind >= FV_DT_VISC_MIN) {
        if (!(ph->mu >= 0.0) || !(ph->pr > 0.0) || !(ph->r > 0.0) || !std::isfinite(ph->cp))
            return fail(FV_ERR_ARG, "Navier-Stokes constants need mu >= 0, pr > 0, r > 0 and a finite cp");
    }
    if (ph->n_groups < n_groups_mesh) return fail(FV_ERR_ARG, "physics has fewer boundary groups than the mesh");
    if (ph->n_groups > kMaxGroups) return fail(FV_ERR_UNSUPPORTED, "more than 16 boundary groups");
    for (int g = 0; g < ph->n_groups; ++g) {
        const int k = ph->group_bc[g];
        if (k < 0 || k > 6) return fail(FV_ERR_UNSUPPORTED, "unknown boundary condition kind");
        if (k == FV_BC_TANGENT && ph->V != 2) return fail(FV_ERR_UNSUPPORTED, "the tangent boundary has V = 2");
        if (ph->V != 4 && k != FV_BC_COPY && k != FV_BC_TANGENT)
            return fail(FV_ERR_UNSUPPORTED, "V = " + std::to_string(ph->V) + " supports the copy boundary only");
    }
    return FV_OK;
}

int fv_solver_create(const fv_mesh* fm, const fv_physics* ph, int32_t precision, int32_t device, fv_solver** out) {
    return fv_solver_create_ex(fm, ph, precision, device, nullptr, out);
}

int fv_solver_create_ex(const fv_mesh* fm, const fv_physics* ph, int32_t precision, int32_t device,
                        const fv_solver_options* opt, fv_solver** out) {
    if (!fm || !out) return fail(FV_ERR_ARG, "fv_solver_create: null");
    const HostMesh& m = fm->m;
    int rc = validate_physics(ph, (int)m.group_names.size());
    if (rc) return rc;
    if (precision < FV_PREC_FP64_EXACT || precision > FV_PREC_FP32) return fail(FV_ERR_ARG, "unknown precision mode");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(FV_ERR_ARG, "no such CUDA device");
    CK(cudaSetDevice(device));
    std::unique_ptr<fv_solver> s(new fv_solver());
    s->device = device;
    s->precision = precision;
    s->f32 = precision == FV_PREC_FP32;
    s->ssz = s->f32 ? 4 : 8;
    s->V = ph->V;
    s->n_real = m.n_real; s->n_total = m.n_total; s->n_bound = m.n_bound;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
    FaceArrays fa;
    build_face_arrays(m, fa);
    TileArrays ta;
    const int tile_cells = (opt && opt->tile_cells) ? opt->tile_cells : 128;
    if (tile_cells != 64 && tile_cells != 128 && tile_cells != 256)
        return fail(FV_ERR_ARG, "tile_cells must be 64, 128 or 256");
    build_tiles(m, fa, tile_cells, ta);
    if (ta.max_halo + tile_cells > 65535 || ta.max_edges > kFaceEdgeMask)
        return fail(FV_ERR_MESH, "tile halo too large for 16-bit local indices");
    s->n_tiles = ta.n_tiles;
    TileParams& TP = s->TP;
    Params& P = TP.P;
    P.n_real = (int)m.n_real; P.n_total = (int)m.n_total; P.n_bound = (int)m.n_bound; P.V = ph->V;
    P.n_own = (int)m.owned_real();
    P.cell0 = fa.cell0;
    if ((rc = upload_v(s.get(), fa.ghost_group, &P.ghost_group))) return rc;
    if ((rc = upload_v(s.get(), fa.ghost_cell, &P.ghost_cell))) return rc;
    if ((rc = upload_v(s.get(), fa.g_nx, &P.g_nx))) return rc;
    if ((rc = upload_v(s.get(), fa.g_ny, &P.g_ny))) return rc;
    if ((rc = upload_v(s.get(), fa.g_le, &P.g_le))) return rc;
    if ((rc = upload_v(s.get(), fa.g_dx, &P.g_dx))) return rc;
    if ((rc = upload_v(s.get(), fa.g_dy, &P.g_dy))) return rc;
    P.flux = ph->flux; P.order2 = ph->order2 ? 1 : 0; P.limiter = ph->limiter; P.dt_kind = ph->dt_kind;
    P.global_dt = ph->global_dt ? 1 : 0;
    P.positivity_guard = ph->positivity_guard ? 1 : 0;
    P.diffusive = ph->diffusive ? 1 : 0;
    P.mu = ph->mu; P.pr = ph->pr; P.cp = ph->cp; P.r = ph->r;
    P.smooth = ph->smooth_residuals ? 1 : 0;
    P.gamma = ph->gamma; P.K = ph->K; P.cfl = ph->cfl; P.dt_const = ph->dt_const;
    P.n_groups = ph->n_groups;
    for (int g = 0; g < ph->n_groups; ++g) {
        P.group_bc[g] = ph->group_bc[g];
        for (int k = 0; k < 4; ++k) P.group_bv[4 * g + k] = ph->group_bv ? ph->group_bv[4 * g + k] : 0.0;
    }
    TP.T = ta.tile_cells; TP.max_halo = ta.max_halo; TP.max_edges = ta.max_edges;
    const int32_t* info; const int32_t* halo; const uint32_t* eij; const uint16_t* face;
    if ((rc = upload_v(s.get(), ta.info, &info))) return rc;
    TP.info = reinterpret_cast<const int4*>(info);
    if ((rc = upload_v(s.get(), ta.halo, &halo))) return rc;
    TP.halo = halo;
    if ((rc = upload_v(s.get(), ta.edge_ij, &eij))) return rc;
    TP.edge_ij = eij;
    if ((rc = upload_v(s.get(), ta.face, &face))) return rc;
    TP.face = face;
    if ((rc = upload_s(s.get(), ta.enx, &TP.enx))) return rc;
    if ((rc = upload_s(s.get(), ta.eny, &TP.eny))) return rc;
    if ((rc = upload_s(s.get(), ta.ele, &TP.ele))) return rc;
    if ((rc = upload_s(s.get(), ta.exf, &TP.exf))) return rc;
    if ((rc = upload_s(s.get(), ta.eyf, &TP.eyf))) return rc;
    if ((rc = upload_s(s.get(), ta.eg, &TP.eg))) return rc;
    {
        std::vector<double> cxy(2 * ta.ccx.size());
        for (size_t i = 0; i < ta.ccx.size(); ++i) { cxy[2 * i] = ta.ccx[i]; cxy[2 * i + 1] = ta.ccy[i]; }
        if ((rc = upload_s(s.get(), cxy, &TP.ccxy))) return rc;
    }
    if ((rc = upload_s(s.get(), fa.area, &TP.area))) return rc;
    const int32_t* n2r;
    if ((rc = upload_v(s.get(), m.new2ref, &n2r))) return rc;
    s->new2ref = const_cast<int32_t*>(n2r);
    CK(tile::prepare(precision, TP));
    {
        // one fused kernel per stage for the second-order Roe kinds
        const int sk = opt ? opt->stage_kernels : FV_STAGE_AUTO;
        if (sk < FV_STAGE_AUTO || sk > FV_STAGE_HYBRID) return fail(FV_ERR_ARG, "unknown stage_kernels");
        const bool can_fuse = ph->V == 4 && ph->order2 && (ph->flux == FV_FLUX_ROE_FS || ph->flux == FV_FLUX_ROE_ST) &&
                              !ph->diffusive && !ph->smooth_residuals;
        if ((sk == FV_STAGE_FUSED || sk == FV_STAGE_HYBRID) && !can_fuse)
            return fail(FV_ERR_UNSUPPORTED, "the fused stage kernel needs a second-order Roe kind without "
                                            "diffusive terms or residual smoothing");
        if (can_fuse && sk != FV_STAGE_SPLIT) {
            Tile2Arrays t2;
            build_tiles2(m, fa, tile_cells, t2);
            FusedParams& F = s->FPm;
            F.T = tile_cells;
            F.max_slots = t2.max_slots; F.max_grad = t2.max_grad;
            F.max_edges = t2.max_edges; F.max_flux = t2.max_flux;
            const bool fits = t2.max_slots <= 65535 && t2.max_edges <= kFaceEdgeMask &&
                              tile::smem_fused(precision, F) <= (size_t)227 * 1024;
            if (!fits && (sk == FV_STAGE_FUSED || sk == FV_STAGE_HYBRID))
                return fail(FV_ERR_MESH, "two-ring tiles too large for the fused stage kernel at this tile size");
            if (fits) {
                const int32_t* i2; const int32_t* h2; const uint32_t* e2; const uint16_t* f2;
                if ((rc = upload_v(s.get(), t2.info, &i2))) return rc;
                F.info = reinterpret_cast<const int4*>(i2);
                if ((rc = upload_v(s.get(), t2.halo, &h2))) return rc;
                F.halo = h2;
                if ((rc = upload_v(s.get(), t2.edge_ij, &e2))) return rc;
                F.edge_ij = e2;
                if ((rc = upload_v(s.get(), t2.face, &f2))) return rc;
                F.face = reinterpret_cast<const uint2*>(f2);
                if ((rc = upload_s(s.get(), t2.enx, &F.enx))) return rc;
                if ((rc = upload_s(s.get(), t2.eny, &F.eny))) return rc;
                if ((rc = upload_s(s.get(), t2.ele, &F.ele))) return rc;
                if ((rc = upload_s(s.get(), t2.exf, &F.exf))) return rc;
                if ((rc = upload_s(s.get(), t2.eyf, &F.eyf))) return rc;
                if ((rc = upload_s(s.get(), t2.eg, &F.eg))) return rc;
                std::vector<double> cca(4 * (size_t)m.n_total, 0.0);
                for (size_t n = 0; n < (size_t)m.n_total; ++n) {
                    cca[4 * n] = ta.ccx[n]; cca[4 * n + 1] = ta.ccy[n]; cca[4 * n + 2] = fa.area[n];
                }
                if ((rc = upload_s(s.get(), cca, &F.cca))) return rc;
                F.threads = tile_cells;
                CK(tile::prepare_fused(precision, F));
                s->fused = true;
                CK(s->alloc(&s->work, kWorkSlots));
                CK(cudaMemset(s->work, 0, kWorkSlots * sizeof(int)));
                s->work_grid = tile::work_grid_fused(precision, F, ta.n_tiles);
                const int sched = opt ? opt->schedule : FV_SCHED_TILE;
                if (sched < FV_SCHED_TILE || sched > FV_SCHED_TILE2) return fail(FV_ERR_ARG, "unknown schedule");
                if (sched == FV_SCHED_TILE2 && tile_cells > kTileMax / 2)
                    return fail(FV_ERR_ARG, "two threads per cell need tiles of at most 128 cells");
                if (sk == FV_STAGE_HYBRID && sched == FV_SCHED_WORKLIST)
                    return fail(FV_ERR_ARG, "the work-list schedule needs the dt kernel of the fused layout");
                s->sched = sched;
                // automatic choice: in FP32 the split first stage (its gradient
                // kernel computes dt) saves more than it costs; in FP64 the
                // fused first stage and the separate dt kernel are faster
                s->split_first = sk == FV_STAGE_HYBRID ||
                                 (sk == FV_STAGE_AUTO && sched != FV_SCHED_WORKLIST && precision == FV_PREC_FP32);
            }
        }
    }
    const size_t nq = (size_t)m.n_total * ph->V;
    CK(s->alloc(&s->qbase[0], nq)); CK(s->alloc(&s->qbase[1], nq));
    if (s->f32) {
        CK(s->alloc(&s->sbase[0], nq, 4)); CK(s->alloc(&s->sbase[1], nq, 4));
    } else {
        s->sbase[0] = s->qbase[0]; s->sbase[1] = s->qbase[1];
    }
    CK(s->alloc(&s->tmp[0], nq, s->ssz)); CK(s->alloc(&s->tmp[1], nq, s->ssz));
    CK(s->alloc(&s->gx, nq, s->ssz)); CK(s->alloc(&s->gy, nq, s->ssz)); CK(s->alloc(&s->lim, nq, s->ssz));
    CK(s->alloc(&s->stage_buf, nq));
    // one more slot: a decomposition's copy of reference cell 0's dt
    CK(s->alloc(&s->dt, (size_t)m.n_total + 1));
    CK(s->alloc(&s->partials, (size_t)ta.n_tiles * ph->V));
    CK(s->alloc(&s->scratch2, 8));
    CK(s->alloc(&s->flag, 4));
    CK(s->alloc(&s->ctrl, 1));
    CK(cudaHostAlloc((void**)&s->hctrl, sizeof(Ctrl), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void**)&s->hctrl_dev, s->hctrl, 0));
    CK(s->alloc(&s->limits, 1));
    s->hist_cap = 4096;
    CK(s->alloc(&s->hist, (size_t)s->hist_cap));
    for (void* p : {(void*)s->qbase[0], (void*)s->qbase[1], s->tmp[0], s->tmp[1], s->gx, s->gy, s->lim})
        CK(cudaMemsetAsync(p, 0, nq * (p == (void*)s->qbase[0] || p == (void*)s->qbase[1] ? 8 : s->ssz), s->stream));
    if (s->f32) {
        CK(cudaMemsetAsync(s->sbase[0], 0, nq * 4, s->stream));
        CK(cudaMemsetAsync(s->sbase[1], 0, nq * 4, s->stream));
    }
    CK(cudaMemsetAsync(s->ctrl, 0, sizeof(Ctrl), s->stream));
    s->keys = s->ctrl->dtkeys;
    if (m.case_real_off.size() > 2) {
        // a batch of independent cases: per-case dt keys, times and lookups
        const int nc = (int)m.case_real_off.size() - 1;
        s->n_cases = nc;
        s->case_real_off = m.case_real_off;
        s->case_bound_off = m.case_bound_off;
        auto case_of_ref = [&](int64_t r) {
            const std::vector<int64_t>& o = r < m.n_real ? m.case_real_off : m.case_bound_off;
            const int64_t x = r < m.n_real ? r : r - m.n_real;
            return (int32_t)(std::upper_bound(o.begin(), o.end(), x) - o.begin() - 1);
        };
        std::vector<int32_t> cell_case(m.n_total), case_cell0(nc), tile_case(ta.n_tiles);
        for (int64_t n = 0; n < m.n_total; ++n) cell_case[n] = case_of_ref(m.new2ref[n]);
        for (int k = 0; k < nc; ++k) case_cell0[k] = m.ref2new[m.case_real_off[k]];
        for (int t = 0; t < ta.n_tiles; ++t) {
            const int64_t a = (int64_t)t * tile_cells, b = std::min<int64_t>(a + tile_cells, m.n_real) - 1;
            tile_case[t] = cell_case[a] == cell_case[b] ? cell_case[a] : -1;
        }
        Params& Pb = s->TP.P;
        Pb.n_cases = nc;
        if ((rc = upload_v(s.get(), cell_case, &Pb.cell_case))) return rc;
        if ((rc = upload_v(s.get(), case_cell0, &Pb.case_cell0))) return rc;
        if ((rc = upload_v(s.get(), tile_case, &Pb.tile_case))) return rc;
        CK(s->alloc(&s->case_time, (size_t)nc));
        CK(cudaMemsetAsync(s->case_time, 0, (size_t)nc * 8, s->stream));
        Pb.case_time = s->case_time;
        CK(s->alloc(&s->keys, (size_t)nc * kDtSlots));
    } else {
        s->TP.P.n_cases = 1;
    }
    if (s->TP.P.smooth) {
        for (auto*& b : s->qts) {
            CK(s->alloc(&b, nq));
            CK(cudaMemsetAsync(b, 0, nq * 8, s->stream));  // ghosts keep qt = 0
        }
        const uint32_t* d;
        if ((rc = upload_v(s.get(), fa.nbr, &d))) return rc;
        s->nbr = const_cast<uint32_t*>(d);
    }
    launch_fill_ghost_grad(s->gx, s->gy, s->lim, (int)m.n_real, (int)m.n_total, ph->V, s->f32, s->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    *out = s.release();
    return FV_OK;
}

int fv_solver_destroy(fv_solver* s) {
    delete s;
    return FV_OK;
}

int fv_solver_create_tuned(const fv_mesh* fm, const fv_physics* ph, int32_t precision, int32_t device,
                           const double* q, const double* alpha, int32_t n_alpha, int32_t n_steps,
                           fv_solver** out, int32_t* tile_cells, double* ms_per_step) {
    if (!fm || !ph || !q || !alpha || n_alpha < 1 || n_steps < 1 || !out)
        return fail(FV_ERR_ARG, "fv_solver_create_tuned: invalid arguments");
    fv_solver* best = nullptr;
    double best_ms = 0.0;
    int best_t = 0;
    // candidates: tile size x edge-tile layout (the split gradient and flux
    // kernels over one-ring tiles, or the fused stage kernel over two-ring
    // tiles where the physics allow it); a solver built for the fused kernel
    // holds both layouts, so each tile size is built once
    for (int t : {64, 128, 256}) {
        fv_solver_options o{t, FV_STAGE_AUTO, FV_SCHED_TILE};
        fv_solver* s = nullptr;
        int rc = fv_solver_create_ex(fm, ph, precision, device, &o, &s);
        if (rc == FV_ERR_MESH) continue;  // tile halo too large for this size
        if (rc) { fv_solver_destroy(best); return rc; }
        const bool can_fuse = s->fused;
        // split; fused with FV_SCHED_TILE, FV_SCHED_WORKLIST, FV_SCHED_TILE2;
        // fused with the split first stage (FV_SCHED_TILE)
        double ms_of[5] = {1e300, 1e300, 1e300, 1e300, 1e300};
        auto set_variant = [&](int v) {
            s->fused = v >= 1;
            s->sched = (v >= 1 && v <= 3) ? v - 1 : FV_SCHED_TILE;
            s->split_first = v == 4;
        };
        for (int variant = can_fuse ? 4 : 0; variant >= 0; --variant) {
            if (variant == 3 && t > kTileMax / 2) continue;
            clear_graphs(s);
            set_variant(variant);
            // one untimed step (graph capture), then n_steps timed on the device
            fv_run_options ro{};
            ro.max_step = 1; ro.max_time = 1e300; ro.tolerance = -1.0; ro.print_interval = 1ull << 62;
            ro.n_alpha = n_alpha; ro.alpha = alpha; ro.restart = 1;
            fv_run_info info{};
            if ((rc = fv_set_state(s, q)) || (rc = fv_run(s, &ro, &info))) { fv_solver_destroy(s); fv_solver_destroy(best); return rc; }
            ro.max_step = 1 + (uint64_t)n_steps; ro.restart = 0;
            if ((rc = fv_run(s, &ro, &info))) { fv_solver_destroy(s); fv_solver_destroy(best); return rc; }
            ms_of[variant] = s->last_ms / n_steps;
        }
        const int v = (int)(std::min_element(ms_of, ms_of + 5) - ms_of);
        const double ms = ms_of[v];
        clear_graphs(s);
        set_variant(v);
        if (!best || ms < best_ms) {
            fv_solver_destroy(best);
            best = s; best_ms = ms; best_t = t;
        } else {
            fv_solver_destroy(s);
        }
    }
    if (!best) return fail(FV_ERR_MESH, "fv_solver_create_tuned: no tile size fits this mesh");
    int rc = fv_set_state(best, q);
    if (rc) { fv_solver_destroy(best); return rc; }
    CK(cudaMemsetAsync(best->ctrl, 0, sizeof(Ctrl), best->stream));
    CK(cudaStreamSynchronize(best->stream));
    *out = best;
    if (tile_cells) *tile_cells = best_t;
    if (ms_per_step) *ms_per_step = best_ms;
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

// after the FP64 base changes, refresh its stage-precision copy
static void sync_shadow(fv_solver* s, int b) {
    if (s->f32) launch_to_float(s->qbase[b], (float*)s->sbase[b], (size_t)s->n_total * s->V, s->stream);
}

static int set_state_common(fv_solver* s, const double* q, cudaMemcpyKind kind) {
    if (!s || !q) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    const size_t nq = (size_t)s->n_total * s->V;
    const double* src = q;
    if (kind != cudaMemcpyDeviceToDevice) {  // device input is permuted in place, without a copy
        CK(cudaMemcpyAsync(s->stage_buf, q, nq * 8, kind, s->stream));
        src = s->stage_buf;
    }
    launch_permute_to_device(src, s->qbase[0], s->new2ref, (int)s->n_total, s->V, s->stream);
    sync_shadow(s, 0);
    CK(cudaGetLastError());
    return FV_OK;
}
static int get_state_common(fv_solver* s, double* q, cudaMemcpyKind kind) {
    if (!s || !q) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    const size_t nq = (size_t)s->n_total * s->V;
    if (kind == cudaMemcpyDeviceToDevice) {  // straight into the caller's device array
        launch_permute_to_ref(s->qbase[0], q, s->new2ref, (int)s->n_total, s->V, s->stream);
        CK(cudaGetLastError());
        return FV_OK;
    }
    launch_permute_to_ref(s->qbase[0], s->stage_buf, s->new2ref, (int)s->n_total, s->V, s->stream);
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

int fv_solver_continue_from(fv_solver* dst, fv_solver* src) {
    if (!dst || !src || dst == src) return fail(FV_ERR_ARG, "fv_solver_continue_from: need two solvers");
    if (dst->device != src->device) return fail(FV_ERR_ARG, "fv_solver_continue_from: solvers on different devices");
    if (dst->n_total != src->n_total || dst->n_real != src->n_real || dst->V != src->V)
        return fail(FV_ERR_ARG, "fv_solver_continue_from: solvers of different meshes");
    CK(cudaSetDevice(dst->device));
    CK(cudaStreamSynchronize(src->stream));
    // through reference numbering, so the two device orders need not agree
    launch_permute_to_ref(src->qbase[0], dst->stage_buf, src->new2ref, (int)src->n_total, src->V, dst->stream);
    launch_permute_to_device(dst->stage_buf, dst->qbase[0], dst->new2ref, (int)dst->n_total, dst->V, dst->stream);
    sync_shadow(dst, 0);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst->ctrl, src->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, dst->stream));
    if (dst->n_cases != src->n_cases) return fail(FV_ERR_ARG, "fv_solver_continue_from: different batches");
    if (dst->case_time)
        CK(cudaMemcpyAsync(dst->case_time, src->case_time, (size_t)dst->n_cases * 8, cudaMemcpyDeviceToDevice,
                           dst->stream));
    CK(cudaStreamSynchronize(dst->stream));
    return FV_OK;
}

int fv_solver_set_ghost_states(fv_solver* s, const double* bv) {
    if (!s) return fail(FV_ERR_ARG, "fv_solver_set_ghost_states: null solver");
    if (s->V != 4) return fail(FV_ERR_UNSUPPORTED, "per-ghost boundary states need V = 4");
    CK(cudaSetDevice(s->device));
    if (!bv) {
        s->TP.P.ghost_bv = nullptr;
    } else {
        if (!s->ghost_bv) CK(s->alloc(&s->ghost_bv, (size_t)s->n_bound * 4));
        // reference ghost order -> device ghost order
        std::vector<int32_t> n2r((size_t)s->n_total);
        CK(cudaMemcpy(n2r.data(), s->new2ref, n2r.size() * 4, cudaMemcpyDeviceToHost));
        std::vector<double> dev((size_t)s->n_bound * 4);
        for (int64_t b = 0; b < s->n_bound; ++b) {
            const int64_t r = (int64_t)n2r[(size_t)(s->n_real + b)] - s->n_real;
            for (int k = 0; k < 4; ++k) dev[(size_t)b * 4 + k] = bv[(size_t)r * 4 + k];
        }
        CK(cudaMemcpy(s->ghost_bv, dev.data(), dev.size() * 8, cudaMemcpyHostToDevice));
        s->TP.P.ghost_bv = s->ghost_bv;
    }
    // captured step graphs hold the old parameters
    for (auto& g : s->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    s->graphs.clear();
    return FV_OK;
}

int fv_batch_times(fv_solver* s, double* times) {
    if (!s || !times) return fail(FV_ERR_ARG, "fv_batch_times: null argument");
    CK(cudaSetDevice(s->device));
    if (s->case_time) {
        CK(cudaMemcpyAsync(times, s->case_time, (size_t)s->n_cases * 8, cudaMemcpyDeviceToHost, s->stream));
    } else {
        Ctrl hc;
        CK(cudaMemcpyAsync(&hc, s->ctrl, sizeof(hc), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        times[0] = hc.time;
    }
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}
int fv_get_state_device(fv_solver* s, double* q) { return get_state_common(s, q, cudaMemcpyDeviceToDevice); }

// ---------------------------------------------------------------- run ----
}  // extern "C"

namespace fvgpu {

int set_error(int code, const std::string& msg) { return fail(code, msg); }

int step_open(fv_solver* s, const std::vector<double>& alpha, int b, bool first, StepCursor& c, EventLog* log,
              bool with_dt) {
    const TileParams& TP = s->TP;
    cudaStream_t st = s->stream;
    int n = 0;
    auto mark = [&](int k) { if (log) log->mark(k); };
    if (first) { launch_step_begin(s->ctrl, s->limits, s->V, s->keys, s->n_cases * kDtSlots, st); ++n; mark(KK_BEGIN); }
    TileIO& io = c.io;
    io = TileIO{};
    io.gx = s->gx; io.gy = s->gy; io.lim = s->lim; io.dt = s->dt; io.ctrl = s->ctrl;
    io.dtkeys = s->keys;
    io.q_stage = s->sbase[b];
    c.b = b;
    // the fused stage kernel computes its gradients itself: the step's dt
    // comes from the dt kernel, as in first order
    c.grads = (TP.P.order2 || TP.P.diffusive) && !s->fused;
    // the split first stage's gradient kernel computes dt
    c.split_first = s->fused && s->split_first;
    // the work-list schedule: one tile counter per stage, zeroed by the dt kernel
    c.worklist = s->fused && s->sched == FV_SCHED_WORKLIST && alpha.size() <= (size_t)kWorkSlots;
    c.FPl = s->FPm;
    c.FPl.P = TP.P;
    c.FPl.threads = (s->sched == FV_SCHED_TILE2) ? 2 * c.FPl.T : c.FPl.T;
    c.in = s->sbase[b];
    c.out = nullptr;
    if (with_dt) n += step_dt(s, c, log);
    return n;
}

int step_dt(fv_solver* s, StepCursor& c, EventLog* log) {
    // every kernel after step_begin is a programmatic dependent of the one
    // before it (its constant tile data is staged during that one's tail)
    if (c.grads || c.split_first) return 0;
    TileIO dio = c.io;
    dio.work_reset = c.worklist ? s->work : nullptr;
    tile::launch_dt(s->precision, s->TP, dio, s->stream, true);
    if (log) log->mark(KK_DT);
    return 1;
}

int step_stage(fv_solver* s, const std::vector<double>& alpha, int k, StepCursor& c, EventLog* log,
               const TileRange* r) {
    const TileParams& TP = s->TP;
    cudaStream_t st = s->stream;
    const bool pdl = true;
    int n = 0;
    auto mark = [&](int kk) { if (log) log->mark(kk); };
    const int ns = (int)alpha.size(), b = c.b;
    const bool last = k == ns - 1;
    TileIO so = c.io;
    so.q_stage = c.in;
    so.q_base = s->qbase[b];
    so.alpha = alpha[k];
    so.partials = last ? s->partials : nullptr;
    void* out_s;
    if (ns == 1) {
        so.q_out = s->qbase[1 - b];
        out_s = s->sbase[1 - b];
    } else if (last) {
        so.q_out = s->qbase[b];
        out_s = s->sbase[b];
    } else {
        out_s = s->tmp[k % 2];
        so.q_out = s->f32 ? nullptr : (double*)out_s;
    }
    so.s_out = s->f32 ? out_s : nullptr;
    so.write_f64 = last ? 1 : 0;
    if (r) {
        if (!s->fused || c.worklist || c.split_first) return -1;
        const PartIO pio{r->t0, nullptr, k, ns};
        if (r->n > 0) {
            tile::launch_fused(s->precision, c.FPl, so, r->stream ? r->stream : st, r->pdl, r->n, r->n, &pio);
            ++n; mark(KK_FUSED);
        }
        c.out = out_s;
        if (r->last) c.in = out_s;
        return n;
    }
    if (c.grads) { tile::launch_gradlim(s->precision, TP, so, st, k == 0, pdl); ++n; mark(KK_GRADLIM); }
    if (TP.P.smooth) {
        // time derivatives, two Jacobi sweeps of smoothing, then the update
        // from the smoothed derivatives (explicit.cpp:742-744)
        so.qt = s->qts[0];
        tile::launch_stage(s->precision, TP, so, st, pdl, 1); ++n; mark(KK_STAGE);
        launch_smooth(TP.P, s->nbr, s->qts[0], s->qts[0], s->qts[1], st); ++n; mark(KK_STAGE);
        launch_smooth(TP.P, s->nbr, s->qts[1], s->qts[0], s->qts[2], st); ++n; mark(KK_STAGE);
        so.qt = s->qts[2];
        tile::launch_stage(s->precision, TP, so, st, pdl, 2); ++n; mark(KK_STAGE);
    } else if (s->fused && c.split_first && k == 0) {
        tile::launch_gradlim(s->precision, TP, so, st, true, pdl); ++n; mark(KK_GRADLIM);
        tile::launch_stage(s->precision, TP, so, st, pdl); ++n; mark(KK_STAGE);
    } else if (s->fused) {
        so.work = c.worklist ? s->work + k : nullptr;
        const PartIO pio{0, c.worklist ? nullptr : c.remote, k, ns};
        tile::launch_fused(s->precision, c.FPl, so, st, pdl, s->n_tiles, s->work_grid, c.part ? &pio : nullptr);
        ++n; mark(KK_FUSED);
    } else {
        tile::launch_stage(s->precision, TP, so, st, pdl); ++n; mark(KK_STAGE);
    }
    c.in = out_s;
    c.out = out_s;
    return n;
}

int step_close(fv_solver* s, const double* partials, int nblocks, EventLog* log) {
    launch_step_end(s->TP.P, s->ctrl, s->limits, partials, nblocks, s->dt, s->keys, s->n_cases * kDtSlots,
                    s->hist, s->hist_cap, s->stream, true);
    if (log) log->mark(KK_END);
    return 1;
}

}  // namespace fvgpu

extern "C" {

// Enqueues one time step (explicit.cpp:715-801) whose base state is
// qbase[b] (RK1 writes its result to qbase[1-b]).  Returns the number of
// kernels launched.
// first: the first step of a launch sequence, which starts with the
// begin-of-step kernel (every step end also begins the next step).
static int enqueue_step(fv_solver* s, const std::vector<double>& alpha, int b, EventLog* log = nullptr,
                        bool first = true) {
    StepCursor c;
    int n = step_open(s, alpha, b, first, c, log);
    for (int k = 0; k < (int)alpha.size(); ++k) n += step_stage(s, alpha, k, c, log);
    n += step_close(s, s->partials, s->n_tiles, log);
    return n;
}

// One captured graph of `len` consecutive steps starting from qbase[0]
// (RK1 alternates qbase[0] and qbase[1] between steps).
static int get_graph(fv_solver* s, const std::vector<double>& alpha, int len, GraphEntry** out) {
    for (auto& g : s->graphs)
        if (g.alpha == alpha && g.chunk == len) { *out = &g; return FV_OK; }
    GraphEntry g;
    g.alpha = alpha;
    g.chunk = len;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    for (int k = 0; k < len; ++k)
        launches += enqueue_step(s, alpha, (alpha.size() == 1 && (k % 2)) ? 1 : 0, nullptr, k == 0);
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

// RK1 leaves the state in qbase[1] after an odd number of steps
static int settle_base(fv_solver* s, unsigned long long steps_taken) {
    if (steps_taken % 2) {
        CK(cudaMemcpyAsync(s->qbase[0], s->qbase[1], (size_t)s->n_total * s->V * 8, cudaMemcpyDeviceToDevice,
                           s->stream));
        if (s->f32)
            CK(cudaMemcpyAsync(s->sbase[0], s->sbase[1], (size_t)s->n_total * s->V * 4, cudaMemcpyDeviceToDevice,
                               s->stream));
    }
    return FV_OK;
}

int fv_run(fv_solver* s, const fv_run_options* o, fv_run_info* info) {
    if (!s || !o) return fail(FV_ERR_ARG, "fv_run: null argument");
    if (o->n_alpha < 1 || o->n_alpha > 16 || !o->alpha) return fail(FV_ERR_ARG, "fv_run: need 1..16 RK stages");
    if (o->print_interval == 0) return fail(FV_ERR_ARG, "fv_run: print_interval must be > 0");
    CK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    std::vector<double> alpha(o->alpha, o->alpha + o->n_alpha);
    // limits and control go through small kernels and mapped memory, never
    // through the copy engines, which callers may keep busy with state
    // transfers on other streams
    const RunLimits L{o->max_step, o->max_time, o->tolerance, o->print_interval};
    launch_set_limits(s->limits, L, st);
    const Ctrl& hc = *s->hctrl;
    if (o->restart) {
        launch_ctrl_reset(s->ctrl, st);
        launch_ctrl_copy(s->ctrl, s->hctrl_dev, st);
        if (s->case_time) CK(cudaMemsetAsync(s->case_time, 0, (size_t)s->n_cases * 8, st));
        // run(): initial ghost fill with zeroed gx, gy, limiters (explicit.cpp:712)
        exact::launch_bounds(s->TP.P, s->qbase[0], nullptr, nullptr, nullptr, 1, st);
        sync_shadow(s, 0);
        CK(cudaGetLastError());
    } else {
        launch_ctrl_copy(s->ctrl, s->hctrl_dev, st);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    const unsigned long long start_step = o->restart ? 0ull : hc.step;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
    std::vector<PrintRec> recs(s->hist_cap);
    double total_ms = 0.0;
    int64_t launches = 0;
    unsigned long long cur = start_step;
    for (;;) {
        // graph length: the largest power of two <= min(chunk, steps left), so
        // runs bounded by max_step launch no idle steps
        const unsigned long long left = o->max_step > cur ? o->max_step - cur : 1ull;
        int len = 1;
        while ((unsigned long long)(len * 2) <= left && len * 2 <= s->chunk) len *= 2;
        GraphEntry* g = nullptr;
        int rc = get_graph(s, alpha, len, &g);
        if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
        CK(cudaEventRecord(e0, st));
        CK(cudaGraphLaunch(g->exec, st));  // its first kernel empties the print records
        CK(cudaEventRecord(e1, st));
        launches += g->launches;
        launch_ctrl_copy(s->ctrl, s->hctrl_dev, st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        total_ms += ms;
        if (alpha.size() == 1 && (rc = settle_base(s, hc.step - cur))) return rc;
        cur = hc.step;
        if (o->on_print && hc.n_hist > 0) {
            CK(cudaMemcpy(recs.data(), s->hist, sizeof(PrintRec) * hc.n_hist, cudaMemcpyDeviceToHost));
            for (int k = 0; k < hc.n_hist; ++k) o->on_print(o->user, recs[k].step, recs[k].time, recs[k].R, s->V);
        }
        double Rmax = 1.0;
        if (hc.step > 0) {
            Rmax = 0.0;
            // std::max(R[k], Rmax) as in explicit.cpp:720 (a NaN residual propagates)
            for (int k = 0; k < s->V; ++k) Rmax = (hc.R[k] < Rmax) ? Rmax : hc.R[k];
        }
        const bool done = !hc.active || hc.step >= o->max_step || hc.time >= o->max_time || Rmax < o->tolerance;
        if (done) break;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
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
    log.mark(-1);
    for (int k = 0; k < n_steps; ++k) enqueue_step(s, a, (a.size() == 1 && (k % 2)) ? 1 : 0, &log, k == 0);
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
    int rc;
    if (a.size() == 1 && (rc = settle_base(s, (unsigned long long)n_steps))) return rc;
    CK(cudaStreamSynchronize(st));
    return FV_OK;
}

int fv_solver_info(fv_solver* s, int64_t* out) {
    if (!s || !out) return fail(FV_ERR_ARG, "null argument");
    out[0] = s->n_tiles; out[1] = s->TP.T; out[2] = s->TP.max_halo; out[3] = s->TP.max_edges;
    out[4] = s->precision; out[5] = (int64_t)s->ssz;
    return FV_OK;
}

int fv_solver_stage_kernels(fv_solver* s) {
    if (!s) return fail(FV_ERR_ARG, "null solver");
    return s->fused ? (s->split_first ? FV_STAGE_HYBRID : FV_STAGE_FUSED) : FV_STAGE_SPLIT;
}

int fv_solver_schedule(fv_solver* s) {
    if (!s) return fail(FV_ERR_ARG, "null solver");
    return s->fused ? s->sched : FV_SCHED_TILE;
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
    launch_check_state(s->TP.P, s->qbase[0], s->flag, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h, s->flag, 4, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (h) return fail(FV_ERR_NONFINITE, "non-finite or non-physical state (rho <= 0 or p <= 0)");
    return FV_OK;
}

int fv_boundary_force(fv_solver* s, int32_t group, double* fx, double* fy) {
    if (!s || !fx || !fy || s->V != 4) return fail(FV_ERR_ARG, "fv_boundary_force: invalid arguments");
    CK(cudaSetDevice(s->device));
    launch_force(s->TP.P, s->qbase[0], group, s->scratch2, s->stream);
    CK(cudaGetLastError());
    double h[2];
    CK(cudaMemcpyAsync(h, s->scratch2, 16, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *fx = h[0]; *fy = h[1];
    return FV_OK;
}

// ------------------------------------------------------- stage entry points --
// Test and debugging paths: host arrays in reference numbering, converted to
// the device numbering and the stage precision.  Temporaries are allocated
// per call.
namespace {
struct DevTmp {
    std::vector<void*> p;
    ~DevTmp() { for (void* x : p) cudaFree(x); }
    cudaError_t get(void** out, size_t bytes) {
        cudaError_t e = cudaMalloc(out, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) p.push_back(*out);
        return e;
    }
};
}  // namespace

int fv_output_fields(fv_solver* s, const double* q, int64_t n, int32_t n_fields, const int32_t* kinds,
                     double* out) {
    if (!s || !kinds || !out || n_fields < 0 || n_fields > 8) return fail(FV_ERR_ARG, "fv_output_fields: invalid arguments");
    if (q && n != s->n_real && n != s->n_total) return fail(FV_ERR_ARG, "fv_output_fields: n must be n_real or n_total");
    OutputPlan plan{};
    plan.n = n_fields;
    int64_t total = 0;
    for (int f = 0; f < n_fields; ++f) {
        const int k = kinds[f];
        const int nc = (k == FV_OUT_PRESSURE || k == FV_OUT_MACH) ? 1 : (k == FV_OUT_VELOCITY || k == FV_OUT_STATE01) ? 2 : 0;
        if (nc == 0) return fail(FV_ERR_UNSUPPORTED, "fv_output_fields: unknown output kind");
        if (s->V < (k == FV_OUT_STATE01 ? 2 : 4)) return fail(FV_ERR_UNSUPPORTED, "fv_output_fields: kind needs more variables");
        plan.kind[f] = k;
        plan.off[f] = total;
        total += nc * s->n_real;
    }
    CK(cudaSetDevice(s->device));
    DevTmp T;
    double* d_out;
    CK(T.get((void**)&d_out, (size_t)std::max<int64_t>(total, 1) * 8));
    if (q) {
        double* d_q;
        CK(T.get((void**)&d_q, (size_t)s->n_real * s->V * 8));
        CK(cudaMemcpyAsync(d_q, q, (size_t)s->n_real * s->V * 8, cudaMemcpyHostToDevice, s->stream));
        launch_output_fields(d_q, s->V, nullptr, (int)s->n_real, s->TP.P.gamma, plan, d_out, s->stream);
    } else {
        launch_output_fields(s->qbase[0], s->V, s->new2ref, (int)s->n_real, s->TP.P.gamma, plan, d_out, s->stream);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d_out, (size_t)total * 8, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

// host (reference order, FP64) -> device (device order, FP64 in d64 and,
// if d_s != nullptr and FP32 mode, an FP32 copy in d_s)
static int h2d(fv_solver* s, const double* h, double* d64, void* d_s, int V) {
    CK(cudaMemcpyAsync(s->stage_buf, h, (size_t)s->n_total * V * 8, cudaMemcpyHostToDevice, s->stream));
    launch_permute_to_device(s->stage_buf, d64, s->new2ref, (int)s->n_total, V, s->stream);
    if (d_s && s->f32) launch_to_float(d64, (float*)d_s, (size_t)s->n_total * V, s->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}
static int d2h(fv_solver* s, const double* d64, double* h, int V) {
    launch_permute_to_ref(d64, s->stage_buf, s->new2ref, (int)s->n_total, V, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h, s->stage_buf, (size_t)s->n_total * V * 8, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}
// device array of the stage precision -> FP64 (in place for FP64 modes)
static const double* as_f64(fv_solver* s, const void* a, double* tmp64, int V) {
    if (!s->f32) return (const double*)a;
    launch_to_double((const float*)a, tmp64, (size_t)s->n_total * V, s->stream);
    return tmp64;
}

int fv_stage_dt(fv_solver* s, const double* q, double* dt, int32_t global_min) {
    if (!s || !q || !dt) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    DevTmp T;
    const size_t nq = (size_t)s->n_total * s->V;
    double* q64; void* qs; unsigned long long* keys;
    CK(T.get((void**)&q64, nq * 8));
    CK(T.get(&qs, nq * s->ssz));
    const size_t nkeys = (size_t)s->n_cases * kDtSlots;
    CK(T.get((void**)&keys, nkeys * 8));
    int rc = h2d(s, q, q64, qs, s->V);
    if (rc) return rc;
    CK(cudaMemsetAsync(keys, 0xFF, nkeys * 8, s->stream));
    TileParams TP = s->TP;
    TP.P.global_dt = global_min ? 1 : 0;
    TileIO io{};
    io.q_stage = s->f32 ? qs : q64;
    io.dt = s->dt;
    io.dtkeys = keys;
    tile::launch_dt(s->precision, TP, io, s->stream);
    CK(cudaGetLastError());
    std::vector<double> dd(s->n_total);
    if ((rc = d2h(s, s->dt, dd.data(), 1))) return rc;
    if (global_min) {
        // per case (one for a single mesh): min over its real and ghost cells;
        // a NaN in the case's dt[0] wins (min_dt, explicit.cpp:555-564)
        std::vector<unsigned long long> hk(nkeys);
        CK(cudaMemcpy(hk.data(), keys, nkeys * 8, cudaMemcpyDeviceToHost));
        std::vector<int64_t> ro = s->case_real_off, bo = s->case_bound_off;
        if (s->n_cases == 1) { ro = {0, s->n_real}; bo = {0, s->n_bound}; }
        for (int k = 0; k < s->n_cases; ++k) {
            unsigned long long key = ~0ull;
            for (int i = 0; i < kDtSlots; ++i) key = hk[(size_t)k * kDtSlots + i] < key ? hk[(size_t)k * kDtSlots + i] : key;
            double mn;
            if (key == ~0ull) {
                mn = std::nan("");
            } else {
                unsigned long long b = (key & 0x8000000000000000ull) ? (key & 0x7fffffffffffffffull) : ~key;
                std::memcpy(&mn, &b, 8);
            }
            const double d0 = dd[(size_t)ro[k]];
            if (d0 != d0) mn = d0;
            for (int64_t r = ro[k]; r < ro[k + 1]; ++r) dd[(size_t)r] = mn;
            for (int64_t b = bo[k]; b < bo[k + 1]; ++b) dd[(size_t)(s->n_real + b)] = mn;
        }
    }
    std::memcpy(dt, dd.data(), dd.size() * 8);
    return FV_OK;
}

// ------------------------------------------ time step without allocation --
// fv_stage_dt_noalloc: the time-step kernel for callers that must not
// allocate device memory.  Its working arrays live in one statically sized
// device array (every GPU that loads this library holds it until exit).
namespace {
constexpr size_t kNoAllocBytes = size_t(8) << 20;  // 8 MiB of scratch per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];
std::mutex g_noalloc_mu;
void* g_noalloc_base[128] = {};  // device address of g_noalloc_scratch, per device ordinal

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// global minimum of the slot keys (min_dt, explicit.cpp:555-564; a NaN in
// dt[0] wins) written to every entry of the caller's output
__global__ void k_noalloc_dt_fill(const unsigned long long* keys, const double* dt_dev, int cell0, double* out, int n) {
    unsigned long long key = ~0ull;
    for (int i = 0; i < kDtSlots; ++i) key = keys[i] < key ? keys[i] : key;
    const double d0 = dt_dev[cell0];
    const double mn = (d0 != d0) ? d0 : tkey_inv(key);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = mn;
}
}  // namespace

int fv_stage_dt_noalloc(fv_solver* s, const double* q_device, double* dt_device, int32_t global_min, void* stream) {
    if (!s || !q_device || !dt_device) return fail(FV_ERR_ARG, "fv_stage_dt_noalloc: null argument");
    if (s->n_cases > 1) return fail(FV_ERR_UNSUPPORTED, "fv_stage_dt_noalloc: batches of cases use fv_stage_dt");
    const size_t nt = (size_t)s->n_total, V = (size_t)s->V;
    const size_t need = align256(kDtSlots * 8) + align256(nt * 8) + align256(nt * V * 8) +
                        (s->f32 ? align256(nt * V * 4) : 0);
    if (need > kNoAllocBytes)
        return fail(FV_ERR_ARG, "fv_stage_dt_noalloc: mesh needs " + std::to_string(need) +
                                    " bytes of scratch, more than the fixed " + std::to_string(kNoAllocBytes) +
                                    " (about 200k cells in FP64, 150k in FP32); use fv_stage_dt");
    if (s->device < 0 || s->device >= 128) return fail(FV_ERR_ARG, "fv_stage_dt_noalloc: device ordinal out of range");
    CK(cudaSetDevice(s->device));
    unsigned char* base = nullptr;
    {
        // one-time set-up per device: the host-side symbol is only a stand-in,
        // the kernels need the scratch array's device address (cached for the
        // life of the device's primary context)
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_base[s->device]) {
            void* p = nullptr;
            CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_noalloc_base[s->device] = p;
        }
        base = (unsigned char*)g_noalloc_base[s->device];
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    unsigned long long* keys = (unsigned long long*)base;
    double* dt_dev = (double*)(base + align256(kDtSlots * 8));
    double* q64 = (double*)((unsigned char*)dt_dev + align256(nt * 8));
    void* qs = s->f32 ? (void*)((unsigned char*)q64 + align256(nt * V * 8)) : (void*)q64;
    // the slots keep the previous call's minimum: they must start at +inf
    CK(cudaMemsetAsync(keys, 0xFF, kDtSlots * 8, st));
    launch_permute_to_device(q_device, q64, s->new2ref, (int)nt, (int)V, st);
    if (s->f32) launch_to_float(q64, (float*)qs, nt * V, st);
    TileParams TP = s->TP;
    TP.P.global_dt = global_min ? 1 : 0;
    TileIO io{};
    io.q_stage = qs;
    io.dt = dt_dev;
    io.dtkeys = keys;
    tile::launch_dt(s->precision, TP, io, st);
    if (global_min) k_noalloc_dt_fill<<<grid_for((int)nt), kBlock, 0, st>>>(keys, dt_dev, TP.P.cell0, dt_device, (int)nt);
    else launch_permute_to_ref(dt_dev, dt_device, s->new2ref, (int)nt, 1, st);
    CK(cudaGetLastError());
    return FV_OK;
}

int fv_stage_gradients_limiters(fv_solver* s, const double* q, double* gx, double* gy, double* lim) {
    if (!s || !q || !gx || !gy || !lim) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    DevTmp T;
    const size_t nq = (size_t)s->n_total * s->V;
    double* q64; void* qs; double* t64;
    CK(T.get((void**)&q64, nq * 8)); CK(T.get(&qs, nq * s->ssz)); CK(T.get((void**)&t64, nq * 8));
    int rc = h2d(s, q, q64, qs, s->V);
    if (rc) return rc;
    TileIO io{};
    io.q_stage = s->f32 ? qs : q64;
    io.gx = s->gx; io.gy = s->gy; io.lim = s->lim;
    tile::launch_gradlim(s->precision, s->TP, io, s->stream);
    CK(cudaGetLastError());
    if ((rc = d2h(s, as_f64(s, s->gx, t64, s->V), gx, s->V))) return rc;
    if ((rc = d2h(s, as_f64(s, s->gy, t64, s->V), gy, s->V))) return rc;
    if (s->precision != FV_PREC_FP64_EXACT && !s->TP.P.diffusive) {  // limiter already folded into gx, gy
        for (size_t i = 0; i < nq; ++i) lim[i] = 1.0;
        return FV_OK;
    }
    return d2h(s, as_f64(s, s->lim, t64, s->V), lim, s->V);
}

int fv_stage_update(fv_solver* s, const double* q_base, const double* q_stage, const double* gx, const double* gy,
                    const double* lim, const double* dt, double alpha, double* q_out) {
    if (!s || !q_base || !q_stage || !gx || !gy || !lim || !dt || !q_out) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    DevTmp T;
    const size_t nq = (size_t)s->n_total * s->V;
    double *b64, *s64, *o64, *t64;
    void *ss, *os;
    CK(T.get((void**)&b64, nq * 8)); CK(T.get((void**)&s64, nq * 8)); CK(T.get((void**)&o64, nq * 8));
    CK(T.get((void**)&t64, nq * 8)); CK(T.get(&ss, nq * s->ssz)); CK(T.get(&os, nq * s->ssz));
    int rc;
    if ((rc = h2d(s, q_base, b64, nullptr, s->V))) return rc;
    if ((rc = h2d(s, q_stage, s64, ss, s->V))) return rc;
    if ((rc = h2d(s, gx, t64, s->gx, s->V))) return rc;
    if (!s->f32) CK(cudaMemcpy(s->gx, t64, nq * 8, cudaMemcpyDeviceToDevice));
    if ((rc = h2d(s, gy, t64, s->gy, s->V))) return rc;
    if (!s->f32) CK(cudaMemcpy(s->gy, t64, nq * 8, cudaMemcpyDeviceToDevice));
    if ((rc = h2d(s, lim, t64, s->lim, s->V))) return rc;
    if (!s->f32) CK(cudaMemcpy(s->lim, t64, nq * 8, cudaMemcpyDeviceToDevice));
    if ((rc = h2d(s, dt, s->dt, nullptr, 1))) return rc;
    // ghosts of the output start as the stage state (every ghost is then overwritten)
    CK(cudaMemcpyAsync(o64, s64, nq * 8, cudaMemcpyDeviceToDevice, s->stream));
    TileIO io{};
    io.q_stage = s->f32 ? ss : s64;
    io.q_base = b64;
    io.q_out = o64;
    io.s_out = s->f32 ? os : nullptr;
    io.write_f64 = 1;
    io.gx = s->gx; io.gy = s->gy; io.lim = s->lim; io.dt = s->dt; io.alpha = alpha;
    tile::launch_stage(s->precision, s->TP, io, s->stream);
    CK(cudaGetLastError());
    rc = d2h(s, o64, q_out, s->V);
    // restore the invariant ghost gradient/limiter values
    launch_fill_ghost_grad(s->gx, s->gy, s->lim, (int)s->n_real, (int)s->n_total, s->V, s->f32, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    return rc;
}

int fv_stage_bounds(fv_solver* s, double* q, const double* gx, const double* gy, const double* lim) {
    if (!s || !q || !gx || !gy || !lim) return fail(FV_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    DevTmp T;
    const size_t nq = (size_t)s->n_total * s->V;
    double *q64, *gx64, *gy64, *l64;
    CK(T.get((void**)&q64, nq * 8)); CK(T.get((void**)&gx64, nq * 8));
    CK(T.get((void**)&gy64, nq * 8)); CK(T.get((void**)&l64, nq * 8));
    int rc;
    if ((rc = h2d(s, q, q64, nullptr, s->V))) return rc;
    if ((rc = h2d(s, gx, gx64, nullptr, s->V))) return rc;
    if ((rc = h2d(s, gy, gy64, nullptr, s->V))) return rc;
    if ((rc = h2d(s, lim, l64, nullptr, s->V))) return rc;
    exact::launch_bounds(s->TP.P, q64, gx64, gy64, l64, 0, s->stream);
    CK(cudaGetLastError());
    return d2h(s, q64, q, s->V);
}

}  // extern "C"

// ------------------------------------------------------------- adjoint ----
// Discrete adjoint of fv_run's FP64_EXACT step for the inflow-parameter
// problem: theta = (M, delta_1..delta_nb) sets the free stream (initial
// state rho_inf, u = M, v = 0, p_inf) and the inflow boundary states (density
// rho_inf (1 + delta_b) on the inflow faces of bin b, velocity M);
// loss = sum_n dt_n sum_{faces of loss_group} p(interior) le.  The forward
// run stores its state every `checkpoint_every` steps.  The reverse sweep
// takes the segments backwards: it recomputes a segment's step states from
// its checkpoint, then, for each step backwards, recomputes that step's
// stage states, gradients and limiters and runs the adjoint kernels of
// fv_adjoint.cu stage by stage backwards.  Device memory therefore holds the
// checkpoints, one segment's step states and one step's stage data.
struct fv_adjoint {
    fv_solver* s = nullptr;
    fv_adjoint_options o{};
    std::vector<double> alpha;
    int S = 0;                        // RK stages
    int nseg = 0;
    double rho_inf = 0, p_inf = 0, gamma = 1.4;
    std::vector<int32_t> ghost_bin;   // reference ghost order: bin, or -1
    std::vector<int32_t> ghost_kind;  // reference ghost order: boundary kind
    AdjFaces F{};
    std::vector<void*> allocs;
    std::vector<double*> ckpt;        // [nseg] states at segment starts
    std::vector<double*> Qn;          // [every + 1] step states of the segment being reversed
    std::vector<double*> Qs;          // [S] inputs of stages 1..S-1 of the step being reversed (Qs[0] unused)
    std::vector<double*> Gx, Gy, Lim; // [S] gradients and limiters of its stages
    double* dtc = nullptr;            // its per-cell dt
    double *tmp[2] = {nullptr, nullptr}, *tgx = nullptr, *tgy = nullptr, *tlim = nullptr;
    double *dt_fill = nullptr, *dt_n = nullptr, *loss = nullptr, *lam_dt = nullptr, *partials = nullptr;
    double *lamA = nullptr, *lamB = nullptr, *lam_qn = nullptr, *lgx = nullptr, *lgy = nullptr, *llim = nullptr;
    double *lam_bv = nullptr;
    unsigned long long* keys = nullptr;
    int* argmin = nullptr;
    int32_t* loss_ghosts = nullptr;   // device ghost indices of the loss group
    int n_loss = 0;
    std::vector<double> theta_last;
    template <class T>
    cudaError_t alloc(T** p, size_t n) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) allocs.push_back((void*)*p);
        return e;
    }
    ~fv_adjoint() {
        if (s) cudaSetDevice(s->device);
        for (void* p : allocs) cudaFree(p);
        delete s;
    }
};

namespace {
// One forward step from q (device numbering, all cells) to q_next.  With
// `store`, the inputs of stages 1..S-1 go to Qs[k], gradients to
// Gx/Gy/Lim[k] and per-cell dt to dtc; otherwise the adjoint's temporaries
// are used.
int adj_forward_step(fv_adjoint* a, const double* q, double* q_next, double* dt_slot, bool store,
                     bool with_loss) {
    fv_solver* s = a->s;
    cudaStream_t st = s->stream;
    const TileParams& TP = s->TP;
    const size_t nt = (size_t)s->n_total;
    double* dtcells = store ? a->dtc : a->dt_fill;
    CK(cudaMemsetAsync(a->keys, 0xFF, kDtSlots * 8, st));
    TileIO io{};
    io.q_stage = q;
    io.dt = dtcells;
    io.dtkeys = a->keys;
    tile::launch_dt(FV_PREC_FP64_EXACT, TP, io, st);
    adj_launch_dt_finalize(a->keys, dtcells, TP.P.cell0, a->dt_fill, (int)nt, dt_slot, st);
    if (with_loss && a->n_loss) adj_launch_loss(TP.P, q, dt_slot, a->loss_ghosts, a->n_loss, a->loss, st);
    const double* in = q;
    if (!store && s->fused) {
        // states only: the fused stage kernel (the same bits as the
        // gradient + stage kernels, without writing the gradients out)
        FusedParams FPl = s->FPm;
        FPl.P = TP.P;
        FPl.threads = (s->sched == FV_SCHED_TILE2) ? 2 * FPl.T : FPl.T;
        for (int k = 0; k < a->S; ++k) {
            double* out = (k == a->S - 1) ? q_next : a->tmp[k % 2];
            TileIO so{};
            so.q_stage = in;
            so.q_base = q;
            so.q_out = out;
            so.dt = a->dt_fill;
            so.alpha = a->alpha[(size_t)k];
            so.write_f64 = 1;
            tile::launch_fused(FV_PREC_FP64_EXACT, FPl, so, st, false, s->n_tiles, s->work_grid);
            in = out;
        }
        CK(cudaGetLastError());
        return FV_OK;
    }
    for (int k = 0; k < a->S; ++k) {
        double* gx = store ? a->Gx[(size_t)k] : a->tgx;
        double* gy = store ? a->Gy[(size_t)k] : a->tgy;
        double* lim = store ? a->Lim[(size_t)k] : a->tlim;
        double* out = (k == a->S - 1) ? q_next : (store ? a->Qs[(size_t)k + 1] : a->tmp[k % 2]);
        TileIO so{};
        so.q_stage = in;
        so.q_base = q;
        so.q_out = out;
        so.gx = gx; so.gy = gy; so.lim = lim;
        so.dt = a->dt_fill;
        so.alpha = a->alpha[(size_t)k];
        so.write_f64 = 1;
        if (TP.P.order2) tile::launch_gradlim(FV_PREC_FP64_EXACT, TP, so, st);
        tile::launch_stage(FV_PREC_FP64_EXACT, TP, so, st);
        in = out;
    }
    CK(cudaGetLastError());
    return FV_OK;
}

int adj_set_theta(fv_adjoint* a, const double* theta, double* q0_dev) {
    fv_solver* s = a->s;
    const double M = theta[0];
    const int nb = a->o.n_bins;
    const double e_inf = a->p_inf / (a->gamma - 1.0);
    // initial state: the free stream (reference numbering, ghosts filled below)
    std::vector<double> q((size_t)s->n_total * 4, 0.0);
    for (int64_t c = 0; c < s->n_total; ++c) {
        q[4 * c] = a->rho_inf; q[4 * c + 1] = a->rho_inf * M; q[4 * c + 2] = 0.0;
        q[4 * c + 3] = e_inf + 0.5 * a->rho_inf * M * M;
    }
    std::vector<double> bv((size_t)s->n_bound * 4, 0.0);
    for (int64_t r = 0; r < s->n_bound; ++r) {
        const int kind = a->ghost_kind[(size_t)r];
        if (kind != FV_BC_INLET_OUTLET && kind != FV_BC_FARFIELD && kind != FV_BC_FARFIELD_B0) continue;
        const int b = a->ghost_bin[(size_t)r];
        const double rho = a->rho_inf * (1.0 + (b >= 0 && b < nb ? theta[1 + b] : 0.0));
        bv[4 * r] = rho; bv[4 * r + 1] = rho * M; bv[4 * r + 2] = 0.0; bv[4 * r + 3] = e_inf + 0.5 * rho * M * M;
    }
    int rc = fv_solver_set_ghost_states(s, bv.data());
    if (rc) return rc;
    if ((rc = fv_set_state(s, q.data()))) return rc;
    CK(cudaMemcpyAsync(q0_dev, s->qbase[0], q.size() * 8, cudaMemcpyDeviceToDevice, s->stream));
    // run(): initial ghost fill with zeroed gradients (explicit.cpp:712)
    exact::launch_bounds(s->TP.P, q0_dev, nullptr, nullptr, nullptr, 1, s->stream);
    CK(cudaGetLastError());
    return FV_OK;
}

// stage k of the step whose input is qn and output qn1 (stages 1..S-1 in Qs)
AdjStage adj_stage(fv_adjoint* a, const double* qn, const double* qn1, int k, double dt) {
    AdjStage S{};
    const size_t i = (size_t)k;
    S.qs = k == 0 ? qn : a->Qs[i];
    S.qs1 = k == a->S - 1 ? qn1 : a->Qs[i + 1];
    S.gx = a->Gx[i]; S.gy = a->Gy[i]; S.lim = a->Lim[i];
    S.dt = dt;
    S.alpha = a->alpha[(size_t)k];
    S.lam_next = a->lamA; S.lam_cur = a->lamB;
    S.lam_gx = a->s->TP.P.order2 ? a->lgx : nullptr;
    S.lam_gy = a->lgy; S.lam_lim = a->llim;
    S.lam_qn = a->lam_qn;
    S.lam_bv = a->lam_bv;
    S.dt_partials = a->partials + (size_t)k * adj_residual_blocks(a->s->TP.P);
    return S;
}
}  // namespace

extern "C" {

int fv_adjoint_create(const fv_mesh* fm, const fv_physics* ph, int32_t device, const fv_adjoint_options* o,
                      fv_adjoint** out) {
    if (!fm || !ph || !o || !out) return fail(FV_ERR_ARG, "fv_adjoint_create: null argument");
    if (ph->V != 4 || (ph->flux != FV_FLUX_ROE_FS && ph->flux != FV_FLUX_ROE_ST))
        return fail(FV_ERR_UNSUPPORTED, "fv_adjoint: Euler with a Roe flux kind only");
    if (!ph->global_dt || (ph->dt_kind != FV_DT_CFL_SUM && ph->dt_kind != FV_DT_CONST))
        return fail(FV_ERR_UNSUPPORTED, "fv_adjoint: the global CFL-sum or constant time step only");
    if (o->n_steps < 1 || o->checkpoint_every < 1 || o->n_alpha < 1 || o->n_alpha > 8 || !o->alpha || o->n_bins < 0)
        return fail(FV_ERR_ARG, "fv_adjoint_create: invalid options");
    const HostMesh& m = fm->m;
    const int ng = (int)m.group_names.size();
    if (o->param_group < 0 || o->param_group >= ng || o->loss_group < 0 || o->loss_group >= ng)
        return fail(FV_ERR_ARG, "fv_adjoint_create: group index out of range");
    if (ph->group_bc[o->param_group] != FV_BC_INLET_OUTLET && ph->group_bc[o->param_group] != FV_BC_FARFIELD &&
        ph->group_bc[o->param_group] != FV_BC_FARFIELD_B0)
        return fail(FV_ERR_ARG, "fv_adjoint_create: the parameter group must be an inflow / far-field boundary");
    if (m.case_real_off.size() > 2) return fail(FV_ERR_UNSUPPORTED, "fv_adjoint: not on batches");
    std::unique_ptr<fv_adjoint> a(new fv_adjoint());
    a->o = *o;
    a->alpha.assign(o->alpha, o->alpha + o->n_alpha);
    a->o.alpha = nullptr;
    a->S = o->n_alpha;
    a->gamma = ph->gamma;
    const double* bv = ph->group_bv + 4 * o->param_group;
    a->rho_inf = bv[0];
    a->p_inf = (ph->gamma - 1) * (bv[3] - 0.5 / bv[0] * (bv[1] * bv[1] + bv[2] * bv[2]));
    int rc = fv_solver_create(fm, ph, FV_PREC_FP64_EXACT, device, &a->s);
    if (rc) return rc;
    fv_solver* s = a->s;
    // parametrisation per reference ghost
    a->ghost_bin.assign((size_t)m.n_bound, -1);
    a->ghost_kind.assign((size_t)m.n_bound, 0);
    for (int64_t r = 0; r < m.n_bound; ++r) {
        const int g = m.bnd_group[(size_t)r];
        a->ghost_kind[(size_t)r] = ph->group_bc[g];
        if (g == o->param_group && o->n_bins > 0) {
            const double y = m.ecy[m.bound_edges[(size_t)r]];
            int b = (int)std::floor((y - o->bin_lo) / (o->bin_hi - o->bin_lo) * o->n_bins);
            a->ghost_bin[(size_t)r] = std::min(std::max(b, 0), o->n_bins - 1);
        }
    }
    // cell-centric face lists for the adjoint kernels
    FaceArrays fa;
    build_face_arrays(m, fa);
    {
        uint32_t* nbr; double *nx, *ny, *le, *g, *dsx, *dsy, *dnx, *dny, *area;
        auto up = [&](auto** d, const auto& v) -> cudaError_t {
            cudaError_t e = a->alloc(d, v.size());
            if (e == cudaSuccess) e = cudaMemcpy(*d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice);
            return e;
        };
        CK(up(&nbr, fa.nbr)); CK(up(&nx, fa.nx)); CK(up(&ny, fa.ny)); CK(up(&le, fa.le)); CK(up(&g, fa.g));
        CK(up(&dsx, fa.dsx)); CK(up(&dsy, fa.dsy)); CK(up(&dnx, fa.dnx)); CK(up(&dny, fa.dny));
        CK(up(&area, fa.area));
        a->F = AdjFaces{nbr, nx, ny, le, g, dsx, dsy, dnx, dny, area};
    }
    std::vector<int32_t> lg;
    for (int64_t b = 0; b < m.n_bound; ++b)
        if (fa.ghost_group[(size_t)b] == o->loss_group) lg.push_back((int32_t)b);
    a->n_loss = (int)lg.size();
    CK(a->alloc(&a->loss_ghosts, lg.size()));
    if (!lg.empty()) CK(cudaMemcpy(a->loss_ghosts, lg.data(), lg.size() * 4, cudaMemcpyHostToDevice));
    // buffers
    const size_t nq = (size_t)m.n_total * 4;
    const int every = std::min(o->checkpoint_every, o->n_steps);
    a->o.checkpoint_every = every;
    a->nseg = (o->n_steps + every - 1) / every;
    a->ckpt.resize((size_t)a->nseg);
    for (auto& p : a->ckpt) CK(a->alloc(&p, nq));
    a->Qn.resize((size_t)every + 1);
    for (auto& p : a->Qn) CK(a->alloc(&p, nq));
    a->Qs.assign((size_t)a->S, nullptr);
    for (int k = 1; k < a->S; ++k) CK(a->alloc(&a->Qs[(size_t)k], nq));
    a->Gx.resize((size_t)a->S); a->Gy.resize((size_t)a->S); a->Lim.resize((size_t)a->S);
    for (int k = 0; k < a->S; ++k) {
        CK(a->alloc(&a->Gx[(size_t)k], nq)); CK(a->alloc(&a->Gy[(size_t)k], nq)); CK(a->alloc(&a->Lim[(size_t)k], nq));
        launch_fill_ghost_grad(a->Gx[(size_t)k], a->Gy[(size_t)k], a->Lim[(size_t)k], (int)m.n_real, (int)m.n_total, 4,
                               false, s->stream);
    }
    CK(a->alloc(&a->dtc, (size_t)m.n_total));
    CK(a->alloc(&a->tmp[0], nq)); CK(a->alloc(&a->tmp[1], nq));
    CK(a->alloc(&a->tgx, nq)); CK(a->alloc(&a->tgy, nq)); CK(a->alloc(&a->tlim, nq));
    launch_fill_ghost_grad(a->tgx, a->tgy, a->tlim, (int)m.n_real, (int)m.n_total, 4, false, s->stream);
    CK(a->alloc(&a->dt_fill, (size_t)m.n_total));
    CK(a->alloc(&a->dt_n, (size_t)o->n_steps));
    CK(a->alloc(&a->loss, 1)); CK(a->alloc(&a->lam_dt, 1));
    CK(a->alloc(&a->partials, (size_t)a->S * adj_residual_blocks(s->TP.P)));
    CK(a->alloc(&a->lamA, nq)); CK(a->alloc(&a->lamB, nq)); CK(a->alloc(&a->lam_qn, nq));
    CK(a->alloc(&a->lgx, nq)); CK(a->alloc(&a->lgy, nq)); CK(a->alloc(&a->llim, nq));
    CK(a->alloc(&a->lam_bv, (size_t)m.n_bound * 4));
    CK(a->alloc(&a->keys, (size_t)kDtSlots));
    CK(a->alloc(&a->argmin, 1));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    *out = a.release();
    return FV_OK;
}

int fv_adjoint_destroy(fv_adjoint* a) {
    delete a;
    return FV_OK;
}

int fv_adjoint_run(fv_adjoint* a, const double* theta, double* loss, double* grad) {
    if (!a || !theta) return fail(FV_ERR_ARG, "fv_adjoint_run: null argument");
    fv_solver* s = a->s;
    CK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    const int N = a->o.n_steps, every = a->o.checkpoint_every, S = a->S;
    const size_t nq = (size_t)s->n_total * 4;
    int rc = adj_set_theta(a, theta, a->ckpt[0]);
    if (rc) return rc;
    a->theta_last.assign(theta, theta + 1 + a->o.n_bins);
    // ---- forward: checkpoints every `every` steps, loss
    CK(cudaMemsetAsync(a->loss, 0, 8, st));
    double* cur = a->ckpt[0];
    double* nxt = a->Qn[0];  // scratch for the non-checkpoint states
    double* alt = a->Qn[1];
    for (int n = 0; n < N; ++n) {
        double* dst = ((n + 1) % every == 0 && (n + 1) / every < a->nseg) ? a->ckpt[(size_t)(n + 1) / every]
                                                                             : (cur == nxt ? alt : nxt);
        if ((rc = adj_forward_step(a, cur, dst, a->dt_n + n, false, true))) return rc;
        cur = dst;
    }
    // final state kept in the solver (fv_adjoint_final_state)
    CK(cudaMemcpyAsync(s->qbase[0], cur, nq * 8, cudaMemcpyDeviceToDevice, st));
    if (loss) {
        CK(cudaMemcpyAsync(loss, a->loss, 8, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    if (!grad) return FV_OK;
    // ---- reverse
    const TileParams& TP = s->TP;
    const int nblk = adj_residual_blocks(TP.P);
    CK(cudaMemsetAsync(a->lamA, 0, nq * 8, st));   // the loss does not depend on q_N
    CK(cudaMemsetAsync(a->lam_bv, 0, (size_t)s->n_bound * 4 * 8, st));
    std::vector<double> dts((size_t)every);
    for (int seg = a->nseg - 1; seg >= 0; --seg) {
        const int n0 = seg * every, len = std::min(every, N - n0);
        // the segment's step states (the same bits as the forward run's)
        CK(cudaMemcpyAsync(a->Qn[0], a->ckpt[(size_t)seg], nq * 8, cudaMemcpyDeviceToDevice, st));
        for (int j = 0; j < len; ++j)
            if ((rc = adj_forward_step(a, a->Qn[(size_t)j], a->Qn[(size_t)j + 1], a->dt_n + n0 + j, false, false)))
                return rc;
        CK(cudaMemcpyAsync(dts.data(), a->dt_n + n0, (size_t)len * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int j = len - 1; j >= 0; --j) {
            // step j's stage states, gradients, limiters and per-cell dt
            if ((rc = adj_forward_step(a, a->Qn[(size_t)j], a->tmp[0], a->dt_n + n0 + j, true, false))) return rc;
            CK(cudaMemsetAsync(a->lam_qn, 0, nq * 8, st));
            for (int k = S - 1; k >= 0; --k) {
                AdjStage stg = adj_stage(a, a->Qn[(size_t)j], a->Qn[(size_t)j + 1], k, dts[(size_t)j]);
                adj_launch_ghosts(TP.P, a->F, stg, st);
                adj_launch_residual(TP.P, a->F, stg, st);
                if (TP.P.order2) adj_launch_gradlim(TP.P, a->F, stg, st);
                std::swap(a->lamA, a->lamB);
            }
            adj_launch_add(a->lam_qn, a->lamA, nq, st);  // q_n is stage 0's input
            adj_launch_sum(a->partials, S * nblk, a->lam_dt, st);
            const double* qn = a->Qn[(size_t)j];
            if (a->n_loss)
                adj_launch_loss_adjoint(TP.P, qn, a->dt_n + n0 + j, a->loss_ghosts, a->n_loss, 1.0, a->lam_qn, a->lam_dt, st);
            if (TP.P.dt_kind == FV_DT_CFL_SUM)
                adj_launch_dt(TP.P, a->F, qn, a->dtc, a->dt_n + n0 + j, a->lam_dt, a->lam_qn, a->argmin, st);
            std::swap(a->lamA, a->lam_qn);
            CK(cudaGetLastError());
        }
    }
    // initial ghost fill (boundary states of q_0 from its interior values)
    {
        AdjStage stg{};
        stg.qs1 = a->ckpt[0];
        stg.zero_grad = 1;
        stg.lam_next = a->lamA;
        stg.lam_bv = a->lam_bv;
        adj_launch_ghosts(TP.P, a->F, stg, st);
    }
    CK(cudaGetLastError());
    std::vector<double> lq(nq), lbv((size_t)s->n_bound * 4);
    std::vector<int32_t> n2r((size_t)s->n_total);
    CK(cudaMemcpyAsync(lq.data(), a->lamA, nq * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(lbv.data(), a->lam_bv, lbv.size() * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(n2r.data(), s->new2ref, n2r.size() * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // dL/dtheta in a fixed order: free stream through the initial state ...
    const double M = theta[0];
    const int nb = a->o.n_bins;
    for (int b = 0; b <= nb; ++b) grad[b] = 0.0;
    for (int64_t c = 0; c < s->n_real; ++c)
        grad[0] += lq[4 * c + 1] * a->rho_inf + lq[4 * c + 3] * a->rho_inf * M;
    // ... and the inflow boundary states (device ghost order -> reference)
    for (int64_t gb = 0; gb < s->n_bound; ++gb) {
        const int64_t r = (int64_t)n2r[(size_t)(s->n_real + gb)] - s->n_real;
        const int kind = a->ghost_kind[(size_t)r];
        if (kind != FV_BC_INLET_OUTLET && kind != FV_BC_FARFIELD && kind != FV_BC_FARFIELD_B0) continue;
        const int b = a->ghost_bin[(size_t)r];
        const double rho = a->rho_inf * (1.0 + (b >= 0 ? theta[1 + b] : 0.0));
        const double* l = &lbv[(size_t)gb * 4];
        grad[0] += l[1] * rho + l[3] * rho * M;
        if (b >= 0) grad[1 + b] += a->rho_inf * (l[0] + l[1] * M + l[3] * 0.5 * M * M);
    }
    return FV_OK;
}

int fv_adjoint_final_state(fv_adjoint* a, double* q) {
    if (!a || !q) return fail(FV_ERR_ARG, "fv_adjoint_final_state: null argument");
    return fv_get_state(a->s, q);
}

}  // extern "C"
