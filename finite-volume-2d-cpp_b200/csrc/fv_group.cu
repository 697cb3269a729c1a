// Domain decomposition of one mesh over parts (fv_group_* in
// include/fvgpu.h): the reference's MPI run (explicit.cpp:657-817 with
// update_comms, validate_dt and the rank sums of calc_residuals,
// explicit.cpp:420-477, 498-550, 567-621) as one process per GPU with NCCL.
//
// Every part is an ordinary solver over its local mesh (build_part: owned
// cells, two rings of halo cells, the boundary ghosts of ring 1), whose
// tiles cover its owned cells only.  A step interleaves the parts' launches
// on one stream:
//   dt kernels -> per-part minimum records -> all-gather -> every part takes
//   the global minimum (and reference cell 0's dt, which carries min_dt's NaN
//   rule and the local-time-step time update);
//   per RK stage: the stage kernels -> pack the halo states other parts read
//   -> NCCL send/recv (device copies between parts of this process) ->
//   unpack into the halo cells;
//   residual partial sums per part -> all-gather -> every part's step end
//   reduces the same [n_parts][V] sums in the same order.
// So every part's run control (step, time, R, stop decision) is bit-identical
// across parts and processes, and every owned cell's arithmetic is the
// single-solver arithmetic on the same inputs: the decomposed state equals
// the single-solver state bit for bit (R differs in summation order only).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "fv_nccl.h"
#include "fv_solver.h"

namespace fvgpu {
namespace {

// parts' minimum dt key and reference cell 0's dt (bits), one record per part
__global__ void k_part_dtrec(const unsigned long long* __restrict__ keys, const double* __restrict__ dt, int cell0,
                             unsigned long long* __restrict__ rec) {
    unsigned long long k = keys[threadIdx.x] < keys[threadIdx.x + 32] ? keys[threadIdx.x] : keys[threadIdx.x + 32];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, k, o);
        k = x < k ? x : k;
    }
    if (threadIdx.x == 0) {
        rec[0] = k;
        rec[1] = cell0 >= 0 ? (unsigned long long)__double_as_longlong(dt[cell0]) : 0ull;
    }
}

// the global minimum into every key slot of a part; reference cell 0's dt
// into the part's extra dt slot when another part owns that cell
__global__ void k_part_dtcombine(const unsigned long long* __restrict__ recs, int n_parts, int owner0, int is_owner,
                                 unsigned long long* __restrict__ keys, double* __restrict__ dt_extra) {
    unsigned long long k = ~0ull;
    for (int p = 0; p < n_parts; ++p) k = recs[2 * p] < k ? recs[2 * p] : k;
    keys[threadIdx.x] = k;
    if (threadIdx.x == 0 && !is_owner) *dt_extra = __longlong_as_double((long long)recs[2 * owner0 + 1]);
}

// a part's residual partial sums, reduced in a fixed order
constexpr int kSumBlock = 256;
__global__ void __launch_bounds__(kSumBlock) k_part_sum(const double* __restrict__ partials, int n, int V,
                                                        double* __restrict__ out) {
    __shared__ double red[kSumBlock / 32][kMaxV];
    double s[kMaxV] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < n; b += blockDim.x)
        for (int k = 0; k < V; ++k) s[k] += partials[(size_t)b * V + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < V; ++k)
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if (lane == 0)
        for (int k = 0; k < V; ++k) red[warp][k] = s[k];
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < V; ++k) {
            s[k] = lane < kSumBlock / 32 ? red[lane][k] : 0.;
            for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
        }
        if (lane == 0)
            for (int k = 0; k < V; ++k) out[k] = s[k];
    }
}

// halo states of `words` 32-bit words per cell: dst[i] = src[idx[i]] (pack)
// or dst[idx[i]] = src[i] (unpack), one thread per word
__global__ void k_pack(const uint32_t* __restrict__ src, const int32_t* __restrict__ idx, uint32_t* __restrict__ dst,
                       int64_t n, int words) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * words) return;
    const int64_t i = t / words;
    const int w = (int)(t - i * words);
    dst[t] = src[(int64_t)idx[i] * words + w];
}
__global__ void k_unpack(const uint32_t* __restrict__ src, const int32_t* __restrict__ idx, uint32_t* __restrict__ dst,
                         int64_t n, int words) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * words) return;
    const int64_t i = t / words;
    const int w = (int)(t - i * words);
    dst[(int64_t)idx[i] * words + w] = src[t];
}
int blocks_of(int64_t n) { return (int)((n + kBlock - 1) / kBlock); }

}  // namespace
}  // namespace fvgpu

struct fv_group {
    int device = 0, precision = 0, V = 4;
    int n_parts = 1, rank = 0, n_ranks = 1, lo = 0, hi = 1;
    bool nccl_local = false;
    int owner0 = 0;
    int64_t g_real = 0, g_total = 0;
    cudaStream_t stream = nullptr;
    const NcclApi* nccl = nullptr;
    ncclComm_t comm = nullptr;
    // local parts [lo, hi): meshes, solvers, plans and exchange buffers
    std::vector<fv_mesh*> meshes;
    std::vector<fv_solver*> parts;
    std::vector<PartPlan> plans;
    std::vector<int32_t*> send_idx, recv_idx;
    std::vector<void*> send_buf, recv_buf;
    unsigned long long* recs = nullptr;  // [n_parts][2]
    double* sums = nullptr;              // [n_parts][V]
    std::vector<void*> allocs;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    int64_t halo_cells = 0;              // halo cells received per stage by the local parts

    int local(int p) const { return p >= lo && p < hi ? p - lo : -1; }
    int rank_of(int p) const { return p / (n_parts / n_ranks); }
    template <class T>
    cudaError_t alloc(T** p, size_t n) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) allocs.push_back((void*)*p);
        return e;
    }
    ~fv_group() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (comm && nccl) nccl->CommDestroy(comm);
        for (fv_solver* s : parts) fv_solver_destroy(s);
        for (fv_mesh* m : meshes) delete m;
        for (void* p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {
using fvgpu::set_error;
#define GK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_error(e_ == cudaErrorMemoryAllocation ? FV_ERR_NOMEM : FV_ERR_CUDA,    \
                             std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)
#define NK(g, call)                                                                           \
    do {                                                                                      \
        ncclResult_t r_ = (g)->nccl->call;                                                    \
        if (r_ != ncclSuccess)                                                                \
            return set_error(FV_ERR_COMM, std::string("NCCL ") + #call + ": " +               \
                                              (g)->nccl->GetErrorString(r_));                 \
    } while (0)

// pack, move and unpack the halo states of the stage outputs out[j]
int halo_exchange(fv_group* g, const std::vector<void*>& out) {
    cudaStream_t st = g->stream;
    const int P = g->n_parts, words = (int)(g->V * g->parts[0]->ssz / 4);
    const size_t cell_bytes = (size_t)words * 4;
    for (size_t j = 0; j < g->parts.size(); ++j) {
        const int64_t n = g->plans[j].send_off[P];
        if (n > 0)
            fvgpu::k_pack<<<fvgpu::blocks_of(n * words), fvgpu::kBlock, 0, st>>>(
                (const uint32_t*)out[j], g->send_idx[j], (uint32_t*)g->send_buf[j], n, words);
    }
    GK(cudaGetLastError());
    // parts of this process: device copies (unless routed through NCCL)
    if (!g->nccl_local) {
        for (int s = g->lo; s < g->hi; ++s)
            for (int r = g->lo; r < g->hi; ++r) {
                if (s == r) continue;
                const PartPlan &ps = g->plans[s - g->lo], &pr = g->plans[r - g->lo];
                const int64_t n = ps.send_off[r + 1] - ps.send_off[r];
                if (n == 0) continue;
                GK(cudaMemcpyAsync((char*)g->recv_buf[r - g->lo] + pr.recv_off[s] * cell_bytes,
                                   (const char*)g->send_buf[s - g->lo] + ps.send_off[r] * cell_bytes, n * cell_bytes,
                                   cudaMemcpyDeviceToDevice, st));
            }
    }
    if (g->comm) {
        // every pair (s, r) in the same order on every process, so that the
        // k-th send to a peer meets the k-th receive from it
        NK(g, GroupStart());
        for (int s = 0; s < P; ++s)
            for (int r = 0; r < P; ++r) {
                if (s == r) continue;
                const int ls = g->local(s), lr = g->local(r);
                if (ls >= 0 && lr >= 0 && !g->nccl_local) continue;
                if (ls >= 0) {
                    const PartPlan& ps = g->plans[ls];
                    const int64_t n = ps.send_off[r + 1] - ps.send_off[r];
                    if (n > 0)
                        NK(g, Send((const char*)g->send_buf[ls] + ps.send_off[r] * cell_bytes, n * cell_bytes, ncclUint8,
                                   g->rank_of(r), g->comm, st));
                }
                if (lr >= 0) {
                    const PartPlan& pr = g->plans[lr];
                    const int64_t n = pr.recv_off[s + 1] - pr.recv_off[s];
                    if (n > 0)
                        NK(g, Recv((char*)g->recv_buf[lr] + pr.recv_off[s] * cell_bytes, n * cell_bytes, ncclUint8,
                                   g->rank_of(s), g->comm, st));
                }
            }
        NK(g, GroupEnd());
    }
    for (size_t j = 0; j < g->parts.size(); ++j) {
        const int64_t n = g->plans[j].recv_off[P];
        if (n > 0)
            fvgpu::k_unpack<<<fvgpu::blocks_of(n * words), fvgpu::kBlock, 0, st>>>(
                (const uint32_t*)g->recv_buf[j], g->recv_idx[j], (uint32_t*)out[j], n, words);
    }
    GK(cudaGetLastError());
    return FV_OK;
}

// one time step of every local part; returns the kernel launches, or a
// negative status
int64_t group_step(fv_group* g, const std::vector<double>& alpha, int b, bool first) {
    cudaStream_t st = g->stream;
    const int P = g->n_parts, nl = (int)g->parts.size();
    std::vector<StepCursor> cur(nl);
    int64_t n = 0;
    for (int j = 0; j < nl; ++j) n += step_open(g->parts[j], alpha, b, first, cur[j], nullptr);
    for (int j = 0; j < nl; ++j) {
        fv_solver* s = g->parts[j];
        fvgpu::k_part_dtrec<<<1, 32, 0, st>>>(s->keys, s->dt, g->plans[j].cell0, g->recs + 2 * (g->lo + j));
        ++n;
    }
    if (g->comm) NK(g, AllGather(g->recs + 2 * g->lo, g->recs, (size_t)2 * nl, ncclUint64, g->comm, st));
    for (int j = 0; j < nl; ++j) {
        fv_solver* s = g->parts[j];
        fvgpu::k_part_dtcombine<<<1, fvgpu::kDtSlots, 0, st>>>(g->recs, P, g->owner0, g->plans[j].cell0 >= 0 ? 1 : 0,
                                                              s->keys, s->dt + s->n_total);
        ++n;
    }
    GK(cudaGetLastError());
    std::vector<void*> out(nl);
    for (int k = 0; k < (int)alpha.size(); ++k) {
        for (int j = 0; j < nl; ++j) {
            n += step_stage(g->parts[j], alpha, k, cur[j], nullptr);
            out[j] = cur[j].out;
        }
        int rc = halo_exchange(g, out);
        if (rc) return rc;
        n += 2 * nl;
    }
    for (int j = 0; j < nl; ++j) {
        fv_solver* s = g->parts[j];
        fvgpu::k_part_sum<<<1, fvgpu::kSumBlock, 0, st>>>(s->partials, s->n_tiles, g->V, g->sums + (size_t)g->V * (g->lo + j));
        ++n;
    }
    if (g->comm)
        NK(g, AllGather(g->sums + (size_t)g->V * g->lo, g->sums, (size_t)g->V * nl, ncclFloat64, g->comm, st));
    for (int j = 0; j < nl; ++j) n += step_close(g->parts[j], g->sums, P, nullptr);
    GK(cudaGetLastError());
    return n;
}

// RK1 leaves the state in qbase[1] after an odd number of steps
int settle(fv_solver* s, unsigned long long steps) {
    if (steps % 2) {
        GK(cudaMemcpyAsync(s->qbase[0], s->qbase[1], (size_t)s->n_total * s->V * 8, cudaMemcpyDeviceToDevice,
                           s->stream));
        if (s->f32)
            GK(cudaMemcpyAsync(s->sbase[0], s->sbase[1], (size_t)s->n_total * s->V * 4, cudaMemcpyDeviceToDevice,
                               s->stream));
    }
    return FV_OK;
}
}  // namespace

extern "C" {

int fv_group_nccl_id(void* id) {
    if (!id) return set_error(FV_ERR_ARG, "fv_group_nccl_id: null argument");
    std::string why;
    const NcclApi* api = nccl_api(&why);
    if (!api) return set_error(FV_ERR_COMM, why);
    ncclUniqueId u;
    ncclResult_t r = api->GetUniqueId(&u);
    if (r != ncclSuccess) return set_error(FV_ERR_COMM, std::string("ncclGetUniqueId: ") + api->GetErrorString(r));
    std::memcpy(id, &u, sizeof(u));
    return FV_OK;
}

int fv_mesh_partition_sizes(const fv_mesh* m, int32_t n_parts, int32_t part, int64_t* sizes) {
    if (!m || !sizes) return set_error(FV_ERR_ARG, "fv_mesh_partition_sizes: null argument");
    HostMesh L;
    PartPlan plan;
    std::string err = build_part(m->m, n_parts, part, L, plan);
    if (!err.empty()) return set_error(FV_ERR_ARG, err);
    sizes[0] = L.n_real; sizes[1] = L.n_total; sizes[2] = L.n_edges;
    sizes[3] = plan.n_own; sizes[4] = plan.n_own_ghost;
    sizes[5] = plan.cell0; sizes[6] = plan.owner0;
    sizes[7] = plan.recv_off[n_parts]; sizes[8] = plan.send_off[n_parts];
    sizes[9] = L.n_bound;
    return FV_OK;
}

int fv_mesh_partition(const fv_mesh* m, int32_t n_parts, int32_t part, int32_t* local2ref, int32_t* local_edges,
                      int64_t* recv_off, int32_t* recv_idx, int64_t* send_off, int32_t* send_idx) {
    if (!m) return set_error(FV_ERR_ARG, "fv_mesh_partition: null mesh");
    HostMesh L;
    PartPlan plan;
    std::string err = build_part(m->m, n_parts, part, L, plan);
    if (!err.empty()) return set_error(FV_ERR_ARG, err);
    auto put = [](const auto& v, auto* dst) { if (dst) std::copy(v.begin(), v.end(), dst); };
    put(plan.local2ref, local2ref);
    put(plan.local_edges, local_edges);
    put(plan.recv_off, recv_off);
    put(plan.recv_idx, recv_idx);
    put(plan.send_off, send_off);
    put(plan.send_idx, send_idx);
    return FV_OK;
}

int fv_group_create(const fv_mesh* fm, const fv_physics* ph, int32_t precision, int32_t device,
                    const fv_group_options* o, fv_group** out) {
    if (!fm || !ph || !o || !out) return set_error(FV_ERR_ARG, "fv_group_create: null argument");
    const int P = o->n_parts, R = o->n_ranks;
    if (P < 1 || R < 1 || o->rank < 0 || o->rank >= R || P % R != 0)
        return set_error(FV_ERR_ARG, "fv_group_create: need n_parts >= 1, a multiple of n_ranks, and 0 <= rank < n_ranks");
    if (R > 1 && !o->nccl_id) return set_error(FV_ERR_ARG, "fv_group_create: several processes need an NCCL id");
    if (ph->diffusive || ph->smooth_residuals)
        return set_error(FV_ERR_UNSUPPORTED, "a decomposition exchanges stage states only: no diffusive gradients "
                                             "or residual smoothing");
    if (fm->m.case_real_off.size() > 2) return set_error(FV_ERR_UNSUPPORTED, "a batch of cases cannot be decomposed");
    if (ph->order2 && o->solver.stage_kernels == FV_STAGE_SPLIT)
        return set_error(FV_ERR_UNSUPPORTED, "second order in a decomposition needs the fused stage kernel");
    GK(cudaSetDevice(device));
    std::unique_ptr<fv_group> g(new fv_group());
    g->device = device; g->precision = precision; g->V = ph->V;
    g->n_parts = P; g->rank = o->rank; g->n_ranks = R;
    g->lo = o->rank * (P / R); g->hi = g->lo + P / R;
    g->nccl_local = o->nccl_local != 0;
    g->g_real = fm->m.n_real; g->g_total = fm->m.n_total;
    GK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    fv_solver_options so = o->solver;
    if (ph->order2) so.stage_kernels = FV_STAGE_FUSED;
    for (int p = g->lo; p < g->hi; ++p) {
        std::unique_ptr<fv_mesh> lm(new fv_mesh());
        PartPlan plan;
        std::string err = build_part(fm->m, P, p, lm->m, plan);
        if (!err.empty()) return set_error(FV_ERR_ARG, err);
        fv_solver* s = nullptr;
        int rc = fv_solver_create_ex(lm.get(), ph, precision, device, &so, &s);
        if (rc) return rc;
        g->meshes.push_back(lm.release());
        g->parts.push_back(s);
        // reference cell 0: its own dt where this part owns it, else the
        // extra dt slot past the ghosts that the combine kernel fills
        s->TP.P.cell0 = plan.cell0 >= 0 ? plan.cell0 : (int)s->n_total;
        g->owner0 = plan.owner0;
        if ((rc = fv_solver_set_stream(s, g->stream))) return rc;
        int32_t *si = nullptr, *ri = nullptr;
        void *sb = nullptr, *rb = nullptr;
        const size_t cell_bytes = (size_t)ph->V * s->ssz;
        GK(g->alloc(&si, plan.send_idx.size()));
        GK(g->alloc(&ri, plan.recv_idx.size()));
        GK(g->alloc((char**)&sb, plan.send_idx.size() * cell_bytes));
        GK(g->alloc((char**)&rb, plan.recv_idx.size() * cell_bytes));
        if (!plan.send_idx.empty())
            GK(cudaMemcpy(si, plan.send_idx.data(), plan.send_idx.size() * 4, cudaMemcpyHostToDevice));
        if (!plan.recv_idx.empty())
            GK(cudaMemcpy(ri, plan.recv_idx.data(), plan.recv_idx.size() * 4, cudaMemcpyHostToDevice));
        g->send_idx.push_back(si); g->recv_idx.push_back(ri);
        g->send_buf.push_back(sb); g->recv_buf.push_back(rb);
        g->halo_cells += (int64_t)plan.recv_idx.size();
        g->plans.push_back(std::move(plan));
    }
    for (fv_solver* s : g->parts)
        if (ph->order2 && !s->fused)
            return set_error(FV_ERR_MESH, "a part's two-ring tiles do not fit the fused stage kernel");
    GK(g->alloc(&g->recs, (size_t)2 * P));
    GK(g->alloc(&g->sums, (size_t)ph->V * P));
    GK(cudaMemset(g->sums, 0, sizeof(double) * ph->V * P));
    if (R > 1 || g->nccl_local) {
        std::string why;
        g->nccl = nccl_api(&why);
        if (!g->nccl) return set_error(FV_ERR_COMM, why);
        ncclUniqueId id;
        if (o->nccl_id) {
            std::memcpy(&id, o->nccl_id, sizeof(id));
        } else {
            ncclResult_t r = g->nccl->GetUniqueId(&id);
            if (r != ncclSuccess) return set_error(FV_ERR_COMM, std::string("ncclGetUniqueId: ") + g->nccl->GetErrorString(r));
        }
        ncclResult_t r = g->nccl->CommInitRank(&g->comm, R, id, o->rank);
        if (r != ncclSuccess) {
            g->comm = nullptr;
            return set_error(FV_ERR_COMM, std::string("ncclCommInitRank: ") + g->nccl->GetErrorString(r));
        }
    }
    GK(cudaStreamSynchronize(g->stream));
    *out = g.release();
    return FV_OK;
}

int fv_group_destroy(fv_group* g) {
    delete g;
    return FV_OK;
}

int fv_group_set_state(fv_group* g, const double* q) {
    if (!g || !q) return set_error(FV_ERR_ARG, "fv_group_set_state: null argument");
    GK(cudaSetDevice(g->device));
    const int V = g->V;
    for (size_t j = 0; j < g->parts.size(); ++j) {
        const PartPlan& pl = g->plans[j];
        std::vector<double> ql(pl.local2ref.size() * V);
        for (size_t i = 0; i < pl.local2ref.size(); ++i)
            for (int k = 0; k < V; ++k) ql[i * V + k] = q[(size_t)pl.local2ref[i] * V + k];
        int rc = fv_set_state(g->parts[j], ql.data());
        if (rc) return rc;
    }
    return FV_OK;
}

int fv_group_get_state(fv_group* g, double* q) {
    if (!g || !q) return set_error(FV_ERR_ARG, "fv_group_get_state: null argument");
    GK(cudaSetDevice(g->device));
    const int V = g->V;
    for (size_t j = 0; j < g->parts.size(); ++j) {
        const PartPlan& pl = g->plans[j];
        fv_solver* s = g->parts[j];
        std::vector<double> ql(pl.local2ref.size() * V);
        int rc = fv_get_state(s, ql.data());
        if (rc) return rc;
        auto put = [&](int64_t i) {
            for (int k = 0; k < V; ++k) q[(size_t)pl.local2ref[i] * V + k] = ql[(size_t)i * V + k];
        };
        for (int64_t i = 0; i < pl.n_own; ++i) put(i);
        for (int64_t i = 0; i < pl.n_own_ghost; ++i) put(s->n_real + i);
    }
    return FV_OK;
}

int fv_group_run(fv_group* g, const fv_run_options* o, fv_run_info* info) {
    if (!g || !o) return set_error(FV_ERR_ARG, "fv_group_run: null argument");
    if (o->n_alpha < 1 || o->n_alpha > 16 || !o->alpha) return set_error(FV_ERR_ARG, "fv_group_run: need 1..16 RK stages");
    if (o->print_interval == 0) return set_error(FV_ERR_ARG, "fv_group_run: print_interval must be > 0");
    GK(cudaSetDevice(g->device));
    cudaStream_t st = g->stream;
    std::vector<double> alpha(o->alpha, o->alpha + o->n_alpha);
    const RunLimits L{o->max_step, o->max_time, o->tolerance, o->print_interval};
    for (fv_solver* s : g->parts) {
        launch_set_limits(s->limits, L, st);
        if (o->restart) {
            launch_ctrl_reset(s->ctrl, st);
            // run(): initial ghost fill with zeroed gx, gy, limiters
            // (explicit.cpp:712); the halo ghosts get the values their
            // owners compute, from the same states
            exact::launch_bounds(s->TP.P, s->qbase[0], nullptr, nullptr, nullptr, 1, st);
            if (s->f32) launch_to_float(s->qbase[0], (float*)s->sbase[0], (size_t)s->n_total * s->V, st);
        }
    }
    fv_solver* s0 = g->parts[0];
    launch_ctrl_copy(s0->ctrl, s0->hctrl_dev, st);
    GK(cudaGetLastError());
    GK(cudaStreamSynchronize(st));
    const Ctrl& hc = *s0->hctrl;
    const unsigned long long start = o->restart ? 0ull : hc.step;
    cudaEvent_t e0, e1;
    GK(cudaEventCreate(&e0)); GK(cudaEventCreate(&e1));
    std::vector<PrintRec> recs(s0->hist_cap);
    double total_ms = 0.0;
    int64_t launches = 0;
    unsigned long long cur = start;
    int rc = FV_OK;
    for (;;) {
        const unsigned long long left = o->max_step > cur ? o->max_step - cur : 1ull;
        const int len = (int)std::min<unsigned long long>(left, (unsigned long long)s0->chunk);
        cudaEventRecord(e0, st);
        for (int k = 0; k < len && rc == FV_OK; ++k) {
            const int64_t n = group_step(g, alpha, (alpha.size() == 1 && (k % 2)) ? 1 : 0, k == 0);
            if (n < 0) rc = (int)n;
            else launches += n;
        }
        if (rc) break;
        cudaEventRecord(e1, st);
        launch_ctrl_copy(s0->ctrl, s0->hctrl_dev, st);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
            rc = set_error(FV_ERR_CUDA, "fv_group_run: a step failed on the device");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total_ms += ms;
        if (alpha.size() == 1)
            for (fv_solver* s : g->parts)
                if ((rc = settle(s, hc.step - cur))) break;
        if (rc) break;
        cur = hc.step;
        if (o->on_print && hc.n_hist > 0) {
            if (cudaMemcpy(recs.data(), s0->hist, sizeof(PrintRec) * hc.n_hist, cudaMemcpyDeviceToHost) != cudaSuccess) {
                rc = set_error(FV_ERR_CUDA, "fv_group_run: print records");
                break;
            }
            for (int k = 0; k < hc.n_hist; ++k) o->on_print(o->user, recs[k].step, recs[k].time, recs[k].R, g->V);
        }
        double Rmax = 1.0;
        if (hc.step > 0) {
            Rmax = 0.0;
            for (int k = 0; k < g->V; ++k) Rmax = (hc.R[k] < Rmax) ? Rmax : hc.R[k];
        }
        if (!hc.active || hc.step >= o->max_step || hc.time >= o->max_time || Rmax < o->tolerance) break;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    if (rc) return rc;
    GK(cudaStreamSynchronize(st));
    g->last_ms = total_ms;
    g->last_launches = launches;
    if (info) {
        info->step = hc.step;
        info->time = hc.time;
        for (int k = 0; k < kMaxV; ++k) { info->R[k] = hc.R[k]; info->R0[k] = hc.R0[k]; }
        for (int k = kMaxV; k < 8; ++k) { info->R[k] = 0; info->R0[k] = 0; }
    }
    return FV_OK;
}

int fv_group_info(fv_group* g, int64_t* out) {
    if (!g || !out) return set_error(FV_ERR_ARG, "fv_group_info: null argument");
    int64_t own = 0, tiles = 0, sent = 0;
    for (size_t j = 0; j < g->parts.size(); ++j) {
        own += g->plans[j].n_own;
        tiles += g->parts[j]->n_tiles;
        sent += g->plans[j].send_off[g->n_parts];
    }
    out[0] = (int64_t)g->parts.size();
    out[1] = own;
    out[2] = g->halo_cells;
    out[3] = sent;
    out[4] = tiles;
    out[5] = g->comm != nullptr ? 1 : 0;
    return FV_OK;
}

int fv_group_last_run_stats(fv_group* g, double* device_ms, int64_t* kernel_launches) {
    if (!g) return set_error(FV_ERR_ARG, "fv_group_last_run_stats: null group");
    if (device_ms) *device_ms = g->last_ms;
    if (kernel_launches) *kernel_launches = g->last_launches;
    return FV_OK;
}

}  // extern "C"
