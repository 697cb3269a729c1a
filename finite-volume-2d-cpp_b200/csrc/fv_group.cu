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
#include <chrono>
#include <cstring>
#include <map>
#include <thread>
#include <memory>
#include <string>
#include <vector>

#include "fv_nccl.h"
#include "fv_solver.h"

namespace fvgpu {
namespace {

// Per-part pointers of the local parts, passed by value to the merged
// small kernels (block j serves local part j).
constexpr int kMaxLocal = 16;
struct PartPtrs {
    unsigned long long* keys[kMaxLocal];   // the part's dt key slots
    double* dt[kMaxLocal];                 // its dt array (extra slot at n_total)
    const double* partials[kMaxLocal];     // its residual partial sums [n_tiles][V]
    uint32_t* out[kMaxLocal];              // this stage's output state
    int n_total[kMaxLocal];
    int cell0[kMaxLocal];                  // local index of reference cell 0, -1: not here
    int n_tiles[kMaxLocal];
};

__device__ __forceinline__ unsigned long long warp_kmin(unsigned long long k) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, k, o);
        k = x < k ? x : k;
    }
    return k;
}

// each local part's minimum dt key and reference cell 0's dt (bits): one
// record per part, block j = local part j (32 threads)
__global__ void k_group_dtrec(PartPtrs pp, unsigned long long* __restrict__ recs) {
    const int j = blockIdx.x;
    const unsigned long long* keys = pp.keys[j];
    unsigned long long k = keys[threadIdx.x] < keys[threadIdx.x + 32] ? keys[threadIdx.x] : keys[threadIdx.x + 32];
    k = warp_kmin(k);
    if (threadIdx.x == 0) {
        recs[2 * j] = k;
        recs[2 * j + 1] = pp.cell0[j] >= 0 ? (unsigned long long)__double_as_longlong(pp.dt[j][pp.cell0[j]]) : 0ull;
    }
}

// the minimum over every part's record into every key slot of local part j,
// and reference cell 0's dt into its extra dt slot when another part owns
// that cell (block j, kDtSlots threads)
__global__ void k_group_dtcombine(PartPtrs pp, const unsigned long long* __restrict__ recs, int n_parts, int owner0) {
    const int j = blockIdx.x;
    unsigned long long k = ~0ull;
    for (int p = 0; p < n_parts; ++p) k = recs[2 * p] < k ? recs[2 * p] : k;
    pp.keys[j][threadIdx.x] = k;
    if (threadIdx.x == 0 && pp.cell0[j] < 0)
        pp.dt[j][pp.n_total[j]] = __longlong_as_double((long long)recs[2 * owner0 + 1]);
}

// without a communicator: records and combine in one block over all local
// parts (kDtSlots threads, thread t reads key slot t of every part)
__global__ void k_group_dt_local(PartPtrs pp, int nl) {
    __shared__ unsigned long long wmin[kDtSlots / 32];
    __shared__ unsigned long long d0;
    unsigned long long k = ~0ull;
    for (int j = 0; j < nl; ++j) {
        const unsigned long long x = pp.keys[j][threadIdx.x];
        k = x < k ? x : k;
        if (threadIdx.x == 0 && pp.cell0[j] >= 0) d0 = (unsigned long long)__double_as_longlong(pp.dt[j][pp.cell0[j]]);
    }
    k = warp_kmin(k);
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = k;
    __syncthreads();
    k = wmin[0];
    for (int w = 1; w < kDtSlots / 32; ++w) k = wmin[w] < k ? wmin[w] : k;
    for (int j = 0; j < nl; ++j) {
        pp.keys[j][threadIdx.x] = k;
        if (threadIdx.x == 0 && pp.cell0[j] < 0) pp.dt[j][pp.n_total[j]] = __longlong_as_double((long long)d0);
    }
}

// each local part's residual partial sums, reduced in a fixed order (block j)
constexpr int kSumBlock = 1024;
__global__ void __launch_bounds__(kSumBlock) k_group_psum(PartPtrs pp, int V, double* __restrict__ out) {
    __shared__ double red[kSumBlock / 32][kMaxV];
    const int j = blockIdx.x;
    const double* partials = pp.partials[j];
    const int n = pp.n_tiles[j];
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
            for (int k = 0; k < V; ++k) out[(size_t)j * V + k] = s[k];
    }
}

// halo states of `words` 32-bit words per cell.  Pack: send[i] = the state
// of local cell src[i] of local part part[i].  Unpack: the state of local
// cell dst[i] of local part part[i] = recv[from[i]] (from >= 0) or
// send[~from[i]] (a part of this process, read straight from its pack).
// One thread per word.
__global__ void k_group_pack(PartPtrs pp, const int32_t* __restrict__ part, const int32_t* __restrict__ src,
                             uint32_t* __restrict__ send, int64_t n, int words) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * words) return;
    const int64_t i = t / words;
    const int w = (int)(t - i * words);
    send[t] = pp.out[part[i]][(int64_t)src[i] * words + w];
}
__global__ void k_group_unpack(PartPtrs pp, const int32_t* __restrict__ part, const int32_t* __restrict__ dst,
                               const int64_t* __restrict__ from, const uint32_t* __restrict__ send,
                               const uint32_t* __restrict__ recv, int64_t n, int words) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * words) return;
    const int64_t i = t / words;
    const int w = (int)(t - i * words);
    const int64_t f = from[i];
    const uint32_t v = f >= 0 ? recv[f * words + w] : send[(~f) * words + w];
    pp.out[part[i]][(int64_t)dst[i] * words + w] = v;
}
int blocks_of(int64_t n) { return (int)((n + kBlock - 1) / kBlock); }

// ---- the P2P transport: stores into the reading parts' memory, epoch flags
// A part's flag word for source part s holds the last epoch s published:
// s's outputs of stage k of step n are complete in this part's buffers once
// it reads n * stages + k + 1.  Epochs come from the step counter in device
// memory, so captured graphs replay them.
__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_sys(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ bool ctrl_inactive(const Ctrl* c) { return *(volatile const int*)&c->active == 0; }

struct PushParams {
    const uint32_t* src;                   // the local part's output of this stage
    uint32_t* dst[kMaxPeers];              // the same stage buffer of each reading part
    unsigned long long* flag[kMaxPeers];   // this part's flag word in each reading part
    int n_dst;
    const int32_t* slot;                   // [n] reading part (slot) of entry i
    const int32_t* from;                   // [n] local cell (real or ghost)
    const int32_t* to;                     // [n] that cell's index in the reading part
    int64_t n;
    int words;                             // 32-bit words per cell state
    unsigned long long* ctr;               // CTAs of this part's pushes that have completed
    const Ctrl* ctrl;
    int stages, stage;
};
// The states other parts read, stored straight into their buffers; the last
// CTA of the launch then releases the stage's epoch into each reader's flag
// word, after every CTA's stores are visible at system scope (the barrier
// orders a CTA's stores before its thread 0, whose system-scope fence and
// count make them visible before any later release).
__global__ void k_p2p_push(PushParams pp) {
    if (ctrl_inactive(pp.ctrl)) return;
    const unsigned long long epoch = pp.ctrl->step * (unsigned long long)pp.stages + pp.stage + 1;
    const int64_t total = pp.n * pp.words;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / pp.words;
        const int w = (int)(t - i * pp.words);
        pp.dst[pp.slot[i]][(int64_t)pp.to[i] * pp.words + w] = pp.src[(int64_t)pp.from[i] * pp.words + w];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence_system();
        const unsigned long long done = atomicAdd(pp.ctr, 1ull) + 1ull;
        if (done == epoch * gridDim.x) {
            __threadfence_system();
            for (int d = 0; d < pp.n_dst; ++d) st_release_sys(pp.flag[d], epoch);
        }
    }
}

// Waits until every part that sends to local part j (block j) has released
// the epoch this stage needs.  Each wait gives up after `limit` polls: it
// then records the failure in err[j] and returns, and the host reports it.
struct WaitParams {
    const unsigned long long* flags[kMaxLocal];  // part j's flag words [n_parts]
    const int32_t* src[kMaxLocal];               // parts that send to part j
    int n_src[kMaxLocal];
    int* err;                                    // [local parts]
    const Ctrl* ctrl;
    int stages, stage;                           // needed epoch: step * stages + stage
    long long limit;
};
__global__ void k_p2p_wait(WaitParams wp) {
    const int j = blockIdx.x;
    if (ctrl_inactive(wp.ctrl)) return;
    const unsigned long long need = wp.ctrl->step * (unsigned long long)wp.stages + wp.stage;
    for (int i = threadIdx.x; i < wp.n_src[j]; i += blockDim.x) {
        const unsigned long long* f = wp.flags[j] + wp.src[j][i];
        long long polls = 0;
        while (ld_acquire_sys(f) < need) {
            if (++polls > wp.limit) {
                atomicExch(wp.err + j, 1);
                break;
            }
            __nanosleep(256);
        }
    }
}

}  // namespace
}  // namespace fvgpu

struct fv_group {
    int device = 0, precision = 0, V = 4;
    int n_parts = 1, rank = 0, n_ranks = 1, lo = 0, hi = 1;
    bool nccl_local = false;
    int owner0 = 0;
    cudaStream_t stream = nullptr;
    // overlap: each stage computes the band tiles (every state another part
    // reads) and then the exchange on cstream (high priority) while the
    // interior tiles compute on stream
    bool overlap = false;
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_halo = nullptr;
    std::vector<int> band_tiles;         // per local part
    const NcclApi* nccl = nullptr;
    ncclComm_t comm = nullptr;
    double timeout_ms = 300000.0;        // a chunk's wait limit with a communicator
    bool aborted = false;                // the communicator was aborted: the group is unusable
    // local parts [lo, hi): meshes, solvers, plans and exchange buffers
    std::vector<fv_mesh*> meshes;
    std::vector<fv_solver*> parts;
    std::vector<PartPlan> plans;
    // the flat pack / unpack lists over the local parts and their buffers
    int64_t n_pack = 0, n_unpack = 0, n_recv = 0;
    int32_t *pack_part = nullptr, *pack_src = nullptr, *unpack_part = nullptr, *unpack_dst = nullptr;
    int64_t* unpack_from = nullptr;
    void *send_all = nullptr, *recv_all = nullptr;
    std::vector<int64_t> pack_off;       // [local parts + 1] each part's run of the pack list
    // NCCL messages in the order every process issues them: (peer rank,
    // send (1) or receive (0), offset in cells into send_all / recv_all, cells)
    struct Msg { int peer, send; int64_t off, n; };
    std::vector<Msg> msgs;
    fvgpu::PartPtrs pp{};
    // the P2P transport: per local part, what it pushes where (entries of
    // reading-part slot, local cell, cell in the reader), the reader's stage
    // buffers by role (tmp[0], tmp[1], sbase[0], sbase[1]) and flag word per
    // slot, and the count of its completed push CTAs
    bool p2p = false;
    // fused parts: the exchange inside each stage launch (RemoteIO per local
    // part and output role, device memory), no push or wait launches per stage
    bool fused_p2p = false;
    fvgpu::RemoteIO* rio = nullptr;       // [local parts][4]
    struct Push {
        int32_t *slot = nullptr, *from = nullptr, *to = nullptr;
        int64_t n = 0;
        int n_dst = 0;
        uint32_t* buf[4][fvgpu::kMaxPeers] = {};
        unsigned long long* flag[fvgpu::kMaxPeers] = {};
        unsigned long long* ctr = nullptr;
    };
    std::vector<Push> push;
    unsigned long long* flags = nullptr;  // [local parts][n_parts] flag words the senders write
    int* err = nullptr;                   // [local parts] a wait that ran out
    fvgpu::WaitParams wp{};
    std::vector<void*> ipc_opened;        // other processes' allocations mapped here
    std::vector<GraphEntry> graphs;
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
        if (stream && !aborted) cudaStreamSynchronize(stream);
        // graphs that hold NCCL calls go before their communicator
        for (auto& e : graphs)
            if (e.exec) cudaGraphExecDestroy(e.exec);
        if (comm && nccl) nccl->CommDestroy(comm);
        for (void* q : ipc_opened) cudaIpcCloseMemHandle(q);
        for (fv_solver* s : parts) fv_solver_destroy(s);
        for (fv_mesh* m : meshes) delete m;
        for (void* p : allocs) cudaFree(p);
        if (ev_start) cudaEventDestroy(ev_start);
        if (ev_halo) cudaEventDestroy(ev_halo);
        if (cstream) cudaStreamDestroy(cstream);
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

int p2p_push(fv_group* g, int j, const void* out, int role, int stages, int k, cudaStream_t st);
int p2p_wait(fv_group* g, int stages, int k, cudaStream_t st);

// pack, move and unpack the halo states of this stage's outputs (pp.out) on st
int halo_exchange(fv_group* g, cudaStream_t st) {
    const int words = (int)(g->V * g->parts[0]->ssz / 4);
    const size_t cell_bytes = (size_t)words * 4;
    if (g->n_pack > 0)
        fvgpu::k_group_pack<<<fvgpu::blocks_of(g->n_pack * words), fvgpu::kBlock, 0, st>>>(
            g->pp, g->pack_part, g->pack_src, (uint32_t*)g->send_all, g->n_pack, words);
    GK(cudaGetLastError());
    if (!g->msgs.empty()) {
        NK(g, GroupStart());
        for (const auto& m : g->msgs) {
            if (m.send)
                NK(g, Send((const char*)g->send_all + m.off * cell_bytes, m.n * cell_bytes, ncclUint8, m.peer, g->comm, st));
            else
                NK(g, Recv((char*)g->recv_all + m.off * cell_bytes, m.n * cell_bytes, ncclUint8, m.peer, g->comm, st));
        }
        NK(g, GroupEnd());
    }
    if (g->n_unpack > 0)
        fvgpu::k_group_unpack<<<fvgpu::blocks_of(g->n_unpack * words), fvgpu::kBlock, 0, st>>>(
            g->pp, g->unpack_part, g->unpack_dst, g->unpack_from, (const uint32_t*)g->send_all,
            (const uint32_t*)g->recv_all, g->n_unpack, words);
    GK(cudaGetLastError());
    return FV_OK;
}

// one time step of every local part; returns the kernel launches, or a
// negative status
int64_t group_step(fv_group* g, const std::vector<double>& alpha, int b, bool first) {
    cudaStream_t st = g->stream;
    const int P = g->n_parts, nl = (int)g->parts.size();
    std::vector<StepCursor> cur(nl);
    const int S = (int)alpha.size();
    // the buffer role of stage k's output (tmp[0], tmp[1], sbase[0], sbase[1])
    auto role_of = [&](int k) { return S == 1 ? 2 + (1 - b) : (k == S - 1 ? 2 + b : k % 2); };
    int64_t n = 0;
    for (int j = 0; j < nl; ++j) {
        n += step_open(g->parts[j], alpha, b, first, cur[j], nullptr, !g->p2p);
        cur[j].part = true;
    }
    if (g->p2p) {
        // the previous step's last stage must have reached the halo before
        // the dt kernel reads it
        int rc = p2p_wait(g, S, 0, st);
        if (rc) return rc;
        ++n;
        for (int j = 0; j < nl; ++j) n += step_dt(g->parts[j], cur[j], nullptr);
    }
    if (g->comm) {
        fvgpu::k_group_dtrec<<<nl, 32, 0, st>>>(g->pp, g->recs + 2 * g->lo);
        NK(g, AllGather(g->recs + 2 * g->lo, g->recs, (size_t)2 * nl, ncclUint64, g->comm, st));
        fvgpu::k_group_dtcombine<<<nl, fvgpu::kDtSlots, 0, st>>>(g->pp, g->recs, P, g->owner0);
        n += 2;
    } else {
        fvgpu::k_group_dt_local<<<1, fvgpu::kDtSlots, 0, st>>>(g->pp, nl);
        n += 1;
    }
    GK(cudaGetLastError());
    for (int k = 0; k < S; ++k) {
        if (g->fused_p2p) {
            // one launch per part: its band tiles wait for the senders,
            // compute, store into the readers' buffers and release the epoch
            for (int j = 0; j < nl; ++j) {
                cur[j].remote = g->rio + (size_t)j * 4 + role_of(k);
                n += step_stage(g->parts[j], alpha, k, cur[j], nullptr);
            }
            continue;
        }
        if (g->p2p && k > 0) {
            int rc = p2p_wait(g, S, k, st);
            if (rc) return rc;
            ++n;
        }
        if (g->overlap) {
            // band tiles, pack, exchange and unpack on cstream, beside the
            // interior tiles on st; both start once the previous stage and
            // its exchange are complete (the first launch on each stream
            // follows a join, so it waits without PDL).  The two write
            // disjoint cells and read only the stage's input.
            GK(cudaEventRecord(g->ev_start, st));
            GK(cudaStreamWaitEvent(g->cstream, g->ev_start, 0));
            for (int j = 0; j < nl; ++j) {
                const TileRange r{0, g->band_tiles[j], j > 0, false, g->cstream};
                const int m = step_stage(g->parts[j], alpha, k, cur[j], nullptr, &r);
                if (m < 0) return set_error(FV_ERR_ARG, "internal error: ranged stage launch");
                n += m;
                g->pp.out[j] = (uint32_t*)cur[j].out;
            }
            int rc = FV_OK;
            if (g->p2p) {
                for (int j = 0; j < nl && rc == FV_OK; ++j)
                    rc = p2p_push(g, j, cur[j].out, role_of(k), S, k, g->cstream);
            } else {
                rc = halo_exchange(g, g->cstream);
            }
            if (rc) return rc;
            GK(cudaEventRecord(g->ev_halo, g->cstream));
            for (int j = 0; j < nl; ++j) {
                const TileRange r{g->band_tiles[j], g->parts[j]->n_tiles - g->band_tiles[j], j > 0, true, st};
                const int m = step_stage(g->parts[j], alpha, k, cur[j], nullptr, &r);
                if (m < 0) return set_error(FV_ERR_ARG, "internal error: ranged stage launch");
                n += m;
            }
            GK(cudaStreamWaitEvent(st, g->ev_halo, 0));
        } else {
            for (int j = 0; j < nl; ++j) {
                n += step_stage(g->parts[j], alpha, k, cur[j], nullptr);
                g->pp.out[j] = (uint32_t*)cur[j].out;
            }
            int rc = FV_OK;
            if (g->p2p) {
                for (int j = 0; j < nl && rc == FV_OK; ++j) rc = p2p_push(g, j, cur[j].out, role_of(k), S, k, st);
            } else {
                rc = halo_exchange(g, st);
            }
            if (rc) return rc;
        }
        if (g->p2p) {
            for (int j = 0; j < nl; ++j) n += g->push[j].n > 0;
        } else {
            n += (g->n_pack > 0) + (g->n_unpack > 0);
        }
    }
    fvgpu::k_group_psum<<<nl, fvgpu::kSumBlock, 0, st>>>(g->pp, g->V, g->sums + (size_t)g->V * g->lo);
    ++n;
    if (g->comm)
        NK(g, AllGather(g->sums + (size_t)g->V * g->lo, g->sums, (size_t)g->V * nl, ncclFloat64, g->comm, st));
    for (int j = 0; j < nl; ++j) n += step_close(g->parts[j], g->sums, P, nullptr);
    GK(cudaGetLastError());
    return n;
}

// One captured graph of `len` consecutive steps (the first begins with the
// begin-of-step kernel; RK1 alternates the base state between steps).
int group_graph(fv_group* g, const std::vector<double>& alpha, int len, GraphEntry** out) {
    for (auto& e : g->graphs)
        if (e.alpha == alpha && e.chunk == len) { *out = &e; return FV_OK; }
    GraphEntry e;
    e.alpha = alpha;
    e.chunk = len;
    cudaGraph_t graph;
    GK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
    int64_t launches = 0;
    int rc = FV_OK;
    for (int k = 0; k < len && rc == FV_OK; ++k) {
        const int64_t n = group_step(g, alpha, (alpha.size() == 1 && (k % 2)) ? 1 : 0, k == 0);
        if (n < 0) rc = (int)n;
        else launches += n;
    }
    cudaError_t ce = cudaStreamEndCapture(g->stream, &graph);
    if (rc) {
        if (ce == cudaSuccess) cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess) return set_error(FV_ERR_CUDA, std::string("group graph capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return set_error(FV_ERR_CUDA, std::string("group graph instantiate: ") + cudaGetErrorString(ce));
    e.launches = (int)launches;
    g->graphs.push_back(e);
    *out = &g->graphs.back();
    return FV_OK;
}

// Waits for the launched chunk.  With a communicator, the wait has a limit
// (fv_group_options.timeout_ms) and watches NCCL's asynchronous error: a
// process that died or never launched its part of a collective ends the
// wait with FV_ERR_COMM after aborting the communicator (NCCL's kernels then
// return), instead of a wait without end.
int wait_chunk(fv_group* g) {
    if (!g->comm) {
        GK(cudaStreamSynchronize(g->stream));
        return FV_OK;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaStreamQuery(g->stream);
        if (q == cudaSuccess) return FV_OK;
        if (q != cudaErrorNotReady) return set_error(FV_ERR_CUDA, std::string("fv_group_run: ") + cudaGetErrorString(q));
        ncclResult_t ae = ncclSuccess;
        g->nccl->CommGetAsyncError(g->comm, &ae);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ae != ncclSuccess || ms > g->timeout_ms) {
            std::string why = ae != ncclSuccess ? std::string("NCCL error: ") + g->nccl->GetErrorString(ae)
                                                : "no progress within " + std::to_string((long long)g->timeout_ms) + " ms";
            g->nccl->CommAbort(g->comm);
            g->comm = nullptr;
            g->aborted = true;
            return set_error(FV_ERR_COMM, "fv_group_run: " + why + "; the communicator was aborted");
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// A local part's stage buffer by role: tmp[0], tmp[1], sbase[0], sbase[1].
void* role_buffer(fv_solver* s, int role) { return role < 2 ? s->tmp[role] : s->sbase[role - 2]; }

// The P2P transport's plan: every push entry of the local parts, the
// readers' buffers (this process's parts directly; other processes' parts
// through CUDA IPC handles all-gathered over NCCL) and the wait lists.
int setup_p2p(fv_group* g, const HostMesh& gm, long long wait_limit) {
    const int P = g->n_parts, nl = (int)g->parts.size();
    GK(g->alloc(&g->flags, (size_t)nl * P));
    GK(cudaMemset(g->flags, 0, sizeof(unsigned long long) * nl * P));
    GK(g->alloc(&g->err, (size_t)nl));
    GK(cudaMemset(g->err, 0, sizeof(int) * nl));
    // IPC handles of every part's stage buffers and of its process's flag words
    struct Handles { cudaIpcMemHandle_t h[5]; };
    std::vector<Handles> all(P);
    if (g->n_ranks > 1) {
        for (int j = 0; j < nl; ++j) {
            Handles& hj = all[g->lo + j];
            for (int role = 0; role < 4; ++role) GK(cudaIpcGetMemHandle(&hj.h[role], role_buffer(g->parts[j], role)));
            GK(cudaIpcGetMemHandle(&hj.h[4], g->flags));
        }
        char* dev = nullptr;
        GK(g->alloc(&dev, sizeof(Handles) * P));
        GK(cudaMemcpy(dev + sizeof(Handles) * g->lo, &all[g->lo], sizeof(Handles) * nl, cudaMemcpyHostToDevice));
        NK(g, AllGather(dev + sizeof(Handles) * g->lo, dev, sizeof(Handles) * nl, ncclUint8, g->comm, g->stream));
        GK(cudaStreamSynchronize(g->stream));
        GK(cudaMemcpy(all.data(), dev, sizeof(Handles) * P, cudaMemcpyDeviceToHost));
    }
    std::map<std::string, void*> opened;  // one mapping per handle
    auto open = [&](const cudaIpcMemHandle_t& h, void** ptr) -> int {
        const std::string key(reinterpret_cast<const char*>(&h), sizeof(h));
        auto it = opened.find(key);
        if (it == opened.end()) {
            void* q = nullptr;
            GK(cudaIpcOpenMemHandle(&q, h, cudaIpcMemLazyEnablePeerAccess));
            g->ipc_opened.push_back(q);
            it = opened.emplace(key, q).first;
        }
        *ptr = it->second;
        return FV_OK;
    };
    std::map<int, PartPlan> other;  // plans of other processes' parts
    auto plan_of = [&](int r) -> const PartPlan* {
        if (g->local(r) >= 0) return &g->plans[g->local(r)];
        auto it = other.find(r);
        if (it == other.end()) {
            HostMesh L;
            PartPlan pl;
            if (!build_part(gm, P, r, L, pl).empty()) return nullptr;
            it = other.emplace(r, std::move(pl)).first;
        }
        return &it->second;
    };
    g->push.resize(nl);
    for (int j = 0; j < nl; ++j) {
        const int p = g->lo + j;
        const PartPlan& pp = g->plans[j];
        fv_group::Push& ps = g->push[j];
        std::vector<int32_t> slot, from, to;
        for (int r = 0; r < P; ++r) {
            if (r == p) continue;
            const int64_t n = pp.send_off[r + 1] - pp.send_off[r];
            if (n == 0) continue;
            const PartPlan* pr = plan_of(r);
            if (!pr || pr->recv_off[p + 1] - pr->recv_off[p] != n)
                return set_error(FV_ERR_ARG, "internal error: send and receive lists differ");
            if (ps.n_dst == fvgpu::kMaxPeers) return set_error(FV_ERR_UNSUPPORTED, "a part reaches more than 16 parts");
            const int sl = ps.n_dst++;
            for (int64_t i = 0; i < n; ++i) {
                slot.push_back(sl);
                from.push_back(pp.send_idx[pp.send_off[r] + i]);
                to.push_back(pr->recv_idx[pr->recv_off[p] + i]);
            }
            const int lr = g->local(r);
            if (lr >= 0) {
                for (int role = 0; role < 4; ++role) ps.buf[role][sl] = (uint32_t*)role_buffer(g->parts[lr], role);
                ps.flag[sl] = g->flags + (size_t)lr * P + p;
            } else {
                for (int role = 0; role < 4; ++role) {
                    void* q = nullptr;
                    int rc = open(all[r].h[role], &q);
                    if (rc) return rc;
                    ps.buf[role][sl] = (uint32_t*)q;
                }
                void* fq = nullptr;
                int rc = open(all[r].h[4], &fq);
                if (rc) return rc;
                const int r_lo = g->rank_of(r) * (P / g->n_ranks);
                ps.flag[sl] = (unsigned long long*)fq + (size_t)(r - r_lo) * P + p;
            }
        }
        ps.n = (int64_t)from.size();
        auto up = [&](int32_t** d, const std::vector<int32_t>& v) -> int {
            GK(g->alloc(d, v.size()));
            if (!v.empty()) GK(cudaMemcpy(*d, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
            return FV_OK;
        };
        int rc;
        if ((rc = up(&ps.slot, slot)) || (rc = up(&ps.from, from)) || (rc = up(&ps.to, to))) return rc;
        GK(g->alloc(&ps.ctr, 1));
        GK(cudaMemset(ps.ctr, 0, sizeof(unsigned long long)));
        // what part p waits for: the parts that send to it
        std::vector<int32_t> src;
        for (int s2 = 0; s2 < P; ++s2)
            if (s2 != p && pp.recv_off[s2 + 1] > pp.recv_off[s2]) src.push_back(s2);
        int32_t* d_src = nullptr;
        if ((rc = up(&d_src, src))) return rc;
        g->wp.flags[j] = g->flags + (size_t)j * P;
        g->wp.src[j] = d_src;
        g->wp.n_src[j] = (int)src.size();
    }
    g->wp.err = g->err;
    g->wp.ctrl = g->parts[0]->ctrl;
    g->wp.limit = wait_limit;
    // fused parts with one CTA per tile: the stage launches exchange the
    // halo themselves (destinations by sending cell and by sending ghost)
    g->fused_p2p = true;
    for (fv_solver* s : g->parts)
        if (!s->fused || s->sched == FV_SCHED_WORKLIST) g->fused_p2p = false;
    if (!g->fused_p2p) return FV_OK;
    GK(g->alloc(&g->rio, (size_t)nl * 4));
    for (int j = 0; j < nl; ++j) {
        const PartPlan& pp = g->plans[j];
        const fv_group::Push& ps = g->push[j];
        std::vector<int32_t> slot((size_t)ps.n), from((size_t)ps.n), to((size_t)ps.n);
        if (ps.n) {
            GK(cudaMemcpy(slot.data(), ps.slot, ps.n * 4, cudaMemcpyDeviceToHost));
            GK(cudaMemcpy(from.data(), ps.from, ps.n * 4, cudaMemcpyDeviceToHost));
            GK(cudaMemcpy(to.data(), ps.to, ps.n * 4, cudaMemcpyDeviceToHost));
        }
        const int64_t nr = g->parts[j]->n_real;
        std::vector<int32_t> coff(pp.n_band + 1, 0), goff(pp.n_own_ghost + 1, 0);
        for (int64_t i = 0; i < ps.n; ++i) {
            if (from[i] < nr) {
                if (from[i] >= pp.n_band) return set_error(FV_ERR_ARG, "internal error: a sent cell outside the band");
                ++coff[from[i] + 1];
            } else {
                if (from[i] - nr >= pp.n_own_ghost) return set_error(FV_ERR_ARG, "internal error: a sent ghost not owned");
                ++goff[from[i] - nr + 1];
            }
        }
        for (size_t i = 1; i < coff.size(); ++i) coff[i] += coff[i - 1];
        for (size_t i = 1; i < goff.size(); ++i) goff[i] += goff[i - 1];
        std::vector<int2> cdst((size_t)coff.back()), gdst((size_t)goff.back());
        std::vector<int32_t> cfill(coff.begin(), coff.end() - 1), gfill(goff.begin(), goff.end() - 1);
        for (int64_t i = 0; i < ps.n; ++i) {
            if (from[i] < nr) cdst[(size_t)cfill[from[i]]++] = make_int2(slot[i], to[i]);
            else gdst[(size_t)gfill[from[i] - nr]++] = make_int2(slot[i], to[i]);
        }
        int32_t *d_coff = nullptr, *d_goff = nullptr;
        int2 *d_cdst = nullptr, *d_gdst = nullptr;
        GK(g->alloc(&d_coff, coff.size()));
        GK(g->alloc(&d_goff, goff.size()));
        GK(g->alloc(&d_cdst, cdst.size()));
        GK(g->alloc(&d_gdst, gdst.size()));
        GK(cudaMemcpy(d_coff, coff.data(), coff.size() * 4, cudaMemcpyHostToDevice));
        GK(cudaMemcpy(d_goff, goff.data(), goff.size() * 4, cudaMemcpyHostToDevice));
        if (!cdst.empty()) GK(cudaMemcpy(d_cdst, cdst.data(), cdst.size() * sizeof(int2), cudaMemcpyHostToDevice));
        if (!gdst.empty()) GK(cudaMemcpy(d_gdst, gdst.data(), gdst.size() * sizeof(int2), cudaMemcpyHostToDevice));
        for (int role = 0; role < 4; ++role) {
            fvgpu::RemoteIO R{};
            R.n_dst = ps.n_dst;
            for (int d = 0; d < ps.n_dst; ++d) { R.dst[d] = ps.buf[role][d]; R.flag[d] = ps.flag[d]; }
            R.cell_off = d_coff; R.cell_dst = d_cdst; R.ghost_off = d_goff; R.ghost_dst = d_gdst;
            R.n_band = (int)pp.n_band;
            R.n_band_tiles = g->band_tiles[j];
            R.n_own_ghost = (int)pp.n_own_ghost;
            R.ctr = ps.ctr;
            R.my_flags = g->wp.flags[j];
            R.src = g->wp.src[j];
            R.n_src = g->wp.n_src[j];
            R.err = g->err + j;
            R.limit = wait_limit;
            GK(cudaMemcpy(g->rio + (size_t)j * 4 + role, &R, sizeof(R), cudaMemcpyHostToDevice));
        }
    }
    return FV_OK;
}

// P2P: push local part j's outputs of stage k to the parts that read them (on st)
int p2p_push(fv_group* g, int j, const void* out, int role, int stages, int k, cudaStream_t st) {
    const fv_group::Push& ps = g->push[j];
    if (ps.n == 0) return FV_OK;
    fvgpu::PushParams pa{};
    pa.src = (const uint32_t*)out;
    for (int d = 0; d < ps.n_dst; ++d) { pa.dst[d] = ps.buf[role][d]; pa.flag[d] = ps.flag[d]; }
    pa.n_dst = ps.n_dst;
    pa.slot = ps.slot; pa.from = ps.from; pa.to = ps.to; pa.n = ps.n;
    pa.words = (int)(g->V * g->parts[j]->ssz / 4);
    pa.ctr = ps.ctr;
    pa.ctrl = g->parts[j]->ctrl;
    pa.stages = stages; pa.stage = k;
    const int blocks = (int)std::min<int64_t>(std::max<int64_t>(fvgpu::blocks_of(ps.n * pa.words), 1), 148);
    fvgpu::k_p2p_push<<<blocks, fvgpu::kBlock, 0, st>>>(pa);
    GK(cudaGetLastError());
    return FV_OK;
}
// P2P: every local part waits for the epoch of stage k's input (on st)
int p2p_wait(fv_group* g, int stages, int k, cudaStream_t st) {
    fvgpu::WaitParams w = g->wp;
    w.stages = stages; w.stage = k;
    fvgpu::k_p2p_wait<<<(int)g->parts.size(), 32, 0, st>>>(w);
    GK(cudaGetLastError());
    return FV_OK;
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
    sizes[10] = plan.n_band;
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
    if (o->timeout_ms > 0) g->timeout_ms = o->timeout_ms;
    GK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    // the communicator first: every later failure of one process then ends
    // in the others' bounded waits, not in an unbounded initialisation
    const bool use_comm = R > 1 || g->nccl_local;
    if (use_comm) {
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
    fv_solver_options so = o->solver;
    if (ph->order2) so.stage_kernels = FV_STAGE_FUSED;
    for (int p = g->lo; p < g->hi; ++p) {
        std::unique_ptr<fv_mesh> lm(new fv_mesh());
        PartPlan plan;
        std::string err = build_part(fm->m, P, p, lm->m, plan);
        if (!err.empty()) return set_error(FV_ERR_ARG, err);
        fv_solver* s = nullptr;
        int rc0 = fv_solver_create_ex(lm.get(), ph, precision, device, &so, &s);
        if (rc0) return rc0;
        g->meshes.push_back(lm.release());
        g->parts.push_back(s);
        // reference cell 0: its own dt where this part owns it, else the
        // extra dt slot past the ghosts that the combine kernel fills
        s->TP.P.cell0 = plan.cell0 >= 0 ? plan.cell0 : (int)s->n_total;
        g->owner0 = plan.owner0;
        if ((rc0 = fv_solver_set_stream(s, g->stream))) return rc0;
        g->halo_cells += (int64_t)plan.recv_idx.size();
        g->plans.push_back(std::move(plan));
    }
    const int nl = (int)g->parts.size();
    if (nl > fvgpu::kMaxLocal) return set_error(FV_ERR_ARG, "at most 16 parts per process");
    for (int j = 0; j < nl; ++j) {
        fv_solver* s = g->parts[j];
        if (ph->order2 && !s->fused)
            return set_error(FV_ERR_MESH, "a part's two-ring tiles do not fit the fused stage kernel");
        g->pp.keys[j] = s->keys;
        g->pp.dt[j] = s->dt;
        g->pp.partials[j] = s->partials;
        g->pp.n_total[j] = (int)s->n_total;
        g->pp.cell0[j] = g->plans[j].cell0;
        g->pp.n_tiles[j] = s->n_tiles;
    }
    // the pack list: each local part's send list (by destination), in turn
    std::vector<int32_t> pk_part, pk_src, up_part, up_dst;
    std::vector<int64_t> up_from;
    g->pack_off.assign(nl + 1, 0);
    for (int j = 0; j < nl; ++j) {
        g->pack_off[j] = (int64_t)pk_src.size();
        for (int32_t c : g->plans[j].send_idx) { pk_part.push_back(j); pk_src.push_back(c); }
    }
    g->pack_off[nl] = (int64_t)pk_src.size();
    // messages and receive slots, pair (s, r) in the same order on every
    // process; pairs within this process read the sender's pack directly
    int64_t n_recv = 0;
    for (int sp = 0; sp < P; ++sp)
        for (int rp = 0; rp < P; ++rp) {
            if (sp == rp) continue;
            const int ls = g->local(sp), lr = g->local(rp);
            const bool wire = use_comm && !(ls >= 0 && lr >= 0 && !g->nccl_local);
            if (ls >= 0 && wire) {
                const PartPlan& ps = g->plans[ls];
                const int64_t n = ps.send_off[rp + 1] - ps.send_off[rp];
                if (n > 0) g->msgs.push_back({g->rank_of(rp), 1, g->pack_off[ls] + ps.send_off[rp], n});
            }
            if (lr >= 0) {
                const PartPlan& pr = g->plans[lr];
                const int64_t n = pr.recv_off[sp + 1] - pr.recv_off[sp];
                if (n == 0) continue;
                for (int64_t i = 0; i < n; ++i) {
                    up_part.push_back(lr);
                    up_dst.push_back(pr.recv_idx[pr.recv_off[sp] + i]);
                }
                if (wire) {
                    g->msgs.push_back({g->rank_of(sp), 0, n_recv, n});
                    for (int64_t i = 0; i < n; ++i) up_from.push_back(n_recv + i);
                    n_recv += n;
                } else {
                    const PartPlan& ps = g->plans[ls];
                    if (ps.send_off[rp + 1] - ps.send_off[rp] != n)
                        return set_error(FV_ERR_ARG, "internal error: send and receive lists differ");
                    for (int64_t i = 0; i < n; ++i) up_from.push_back(~(g->pack_off[ls] + ps.send_off[rp] + i));
                }
            }
        }
    g->n_pack = (int64_t)pk_src.size();
    g->n_unpack = (int64_t)up_dst.size();
    g->n_recv = n_recv;
    const size_t cell_bytes = (size_t)ph->V * g->parts[0]->ssz;
    auto up = [&](auto** d, const auto& v) -> int {
        GK(g->alloc(d, v.size()));
        if (!v.empty()) GK(cudaMemcpy(*d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice));
        return FV_OK;
    };
    int rc;
    if ((rc = up(&g->pack_part, pk_part)) || (rc = up(&g->pack_src, pk_src)) || (rc = up(&g->unpack_part, up_part)) ||
        (rc = up(&g->unpack_dst, up_dst)) || (rc = up(&g->unpack_from, up_from)))
        return rc;
    GK(g->alloc((char**)&g->send_all, (size_t)g->n_pack * cell_bytes));
    GK(g->alloc((char**)&g->recv_all, (size_t)n_recv * cell_bytes));
    // the band-first stage: fused parts with one CTA per tile, and
    // something to exchange
    g->overlap = o->serial_exchange == 0 && (g->n_pack > 0 || g->n_unpack > 0);
    for (int j = 0; j < nl; ++j) {
        fv_solver* s = g->parts[j];
        if (!s->fused || s->sched == FV_SCHED_WORKLIST) g->overlap = false;
        const int T = s->fused ? s->FPm.T : 1;
        g->band_tiles.push_back((int)std::min<int64_t>((g->plans[j].n_band + T - 1) / T, s->n_tiles));
    }
    if (o->transport == FV_EXCHANGE_P2P && (g->n_pack > 0 || g->n_unpack > 0)) {
        g->p2p = true;
        int rc2 = setup_p2p(g.get(), fm->m, o->wait_polls > 0 ? o->wait_polls : (1ll << 24));
        if (rc2) return rc2;
        // the in-launch exchange overlaps the interior tiles by itself
        if (g->fused_p2p) g->overlap = false;
    } else if (o->transport != FV_EXCHANGE_COPY && o->transport != FV_EXCHANGE_P2P) {
        return set_error(FV_ERR_ARG, "unknown transport");
    }
    if (g->overlap) {
        int lo_pri = 0, hi_pri = 0;
        GK(cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
        GK(cudaStreamCreateWithPriority(&g->cstream, cudaStreamNonBlocking, hi_pri));
        GK(cudaEventCreateWithFlags(&g->ev_start, cudaEventDisableTiming));
        GK(cudaEventCreateWithFlags(&g->ev_halo, cudaEventDisableTiming));
    }
    GK(g->alloc(&g->recs, (size_t)2 * P));
    GK(g->alloc(&g->sums, (size_t)ph->V * P));
    GK(cudaMemset(g->sums, 0, sizeof(double) * ph->V * P));
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
    if (g->aborted) return set_error(FV_ERR_COMM, "fv_group_run: the communicator was aborted by an earlier run");
    GK(cudaSetDevice(g->device));
    cudaStream_t st = g->stream;
    std::vector<double> alpha(o->alpha, o->alpha + o->n_alpha);
    const RunLimits L{o->max_step, o->max_time, o->tolerance, o->print_interval};
    if (g->p2p && o->restart) {
        // epochs count from step 0 again: flags, failures and push counts
        // restart at zero (before this process's first dt all-gather, which
        // no process passes before every process has reset)
        GK(cudaMemsetAsync(g->flags, 0, sizeof(unsigned long long) * g->parts.size() * g->n_parts, st));
        GK(cudaMemsetAsync(g->err, 0, sizeof(int) * g->parts.size(), st));
        for (auto& ps : g->push)
            if (ps.ctr) GK(cudaMemsetAsync(ps.ctr, 0, sizeof(unsigned long long), st));
    }
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
        // graph length: the largest power of two <= min(chunk, steps left)
        const unsigned long long left = o->max_step > cur ? o->max_step - cur : 1ull;
        int len = 1;
        while ((unsigned long long)(len * 2) <= left && len * 2 <= s0->chunk) len *= 2;
        GraphEntry* ge = nullptr;
        if ((rc = group_graph(g, alpha, len, &ge))) break;
        cudaEventRecord(e0, st);
        if (cudaGraphLaunch(ge->exec, st) != cudaSuccess) {
            rc = set_error(FV_ERR_CUDA, "fv_group_run: graph launch");
            break;
        }
        launches += ge->launches;
        cudaEventRecord(e1, st);
        launch_ctrl_copy(s0->ctrl, s0->hctrl_dev, st);
        if (cudaGetLastError() != cudaSuccess) {
            rc = set_error(FV_ERR_CUDA, "fv_group_run: a launch failed");
            break;
        }
        if ((rc = wait_chunk(g))) break;
        if (g->p2p) {
            std::vector<int> errs(g->parts.size());
            if (cudaMemcpy(errs.data(), g->err, errs.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
                rc = set_error(FV_ERR_CUDA, "fv_group_run: halo wait status");
                break;
            }
            if (std::find(errs.begin(), errs.end(), 1) != errs.end()) {
                rc = set_error(FV_ERR_COMM, "fv_group_run: a halo wait gave up before its senders' epoch arrived");
                break;
            }
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
    int64_t band = 0;
    for (int b : g->band_tiles) band += b;
    out[6] = (g->overlap || g->fused_p2p) ? band : -1;
    out[7] = g->p2p ? FV_EXCHANGE_P2P : FV_EXCHANGE_COPY;
    return FV_OK;
}

int fv_group_last_run_stats(fv_group* g, double* device_ms, int64_t* kernel_launches) {
    if (!g) return set_error(FV_ERR_ARG, "fv_group_last_run_stats: null group");
    if (device_ms) *device_ms = g->last_ms;
    if (kernel_launches) *kernel_launches = g->last_launches;
    return FV_OK;
}

}  // extern "C"
