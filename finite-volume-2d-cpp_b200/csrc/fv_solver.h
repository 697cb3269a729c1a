// The solver object behind the C ABI's fv_solver handle, and one time step
// split into the launches a domain decomposition interleaves across its
// parts (internal to the library).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/fvgpu.h"
#include "fv_fused.cuh"
#include "fv_launch.h"
#include "fv_mesh.h"
#include "fv_tile.cuh"

using namespace fvgpu;

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
    bool f32 = false;
    size_t ssz = 8;                 // bytes of one stored stage value
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int V = 4;
    int64_t n_real = 0, n_total = 0, n_bound = 0;
    int n_tiles = 0;
    TileParams TP{};
    // the fused stage kernel over two-ring tiles (its Params are TP.P at launch)
    bool fused = false;
    // with fused: the first stage of each step runs the split kernels, whose
    // gradient kernel also computes dt (no separate dt kernel)
    bool split_first = false;
    FusedParams FPm{};
    // its schedule (FV_SCHED_*); the work list's per-stage tile counters and
    // CTAs per launch
    int sched = 0;
    int* work = nullptr;
    int work_grid = 0;
    // device buffers
    std::vector<void*> allocs;
    double* qbase[2] = {nullptr, nullptr};   // FP64 step-start state (RK1 alternates)
    void* sbase[2] = {nullptr, nullptr};     // stage-precision copy of the base (== qbase unless FP32)
    void* tmp[2] = {nullptr, nullptr};       // intermediate stage outputs
    void *gx = nullptr, *gy = nullptr, *lim = nullptr;
    double* dt = nullptr;
    double* stage_buf = nullptr;   // [n_total*V] staging for host transfers
    double* partials = nullptr;
    double* scratch2 = nullptr;
    int* flag = nullptr;
    int32_t* new2ref = nullptr;
    Ctrl* ctrl = nullptr;
    RunLimits* limits = nullptr;
    PrintRec* hist = nullptr;
    int hist_cap = 0;
    int chunk = 16;
    std::vector<GraphEntry> graphs;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    // dt minimum key slots: [n_cases][kDtSlots] (one case: inside ctrl)
    unsigned long long* keys = nullptr;
    int n_cases = 1;
    double* case_time = nullptr;                           // batches: [n_cases]
    double* ghost_bv = nullptr;                            // per-ghost boundary states [n_bound][4]
    Ctrl* hctrl = nullptr;      // mapped pinned host copy of the run control, written by a kernel
    Ctrl* hctrl_dev = nullptr;  // its device address
    std::vector<int64_t> case_real_off, case_bound_off;    // batches: host copies
    // residual smoothing: time derivatives before / after each Jacobi sweep
    // ([n_total][V], ghosts 0) and the real cells' neighbours ([4][n_real])
    double* qts[3] = {nullptr, nullptr, nullptr};
    uint32_t* nbr = nullptr;

    template <class T>
    cudaError_t alloc(T** p, size_t n, size_t elem = sizeof(T)) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * elem);
        if (e == cudaSuccess) allocs.push_back((void*)*p);
        return e;
    }
    ~fv_solver() {
        cudaSetDevice(device);
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        for (void* p : allocs) cudaFree(p);
        if (hctrl) cudaFreeHost(hctrl);  // allocated with cudaHostAlloc
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace fvgpu {

// Kernel kinds for per-kernel timing.
enum { KK_BEGIN = 0, KK_DT = 1, KK_GRADLIM = 2, KK_STAGE = 3, KK_END = 4, KK_FUSED = 5, KK_N = 6 };

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

// One time step whose base state is qbase[b] (explicit.cpp:715-801), as
// three launch phases: step_open (the begin-of-step kernel when `first`, and
// the dt kernel), step_stage for each RK stage k (whose output state, in the
// stage precision, is c.out afterwards), and step_close (residual norms from
// `nblocks` partial sums, time, stop criteria, the next step's start).
// Each returns the number of kernels it launched.
struct StepCursor {
    TileIO io{};
    FusedParams FPl{};
    bool grads = false, worklist = false, split_first = false;
    int b = 0;
    const void* in = nullptr;
    void* out = nullptr;
    // a decomposition part: its fused launches use the part kernel (owned
    // count from the tile info); remote: the next one exchanges its halo
    // inside (device memory), or nullptr
    bool part = false;
    const RemoteIO* remote = nullptr;
};
// with_dt = false: step_open leaves the dt kernel to a later step_dt (a
// decomposition waits for its halo in between).
int step_open(fv_solver* s, const std::vector<double>& alpha, int b, bool first, StepCursor& c, EventLog* log,
              bool with_dt = true);
int step_dt(fv_solver* s, StepCursor& c, EventLog* log);
// r: only tiles [r->t0, r->t0 + r->n) of the fused stage kernel (one CTA
// per tile) on r->stream (nullptr: the solver's stream), with programmatic
// dependent launch when r->pdl; the stage's output becomes the next stage's
// input after the range with r->last set.
struct TileRange {
    int t0, n;
    bool pdl, last;
    cudaStream_t stream;
};
int step_stage(fv_solver* s, const std::vector<double>& alpha, int k, StepCursor& c, EventLog* log,
               const TileRange* r = nullptr);
int step_close(fv_solver* s, const double* partials, int nblocks, EventLog* log);

// The library's last-error slot (fv_last_error) and its codes.
int set_error(int code, const std::string& msg);

}  // namespace fvgpu
