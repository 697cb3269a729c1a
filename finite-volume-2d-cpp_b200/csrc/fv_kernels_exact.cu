// FP64 kernels of the explicit FV step in the reference's exact evaluation
// order (compile with -fmad=false).  One thread per real cell; each cell
// gathers its faces in increasing reference edge order, so every per-cell
// sum is accumulated in the same order as the reference's edge-scatter loops
// and the results are bit-identical -- with no atomics anywhere.
#include <cuda_runtime.h>

#include "fv_launch.h"
#include "fv_physics_exact.cuh"

namespace fvgpu {

__device__ __forceinline__ unsigned long long dkey(double x) {
    if (x != x) return ~0ull;  // NaN never wins the minimum
    const long long b = __double_as_longlong(x);
    return b < 0 ? ~(unsigned long long)b : ((unsigned long long)b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
    if (k == ~0ull) return __longlong_as_double(0x7ff8000000000000ll);
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}
__device__ __forceinline__ bool inactive(const Ctrl* c) {
    return c != nullptr && *(volatile const int*)&c->active == 0;
}
template <int V>
__device__ __forceinline__ void load_cell(const double* __restrict__ a, int c, double* v) {
    if (V == 4) {
        const double2* p = reinterpret_cast<const double2*>(a + 4 * (size_t)c);
        double2 x = p[0], y = p[1];
        v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = a[(size_t)V * c + k];
    }
}
template <int V>
__device__ __forceinline__ void store_cell(double* __restrict__ a, int c, const double* v) {
    if (V == 4) {
        double2* p = reinterpret_cast<double2*>(a + 4 * (size_t)c);
        p[0] = make_double2(v[0], v[1]);
        p[1] = make_double2(v[2], v[3]);
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) a[(size_t)V * c + k] = v[k];
    }
}

// ------------------------------------------------------------ step control --
// Stop criteria of the step about to start (explicit.cpp:717-726), one thread.
__device__ __forceinline__ void step_start(unsigned long long step, double time, const double* R, int V,
                                           const RunLimits& L, int* active, int* need_R) {
    double Rmax;
    if (step > 0) {
        Rmax = 0.0;
        for (int k = 0; k < V; ++k) Rmax = exact::dmax(R[k], Rmax);
    } else {
        Rmax = 1.0;
    }
    const int stop = (step >= L.max_step) | (time >= L.max_time) | (Rmax < L.tolerance);
    *active = !stop;
    *need_R = !stop && (step == 0 || (step % L.print_interval) == 0 || (L.tolerance > 1.01e-16));
}
__device__ void begin_step(Ctrl* c, const RunLimits* L, int V) {
    int active, need_R;
    step_start(c->step, c->time, c->R, V, *L, &active, &need_R);
    c->active = active;
    c->need_R = need_R;
}

// First kernel of every launch sequence (graph): the step's start, and an
// empty print-record list for this sequence.
__global__ void k_step_begin(Ctrl* c, const RunLimits* L, int V, unsigned long long* keys, int nkeys) {
    for (int i = threadIdx.x; i < nkeys; i += blockDim.x) keys[i] = ~0ull;
    if (threadIdx.x == 0) {
        c->n_hist = 0;
        begin_step(c, L, V);
    }
}

// Run control set and read by small kernels, not by copies: a copy would
// queue behind state transfers that other streams keep the copy engines busy
// with (the host reads the control through mapped pinned memory).
static_assert(sizeof(Ctrl) % 8 == 0, "Ctrl is copied in 8-byte words");
__global__ void k_ctrl_reset(Ctrl* c) {
    unsigned long long* w = reinterpret_cast<unsigned long long*>(c);
    for (int i = threadIdx.x; i < (int)(sizeof(Ctrl) / 8); i += blockDim.x) w[i] = 0ull;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < kMaxV; ++k) c->R[k] = 1.0;
        c->active = 1;
    }
}
__global__ void k_ctrl_copy(const Ctrl* src, Ctrl* dst) {
    const unsigned long long* a = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* b = reinterpret_cast<unsigned long long*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(Ctrl) / 8); i += blockDim.x) b[i] = a[i];
}
__global__ void k_set_limits(RunLimits* d, RunLimits v) {
    if (threadIdx.x == 0) *d = v;
}
void launch_ctrl_reset(Ctrl* c, cudaStream_t st) { k_ctrl_reset<<<1, 64, 0, st>>>(c); }
void launch_ctrl_copy(const Ctrl* src, Ctrl* dst, cudaStream_t st) { k_ctrl_copy<<<1, 64, 0, st>>>(src, dst); }
void launch_set_limits(RunLimits* d, const RunLimits& v, cudaStream_t st) { k_set_limits<<<1, 32, 0, st>>>(d, v); }

// Residual norms, step/time bookkeeping and print records
// (explicit.cpp:752-800), then the next step's start: its stop criteria and
// fresh dt key slots, so that consecutive steps need no separate begin
// kernel.  Partial sums are reduced in a fixed order.
constexpr int kEndBlock = 1024;  // threads of the step-end kernel (one block)
__global__ void __launch_bounds__(kEndBlock) k_step_end(Params P, Ctrl* c, const RunLimits* L, const double* partials, int nblocks,
                           const double* dt, unsigned long long* keys, int nkeys, PrintRec* hist, int hist_cap) {
    // launched as a programmatic dependent of the last stage kernel: wait for
    // it to complete before reading anything
    asm volatile("griddepcontrol.wait;" ::: "memory");
    // every thread reads the step's control words before thread 0 rewrites
    // them for the next step
    const bool act = c->active != 0, need_R = c->need_R != 0;
    __syncthreads();
    if (!act) return;
    if (P.n_cases > 1) {
        // each case of a batch keeps its own time: time += dt[0] of that case
        for (int k = threadIdx.x; k < P.n_cases; k += blockDim.x) {
            const double d0 = dt[P.case_cell0[k]];
            double dk = d0;
            if (P.global_dt && d0 == d0) {
                unsigned long long key = ~0ull;
                for (int i = 0; i < 64; ++i) key = keys[(size_t)k * 64 + i] < key ? keys[(size_t)k * 64 + i] : key;
                dk = dkey_inv(key);
            }
            P.case_time[k] += dk;
        }
    }
    // residual sums: per-thread strided sums over the tile partials, then a
    // fixed butterfly inside each warp and over the warps (deterministic)
    __shared__ double red[kEndBlock / 32][kMaxV];
    const int V = P.V;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double s[kMaxV] = {0, 0, 0, 0};
    if (need_R) {
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
            for (int k = 0; k < V; ++k) s[k] += partials[(size_t)b * V + k];
        for (int k = 0; k < V; ++k)
            for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
        if (lane == 0)
            for (int k = 0; k < V; ++k) red[warp][k] = s[k];
        __syncthreads();
        if (warp == 0) {
            for (int k = 0; k < V; ++k) {
                s[k] = lane < (int)(blockDim.x >> 5) ? red[lane][k] : 0.;
                for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
            }
        }
    }
    // the global dt minimum of the step (case 0 of a batch: its keys come first)
    unsigned long long kmin = ~0ull;
    if (P.global_dt && warp == 0) {
        kmin = keys[lane] < keys[lane + 32] ? keys[lane] : keys[lane + 32];
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, kmin, o);
            kmin = x < kmin ? x : kmin;
        }
    }
    if (threadIdx.x == 0) {
        // every control value of the step, loaded together
        const unsigned long long step = c->step;
        const double time = c->time;
        double R[kMaxV], R0[kMaxV];
        for (int k = 0; k < V; ++k) { R[k] = c->R[k]; R0[k] = c->R0[k]; }
        const int n_hist = c->n_hist;
        const RunLimits lim = *L;
        // min_dt (explicit.cpp:555-564): a NaN in dt[0] wins
        const double d0 = dt[P.cell0];
        if (need_R) {
            for (int k = 0; k < V; ++k) {
                const double r = sqrt(s[k]);
                c->Rraw[k] = r;
                if (step == 0) R0[k] = r;
                R[k] = step == 0 ? r : r / R0[k];
                c->R0[k] = R0[k];
                c->R[k] = R[k];
            }
        }
        const bool print = (step == 0) || (step % lim.print_interval) == 0;
        if (print && n_hist < hist_cap) {
            PrintRec& r = hist[n_hist];
            r.step = step;
            r.time = time;
            for (int k = 0; k < V; ++k) r.R[k] = (step == 0) ? 1.0 : R[k];
            c->n_hist = n_hist + 1;
        }
        const double dt0 = P.global_dt ? ((d0 != d0) ? d0 : dkey_inv(kmin)) : d0;
        c->step = step + 1;
        c->time = time + dt0;
        int active, next_R;
        step_start(step + 1, time + dt0, R, V, lim, &active, &next_R);
        c->active = active;
        c->need_R = next_R;
    }
    __syncthreads();  // the keys have been read
    for (int i = threadIdx.x; i < nkeys; i += blockDim.x) keys[i] = ~0ull;
}

void launch_step_begin(Ctrl* c, const RunLimits* lim, int V, unsigned long long* keys, int nkeys, cudaStream_t st) {
    k_step_begin<<<1, 128, 0, st>>>(c, lim, V, keys, nkeys);
}
void launch_step_end(const Params& P, Ctrl* c, const RunLimits* lim, const double* partials, int nblocks,
                     const double* dt, unsigned long long* keys, int nkeys, PrintRec* hist, int hist_cap,
                     cudaStream_t st, bool pdl) {
    if (!pdl) {
        k_step_end<<<1, kEndBlock, 0, st>>>(P, c, lim, partials, nblocks, dt, keys, nkeys, hist, hist_cap);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(kEndBlock);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_step_end, P, c, lim, partials, nblocks, dt, keys, nkeys, hist, hist_cap);
}

namespace exact {

// Standalone ghost fill (update_bounds, explicit.cpp:380-417), one thread
// per ghost.  zero_grad: the initial fill run() does before the loop with
// freshly zeroed gx, gy, limiters (explicit.cpp:712).
template <int V>
__global__ void k_bounds(Params P, double* __restrict__ q, const double* __restrict__ gx,
                         const double* __restrict__ gy, const double* __restrict__ lim, int zero_grad) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= P.n_bound) return;
    const int N = P.n_real;
    const int c = P.ghost_cell[b];
    const double nx = P.g_nx[b], ny = P.g_ny[b];
    double qc[V], qint[V], out[V];
    load_cell<V>(q, c, qc);
    if (P.order2) {
        const double d0 = P.g_dx[b], d1 = P.g_dy[b];
        double gxc[V], gyc[V], lc[V];
        if (zero_grad) {
#pragma unroll
            for (int k = 0; k < V; ++k) { gxc[k] = 0.; gyc[k] = 0.; lc[k] = 0.; }
        } else {
            load_cell<V>(gx, c, gxc); load_cell<V>(gy, c, gyc); load_cell<V>(lim, c, lc);
        }
#pragma unroll
        for (int k = 0; k < V; ++k) qint[k] = qc[k] + (gxc[k] * d0 + gyc[k] * d1) * lc[k];
        if (V == 4 && P.positivity_guard) {  // optional guard, see fv_tile.cuh
            const double p = (P.gamma - 1) * (qint[3] - 0.5 / qint[0] * (qint[1] * qint[1] + qint[2] * qint[2]));
            if (!(qint[0] > 0.) || !(p > 0.))
                for (int k = 0; k < V; ++k) qint[k] = qc[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) qint[k] = qc[k];
    }
    bc<V>(P, P.ghost_group[b], b, out, qint, nx, ny);
    store_cell<V>(q, N + b, out);
}

}  // namespace exact

namespace exact {
void launch_bounds(const Params& P, double* q, const double* gx, const double* gy, const double* lim,
                   int zero_grad, cudaStream_t st) {
    if (P.n_bound == 0) return;
    const int g = grid_for(P.n_bound);
    if (P.V == 4) k_bounds<4><<<g, kBlock, 0, st>>>(P, q, gx, gy, lim, zero_grad);
    else if (P.V == 2) k_bounds<2><<<g, kBlock, 0, st>>>(P, q, gx, gy, lim, zero_grad);
    else k_bounds<1><<<g, kBlock, 0, st>>>(P, q, gx, gy, lim, zero_grad);
}
}  // namespace exact

// ------------------------------------------------------ residual smoothing --
// One Jacobi sweep (explicit.cpp:46-64, epsilon 0.6), one thread per real
// cell, neighbours gathered in increasing reference edge order: the same
// operations in the same order as the reference's edge scatter.
template <int V>
__global__ void k_smooth(int n_real, const uint32_t* __restrict__ nbr, const double* __restrict__ qt_in,
                         const double* __restrict__ qt0, double* __restrict__ qt_out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_real) return;
    const double epsilon = 0.6;
    double s[V];
#pragma unroll
    for (int k = 0; k < V; ++k) s[k] = 0.;
    int ne = 0;
#pragma unroll
    for (int f = 0; f < kMaxFaces; ++f) {
        const uint32_t w = nbr[(size_t)f * n_real + c];
        if (w == kNoFace) continue;
        ++ne;
        const int nb = (int)(w & 0x7FFFFFFFu);
        double qn[V];
        load_cell<V>(qt_in, nb, qn);
#pragma unroll
        for (int k = 0; k < V; ++k) s[k] -= qn[k] * epsilon;
    }
    const double nf = ne == 3 ? 3 : 4;  // cellsIsTriangle ? 3 : 4
    double q0[V], out[V];
    load_cell<V>(qt0, c, q0);
#pragma unroll
    for (int k = 0; k < V; ++k) out[k] = (q0[k] - s[k]) / (1. + nf * epsilon);
    store_cell<V>(qt_out, c, out);
}
void launch_smooth(const Params& P, const uint32_t* nbr, const double* qt_in, const double* qt0, double* qt_out,
                   cudaStream_t st) {
    const int g = grid_for(P.n_real);
    if (P.V == 4) k_smooth<4><<<g, kBlock, 0, st>>>(P.n_real, nbr, qt_in, qt0, qt_out);
    else if (P.V == 2) k_smooth<2><<<g, kBlock, 0, st>>>(P.n_real, nbr, qt_in, qt0, qt_out);
    else k_smooth<1><<<g, kBlock, 0, st>>>(P.n_real, nbr, qt_in, qt0, qt_out);
}

// ----------------------------------------------------------------- utilities --
__global__ void k_permute_to_device(const double* __restrict__ qr, double* __restrict__ qd,
                                    const int32_t* __restrict__ new2ref, int n, int V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = new2ref[i];
    for (int k = 0; k < V; ++k) qd[(size_t)V * i + k] = qr[(size_t)V * r + k];
}
__global__ void k_permute_to_ref(const double* __restrict__ qd, double* __restrict__ qr,
                                 const int32_t* __restrict__ new2ref, int n, int V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = new2ref[i];
    for (int k = 0; k < V; ++k) qr[(size_t)V * r + k] = qd[(size_t)V * i + k];
}
void launch_permute_to_device(const double* q_ref, double* q_dev, const int32_t* new2ref, int n, int V,
                              cudaStream_t st) {
    k_permute_to_device<<<grid_for(n), kBlock, 0, st>>>(q_ref, q_dev, new2ref, n, V);
}
void launch_permute_to_ref(const double* q_dev, double* q_ref, const int32_t* new2ref, int n, int V,
                           cudaStream_t st) {
    k_permute_to_ref<<<grid_for(n), kBlock, 0, st>>>(q_dev, q_ref, new2ref, n, V);
}

// Extra output fields of real cells (exact::output_field) into reference
// order: field f of cell r at out[off[f] + nc[f] * r + j].  q is in device
// numbering (new2ref given) or in reference numbering (new2ref null).
__global__ void k_output_fields(const double* __restrict__ q, int V, const int32_t* __restrict__ new2ref, int n_real,
                                double gamma, OutputPlan plan, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_real) return;
    const int r = new2ref ? new2ref[i] : i;
    double qc[kMaxV] = {0., 0., 0., 0.};
    for (int k = 0; k < V; ++k) qc[k] = q[(size_t)V * i + k];
    for (int f = 0; f < plan.n; ++f) {
        double v[2];
        const int nc = exact::output_field(plan.kind[f], gamma, qc, v);
        for (int j = 0; j < nc; ++j) out[plan.off[f] + (size_t)nc * r + j] = v[j];
    }
}
void launch_output_fields(const double* q, int V, const int32_t* new2ref, int n_real, double gamma,
                          const OutputPlan& plan, double* out, cudaStream_t st) {
    k_output_fields<<<grid_for(n_real), kBlock, 0, st>>>(q, V, new2ref, n_real, gamma, plan, out);
}

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void k_to_double(const float* __restrict__ a, double* __restrict__ b, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}
void launch_to_float(const double* a, float* b, size_t n, cudaStream_t st) {
    if (n) k_to_float<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, st>>>(a, b, n);
}
void launch_to_double(const float* a, double* b, size_t n, cudaStream_t st) {
    if (n) k_to_double<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, st>>>(a, b, n);
}

template <class S>
__global__ void k_fill_ghost_grad_t(S* gx, S* gy, S* lim, int n_real, int n_total, int V) {
    const int i = n_real + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total) return;
    for (int k = 0; k < V; ++k) {
        gx[(size_t)V * i + k] = 0.;
        gy[(size_t)V * i + k] = 0.;
        lim[(size_t)V * i + k] = 1.;
    }
}
// Ghost cells keep gx = gy = 0 and lim = 1 (the reference never updates them).
void launch_fill_ghost_grad(void* gx, void* gy, void* lim, int n_real, int n_total, int V, bool f32,
                            cudaStream_t st) {
    if (n_total <= n_real) return;
    const int g = grid_for(n_total - n_real);
    if (f32) k_fill_ghost_grad_t<float><<<g, kBlock, 0, st>>>((float*)gx, (float*)gy, (float*)lim, n_real, n_total, V);
    else k_fill_ghost_grad_t<double><<<g, kBlock, 0, st>>>((double*)gx, (double*)gy, (double*)lim, n_real, n_total, V);
}

__global__ void k_check_state(Params P, const double* __restrict__ q, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_real) return;
    bool bad = false;
    const int V = P.V;
    for (int k = 0; k < V; ++k) {
        const double v = q[(size_t)V * i + k];
        bad |= !(v == v) || fabs(v) > 1.7e308;
    }
    if (V == 4 && !bad) {
        double s[4];
        for (int k = 0; k < 4; ++k) s[k] = q[(size_t)4 * i + k];
        bad = !(s[0] > 0.) || !(exact::pres(P.gamma, s) > 0.);
    }
    if (bad) atomicExch(flag, 1);
}
void launch_check_state(const Params& P, const double* q, int* flag, cudaStream_t st) {
    k_check_state<<<grid_for(P.n_real), kBlock, 0, st>>>(P, q, flag);
}

// Pressure force over one boundary group; one block, fixed summation order.
__global__ void k_force(Params P, const double* __restrict__ q, int group, double* out) {
    __shared__ double sx[kBlock], sy[kBlock];
    double ax = 0., ay = 0.;
    for (int b = threadIdx.x; b < P.n_bound; b += blockDim.x) {
        if (P.ghost_group[b] != group) continue;
        double s[4];
        load_cell<4>(q, P.ghost_cell[b], s);
        const double p = exact::pres(P.gamma, s);
        const double le = P.g_le[b];
        ax += p * P.g_nx[b] * le;
        ay += p * P.g_ny[b] * le;
    }
    sx[threadIdx.x] = ax; sy[threadIdx.x] = ay;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) { sx[threadIdx.x] += sx[threadIdx.x + w]; sy[threadIdx.x] += sy[threadIdx.x + w]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = sx[0]; out[1] = sy[0]; }
}
void launch_force(const Params& P, const double* q, int group, double* out2, cudaStream_t st) {
    k_force<<<1, kBlock, 0, st>>>(P, q, group, out2);
}

}  // namespace fvgpu
