// Tile kernels of the explicit FV step.
//
// The device-numbered (Hilbert-ordered) real cells are cut into tiles of T
// consecutive cells; one CTA of T threads owns one tile.  A CTA stages the
// records of its cells and their halo (state, gradients, centroid) into
// shared memory, computes every edge flux touching the tile once, and then
// lets each thread sum its cell's faces from shared memory in increasing
// reference edge order -- deterministic, atomic-free, and (with the Exact
// policy) bit-identical to the reference's edge-scatter loops.
//
// Math policies: MExact (FP64, reference evaluation order; instantiated in a
// -fmad=false translation unit), MF64 (FP64, fast algebra), MF32 (FP32 bulk
// arithmetic and storage of stage states, gradients and geometry; FP64
// conserved state, per-cell flux sums, RK accumulation and residuals).  The
// fast policies store the limiter already multiplied into the gradients.
//
// Face words (uint16, [4][n_real]): bits 0-13 tile-local edge, bit 14 the
// neighbour is a boundary ghost, bit 15 the cell is the edge's second cell;
// 0xFFFF = no face.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <type_traits>

#include "fv_internal.h"
#include "fv_physics_exact.cuh"
#include "fv_physics_fast.cuh"

namespace fvgpu {

struct MExact { using S = double; static constexpr bool exact = true; };
struct MF64 { using S = double; static constexpr bool exact = false; };
struct MF32 { using S = float; static constexpr bool exact = false; };

constexpr int kDtSlots = 64;        // atomic slots of the global dt minimum
constexpr int kTileMax = 256;       // threads (= cells) per tile at most
constexpr uint16_t kFaceNone = 0xFFFF;
constexpr int kFaceEdgeMask = 0x3FFF;

struct TileParams {
    Params P;                  // sizes, ghost metadata and physics
    int T;                     // cells per tile (= threads per CTA)
    int max_halo, max_edges;
    const int4* info;          // [n_tiles]: edge_off, n_edges, halo_off, n_halo
    const int32_t* halo;       // device cell index per halo slot
    const uint32_t* edge_ij;   // local i | local j << 16
    const void* enx;           // S [tile edges]: normal, length, face centre, GG weight
    const void* eny;
    const void* ele;
    const void* exf;
    const void* eyf;
    const void* eg;
    const uint16_t* face;      // [4][n_real] face words
    const void* ccxy;          // S [n_total][2] centroids
    const void* area;          // S [n_total]
};

struct TileIO {
    const void* q_stage;       // S [n_total][V] stage input
    const double* q_base;      // [n_total][V] step-start state (FP64)
    double* q_out;             // FP64 output (FP64 modes: every stage; FP32: last stage only)
    void* s_out;               // FP32 mode: FP32 stage output (the next stage's input)
    void* gx;                  // S [n_total][V]; fast modes: limited gradients; ghosts hold 0
    void* gy;
    void* lim;                 // exact mode only; ghosts hold 1
    double* dt;                // [n_total]
    double alpha;
    Ctrl* ctrl;                // nullptr: always active, dt from dt[]
    double* partials;          // [n_tiles][V] or nullptr
    unsigned long long* dtkeys;  // [n_cases][kDtSlots] ordered keys of the global dt minimum
    int write_f64;             // FP32 mode: also write q_out (last stage)
    double* qt;                // [n_total][V] time derivatives of the smoothing phases (FP64)
    int* work;                 // fused stage kernel, work-list schedule: this launch's tile counter
    int* work_reset;           // dt kernel: tile counters zeroed after the dependency wait, or nullptr
};
constexpr int kWorkSlots = 8;  // tile counters of the work-list schedule (one per RK stage)

// A decomposition part's halo exchange inside its fused stage launches (the
// P2P transport).  Tiles [0, n_band_tiles) hold every owned cell other parts
// read (local cells [0, n_band)).  Those tiles, and only those, read halo
// cells: after the dependency wait their thread 0 polls the flag word of
// every sending part until it holds the epoch of the stage's input
// (step * stages + stage), giving up after `limit` polls (err, and the tile
// is skipped).  After the update each such tile stores its cells' and
// ghosts' new states into the reading parts' buffers of this stage's
// output, and the last of them to finish releases step * stages + stage + 1
// into each reader's flag word for this part.
constexpr int kMaxPeers = 16;
struct RemoteIO {
    int n_dst;
    void* dst[kMaxPeers];                     // each reader's buffer of this stage's output
    unsigned long long* flag[kMaxPeers];      // this part's flag word in each reader
    const int32_t* cell_off;                  // [n_band + 1] destinations of owned cell c
    const int2* cell_dst;                     // (reader slot, the cell's index there)
    const int32_t* ghost_off;                 // [n_own_ghost + 1] destinations of owned ghost g - n_real
    const int2* ghost_dst;
    int n_band, n_band_tiles, n_own_ghost;
    unsigned long long* ctr;                  // band tiles completed (monotonic)
    const unsigned long long* my_flags;       // [n_parts] flag words the senders write here
    const int32_t* src;                       // the parts that send to this one
    int n_src;
    int* err;
    long long limit;
};
// A decomposition part's fused stage launch, passed beside TileIO (whose
// layout the single-solver kernel keeps: a larger TileIO made the FP64
// fused kernel 1.1 % slower).
struct PartIO {
    int t0;                    // the launch's first tile
    const RemoteIO* remote;    // the halo exchange inside the launch (device memory), or nullptr
    int stage, stages;         // with remote: this launch's RK stage, and the step's stages
};
__device__ __forceinline__ unsigned long long ld_acquire_sys_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_sys_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long tkey(double x) {
    if (x != x) return ~0ull;
    const long long b = __double_as_longlong(x);
    return b < 0 ? ~(unsigned long long)b : ((unsigned long long)b | 0x8000000000000000ull);
}
__device__ __forceinline__ double tkey_inv(unsigned long long k) {
    if (k == ~0ull) return __longlong_as_double(0x7ff8000000000000ll);
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}
__device__ __forceinline__ bool t_inactive(const Ctrl* c) { return c != nullptr && *(volatile const int*)&c->active == 0; }

// Programmatic dependent launch.  Step kernels let the next kernel of the
// stream start as soon as all of their CTAs run (pdl_trigger), so its CTAs
// stage the constant tile data (geometry, face words) while this kernel's
// last CTAs finish; pdl_wait() then blocks until the previous kernel has
// completed and its writes are visible.  Nothing a previous kernel writes
// is read, and nothing is written to global memory, before pdl_wait().
// Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ unsigned long long kmin_(unsigned long long a, unsigned long long b) { return b < a ? b : a; }

template <class S, int V>
__device__ __forceinline__ void ld(const S* __restrict__ a, int c, S* v) {
    if (V == 4 && sizeof(S) == 8) {
        const double2* p = reinterpret_cast<const double2*>(a + 4 * (size_t)c);
        const double2 x = p[0], y = p[1];
        v[0] = (S)x.x; v[1] = (S)x.y; v[2] = (S)y.x; v[3] = (S)y.y;
    } else if (V == 4) {
        const float4 x = *reinterpret_cast<const float4*>(a + 4 * (size_t)c);
        v[0] = (S)x.x; v[1] = (S)x.y; v[2] = (S)x.z; v[3] = (S)x.w;
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = a[(size_t)V * c + k];
    }
}
template <class S, int V>
__device__ __forceinline__ void st(S* __restrict__ a, int c, const S* v) {
    if (V == 4 && sizeof(S) == 8) {
        double2* p = reinterpret_cast<double2*>(a + 4 * (size_t)c);
        p[0] = make_double2((double)v[0], (double)v[1]);
        p[1] = make_double2((double)v[2], (double)v[3]);
    } else if (V == 4) {
        *reinterpret_cast<float4*>(a + 4 * (size_t)c) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) a[(size_t)V * c + k] = v[k];
    }
}
// V consecutive values at a 16-byte aligned shared-memory address
template <class S, int V>
__device__ __forceinline__ void lds(const S* p, S* v) {
    if (V == 4 && sizeof(S) == 8) {
        const double2 x = reinterpret_cast<const double2*>(p)[0], y = reinterpret_cast<const double2*>(p)[1];
        v[0] = (S)x.x; v[1] = (S)x.y; v[2] = (S)y.x; v[3] = (S)y.y;
    } else if (V == 4) {
        const float4 x = reinterpret_cast<const float4*>(p)[0];
        v[0] = (S)x.x; v[1] = (S)x.y; v[2] = (S)x.z; v[3] = (S)x.w;
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = p[k];
    }
}

// Shared-memory record of one tile-local cell: q[V], then (with gradients)
// gx[V], gy[V], (LIM: exact mode, or a flux that needs the raw gradients)
// lim[V], then the centroid on an even word (one 2-word copy); padded to 16
// bytes.
template <class M, int V, bool ORDER2, bool CENTROID, bool LIM = M::exact>
struct Rec {
    using S = typename M::S;
    static constexpr int NG = ORDER2 ? (LIM ? 3 : 2) : 0;
    static constexpr int OGX = V, OGY = 2 * V, OLM = 3 * V;
    static constexpr int OC = (V * (1 + NG) + 1) / 2 * 2;
    static constexpr int RAW = OC + (CENTROID ? 2 : 0);
    static constexpr int AL = 16 / (int)sizeof(S);
    // an odd number of 16-byte units, so that 128-bit reads of records of
    // random cells spread over all eight shared-memory bank groups
    static constexpr int U = (RAW + AL - 1) / AL;
    static constexpr int NR = ((U % 2) ? U : U + 1) * AL;
};

// Optional positivity guard (not in the reference): a reconstructed Euler
// face state with rho <= 0 or p <= 0 is replaced by the cell value.  The
// exact mode evaluates p as the oracle does; the fast modes test the same
// sign without a division: for rho > 0 and gamma > 1,
// p > 0  <=>  2 rho E - (m_x^2 + m_y^2) > 0.
template <class S, int V, bool EXACT = true>
__device__ __forceinline__ void guard_face(const Params& P, S* qf, const S* qc) {
    if (V != 4 || !P.positivity_guard) return;
    bool bad;
    if constexpr (EXACT) {
        const S p = ((S)P.gamma - S(1)) * (qf[3] - S(0.5) / qf[0] * (qf[1] * qf[1] + qf[2] * qf[2]));
        bad = !(qf[0] > S(0)) || !(p > S(0));
    } else {
        const S m2 = qf[1] * qf[1] + qf[2] * qf[2];
        bad = !(qf[0] > S(0)) || !(S(2) * qf[0] * qf[3] - m2 > S(0));
    }
    if (bad) {
#pragma unroll
        for (int k = 0; k < V; ++k) qf[k] = qc[k];
    }
}

// Asynchronous global -> shared copies (no register round trip); a thread
// issues all of its copies and waits once, so a whole tile is in flight.
__device__ __forceinline__ void cpa16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Groups: the constant tile data staged before the dependency wait is one
// group; cpa_wait_prior() waits for it while the newest group stays in flight.
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
template <int BYTES>
__device__ __forceinline__ void cpa(void* dst, const void* src) {
    if (BYTES == 32) { cpa16(dst, src); cpa16((char*)dst + 16, (const char*)src + 16); }
    else if (BYTES == 16) cpa16(dst, src);
    else if (BYTES == 8) cpa8(dst, src);
    else cpa4(dst, src);
}

// Loads the record of device cell g into shared-memory record r (asynchronously).
template <class M, int V, bool ORDER2, bool CENTROID, bool LIM = M::exact>
__device__ __forceinline__ void stage_record(const TileParams& TP, const TileIO& io, int g, typename M::S* r) {
    using S = typename M::S;
    using R = Rec<M, V, ORDER2, CENTROID, LIM>;
    constexpr int QB = V * (int)sizeof(S);
    cpa<QB>(r, (const S*)io.q_stage + (size_t)V * g);
    if (ORDER2) {
        cpa<QB>(r + R::OGX, (const S*)io.gx + (size_t)V * g);
        cpa<QB>(r + R::OGY, (const S*)io.gy + (size_t)V * g);
        if (LIM) cpa<QB>(r + R::OLM, (const S*)io.lim + (size_t)V * g);
    }
    if (CENTROID) cpa<2 * (int)sizeof(S)>(r + R::OC, (const S*)TP.ccxy + 2 * (size_t)g);
}

// Loads the records of the tile's owned cells and halo (asynchronously), in
// two groups.  The halo cell indices were staged into shalo by stage_halo
// before the dependency wait: the owned records are issued first, then the
// staged indices are awaited (a block barrier) and the halo records issued,
// so no global index load sits on the chain in front of the record copies.
template <class M, int V, bool ORDER2, bool CENTROID, bool LIM = M::exact>
__device__ __forceinline__ void stage_records(const TileParams& TP, const TileIO& io, const int4& inf, int c0,
                                              int nown, typename M::S* rec, const int* shalo) {
    using R = Rec<M, V, ORDER2, CENTROID, LIM>;
    for (int l = threadIdx.x; l < nown; l += blockDim.x)
        stage_record<M, V, ORDER2, CENTROID, LIM>(TP, io, c0 + l, rec + (size_t)l * R::NR);
    cpa_commit();
    cpa_wait_prior();  // the constant group: edges and halo indices
    __syncthreads();
    for (int h = threadIdx.x; h < inf.w; h += blockDim.x)
        stage_record<M, V, ORDER2, CENTROID, LIM>(TP, io, shalo[h], rec + (size_t)(TP.T + h) * R::NR);
}

// Stages the tile's halo cell indices (constant mesh data) into shared memory
// and closes the constant group of copies issued before the dependency wait.
__device__ __forceinline__ void stage_halo(const TileParams& TP, const int4& inf, int* shalo) {
    for (int h = threadIdx.x; h < inf.w; h += blockDim.x) cpa4(shalo + h, TP.halo + inf.z + h);
    cpa_commit();
}

// Loads the tile's edge geometry (contiguous per tile) into shared memory.
template <class S, bool GG, bool XF>
__device__ __forceinline__ void stage_edges(const TileParams& TP, const int4& inf, uint32_t* sij, S* snx, S* sny,
                                            S* sle, S* sg, S* sxf, S* syf) {
    for (int e = threadIdx.x; e < inf.y; e += blockDim.x) {
        const int ge = inf.x + e;
        cpa4(sij + e, TP.edge_ij + ge);
        cpa<(int)sizeof(S)>(snx + e, (const S*)TP.enx + ge);
        cpa<(int)sizeof(S)>(sny + e, (const S*)TP.eny + ge);
        cpa<(int)sizeof(S)>(sle + e, (const S*)TP.ele + ge);
        if (GG) cpa<(int)sizeof(S)>(sg + e, (const S*)TP.eg + ge);
        if (XF) {
            cpa<(int)sizeof(S)>(sxf + e, (const S*)TP.exf + ge);
            cpa<(int)sizeof(S)>(syf + e, (const S*)TP.eyf + ge);
        }
    }
}

__device__ __forceinline__ void load_faces(const TileParams& TP, int c, uint16_t* w) {
    const int N = TP.P.n_real;
#pragma unroll
    for (int f = 0; f < kMaxFaces; ++f) w[f] = TP.face[f * N + c];
}

// ------------------------------------------------------------------ K0: dt --
// Viscous time steps of owned cell c and of its boundary ghosts (C = 2):
// VISC_MIN (dt_kind 3, examples/flatPlate/main.cpp:230-277) and VISC_SUM
// (dt_kind 4, examples/nacaTransient/main.cpp:234-285); the sum kind reads
// the neighbour's area.  Faces are visited in reference edge order.
template <class M, int NR>
__device__ __forceinline__ unsigned long long tile_cell_dt_visc(const TileParams& TP, const TileIO& io,
                                                                const int4& inf, int l, int c, const uint16_t* w,
                                                                const typename M::S* rec, const uint32_t* sij,
                                                                const typename M::S* snx,
                                                                const typename M::S* sny,
                                                                const typename M::S* sle) {
    using S = typename M::S;
    const Params& P = TP.P;
    const int T = TP.T;
    const S* AR = (const S*)TP.area;
    const bool sum = P.dt_kind == 4;
    unsigned long long kmin = ~0ull;
    S qs[4];
    lds<S, 4>(rec + (size_t)l * NR, qs);
    if constexpr (M::exact) {
        const double gamma = P.gamma, gm1 = gamma - 1, cfl = P.cfl, C = 2;
        const double cs = sqrt((gm1 * (qs[3] - 0.5 / qs[0] * (qs[1] * qs[1] + qs[2] * qs[2]))) * gamma / qs[0]);
        const double Ai = AR[c];
        double acc = sum ? 0. : 1.0;
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (w[f] == kFaceNone) continue;
            const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
            const uint32_t ij = sij[el];
            const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
            const double n0 = snx[el], n1 = sny[el], le = sle[el];
            const bool ghost = (w[f] & 0x4000) != 0;
            double qn[4];
            lds<double, 4>(rec + (size_t)o * NR, qn);
            const double cn = sqrt((gm1 * (qn[3] - 0.5 / qn[0] * (qn[1] * qn[1] + qn[2] * qn[2]))) * gamma / qn[0]);
            const double evs = exact::visc_eig(P, qs[0], le, Ai);
            if (sum) {
                const int gn = o < T ? c - l + o : TP.halo[inf.z + o - T];
                const double An = AR[gn];
                const double ts = cs + fabs(qs[1] / qs[0] * n0 + qs[2] / qs[0] * n1) + C * evs;
                const double tn = cn + fabs(qn[1] / qn[0] * n0 + qn[2] / qn[0] * n1) + C * exact::visc_eig(P, qn[0], le, An);
                const double center = side ? exact::dmax(tn, ts) : exact::dmax(ts, tn);
                acc += center * le;
                if (ghost) {
                    double d = 0.;
                    d += center * le;
                    const double dg = cfl * An / d;
                    io.dt[gn] = dg;
                    kmin = kmin_(kmin, tkey(dg));
                }
            } else {
                const double es = (cs + fabs(n0 * qs[1] / qs[0]) + fabs(n1 * qs[2] / qs[0])) * le;
                acc = exact::dmin(acc, cfl * Ai / (es + C * evs));
                if (ghost) {
                    const int gn = TP.halo[inf.z + o - T];
                    const double An = AR[gn];
                    const double en = (cn + fabs(n0 * qn[1] / qn[0]) + fabs(n1 * qn[2] / qn[0])) * le;
                    const double dg = exact::dmin(1.0, cfl * An / (en + C * exact::visc_eig(P, qn[0], le, An)));
                    io.dt[gn] = dg;
                    kmin = kmin_(kmin, tkey(dg));
                }
            }
        }
        const double di = sum ? cfl * Ai / acc : acc;
        io.dt[c] = di;
        kmin = kmin_(kmin, tkey(di));
    } else {
        const S gamma = (S)P.gamma, gm1 = gamma - S(1), cfl = (S)P.cfl;
        const S mp2 = S(2) * (S)(P.mu / P.pr);  // C * mu / pr
        const S ri = fast::rcp(qs[0]);
        const S us = qs[1] * ri, vs = qs[2] * ri;
        const S cs = fast::sqrt_(gamma * gm1 * (qs[3] * ri - S(0.5) * (us * us + vs * vs)));
        const S vs_rho = fast::tmax(S(4.0 / 3.0) * ri, gamma * ri);     // max(4/(3 rho), gamma/rho)
        const S Ai = AR[c], rAi = fast::rcp(Ai);
        S acc = sum ? S(0) : S(1);
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (w[f] == kFaceNone) continue;
            const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
            const uint32_t ij = sij[el];
            const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
            const S n0 = snx[el], n1 = sny[el], le = sle[el];
            const bool ghost = (w[f] & 0x4000) != 0;
            S qn[4];
            lds<S, 4>(rec + (size_t)o * NR, qn);
            const S rn = fast::rcp(qn[0]);
            const S un = qn[1] * rn, vn = qn[2] * rn;
            const S cn = fast::sqrt_(gamma * gm1 * (qn[3] * rn - S(0.5) * (un * un + vn * vn)));
            const S vn_rho = fast::tmax(S(4.0 / 3.0) * rn, gamma * rn);
            const S le2 = le * le;
            if (sum) {
                const int gn = o < T ? c - l + o : TP.halo[inf.z + o - T];
                const S An = AR[gn];
                const S ts = cs + fabs(us * n0 + vs * n1) + mp2 * vs_rho * le2 * rAi;
                const S tn = cn + fabs(un * n0 + vn * n1) + mp2 * vn_rho * le2 * fast::rcp(An);
                const S center = fast::tmax(ts, tn);
                acc += center * le;
                if (ghost) {
                    const double dg = (double)(cfl * An * fast::rcp(center * le));
                    io.dt[gn] = dg;
                    kmin = kmin_(kmin, tkey(dg));
                }
            } else {
                const S es = (cs + fabs(n0 * us) + fabs(n1 * vs)) * le + mp2 * vs_rho * le2 * rAi;
                acc = fast::tmin(acc, cfl * Ai * fast::rcp(es));
                if (ghost) {
                    const int gn = TP.halo[inf.z + o - T];
                    const S An = AR[gn];
                    const S en = (cn + fabs(n0 * un) + fabs(n1 * vn)) * le + mp2 * vn_rho * le2 * fast::rcp(An);
                    const double dg = (double)fast::tmin(S(1), cfl * An * fast::rcp(en));
                    io.dt[gn] = dg;
                    kmin = kmin_(kmin, tkey(dg));
                }
            }
        }
        const double di = (double)(sum ? cfl * Ai * fast::rcp(acc) : acc);
        io.dt[c] = di;
        kmin = kmin_(kmin, tkey(di));
    }
    return kmin;
}

// CFL time step of owned cell c (tile-local l) and of its boundary ghosts,
// from staged records (stride NR) and edges (calc_dt of
// examples/forwardStep/main.cpp:140-185 and examples/naca/main.cpp:142-183);
// returns the ordered-key minimum of the values written.
// VISC: the viscous kinds (dt_kind 3, 4) only, a separate instantiation so
// that the CFL kinds keep their register budget.
template <class M, int V, int NR, bool VISC = false>
__device__ __forceinline__ unsigned long long tile_cell_dt(const TileParams& TP, const TileIO& io, const int4& inf,
                                                           int l, int c, const uint16_t* w,
                                                           const typename M::S* rec, const uint32_t* sij,
                                                           const typename M::S* snx, const typename M::S* sny,
                                                           const typename M::S* sle) {
    using S = typename M::S;
    const Params& P = TP.P;
    const int T = TP.T;
    unsigned long long kmin = ~0ull;
    const S* AR = (const S*)TP.area;
    if (P.dt_kind == 0) {
        io.dt[c] = P.dt_const;
        kmin = tkey(P.dt_const);
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (w[f] == kFaceNone || !(w[f] & 0x4000)) continue;
            const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
            const uint32_t ij = sij[el];
            const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
            io.dt[TP.halo[inf.z + o - T]] = P.dt_const;
        }
    } else if (VISC) {
        if (V == 4) kmin = tile_cell_dt_visc<M, NR>(TP, io, inf, l, c, w, rec, sij, snx, sny, sle);
    } else if (V == 4) {
        S qs[4];
        lds<S, 4>(rec + (size_t)l * NR, qs);
        const bool sum = P.dt_kind == 1;
        if constexpr (M::exact) {
            const double gamma = P.gamma, gm1 = gamma - 1, cfl = P.cfl;
            const double cs = sqrt((gm1 * (qs[3] - 0.5 / qs[0] * (qs[1] * qs[1] + qs[2] * qs[2]))) * gamma / qs[0]);
            const double Ai = AR[c];
            double acc = sum ? 0. : 1.0;
#pragma unroll
            for (int f = 0; f < kMaxFaces; ++f) {
                if (w[f] == kFaceNone) continue;
                const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
                const uint32_t ij = sij[el];
                const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
                const double n0 = snx[el], n1 = sny[el], le = sle[el];
                double qn[4];
                lds<double, 4>(rec + (size_t)o * NR, qn);
                const double cn = sqrt((gm1 * (qn[3] - 0.5 / qn[0] * (qn[1] * qn[1] + qn[2] * qn[2]))) * gamma / qn[0]);
                const bool ghost = (w[f] & 0x4000) != 0;
                if (sum) {
                    const double es = cs + fabs(qs[1] / qs[0] * n0 + qs[2] / qs[0] * n1);
                    const double en = cn + fabs(qn[1] / qn[0] * n0 + qn[2] / qn[0] * n1);
                    const double center = side ? exact::dmax(en, es) : exact::dmax(es, en);
                    acc += center * le;
                    if (ghost) {
                        const int g = TP.halo[inf.z + o - T];
                        double d = 0.;
                        d += center * le;
                        const double dg = cfl * AR[g] / d;
                        io.dt[g] = dg;
                        kmin = kmin_(kmin, tkey(dg));
                    }
                } else {
                    const double es = (cs + fabs(qs[1] / qs[0])) * n0 + (cs + fabs(qs[2] / qs[0])) * n1;
                    acc = exact::dmin(acc, cfl * (Ai / le) / fabs(es));
                    if (ghost) {
                        const int g = TP.halo[inf.z + o - T];
                        const double en = (cn + fabs(qn[1] / qn[0])) * n0 + (cn + fabs(qn[2] / qn[0])) * n1;
                        const double dg = exact::dmin(1.0, cfl * (AR[g] / le) / fabs(en));
                        io.dt[g] = dg;
                        kmin = kmin_(kmin, tkey(dg));
                    }
                }
            }
            const double di = sum ? cfl * Ai / acc : acc;
            io.dt[c] = di;
            kmin = kmin_(kmin, tkey(di));
        } else {
            const S gamma = (S)P.gamma, gm1 = gamma - S(1), cfl = (S)P.cfl;
            const S ri = fast::rcp(qs[0]);
            const S us = qs[1] * ri, vs = qs[2] * ri;
            const S cs = fast::sqrt_(gamma * gm1 * (qs[3] * ri - S(0.5) * (us * us + vs * vs)));
            const S Ai = AR[c];
            S acc = sum ? S(0) : S(1);
#pragma unroll
            for (int f = 0; f < kMaxFaces; ++f) {
                if (w[f] == kFaceNone) continue;
                const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
                const uint32_t ij = sij[el];
                const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
                const S n0 = snx[el], n1 = sny[el], le = sle[el];
                S qn[4];
                lds<S, 4>(rec + (size_t)o * NR, qn);
                const S rn = fast::rcp(qn[0]);
                const S un = qn[1] * rn, vn = qn[2] * rn;
                const S cn = fast::sqrt_(gamma * gm1 * (qn[3] * rn - S(0.5) * (un * un + vn * vn)));
                const bool ghost = (w[f] & 0x4000) != 0;
                if (sum) {
                    const S center = fast::tmax(cs + fabs(us * n0 + vs * n1), cn + fabs(un * n0 + vn * n1));
                    acc += center * le;
                    if (ghost) {
                        const int g = TP.halo[inf.z + o - T];
                        const double dg = (double)(cfl * AR[g] * fast::rcp(center * le));
                        io.dt[g] = dg;
                        kmin = kmin_(kmin, tkey(dg));
                    }
                } else {
                    const S es = (cs + fabs(us)) * n0 + (cs + fabs(vs)) * n1;
                    acc = fast::tmin(acc, cfl * Ai * fast::rcp(le * fabs(es)));
                    if (ghost) {
                        const int g = TP.halo[inf.z + o - T];
                        const S en = (cn + fabs(un)) * n0 + (cn + fabs(vn)) * n1;
                        const double dg = (double)fast::tmin(S(1), cfl * (S)AR[g] * fast::rcp(le * fabs(en)));
                        io.dt[g] = dg;
                        kmin = kmin_(kmin, tkey(dg));
                    }
                }
            }
            const double di = (double)(sum ? cfl * Ai * fast::rcp(acc) : acc);
            io.dt[c] = di;
            kmin = kmin_(kmin, tkey(di));
        }
    }
    return kmin;
}

// min_dt's global minimum (explicit.cpp:555-564): a block minimum, then one
// atomic per block spread over kDtSlots slots of the tile's case.  Every
// thread of the block calls it.
__device__ __forceinline__ void tile_dt_reduce(const TileParams& TP, const TileIO& io, int t, int l, int nown,
                                               unsigned long long kmin) {
    __shared__ unsigned long long wmin[kTileMax / 32];
    const Params& P = TP.P;
    const int T = TP.T;
    if (P.global_dt && io.dtkeys != nullptr) {
        const int tc = P.n_cases > 1 ? P.tile_case[t] : 0;
        if (tc >= 0) {
            // block minimum, then one atomic per block spread over kDtSlots slots
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) kmin = kmin_(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
            if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = kmin;
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned long long b = ~0ull;
                for (int i = 0; i < (int)(blockDim.x >> 5); ++i) b = kmin_(b, wmin[i]);
                if (b != ~0ull) atomicMin(io.dtkeys + (size_t)tc * kDtSlots + (blockIdx.x % kDtSlots), b);
            }
        } else if (l < nown && kmin != ~0ull) {
            // a tile across two cases of a batch: each cell (and its ghosts) to its own case
            atomicMin(io.dtkeys + (size_t)P.cell_case[t * T + l] * kDtSlots + (l % kDtSlots), kmin);
        }
    }
}

template <class M, int V, bool VISC = false>
__global__ void __launch_bounds__(kTileMax) k_tile_dt(TileParams TP, TileIO io) {
    using S = typename M::S;
    using R = Rec<M, V, false, false>;
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Params& P = TP.P;
    const int T = TP.T, t = blockIdx.x;
    const int4 inf = TP.info[t];
    const int c0 = t * T, nown = min(T, P.n_own - c0);
    const int LT = T + TP.max_halo;
    S* rec = reinterpret_cast<S*>(smem_raw);
    S* snx = rec + (size_t)LT * R::NR;
    S* sny = snx + TP.max_edges;
    S* sle = sny + TP.max_edges;
    uint32_t* sij = reinterpret_cast<uint32_t*>(sle + TP.max_edges);
    int* shalo = reinterpret_cast<int*>(sij + TP.max_edges);
    const int l = threadIdx.x;
    uint16_t w[kMaxFaces];
    // constant tile data first (may overlap the previous kernel's tail)
    if (l < nown) load_faces(TP, c0 + l, w);
    stage_edges<S, false, false>(TP, inf, sij, snx, sny, sle, nullptr, nullptr, nullptr);
    stage_halo(TP, inf, shalo);
    pdl_wait();
    // the step's first kernel: the work-list tile counters of its stage
    // kernels start at zero (every kernel that used them has completed)
    if (io.work_reset != nullptr && blockIdx.x == 0 && threadIdx.x < kWorkSlots) io.work_reset[threadIdx.x] = 0;
    // the step-control flag is read while the records load; an inactive
    // step's kernels write nothing
    const bool inactive = t_inactive(io.ctrl);
    stage_records<M, V, false, false>(TP, io, inf, c0, nown, rec, shalo);
    cpa_wait();
    if (inactive) return;
    __syncthreads();
    unsigned long long kmin = ~0ull;
    if (l < nown) kmin = tile_cell_dt<M, V, R::NR, VISC>(TP, io, inf, l, c0 + l, w, rec, sij, snx, sny, sle);
    if (P.global_dt && io.dtkeys != nullptr) tile_dt_reduce(TP, io, t, l, nown, kmin);
}

// ------------------------------------------------ K1: gradients + limiters --
// DT: the first stage of a step also computes the step's time step here, from
// the same staged state and edges (k_tile_dt's work without a second pass):
// 0 none, 1 the CFL / constant kinds, 2 the viscous kinds.
template <class M, int V, int DT>
__global__ void __launch_bounds__(kTileMax) k_tile_gradlim(TileParams TP, TileIO io) {
    using S = typename M::S;
    using R = Rec<M, V, false, true>;
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Params& P = TP.P;
    const int T = TP.T, t = blockIdx.x;
    const int4 inf = TP.info[t];
    const int c0 = t * T, nown = min(T, P.n_own - c0);
    const int LT = T + TP.max_halo, EM = TP.max_edges;
    S* rec = reinterpret_cast<S*>(smem_raw);
    S* snx = rec + (size_t)LT * R::NR;
    S* sny = snx + EM; S* sle = sny + EM; S* sg = sle + EM; S* sxf = sg + EM; S* syf = sxf + EM;
    uint32_t* sij = reinterpret_cast<uint32_t*>(syf + EM);
    int* shalo = reinterpret_cast<int*>(sij + EM);
    const int l = threadIdx.x;
    const int c = c0 + l;
    uint16_t w[kMaxFaces];
    S A = S(1);
    if (l < nown) {  // constant tile data first (may overlap the previous kernel's tail)
        load_faces(TP, c, w);
        A = ((const S*)TP.area)[c];
    }
    stage_edges<S, true, true>(TP, inf, sij, snx, sny, sle, sg, sxf, syf);
    stage_halo(TP, inf, shalo);
    pdl_wait();
    const bool inactive = t_inactive(io.ctrl);
    stage_records<M, V, false, true>(TP, io, inf, c0, nown, rec, shalo);
    cpa_wait();
    if (inactive) return;
    __syncthreads();
    if constexpr (DT != 0) {
        unsigned long long kmin = ~0ull;
        if (l < nown) kmin = tile_cell_dt<M, V, R::NR, DT == 2>(TP, io, inf, l, c, w, rec, sij, snx, sny, sle);
        if (P.global_dt && io.dtkeys != nullptr) tile_dt_reduce(TP, io, t, l, nown, kmin);
    }
    if (l >= nown) return;
    const S* rs = rec + (size_t)l * R::NR;
    S qs[V], gx[V], gy[V], qmn[V], qmx[V], lim[V];
    lds<S, V>(rs, qs);
#pragma unroll
    for (int k = 0; k < V; ++k) { gx[k] = 0; gy[k] = 0; qmn[k] = qs[k]; qmx[k] = qs[k]; lim[k] = 1; }
#pragma unroll
    for (int f = 0; f < kMaxFaces; ++f) {
        if (w[f] == kFaceNone) continue;
        const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
        const uint32_t ij = sij[el];
        const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
        const S nx = snx[el], ny = sny[el], le = sle[el], g = sg[el];
        S qn[V];
        lds<S, V>(rec + (size_t)o * R::NR, qn);
#pragma unroll
        for (int k = 0; k < V; ++k) {
            if constexpr (M::exact) {
                if (!side) {
                    const double fl = (qs[k] * (1.0 - g) + qn[k] * g) * le;
                    gx[k] += fl * nx; gy[k] += fl * ny;
                } else {
                    const double fl = (qn[k] * (1.0 - g) + qs[k] * g) * le;
                    gx[k] -= fl * nx; gy[k] -= fl * ny;
                }
                qmn[k] = exact::dmin(qmn[k], qn[k]); qmx[k] = exact::dmax(qmx[k], qn[k]);
            } else {
                const S qi = side ? qn[k] : qs[k], qj = side ? qs[k] : qn[k];
                const S fl = (qi + (qj - qi) * g) * (side ? -le : le);
                gx[k] += fl * nx; gy[k] += fl * ny;
                qmn[k] = fast::tmin(qmn[k], qn[k]); qmx[k] = fast::tmax(qmx[k], qn[k]);
            }
        }
    }
    const S xc = rs[R::OC], yc = rs[R::OC + 1];
    // gradients without limiters (diffusive fluxes, first order): lim = 1
    const bool limit = P.order2 != 0;
    if constexpr (M::exact) {
        const double invA = 1. / A;
#pragma unroll
        for (int k = 0; k < V; ++k) { gx[k] *= invA; gy[k] *= invA; }
        const double sqrt_area = sqrt(A);
        const double tol = 1e-15;
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (!limit || w[f] == kFaceNone) continue;
            const int el = w[f] & kFaceEdgeMask;
            const double dx = sxf[el] - xc, dy = syf[el] - yc;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const double dqg = gx[k] * dx + gy[k] * dy;
                const double delta_max = qmx[k] - qs[k];
                const double delta_min = qmn[k] - qs[k];
                const double Ka = P.K * sqrt_area;
                const double K3a = Ka * Ka * Ka;
                const double d2 = (delta_max - delta_min) * (delta_max - delta_min);
                double sig;
                if (d2 <= K3a) sig = 1.;
                else if (d2 <= 2 * K3a) {
                    const double y = (d2 / K3a - 1.0);
                    sig = 2.0 * y * y * y - 3.0 * y * y + 1.0;
                } else sig = 0.;
                double lv = 1.0;
                if (sig < 1.0) {
                    if (dqg > tol) lv = exact::limiter_func(P.limiter, delta_max / dqg);
                    else if (dqg < -tol) lv = exact::limiter_func(P.limiter, delta_min / dqg);
                    else lv = 1.0;
                }
                lv = sig + (1.0 - sig) * lv;
                lim[k] = exact::dmin(lim[k], lv);
            }
        }
        st<S, V>((S*)io.gx, c, gx);
        st<S, V>((S*)io.gy, c, gy);
        st<S, V>((S*)io.lim, c, lim);
    } else {
        const S invA = fast::rcp(A);
#pragma unroll
        for (int k = 0; k < V; ++k) { gx[k] *= invA; gy[k] *= invA; }
        const S Ka = (S)P.K * fast::sqrt_(A);
        const S K3a = Ka * Ka * Ka, rK3a = fast::rcp(K3a);
        const S tol = S(1e-15);
        // the smooth switch sigma depends on the cell and variable only
        S sig[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const S d = qmx[k] - qmn[k];
            const S d2 = d * d;
            if (d2 <= K3a) sig[k] = 1;
            else if (d2 <= 2 * K3a) {
                const S y = d2 * rK3a - S(1);
                sig[k] = (S(2) * y - S(3)) * y * y + S(1);
            } else sig[k] = 0;
        }
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (!limit || w[f] == kFaceNone) continue;
            const int el = w[f] & kFaceEdgeMask;
            const S dx = sxf[el] - xc, dy = syf[el] - yc;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                if (sig[k] < S(1)) {
                    const S dqg = gx[k] * dx + gy[k] * dy;
                    S phi = 1;
                    if (dqg > tol) phi = fast::limiter_ratio(P.limiter, qmx[k] - qs[k], dqg);
                    else if (dqg < -tol) phi = fast::limiter_ratio(P.limiter, qmn[k] - qs[k], dqg);
                    lim[k] = fast::tmin(lim[k], sig[k] + (S(1) - sig[k]) * phi);
                }
            }
        }
        if (P.diffusive) {
            // the face gradient of a diffusive flux needs the raw gradients:
            // the limiter is stored apart, as in the exact mode
            st<S, V>((S*)io.lim, c, lim);
        } else {
            // limited gradients
#pragma unroll
            for (int k = 0; k < V; ++k) { gx[k] *= lim[k]; gy[k] *= lim[k]; }
        }
        st<S, V>((S*)io.gx, c, gx);
        st<S, V>((S*)io.gy, c, gy);
    }
}

// Flux of one tile edge for the diffusive kinds with raw gradients and
// limiters staged apart in every mode: FLUX 5 (Navier-Stokes, V = 4) and
// FLUX 6 (Burgers + diffusion, V = 2).  MUSCL face states when P.order2, the
// corrected face gradient from the cell states, then the convective flux
// (roe<false> / burgers) with the viscous or diffusive terms.  Fast modes
// return f * le.
template <class M, int V, int FLUX, class R>
__device__ __forceinline__ void diffusive_edge_flux(const Params& P, const typename M::S* ri, const typename M::S* rj,
                                                    typename M::S n0, typename M::S n1, typename M::S xf,
                                                    typename M::S yf, typename M::S le,
                                                    typename std::conditional<M::exact, double, typename M::S>::type* f) {
    using S = typename M::S;
    S qci[V], qcj[V], gxi[V], gyi[V], gxj[V], gyj[V], qL[V], qR[V];
    lds<S, V>(ri, qci); lds<S, V>(rj, qcj);
    lds<S, V>(ri + R::OGX, gxi); lds<S, V>(ri + R::OGY, gyi);
    lds<S, V>(rj + R::OGX, gxj); lds<S, V>(rj + R::OGY, gyj);
    const S cix = ri[R::OC], ciy = ri[R::OC + 1], cjx = rj[R::OC], cjy = rj[R::OC + 1];
    if (P.order2) {
        S li_[V], lj_[V];
        lds<S, V>(ri + R::OLM, li_); lds<S, V>(rj + R::OLM, lj_);
        const S di0 = xf - cix, di1 = yf - ciy, dj0 = xf - cjx, dj1 = yf - cjy;
#pragma unroll
        for (int k = 0; k < V; ++k) {
            qL[k] = qci[k] + (gxi[k] * di0 + gyi[k] * di1) * li_[k];
            qR[k] = qcj[k] + (gxj[k] * dj0 + gyj[k] * dj1) * lj_[k];
        }
        guard_face<S, V, M::exact>(P, qL, qci);
        guard_face<S, V, M::exact>(P, qR, qcj);
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) { qL[k] = qci[k]; qR[k] = qcj[k]; }
    }
    if constexpr (M::exact) {
        double gxf[V], gyf[V];
        exact::face_gradient<V>(gxf, gyf, gxi, gyi, gxj, gyj, qci, qcj, cix, ciy, cjx, cjy);
        if constexpr (FLUX == 5) {
            exact::roe<false>(P.gamma, f, qL, qR, n0, n1);
            exact::ns_viscous(P, f, qL, qR, gxf, gyf, n0, n1);
        } else {
            exact::burgers_diffusion(f, qL, qR, gxf, gyf, n0, n1);
        }
    } else {
        S t0 = cix - cjx, t1 = ciy - cjy;
        const S rl = fast::rcp(fast::sqrt_(t0 * t0 + t1 * t1));
        t0 *= rl;
        t1 *= rl;
        S gxf[V], gyf[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const S bx = S(0.5) * (gxi[k] + gxj[k]), by = S(0.5) * (gyi[k] + gyj[k]);
            const S corr = bx * t0 + by * t1 - (qci[k] - qcj[k]) * rl;
            gxf[k] = bx - corr * t0;
            gyf[k] = by - corr * t1;
        }
        if constexpr (FLUX == 5) {
            fast::roe<S>((S)P.gamma, f, qL, qR, n0, n1);
            fast::ns_viscous<S>(P, f, qL, qR, gxf, gyf, n0, n1);
        } else {
            fast::burgers<S>(f, qL, qR, n0, n1);
#pragma unroll
            for (int k = 0; k < V; ++k) f[k] -= gxf[k] * n0 + gyf[k] * n1;
        }
#pragma unroll
        for (int k = 0; k < V; ++k) f[k] *= le;
    }
}

// ------------------------------------- K2: flux + RK update + ghost fill --
// ORDER2: the records carry gradients and centroids.  They feed the MUSCL
// face states, or (FLUX 4, diffusion) the face gradient of the flux, whose
// face states are the cell values (first order).
// PH (residual smoothing, FLUX 6 only): 0 the whole stage; 1 the time
// derivatives only, written to io.qt; 2 the update from the smoothed io.qt
// (RK update, ghost fill, residual partials) without fluxes.
template <class M, int V, bool ORDER2, int FLUX, int PH>
__device__ __forceinline__ void tile_stage(const TileParams& TP, const TileIO& io) {
    using S = typename M::S;
    using FT = typename std::conditional<M::exact, double, S>::type;  // flux storage
    // FLUX 5 and 6 keep raw gradients and limiters apart in every mode
    constexpr bool LIMREC = M::exact || FLUX == 5 || FLUX == 6;
    using R = Rec<M, V, ORDER2, ORDER2, LIMREC>;
    constexpr bool MUSCL = ORDER2 && FLUX != 4;
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long s_dtkey;
    const Params& P = TP.P;
    const int N = P.n_real, T = TP.T, t = blockIdx.x;
    const int4 inf = TP.info[t];
    const int c0 = t * T, nown = min(T, P.n_own - c0);
    const int LT = T + TP.max_halo, EM = TP.max_edges;
    S* rec = reinterpret_cast<S*>(smem_raw);
    FT* sF = reinterpret_cast<FT*>(rec + (size_t)LT * R::NR);
    // the flux store's size as smem_stage lays it out
    const size_t fbytes = max(max((size_t)EM * V * sizeof(FT), (size_t)TP.max_halo * 4),
                              (size_t)(kTileMax / 32) * V * sizeof(double));
    S* snx = reinterpret_cast<S*>(reinterpret_cast<unsigned char*>(sF) + (fbytes + 15) / 16 * 16);
    S* sny = snx + EM; S* sle = sny + EM; S* sxf = sle + EM; S* syf = sxf + EM;
    uint32_t* sij = reinterpret_cast<uint32_t*>(syf + EM);
    // the halo indices are read only while the records are staged, before the
    // first flux is stored: they share the flux store
    int* shalo = reinterpret_cast<int*>(sF);
    const bool global_dt = io.ctrl != nullptr && P.global_dt;
    // ---- issue this thread's cell loads first: their latency overlaps the staging
    const int l = threadIdx.x;
    const int c = c0 + l;
    uint16_t w[kMaxFaces];
    double qb[V];
    double A = 1.0, dtc = 0.0;
    if (l < nown) {  // constant tile data first (may overlap the previous kernel's tail)
        load_faces(TP, c, w);
        A = (double)((const S*)TP.area)[c];
    }
    if (MUSCL) stage_edges<S, false, true>(TP, inf, sij, snx, sny, sle, nullptr, sxf, syf);
    else stage_edges<S, false, false>(TP, inf, sij, snx, sny, sle, nullptr, nullptr, nullptr);
    stage_halo(TP, inf, shalo);
    // the tile's case (batches); -1: the tile spans two cases
    const int tc = (global_dt && P.n_cases > 1) ? P.tile_case[t] : 0;
    // reference cell 0 of the tile's case, whose dt carries the NaN rule of min_dt
    const int cell0 = (P.n_cases > 1 && tc >= 0) ? P.case_cell0[tc] : P.cell0;
    pdl_wait();
    // every load of data written by earlier kernels is issued here together,
    // ahead of the record copies: the step-control flag, the base state, the
    // local time step or the dt of reference cell 0
    const bool inactive = t_inactive(io.ctrl);
    double d0 = 0.;
    if (global_dt && tc >= 0) d0 = io.dt[cell0];
    if (l < nown) {
        ld<double, V>(io.q_base, c, qb);
        if (!global_dt) dtc = io.dt[c];
    }
    stage_records<M, V, ORDER2, ORDER2, LIMREC>(TP, io, inf, c0, nown, rec, shalo);
    // MUSCL face states: FLUX 5 and 6 run with and without them (P.order2)
    const bool muscl = MUSCL && ((FLUX != 5 && FLUX != 6) || P.order2 != 0);
    if (global_dt && tc >= 0 && threadIdx.x < 32) {
        const unsigned long long* keys = io.dtkeys + (size_t)tc * kDtSlots;
        unsigned long long k = kmin_(keys[threadIdx.x], keys[threadIdx.x + 32]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) k = kmin_(k, __shfl_xor_sync(0xffffffffu, k, o));
        if (threadIdx.x == 0) s_dtkey = k;
    }
    cpa_wait();
    if (inactive) return;
    __syncthreads();
    // ---- one flux per tile edge
    for (int el = threadIdx.x; el < (PH == 2 ? 0 : inf.y); el += blockDim.x) {
        const uint32_t ij = sij[el];
        const int li = (int)(ij & 0xffff), lj = (int)(ij >> 16);
        const S n0 = snx[el], n1 = sny[el];
        const S* ri = rec + (size_t)li * R::NR;
        const S* rj = rec + (size_t)lj * R::NR;
        FT f[V];
        if constexpr (FLUX == 5 || FLUX == 6) {
            diffusive_edge_flux<M, V, FLUX, R>(P, ri, rj, n0, n1, sxf[el], syf[el], sle[el], f);
        } else {
            S qL[V], qR[V];
            lds<S, V>(ri, qL);
            lds<S, V>(rj, qR);
            if (MUSCL) {
                const S xf = sxf[el], yf = syf[el];
                const S di0 = xf - ri[R::OC], di1 = yf - ri[R::OC + 1];
                const S dj0 = xf - rj[R::OC], dj1 = yf - rj[R::OC + 1];
                S gxi[V], gyi[V], gxj[V], gyj[V];
                lds<S, V>(ri + R::OGX, gxi); lds<S, V>(ri + R::OGY, gyi);
                lds<S, V>(rj + R::OGX, gxj); lds<S, V>(rj + R::OGY, gyj);
                S ci[V], cj[V];
#pragma unroll
                for (int k = 0; k < V; ++k) { ci[k] = qL[k]; cj[k] = qR[k]; }
                if constexpr (M::exact) {
                    S li_[V], lj_[V];
                    lds<S, V>(ri + R::OLM, li_); lds<S, V>(rj + R::OLM, lj_);
#pragma unroll
                    for (int k = 0; k < V; ++k) {
                        qL[k] = ci[k] + (gxi[k] * di0 + gyi[k] * di1) * li_[k];
                        qR[k] = cj[k] + (gxj[k] * dj0 + gyj[k] * dj1) * lj_[k];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < V; ++k) {
                        qL[k] = ci[k] + gxi[k] * di0 + gyi[k] * di1;
                        qR[k] = cj[k] + gxj[k] * dj0 + gyj[k] * dj1;
                    }
                }
                guard_face<S, V, M::exact>(P, qL, ci);
                guard_face<S, V, M::exact>(P, qR, cj);
            }
            if constexpr (FLUX == 4) {
                S gxi[V], gyi[V], gxj[V], gyj[V];
                lds<S, V>(ri + R::OGX, gxi); lds<S, V>(ri + R::OGY, gyi);
                lds<S, V>(rj + R::OGX, gxj); lds<S, V>(rj + R::OGY, gyj);
                if constexpr (M::exact) {
                    double gxf[V], gyf[V];
                    exact::face_gradient<V>(gxf, gyf, gxi, gyi, gxj, gyj, qL, qR, ri[R::OC], ri[R::OC + 1], rj[R::OC],
                                            rj[R::OC + 1]);
                    exact::diffusion(f, gxf, gyf, n0, n1);
                } else {
                    fast::diffusion<V, S>(f, gxi, gyi, gxj, gyj, qL, qR, ri[R::OC] - rj[R::OC],
                                          ri[R::OC + 1] - rj[R::OC + 1], n0, n1);
                }
            } else if constexpr (M::exact) {
                exact::flux<FLUX>(P.gamma, f, qL, qR, n0, n1);
            } else {
                fast::flux<FLUX, S>((S)P.gamma, f, qL, qR, n0, n1);
            }
            if constexpr (!M::exact) {
                const S le = sle[el];
#pragma unroll
                for (int k = 0; k < V; ++k) f[k] *= le;
            }
        }
        if (V == 4 && sizeof(FT) == 4) {
            reinterpret_cast<float4*>(sF)[el] = make_float4((float)f[0], (float)f[1], (float)f[2], (float)f[3]);
        } else {
#pragma unroll
            for (int k = 0; k < V; ++k) sF[el * V + k] = f[k];
        }
    }
    __syncthreads();
    // ---- per-cell sums in reference edge order, RK update, ghost fill
    double res[V];
#pragma unroll
    for (int k = 0; k < V; ++k) res[k] = 0.;
    if (l < nown) {
        double qt[V];
#pragma unroll
        for (int k = 0; k < V; ++k) qt[k] = 0.;
        bool has_ghost = false;
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (w[f] == kFaceNone) continue;
            const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
            has_ghost |= (w[f] & 0x4000) != 0;
            if (PH == 2) continue;  // the smoothed time derivatives are read below
            FT fe[V];
            lds<FT, V>(sF + (size_t)el * V, fe);
            if constexpr (M::exact) {
                const double le = sle[el];
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    if (!side) qt[k] -= fe[k] * le / A;
                    else qt[k] += fe[k] * le / A;
                }
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k) qt[k] += side ? (double)fe[k] : -(double)fe[k];
            }
        }
        if constexpr (!M::exact) {
            if (PH != 2) {
                const double rA = 1.0 / A;
#pragma unroll
                for (int k = 0; k < V; ++k) qt[k] *= rA;
            }
        }
        if constexpr (PH == 1) {
            st<double, V>(io.qt, c, qt);
        } else {
        if constexpr (PH == 2) ld<double, V>(io.qt, c, qt);
        if (global_dt) {
            // min_dt (explicit.cpp:555-564) of this cell's case; a NaN in its dt[0] wins
            unsigned long long key = s_dtkey;
            if (tc < 0) {  // a tile across two cases of a batch: this cell's case
                const int k = P.cell_case[c];
                key = ~0ull;
                for (int i = 0; i < kDtSlots; ++i) key = kmin_(key, io.dtkeys[(size_t)k * kDtSlots + i]);
                d0 = io.dt[P.case_cell0[k]];
            }
            dtc = (d0 != d0) ? d0 : tkey_inv(key);
        }
        double qnew[V];
        if constexpr (M::exact) {
#pragma unroll
            for (int k = 0; k < V; ++k) qnew[k] = qb[k] + qt[k] * dtc * io.alpha;
        } else {
            const double da = dtc * io.alpha;
#pragma unroll
            for (int k = 0; k < V; ++k) qnew[k] = fma(qt[k], da, qb[k]);
        }
        if (sizeof(S) == 8) {
            st<double, V>(io.q_out, c, qnew);
        } else {
            S qs[V];
#pragma unroll
            for (int k = 0; k < V; ++k) qs[k] = (S)qnew[k];
            st<S, V>((S*)io.s_out, c, qs);
            if (io.write_f64) st<double, V>(io.q_out, c, qnew);
        }
        if (has_ghost) {
            const S* rs = rec + (size_t)l * R::NR;
#pragma unroll
            for (int f = 0; f < kMaxFaces; ++f) {
                if (w[f] == kFaceNone || !(w[f] & 0x4000)) continue;
                const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
                const uint32_t ij = sij[el];
                const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
                const int g = TP.halo[inf.z + o - T];
                const S n0 = snx[el], n1 = sny[el];
                S qint[V], qc[V], b[V];
#pragma unroll
                for (int k = 0; k < V; ++k) { qc[k] = (S)qnew[k]; qint[k] = qc[k]; }
                if (muscl) {
                    const S d0 = sxf[el] - rs[R::OC], d1 = syf[el] - rs[R::OC + 1];
                    S gxs[V], gys[V];
                    lds<S, V>(rs + R::OGX, gxs); lds<S, V>(rs + R::OGY, gys);
                    if constexpr (LIMREC) {
                        S lms[V];
                        lds<S, V>(rs + R::OLM, lms);
#pragma unroll
                        for (int k = 0; k < V; ++k) qint[k] = qc[k] + (gxs[k] * d0 + gys[k] * d1) * lms[k];
                    } else {
#pragma unroll
                        for (int k = 0; k < V; ++k) qint[k] = qc[k] + gxs[k] * d0 + gys[k] * d1;
                    }
                    guard_face<S, V, M::exact>(P, qint, qc);
                }
                if constexpr (M::exact) exact::bc<V>(P, P.ghost_group[g - N], g - N, b, qint, n0, n1);
                else fast::bc<V, S>(P, P.ghost_group[g - N], g - N, b, qint, n0, n1);
                if (sizeof(S) == 8) {
                    st<double, V>(io.q_out, g, (const double*)b);
                } else {
                    st<S, V>((S*)io.s_out, g, b);
                    if (io.write_f64) {
                        double bd[V];
#pragma unroll
                        for (int k = 0; k < V; ++k) bd[k] = (double)b[k];
                        st<double, V>(io.q_out, g, bd);
                    }
                }
            }
        }
        if (io.partials != nullptr) {
#pragma unroll
            for (int k = 0; k < V; ++k) res[k] = qt[k] * qt[k] * A;
        }
        }  // PH != 1
    }
    if (PH != 1 && io.partials != nullptr) {
#pragma unroll
        for (int k = 0; k < V; ++k)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) res[k] += __shfl_xor_sync(0xffffffffu, res[k], o);
        // the warp sums share the flux store once every thread has read its fluxes
        double* red = reinterpret_cast<double*>(sF);
        __syncthreads();
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int k = 0; k < V; ++k) red[(threadIdx.x >> 5) * V + k] = res[k];
        __syncthreads();
        if (threadIdx.x == 0) {
            const int nw = blockDim.x >> 5;
            for (int k = 0; k < V; ++k) {
                double s = 0.;
                for (int w = 0; w < nw; ++w) s += red[w * V + k];
                io.partials[(size_t)blockIdx.x * V + k] = s;
            }
        }
    }
}

template <class M, int V, bool ORDER2, int FLUX, int PH = 0>
__global__ void __launch_bounds__(kTileMax) k_tile_stage(TileParams TP, TileIO io) {
    tile_stage<M, V, ORDER2, FLUX, PH>(TP, io);
}
// The Roe kinds of the fast modes on tiles of at most 128 cells, with the
// register budget that the shared memory of such tiles allows blocks for:
// FP32 56 registers (9 blocks of 128 threads per SM), FP64 96 (5 blocks).
template <class M>
struct T128Regs { static constexpr int v = sizeof(typename M::S) == 4 ? 56 : 96; };
template <class M, int V, bool ORDER2, int FLUX>
__global__ void __launch_bounds__(128) __maxnreg__(T128Regs<M>::v) k_tile_stage_t128(TileParams TP, TileIO io) {
    tile_stage<M, V, ORDER2, FLUX, 0>(TP, io);
}

// shared memory bytes of each kernel for a tile layout
template <class M, int V>
inline size_t smem_dt(const TileParams& TP) {
    using S = typename M::S;
    return (size_t)(TP.T + TP.max_halo) * Rec<M, V, false, false>::NR * sizeof(S) +
           (size_t)TP.max_edges * (3 * sizeof(S) + 4) + (size_t)TP.max_halo * 4;
}
template <class M, int V>
inline size_t smem_gradlim(const TileParams& TP) {
    using S = typename M::S;
    return (size_t)(TP.T + TP.max_halo) * Rec<M, V, false, true>::NR * sizeof(S) +
           (size_t)TP.max_edges * (6 * sizeof(S) + 4) + (size_t)TP.max_halo * 4;
}
template <class M, int V, bool ORDER2, int FLUX = 0>
inline size_t smem_stage(const TileParams& TP) {
    using S = typename M::S;
    using FT = typename std::conditional<M::exact, double, S>::type;
    // the flux store also holds the halo indices (staging) and the warp sums
    // of the residual partials (after the per-cell sums)
    const size_t flux = std::max({(size_t)TP.max_edges * V * sizeof(FT), (size_t)TP.max_halo * 4,
                                  (size_t)(kTileMax / 32) * V * sizeof(double)});
    return (size_t)(TP.T + TP.max_halo) * Rec<M, V, ORDER2, ORDER2, M::exact || FLUX == 5 || FLUX == 6>::NR * sizeof(S) +
           (flux + 15) / 16 * 16 + (size_t)TP.max_edges * (5 * sizeof(S) + 4);
}

// ------------------------------------------------------------- launchers --
template <class M>
struct TileLaunch {
    static cudaError_t prepare(const TileParams& TP) {
        cudaError_t e = cudaSuccess;
        // solvers created on several host threads at once read and raise the
        // same kernels' limits: one at a time, so a smaller request never
        // overwrites a larger one
        static std::mutex mu;
        std::lock_guard<std::mutex> lock(mu);
        auto set = [&](const void* fn, size_t bytes) {
            // the limit belongs to the kernel, shared by every solver of the
            // process: it is only ever raised, never lowered below what a
            // solver created earlier launches with
            cudaFuncAttributes fa{};
            if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
            if (e == cudaSuccess && (size_t)fa.maxDynamicSharedSizeBytes < bytes)
                e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
        };
        if (TP.P.V == 4) {
            set((const void*)k_tile_dt<M, 4>, smem_dt<M, 4>(TP));
            set((const void*)k_tile_dt<M, 4, true>, smem_dt<M, 4>(TP));
            set((const void*)k_tile_gradlim<M, 4, 0>, smem_gradlim<M, 4>(TP));
            set((const void*)k_tile_gradlim<M, 4, 1>, smem_gradlim<M, 4>(TP));
            set((const void*)k_tile_gradlim<M, 4, 2>, smem_gradlim<M, 4>(TP));
            set((const void*)k_tile_stage<M, 4, true, 1>, smem_stage<M, 4, true>(TP));
            set((const void*)k_tile_stage<M, 4, false, 1>, smem_stage<M, 4, false>(TP));
            set((const void*)k_tile_stage<M, 4, true, 2>, smem_stage<M, 4, true>(TP));
            set((const void*)k_tile_stage<M, 4, false, 2>, smem_stage<M, 4, false>(TP));
            set((const void*)k_tile_stage<M, 4, true, 5>, smem_stage<M, 4, true, 5>(TP));
            if constexpr (kT128) {
                if (use_t128(TP)) {
                    set((const void*)k_tile_stage_t128<M, 4, true, 1>, smem_stage<M, 4, true>(TP));
                    set((const void*)k_tile_stage_t128<M, 4, false, 1>, smem_stage<M, 4, false>(TP));
                    set((const void*)k_tile_stage_t128<M, 4, true, 2>, smem_stage<M, 4, true>(TP));
                    set((const void*)k_tile_stage_t128<M, 4, false, 2>, smem_stage<M, 4, false>(TP));
                }
            }
        } else if (TP.P.V == 2) {
            set((const void*)k_tile_dt<M, 2>, smem_dt<M, 2>(TP));
            set((const void*)k_tile_gradlim<M, 2, 0>, smem_gradlim<M, 2>(TP));
            set((const void*)k_tile_gradlim<M, 2, 1>, smem_gradlim<M, 2>(TP));
            set((const void*)k_tile_stage<M, 2, true, 3>, smem_stage<M, 2, true>(TP));
            set((const void*)k_tile_stage<M, 2, false, 3>, smem_stage<M, 2, false>(TP));
            set((const void*)k_tile_stage<M, 2, true, 6>, smem_stage<M, 2, true, 6>(TP));
            set((const void*)k_tile_stage<M, 2, true, 6, 1>, smem_stage<M, 2, true, 6>(TP));
            set((const void*)k_tile_stage<M, 2, true, 6, 2>, smem_stage<M, 2, true, 6>(TP));
        } else {
            set((const void*)k_tile_dt<M, 1>, smem_dt<M, 1>(TP));
            set((const void*)k_tile_gradlim<M, 1, 0>, smem_gradlim<M, 1>(TP));
            set((const void*)k_tile_gradlim<M, 1, 1>, smem_gradlim<M, 1>(TP));
            set((const void*)k_tile_stage<M, 1, true, 4>, smem_stage<M, 1, true>(TP));
        }
        return e;
    }
    static int grid(const TileParams& TP) { return (TP.P.n_own + TP.T - 1) / TP.T; }
    // the fast modes' Roe flux kernels of tiles up to 128 cells use k_tile_stage_t128
    static constexpr bool kT128 = !M::exact;
    static bool use_t128(const TileParams& TP) { return kT128 && TP.T <= 128; }
    // <<<>>> launch, or with programmatic stream serialisation (pdl)
    template <class... A>
    static void go(void (*k)(A...), int g, int b, size_t smem, cudaStream_t st, bool pdl, const TileParams& TP,
                   const TileIO& io) {
        if (!pdl) {
            k<<<g, b, smem, st>>>(TP, io);
            return;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)g);
        cfg.blockDim = dim3((unsigned)b);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k, TP, io);
    }
    static bool visc(const TileParams& TP) { return TP.P.V == 4 && TP.P.dt_kind >= 3; }
    static void dt(const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl = false) {
        const int g = grid(TP);
        if (TP.P.V == 4) {
            if (visc(TP)) go(k_tile_dt<M, 4, true>, g, TP.T, smem_dt<M, 4>(TP), st, pdl, TP, io);
            else go(k_tile_dt<M, 4>, g, TP.T, smem_dt<M, 4>(TP), st, pdl, TP, io);
        } else if (TP.P.V == 2) {
            go(k_tile_dt<M, 2>, g, TP.T, smem_dt<M, 2>(TP), st, pdl, TP, io);
        } else {
            go(k_tile_dt<M, 1>, g, TP.T, smem_dt<M, 1>(TP), st, pdl, TP, io);
        }
    }
    static void gradlim(const TileParams& TP, const TileIO& io, cudaStream_t st, bool with_dt, bool pdl = false) {
        const int g = grid(TP);
        if (TP.P.V == 4) {
            if (with_dt && visc(TP)) go(k_tile_gradlim<M, 4, 2>, g, TP.T, smem_gradlim<M, 4>(TP), st, pdl, TP, io);
            else if (with_dt) go(k_tile_gradlim<M, 4, 1>, g, TP.T, smem_gradlim<M, 4>(TP), st, pdl, TP, io);
            else go(k_tile_gradlim<M, 4, 0>, g, TP.T, smem_gradlim<M, 4>(TP), st, pdl, TP, io);
        } else if (TP.P.V == 2) {
            if (with_dt) go(k_tile_gradlim<M, 2, 1>, g, TP.T, smem_gradlim<M, 2>(TP), st, pdl, TP, io);
            else go(k_tile_gradlim<M, 2, 0>, g, TP.T, smem_gradlim<M, 2>(TP), st, pdl, TP, io);
        } else {
            if (with_dt) go(k_tile_gradlim<M, 1, 1>, g, TP.T, smem_gradlim<M, 1>(TP), st, pdl, TP, io);
            else go(k_tile_gradlim<M, 1, 0>, g, TP.T, smem_gradlim<M, 1>(TP), st, pdl, TP, io);
        }
    }
    // phase: 0 the whole stage, 1 time derivatives only, 2 update only (residual smoothing, FLUX 6)
    static void stage(const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl = false, int phase = 0) {
        const int g = grid(TP);
        const bool o2 = TP.P.order2 != 0;
        if (TP.P.flux == 6) {
            const size_t sm = smem_stage<M, 2, true, 6>(TP);
            if (phase == 1) go(k_tile_stage<M, 2, true, 6, 1>, g, TP.T, sm, st, pdl, TP, io);
            else if (phase == 2) go(k_tile_stage<M, 2, true, 6, 2>, g, TP.T, sm, st, pdl, TP, io);
            else go(k_tile_stage<M, 2, true, 6>, g, TP.T, sm, st, pdl, TP, io);
        } else if (TP.P.flux == 4) {
            go(k_tile_stage<M, 1, true, 4>, g, TP.T, smem_stage<M, 1, true>(TP), st, pdl, TP, io);
        } else if (TP.P.flux == 5) {
            go(k_tile_stage<M, 4, true, 5>, g, TP.T, smem_stage<M, 4, true, 5>(TP), st, pdl, TP, io);
        } else if (TP.P.flux == 3) {
            if (o2) go(k_tile_stage<M, 2, true, 3>, g, TP.T, smem_stage<M, 2, true>(TP), st, pdl, TP, io);
            else go(k_tile_stage<M, 2, false, 3>, g, TP.T, smem_stage<M, 2, false>(TP), st, pdl, TP, io);
        } else if (TP.P.flux == 1) {
            if constexpr (kT128) {
                if (use_t128(TP)) {
                    if (o2) go(k_tile_stage_t128<M, 4, true, 1>, g, TP.T, smem_stage<M, 4, true>(TP), st, pdl, TP, io);
                    else go(k_tile_stage_t128<M, 4, false, 1>, g, TP.T, smem_stage<M, 4, false>(TP), st, pdl, TP, io);
                    return;
                }
            }
            if (o2) go(k_tile_stage<M, 4, true, 1>, g, TP.T, smem_stage<M, 4, true>(TP), st, pdl, TP, io);
            else go(k_tile_stage<M, 4, false, 1>, g, TP.T, smem_stage<M, 4, false>(TP), st, pdl, TP, io);
        } else {
            if constexpr (kT128) {
                if (use_t128(TP)) {
                    if (o2) go(k_tile_stage_t128<M, 4, true, 2>, g, TP.T, smem_stage<M, 4, true>(TP), st, pdl, TP, io);
                    else go(k_tile_stage_t128<M, 4, false, 2>, g, TP.T, smem_stage<M, 4, false>(TP), st, pdl, TP, io);
                    return;
                }
            }
            if (o2) go(k_tile_stage<M, 4, true, 2>, g, TP.T, smem_stage<M, 4, true>(TP), st, pdl, TP, io);
            else go(k_tile_stage<M, 4, false, 2>, g, TP.T, smem_stage<M, 4, false>(TP), st, pdl, TP, io);
        }
    }
};

// Entry points per precision mode (defined in fv_tile_exact.cu / fv_tile_fast.cu).
namespace tile {
cudaError_t prepare(int precision, const TileParams& TP);
// pdl: launch with programmatic stream serialisation (the step sequence)
void launch_dt(int precision, const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl = false);
// with_dt: also the step's time step (io.dt, io.dtkeys), as launch_dt computes it
void launch_gradlim(int precision, const TileParams& TP, const TileIO& io, cudaStream_t st, bool with_dt = false,
                    bool pdl = false);
void launch_stage(int precision, const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl = false,
                  int phase = 0);
}  // namespace tile

}  // namespace fvgpu
