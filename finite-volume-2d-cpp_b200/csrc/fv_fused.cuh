// Fused stage kernel of the second-order Euler step: Green-Gauss gradients,
// smooth-switch limiter, MUSCL + Roe flux, per-cell sums, RK update, ghost
// fill and residual partials of one tile of T cells in one CTA, one launch
// per RK stage (calc_gradients + calc_limiters + calc_time_derivatives +
// update_cells + update_bounds of explicit.cpp:112-417 for one stage).
//
// A tile stages the states of its cells, of their face neighbours (ring 1)
// and of the ring-1 cells' other neighbours (ring 2), computes the gradients
// and limiters of its cells and of ring 1 into shared memory, and then the
// fluxes of its edges from them.  The limited gradients never leave the
// chip: per stage the kernel reads the stage state, the base state and the
// constant geometry once and writes the new state, with one staging round
// and one kernel boundary instead of two.  Ring-1 gradients are computed by
// every tile that borders the cell (the same arithmetic in each, so the
// results are identical and, in the exact policy, bit-identical to the
// reference's).
//
// Shared-memory records are planes of 16-byte units (one float4, or two
// double2 planes, per 4-vector), so that reads of random slots are free of
// bank conflicts.  The time step of the step comes from k_tile_dt, launched
// before the first stage.
#pragma once
#include "fv_tile.cuh"

namespace fvgpu {

struct FusedParams {
    Params P;
    int T;
    int threads;               // threads per CTA: T, or 2T (at most kTileMax)
    int max_slots, max_grad, max_edges, max_flux;  // max_edges rounded up to a multiple of 4
    const int4* info;          // [n_tiles][2]: {edge_off, n_edges, n_flux, halo_off}, {n1, n2, face_off, 0}
    const int32_t* halo;       // device cell of each ring-1, then ring-2 slot
    const uint32_t* edge_ij;   // local i | local j << 16; each tile's run starts on a multiple of 4
    const void* enx;           // S [local edges]
    const void* eny;
    const void* ele;
    const void* exf;
    const void* eyf;
    const void* eg;
    const uint2* face;         // four face words per gradient slot
    const void* cca;           // S [n_total][4]: centroid x, y, area, 0
};

// 4-vectors in shared-memory planes of 16-byte units: FP32 one float4 plane,
// FP64 two double2 planes `stride` units apart.
template <class S>
struct Planes;
template <>
struct Planes<float> {
    static constexpr int NU = 1;
    __device__ static __forceinline__ void get(const uint4* p, int, int r, float* v) {
        const float4 x = reinterpret_cast<const float4*>(p)[r];
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
    __device__ static __forceinline__ void put(uint4* p, int, int r, const float* v) {
        reinterpret_cast<float4*>(p)[r] = make_float4(v[0], v[1], v[2], v[3]);
    }
    // asynchronous copy of the 4-vector at global g into slot r
    __device__ static __forceinline__ void stage(uint4* p, int, int r, const float* g) { cpa16(p + r, g); }
};
template <>
struct Planes<double> {
    static constexpr int NU = 2;
    __device__ static __forceinline__ void get(const uint4* p, int stride, int r, double* v) {
        const double2 x = reinterpret_cast<const double2*>(p)[r];
        const double2 y = reinterpret_cast<const double2*>(p + stride)[r];
        v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
    }
    __device__ static __forceinline__ void put(uint4* p, int stride, int r, const double* v) {
        reinterpret_cast<double2*>(p)[r] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p + stride)[r] = make_double2(v[2], v[3]);
    }
    __device__ static __forceinline__ void stage(uint4* p, int stride, int r, const double* g) {
        cpa16(p + r, g);
        cpa16(p + stride + r, g + 2);
    }
};

// Shared-memory layout of one fused tile, in bytes from the start.
//  - state planes [max_slots];
//  - centroids [max_grad]: FP32 one float4 plane (x, y, area, 0); FP64 one
//    double2 plane (x, y) and the ring-1 areas [max_grad - T] (an owned
//    cell's area is held by its thread);
//  - gradient planes [max_grad] (and the limiter in the exact policy);
//  - edge indices and normal, length, face centre [max_edges];
//  - the flux store, which before the flux phase holds the Green-Gauss
//    weights [max_edges] (gradient phase) and the halo indices (staging), and
//    after the per-cell sums the residual warp sums.
struct FusedSmem {
    size_t q, c, ar, gx, gy, lm, ij, geo, flux, halo, total;
    int ls, lg, em;  // plane strides (units) and edge-array length
};
template <class M>
__host__ __device__ inline FusedSmem fused_smem(int max_slots, int max_grad, int max_edges, int max_flux, int T) {
    using S = typename M::S;
    using FT = typename std::conditional<M::exact, double, S>::type;
    constexpr int NU = (int)(4 * sizeof(S) / 16);
    FusedSmem L{};
    L.ls = max_slots;
    L.lg = max_grad;
    L.em = max_edges;
    size_t o = 0;
    L.q = o; o += (size_t)16 * NU * max_slots;
    L.c = o; o += (size_t)16 * max_grad;
    L.ar = o; if (sizeof(S) == 8) o += ((size_t)8 * (max_grad - T) + 15) / 16 * 16;
    L.gx = o; o += (size_t)16 * NU * max_grad;
    L.gy = o; o += (size_t)16 * NU * max_grad;
    L.lm = o; if (M::exact) o += (size_t)16 * NU * max_grad;
    L.ij = o; o += (size_t)4 * max_edges;
    L.geo = o; o += (size_t)5 * sizeof(S) * max_edges;
    o = (o + 15) / 16 * 16;
    L.flux = o;
    L.halo = L.flux + ((size_t)sizeof(S) * max_edges + 15) / 16 * 16;
    size_t fb = (size_t)max_flux * 4 * sizeof(FT);
    const size_t before = (L.halo - L.flux) + (size_t)max_slots * 4;
    fb = fb > before ? fb : before;
    fb = fb > (size_t)(kTileMax / 32) * 4 * sizeof(double) ? fb : (size_t)(kTileMax / 32) * 4 * sizeof(double);
    o += (fb + 15) / 16 * 16;
    L.total = o;
    return L;
}

// centroid (x, y) of slot r
template <class S>
__device__ __forceinline__ void cent(const uint4* C, int r, S& x, S& y) {
    if constexpr (sizeof(S) == 4) {
        const float4 v = reinterpret_cast<const float4*>(C)[r];
        x = v.x; y = v.y;
    } else {
        const double2 v = reinterpret_cast<const double2*>(C)[r];
        x = v.x; y = v.y;
    }
}

// One tile t.  Returns false when the step is inactive (nothing written).
// PART: a decomposition part's tile, whose owned cells come from the tile
// info (a part owns fewer real cells than its local mesh holds).
template <class M, int FLUX, bool REMOTE = false, bool PART = false>
__device__ __forceinline__ bool fused_tile(const FusedParams& FP, const TileIO& io, const int t, const PartIO& pio) {
    using S = typename M::S;
    using FT = typename std::conditional<M::exact, double, S>::type;  // flux storage
    using PL = Planes<S>;
    constexpr int V = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long s_dtkey;
    const Params& P = FP.P;
    const int N = P.n_real, T = FP.T;
    const int4 ia = FP.info[2 * t], ib = FP.info[2 * t + 1];
    const int edge_off = ia.x, n_edges = ia.y, n_flux = ia.z, halo_off = ia.w;
    const int n1 = ib.x, n2 = ib.y, face_off = ib.z;
    const int c0 = t * T, nown = PART ? ib.w : min(T, N - c0);
    const FusedSmem L = fused_smem<M>(FP.max_slots, FP.max_grad, FP.max_edges, FP.max_flux, FP.T);
    uint4* Q = reinterpret_cast<uint4*>(smem_raw + L.q);
    uint4* C = reinterpret_cast<uint4*>(smem_raw + L.c);
    S* AR = reinterpret_cast<S*>(smem_raw + L.ar);  // FP64: ring-1 areas
    uint4* GX = reinterpret_cast<uint4*>(smem_raw + L.gx);
    uint4* GY = reinterpret_cast<uint4*>(smem_raw + L.gy);
    uint4* LM = reinterpret_cast<uint4*>(smem_raw + L.lm);
    uint32_t* sij = reinterpret_cast<uint32_t*>(smem_raw + L.ij);
    S* snx = reinterpret_cast<S*>(smem_raw + L.geo);
    S* sny = snx + L.em; S* sle = sny + L.em; S* sxf = sle + L.em; S* syf = sxf + L.em;
    FT* sF = reinterpret_cast<FT*>(smem_raw + L.flux);
    // the Green-Gauss weights (gradient phase) and the halo indices (staging)
    // are dead before the first flux is stored: they share the flux store
    S* sg = reinterpret_cast<S*>(smem_raw + L.flux);
    int* shalo = reinterpret_cast<int*>(smem_raw + L.halo);
    const bool global_dt = io.ctrl != nullptr && P.global_dt;
    const int l = threadIdx.x;
    const int c = c0 + l;
    // ---- constant tile data first (may overlap the previous kernel's tail):
    // edges in 16-byte chunks, halo indices, centroid/area records of the
    // owned cells, face words of this thread's gradient slots
    {
        const int nch = (n_edges + 3) >> 2;  // 4 edges per chunk of the u32 array
        for (int k = l; k < nch; k += blockDim.x) cpa16(sij + 4 * k, FP.edge_ij + edge_off + 4 * k);
        constexpr int EPC = 16 / (int)sizeof(S);  // edges per 16-byte chunk of a geometry array
        const int ncg = (n_edges + EPC - 1) / EPC;
        for (int k = l; k < ncg; k += blockDim.x) {
            const int d = EPC * k, g = edge_off + EPC * k;
            cpa16(snx + d, (const S*)FP.enx + g);
            cpa16(sny + d, (const S*)FP.eny + g);
            cpa16(sle + d, (const S*)FP.ele + g);
            cpa16(sxf + d, (const S*)FP.exf + g);
            cpa16(syf + d, (const S*)FP.eyf + g);
            cpa16(sg + d, (const S*)FP.eg + g);
        }
        for (int h = l; h < n1 + n2; h += blockDim.x) cpa4(shalo + h, FP.halo + halo_off + h);
        for (int r = l; r < nown; r += blockDim.x) cpa16(C + r, (const S*)FP.cca + 4 * (size_t)(c0 + r));
        cpa_commit();
    }
    // the owned cell's area (this thread's gradient slot and update)
    const S A_own = l < nown ? ((const S*)FP.cca)[4 * (size_t)c + 2] : S(1);
    // face words of this thread's gradient slots: slot l (pass 0) and slot
    // l + blockDim.x (pass 1); slots [0, nown) are owned, [T, T + n1) ring 1
    const uint2 kNoWords = make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
    auto slot_words = [&](int r) {
        const bool has = r < T ? r < nown : r - T < n1;
        return has ? FP.face[face_off + r] : kNoWords;
    };
    const uint2 fw0 = slot_words(l);
    const uint2 fw1 = slot_words(l + blockDim.x);
    // the tile's case (batches); -1: the tile spans two cases
    const int tc = (global_dt && P.n_cases > 1) ? P.tile_case[t] : 0;
    // reference cell 0 of the tile's case, whose dt carries the NaN rule of min_dt
    const int cell0 = (P.n_cases > 1 && tc >= 0) ? P.case_cell0[tc] : P.cell0;
    pdl_wait();
    // every load of data written by earlier kernels is issued here together
    const bool inactive = t_inactive(io.ctrl);
    double d0 = 0., dtc = 0.;
    double qb[V];
    if (global_dt && tc >= 0) d0 = io.dt[cell0];
    if (l < nown) {
        ld<double, V>(io.q_base, c, qb);
        if (!global_dt) dtc = io.dt[c];
    }
    for (int r = l; r < nown; r += blockDim.x) PL::stage(Q, L.ls, r, (const S*)io.q_stage + 4 * (size_t)(c0 + r));
    cpa_commit();
    cpa_wait_prior();  // the constant group: edges, halo indices
    if constexpr (REMOTE) {
        // a band tile reads halo cells: wait for the senders' epoch of this
        // stage's input (bounded; a tile that gives up is skipped)
        __shared__ int s_gave_up;
        const RemoteIO& R = *pio.remote;
        if (threadIdx.x == 0) {
            s_gave_up = 0;
            if (!inactive && t < R.n_band_tiles) {
                const unsigned long long need = io.ctrl->step * (unsigned long long)pio.stages + pio.stage;
                for (int i = 0; i < R.n_src && !s_gave_up; ++i) {
                    const unsigned long long* f = R.my_flags + R.src[i];
                    long long polls = 0;
                    while (ld_acquire_sys_u64(f) < need) {
                        if (++polls > R.limit) {
                            atomicExch(R.err, 1);
                            s_gave_up = 1;
                            break;
                        }
                        __nanosleep(256);
                    }
                }
            }
        }
        __syncthreads();
        if (s_gave_up) {
            cpa_wait();  // this tile's copies in flight land before it leaves
            return false;
        }
    }
    __syncthreads();
    for (int h = l; h < n1 + n2; h += blockDim.x) {
        const int g = shalo[h];
        PL::stage(Q, L.ls, T + h, (const S*)io.q_stage + 4 * (size_t)g);
        if (h < n1) {
            cpa16(C + T + h, (const S*)FP.cca + 4 * (size_t)g);
            if constexpr (sizeof(S) == 8) cpa8(AR + h, (const S*)FP.cca + 4 * (size_t)g + 2);
        }
    }
    if (global_dt && tc >= 0 && threadIdx.x < 32) {
        const unsigned long long* keys = io.dtkeys + (size_t)tc * kDtSlots;
        unsigned long long k = kmin_(keys[threadIdx.x], keys[threadIdx.x + 32]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) k = kmin_(k, __shfl_xor_sync(0xffffffffu, k, o));
        if (threadIdx.x == 0) s_dtkey = k;
    }
    cpa_wait();
    if (inactive) return false;
    __syncthreads();

    // ---- gradients and limiters of the owned cells and ring 1
    // (calc_gradients + calc_limiters, explicit.cpp:112-258)
    for (int r = l, pass = 0; r < T + n1; r += blockDim.x, ++pass) {
        if (r < T && r >= nown) continue;
        const uint2 fwv = pass == 0 ? fw0 : (pass == 1 ? fw1 : FP.face[face_off + r]);
        uint16_t w[kMaxFaces];
        w[0] = (uint16_t)(fwv.x & 0xFFFF); w[1] = (uint16_t)(fwv.x >> 16);
        w[2] = (uint16_t)(fwv.y & 0xFFFF); w[3] = (uint16_t)(fwv.y >> 16);
        S qs[V], gx[V], gy[V], qmn[V], qmx[V], lim[V];
        PL::get(Q, L.ls, r, qs);
        S xc, yc, A;
        if constexpr (sizeof(S) == 4) {
            const float4 cv = reinterpret_cast<const float4*>(C)[r];
            xc = cv.x; yc = cv.y; A = cv.z;
        } else {
            cent<S>(C, r, xc, yc);
            A = r < T ? A_own : AR[r - T];
        }
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
            PL::get(Q, L.ls, o, qn);
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
        if constexpr (M::exact) {
            const double invA = 1. / A;
#pragma unroll
            for (int k = 0; k < V; ++k) { gx[k] *= invA; gy[k] *= invA; }
            const double sqrt_area = sqrt(A);
            const double tol = 1e-15;
#pragma unroll
            for (int f = 0; f < kMaxFaces; ++f) {
                if (w[f] == kFaceNone) continue;
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
            PL::put(LM, L.lg, r, lim);
        } else {
            const S invA = fast::rcp(A);
#pragma unroll
            for (int k = 0; k < V; ++k) { gx[k] *= invA; gy[k] *= invA; }
            const S Ka = (S)P.K * fast::sqrt_(A);
            const S K3a = Ka * Ka * Ka, rK3a = fast::rcp(K3a);
            const S tol = S(1e-15);
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
                if (w[f] == kFaceNone) continue;
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
            // limited gradients
#pragma unroll
            for (int k = 0; k < V; ++k) { gx[k] *= lim[k]; gy[k] *= lim[k]; }
        }
        PL::put(GX, L.lg, r, gx);
        PL::put(GY, L.lg, r, gy);
    }
    __syncthreads();

    // ---- one flux per flux edge (calc_time_derivatives, explicit.cpp:261-350)
    for (int el = l; el < n_flux; el += blockDim.x) {
        const uint32_t ij = sij[el];
        const int li = (int)(ij & 0xffff), lj = (int)(ij >> 16);
        const S n0 = snx[el], n1v = sny[el];
        FT f[V];
        S qL[V], qR[V], ci[V], cj[V], gxi[V], gyi[V], gxj[V], gyj[V], pi[2], pj[2];
        PL::get(Q, L.ls, li, ci);
        PL::get(Q, L.ls, lj, cj);
        cent<S>(C, li, pi[0], pi[1]);
        cent<S>(C, lj, pj[0], pj[1]);
        PL::get(GX, L.lg, li, gxi); PL::get(GY, L.lg, li, gyi);
        PL::get(GX, L.lg, lj, gxj); PL::get(GY, L.lg, lj, gyj);
        const S xf = sxf[el], yf = syf[el];
        const S di0 = xf - pi[0], di1 = yf - pi[1];
        const S dj0 = xf - pj[0], dj1 = yf - pj[1];
        if constexpr (M::exact) {
            S li_[V], lj_[V];
            PL::get(LM, L.lg, li, li_); PL::get(LM, L.lg, lj, lj_);
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
        if constexpr (M::exact) {
            exact::flux<FLUX>(P.gamma, f, qL, qR, n0, n1v);
        } else {
            fast::flux<FLUX, S>((S)P.gamma, f, qL, qR, n0, n1v);
            const S le = sle[el];
#pragma unroll
            for (int k = 0; k < V; ++k) f[k] *= le;
        }
        if (sizeof(FT) == 4) {
            reinterpret_cast<float4*>(sF)[el] = make_float4((float)f[0], (float)f[1], (float)f[2], (float)f[3]);
        } else {
            reinterpret_cast<double2*>(sF)[2 * el] = make_double2((double)f[0], (double)f[1]);
            reinterpret_cast<double2*>(sF)[2 * el + 1] = make_double2((double)f[2], (double)f[3]);
        }
    }
    __syncthreads();

    // ---- per-cell sums in reference edge order, RK update, ghost fill
    // (update_cells + update_bounds, explicit.cpp:368-417)
    double res[V];
#pragma unroll
    for (int k = 0; k < V; ++k) res[k] = 0.;
    if (l < nown) {  // fw0 holds the owned cell's faces (slot l < T)
        uint16_t w[kMaxFaces];
        w[0] = (uint16_t)(fw0.x & 0xFFFF); w[1] = (uint16_t)(fw0.x >> 16);
        w[2] = (uint16_t)(fw0.y & 0xFFFF); w[3] = (uint16_t)(fw0.y >> 16);
        S cr[2];
        cent<S>(C, l, cr[0], cr[1]);
        const double A = (double)A_own;
        double qt[V];
#pragma unroll
        for (int k = 0; k < V; ++k) qt[k] = 0.;
        bool has_ghost = false;
#pragma unroll
        for (int f = 0; f < kMaxFaces; ++f) {
            if (w[f] == kFaceNone) continue;
            const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
            has_ghost |= (w[f] & 0x4000) != 0;
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
            const double rA = 1.0 / A;
#pragma unroll
            for (int k = 0; k < V; ++k) qt[k] *= rA;
        }
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
        if constexpr (REMOTE) {
            // this cell's new state into every part that reads it
            const RemoteIO& R = *pio.remote;
            if (c < R.n_band) {
                S qs[V];
#pragma unroll
                for (int k = 0; k < V; ++k) qs[k] = (S)qnew[k];
                for (int i = R.cell_off[c]; i < R.cell_off[c + 1]; ++i) {
                    const int2 d = R.cell_dst[i];
                    st<S, V>((S*)R.dst[d.x], d.y, qs);
                }
            }
        }
        if (has_ghost) {
            S gxs[V], gys[V];
            PL::get(GX, L.lg, l, gxs);
            PL::get(GY, L.lg, l, gys);
#pragma unroll
            for (int f = 0; f < kMaxFaces; ++f) {
                if (w[f] == kFaceNone || !(w[f] & 0x4000)) continue;
                const int el = w[f] & kFaceEdgeMask, side = w[f] >> 15;
                const uint32_t ij = sij[el];
                const int o = side ? (int)(ij & 0xffff) : (int)(ij >> 16);
                const int g = FP.halo[halo_off + o - T];
                const S n0 = snx[el], n1v = sny[el];
                S qint[V], qc[V], b[V];
#pragma unroll
                for (int k = 0; k < V; ++k) { qc[k] = (S)qnew[k]; qint[k] = qc[k]; }
                const S e0 = sxf[el] - cr[0], e1 = syf[el] - cr[1];
                if constexpr (M::exact) {
                    S lms[V];
                    PL::get(LM, L.lg, l, lms);
#pragma unroll
                    for (int k = 0; k < V; ++k) qint[k] = qc[k] + (gxs[k] * e0 + gys[k] * e1) * lms[k];
                } else {
#pragma unroll
                    for (int k = 0; k < V; ++k) qint[k] = qc[k] + gxs[k] * e0 + gys[k] * e1;
                }
                guard_face<S, V, M::exact>(P, qint, qc);
                if constexpr (M::exact) exact::bc<V>(P, P.ghost_group[g - N], g - N, b, qint, n0, n1v);
                else fast::bc<V, S>(P, P.ghost_group[g - N], g - N, b, qint, n0, n1v);
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
                if constexpr (REMOTE) {
                    const RemoteIO& R = *pio.remote;
                    const int go = g - N;
                    if (go < R.n_own_ghost)
                        for (int i = R.ghost_off[go]; i < R.ghost_off[go + 1]; ++i) {
                            const int2 d = R.ghost_dst[i];
                            st<S, V>((S*)R.dst[d.x], d.y, b);
                        }
                }
            }
        }
        if (io.partials != nullptr) {
#pragma unroll
            for (int k = 0; k < V; ++k) res[k] = qt[k] * qt[k] * A;
        }
    }
    if (io.partials != nullptr) {
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
                io.partials[(size_t)t * V + k] = s;
            }
        }
    }
    if constexpr (REMOTE) {
        // every band tile counts itself once its stores are visible; the
        // last one releases this stage's epoch to the readers
        const RemoteIO& R = *pio.remote;
        if (t < R.n_band_tiles) {
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence_system();
                const unsigned long long epoch = io.ctrl->step * (unsigned long long)pio.stages + pio.stage + 1;
                const unsigned long long done = atomicAdd(R.ctr, 1ull) + 1ull;
                if (done == epoch * (unsigned long long)R.n_band_tiles) {
                    __threadfence_system();
                    for (int d = 0; d < R.n_dst; ++d) st_release_sys_u64(R.flag[d], epoch);
                }
            }
        }
    }
    return true;
}

// One CTA per tile, tiles [0, grid).
template <class M, int FLUX>
__global__ void __launch_bounds__(kTileMax) k_tile_fused(FusedParams FP, TileIO io) {
    pdl_trigger();
    fused_tile<M, FLUX, false, false>(FP, io, (int)blockIdx.x, PartIO{});
}

// A decomposition part's launches, one CTA per tile.  MODE 1: tiles
// [pio.t0, pio.t0 + grid) (the band and interior launches); MODE 2: the halo
// exchange inside the launch (pio.remote).  Kept apart from k_tile_fused,
// whose register allocation the tile offset and the owned count from the
// tile info upset (FP32: 80 registers instead of 64, 5.7 % slower); a
// register cap on these launches restores 64 registers but runs slower
// still, so they keep the compiler's choice.
template <class M, int FLUX, int MODE>
__global__ void __launch_bounds__(kTileMax) k_tile_fused_part(FusedParams FP, TileIO io, PartIO pio) {
    pdl_trigger();
    fused_tile<M, FLUX, MODE == 2, true>(FP, io, (MODE == 1 ? pio.t0 : 0) + (int)blockIdx.x, pio);
}

// Work-list schedule: as many CTAs as fit on the device at once, each taking
// the next tile from the launch's counter (reset by the step's dt kernel)
// until none is left, so no CTA waits at a tail of unevenly sized tiles.
// The counter is read only after the dependency wait.
template <class M, int FLUX>
__global__ void __launch_bounds__(kTileMax) k_tile_fused_work(FusedParams FP, TileIO io, int n_tiles) {
    pdl_trigger();
    pdl_wait();
    __shared__ int s_t;
    for (;;) {
        if (threadIdx.x == 0) s_t = atomicAdd(io.work, 1);
        __syncthreads();
        const int t = s_t;
        if (t >= n_tiles) return;
        if (!fused_tile<M, FLUX, false, true>(FP, io, t, PartIO{})) return;
        __syncthreads();  // every thread is done with this tile's shared memory (and s_t)
    }
}

template <class M>
struct FusedLaunch {
    static size_t smem(const FusedParams& FP) {
        return fused_smem<M>(FP.max_slots, FP.max_grad, FP.max_edges, FP.max_flux, FP.T).total;
    }
    static cudaError_t prepare(const FusedParams& FP) {
        static std::mutex mu;
        std::lock_guard<std::mutex> lock(mu);
        cudaError_t e = cudaSuccess;
        const size_t bytes = smem(FP);
        for (const void* fn : {(const void*)k_tile_fused<M, 1>, (const void*)k_tile_fused<M, 2>,
                               (const void*)k_tile_fused_part<M, 1, 1>, (const void*)k_tile_fused_part<M, 2, 1>,
                               (const void*)k_tile_fused_part<M, 1, 2>, (const void*)k_tile_fused_part<M, 2, 2>,
                               (const void*)k_tile_fused_work<M, 1>, (const void*)k_tile_fused_work<M, 2>}) {
            // only ever raised: a solver created earlier may launch with more
            cudaFuncAttributes fa{};
            if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
            if (e == cudaSuccess && (size_t)fa.maxDynamicSharedSizeBytes < bytes)
                e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
        }
        return e;
    }
    // CTAs of the work-list schedule: the device's resident capacity
    static int work_grid(const FusedParams& FP, int n_tiles) {
        int dev = 0, sms = 0, nb = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_tile_fused_work<M, 1>, FP.threads, smem(FP));
        return std::max(1, std::min(n_tiles, sms * std::max(nb, 1)));
    }
    // io.work != nullptr: the work-list schedule on `grid` CTAs
    // part: a decomposition part's launch (its tile offset, in-launch exchange)
    static void stage(const FusedParams& FP, const TileIO& io, cudaStream_t st, bool pdl, int n_tiles, int grid,
                      const PartIO* part = nullptr) {
        const size_t sm = smem(FP);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(io.work ? grid : n_tiles));
        cfg.blockDim = dim3((unsigned)FP.threads);
        cfg.dynamicSmemBytes = sm;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl ? 1 : 0;
        if (io.work) {
            if (FP.P.flux == 1) cudaLaunchKernelEx(&cfg, k_tile_fused_work<M, 1>, FP, io, n_tiles);
            else cudaLaunchKernelEx(&cfg, k_tile_fused_work<M, 2>, FP, io, n_tiles);
        } else if (part && part->remote) {
            if (FP.P.flux == 1) cudaLaunchKernelEx(&cfg, k_tile_fused_part<M, 1, 2>, FP, io, *part);
            else cudaLaunchKernelEx(&cfg, k_tile_fused_part<M, 2, 2>, FP, io, *part);
        } else if (part) {
            if (FP.P.flux == 1) cudaLaunchKernelEx(&cfg, k_tile_fused_part<M, 1, 1>, FP, io, *part);
            else cudaLaunchKernelEx(&cfg, k_tile_fused_part<M, 2, 1>, FP, io, *part);
        } else {
            if (FP.P.flux == 1) cudaLaunchKernelEx(&cfg, k_tile_fused<M, 1>, FP, io);
            else cudaLaunchKernelEx(&cfg, k_tile_fused<M, 2>, FP, io);
        }
    }
};

namespace tile {
cudaError_t prepare_fused(int precision, const FusedParams& FP);
size_t smem_fused(int precision, const FusedParams& FP);
int work_grid_fused(int precision, const FusedParams& FP, int n_tiles);
void launch_fused(int precision, const FusedParams& FP, const TileIO& io, cudaStream_t st, bool pdl, int n_tiles,
                  int grid, const PartIO* part = nullptr);
}  // namespace tile

}  // namespace fvgpu
