// Internal device-side data structures shared by the kernels and the C ABI.
#pragma once
#include <cstdint>

namespace fvgpu {

constexpr int kMaxFaces = 4;      // triangles and quads
constexpr int kMaxGroups = 16;    // boundary groups per mesh
constexpr int kMaxV = 4;
constexpr uint32_t kNoFace = 0xFFFFFFFFu;
constexpr int kBlock = 256;       // threads per block of the cell kernels

// Run control shared by the kernels of a captured step (device memory).
struct Ctrl {
    unsigned long long step;       // steps taken
    double time;                   // accumulated time
    double R[kMaxV], R0[kMaxV];    // residual norms (run() semantics)
    double Rraw[kMaxV];            // un-normalised R of the last evaluated step
    int active;                    // this step runs
    int need_R;                    // residuals are evaluated this step
    int n_hist;                    // print records written this chunk
    int pad;
    unsigned long long dtkeys[64]; // global dt minimum, spread over atomic slots
};

// One print record (step, time at step start, R as printed).
struct PrintRec {
    unsigned long long step;
    double time;
    double R[kMaxV];
};

struct RunLimits {
    unsigned long long max_step;
    double max_time;
    double tolerance;
    unsigned long long print_interval;
};

// Sizes, boundary-ghost metadata and physics, passed to kernels by value.
struct Params {
    int n_real, n_total, n_bound, V;
    int n_own;                      // tiles cover real cells [0, n_own): n_real, or a part's own cells
    int cell0;                      // device index of reference cell 0 (time += dt[0])
    // boundary ghost b (device cell n_real + b): its interior cell, the face
    // normal/length, and x_f - x_interior (reference arithmetic, FP64)
    const int32_t* ghost_group;     // [n_bound]
    const int32_t* ghost_cell;      // [n_bound]
    const double* g_nx;
    const double* g_ny;
    const double* g_le;
    const double* g_dx;
    const double* g_dy;
    // physics
    int flux, order2, limiter, dt_kind, global_dt, positivity_guard;
    int diffusive;                  // cell gradients feed the face gradient of the flux
    int smooth;                     // residual smoothing after each stage's time derivatives
    double gamma, K, cfl, dt_const;
    double mu, pr, cp, r;           // Navier-Stokes constants (viscous flux and dt kinds)
    int n_groups;
    int group_bc[kMaxGroups];
    double group_bv[kMaxGroups * 4];
    const double* ghost_bv;     // [n_bound][4] per-ghost boundary state (device ghost order) or nullptr
    // batches of independent cases (n_cases > 1): each case has its own
    // global dt minimum (64 key slots per case) and its own time
    int n_cases;
    const int32_t* cell_case;   // [n_total] case of each device cell
    const int32_t* tile_case;   // [n_tiles] case of a tile's cells, -1 if the tile spans two cases
    const int32_t* case_cell0;  // [n_cases] device index of each case's reference cell 0
    double* case_time;          // [n_cases]
};

}  // namespace fvgpu
