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
    unsigned long long dtmin_key;  // ordered key of the global dt minimum
    int active;                    // this step runs
    int need_R;                    // residuals are evaluated this step
    int n_hist;                    // print records written this chunk
    int pad;
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

// Mesh in device numbering + physics, passed to every kernel by value.
struct Params {
    int n_real, n_total, n_bound, V;
    int cell0;                      // device index of reference cell 0 (time += dt[0])
    const uint32_t* face_nbr;       // [kMaxFaces][n_real]: neighbour | side << 31, kNoFace
    const double* f_nx;             // [kMaxFaces][n_real] edge normal (edge orientation)
    const double* f_ny;
    const double* f_le;             // edge length
    const double* f_g;              // Green-Gauss weight |x_f - x_i| / |x_i - x_j| (i = edge cell 0)
    const double* f_dsx;            // x_f - x_self
    const double* f_dsy;
    const double* f_dnx;            // x_f - x_neighbour
    const double* f_dny;
    const double* area;             // [n_total]
    const int32_t* ghost_group;     // [n_bound] group of ghost n_real + b
    const int32_t* ghost_cell;      // [n_bound] interior (real) cell of ghost n_real + b
    const uint8_t* ghost_slot;      // [n_bound] face slot of that boundary face in ghost_cell
    // physics
    int flux, order2, limiter, dt_kind, global_dt;
    double gamma, K, cfl, dt_const;
    int n_groups;
    int group_bc[kMaxGroups];
    double group_bv[kMaxGroups * 4];
};

// Buffers of one RK stage.
struct StageIO {
    const double* q_stage;   // stage input (neighbour gathers)
    const double* q_base;    // step-start state
    double* q_out;           // stage output (may alias q_base on the last stage)
    double* gx;              // [n_total*V]; ghosts hold 0
    double* gy;
    double* lim;             // ghosts hold 1
    const double* dt;        // [n_total]
    double alpha;
    Ctrl* ctrl;              // nullptr: always active, dt from dt[]
    double* partials;        // [grid][V] residual partial sums, or nullptr
};

}  // namespace fvgpu
