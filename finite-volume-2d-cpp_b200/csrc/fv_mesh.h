// Host-side finite-volume mesh: the geometry fvhyper's reader builds
// (fvhyper/src/mesh.cpp:821-853), in the reference numbering, plus the
// device numbering (Hilbert order of real cells) and the per-cell face
// lists the kernels gather through.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace fvgpu {

struct HostMesh {
    // ---- element mesh (as read) ----
    std::vector<double> nodes_x, nodes_y;
    std::vector<int32_t> cells4;        // [n_real][4], -1 pads triangles
    std::vector<int32_t> bnd_nodes;     // [n_bound][2]
    std::vector<int32_t> bnd_group;     // [n_bound]
    std::vector<std::string> group_names;

    // ---- reference-numbered FV geometry (mesh.h:151-171) ----
    int64_t n_real = 0, n_total = 0, n_edges = 0, n_bound = 0;
    std::vector<uint32_t> edge_cells, edge_nodes;        // [E][2]
    std::vector<double> enx, eny, elen, ecx, ecy;        // [E]
    std::vector<double> area, ccx, ccy;                  // [n_total]
    std::vector<uint32_t> bound_edges;                   // [n_bound]

    // ---- batches of independent cases (fv_mesh_create_batch) ----
    // Case k owns reference real cells [case_real_off[k], case_real_off[k+1])
    // and boundary ghosts [case_bound_off[k], case_bound_off[k+1]).  Empty for
    // a single mesh.  Device numbering keeps each case's cells contiguous.
    std::vector<int64_t> case_real_off, case_bound_off;

    // ---- device numbering ----
    // new index of reference cell r: ref2new[r]; reference index of new cell n: new2ref[n].
    // Real cells occupy [0, n_real), ghosts [n_real, n_total) in both numberings.
    std::vector<int32_t> ref2new, new2ref;
    // Faces of each new-numbered real cell, in increasing reference edge order
    // (the order the reference's edge loops accumulate into that cell).
    static constexpr int MAXF = 4;
    std::vector<int32_t> face_edge;  // [n_real][MAXF] reference edge index or -1
    std::vector<uint8_t> face_side;  // [n_real][MAXF] 0: cell is edge_cells(e,0), 1: cell is edge_cells(e,1)
    std::vector<uint8_t> n_faces;    // [n_real]

    // ---- one part of a domain decomposition (build_part) ----
    // The tiles cover device cells [0, n_own); real cells [n_own, n_real) are
    // halo cells whose states other parts compute.  -1: every real cell.
    int64_t n_own = -1;
    int64_t owned_real() const { return n_own >= 0 ? n_own : n_real; }
};

// Per-face arrays of the device kernels, slot-major [MAXF][n_real] in device
// numbering, plus ghost metadata in device ghost order.
struct FaceArrays {
    std::vector<uint32_t> nbr;            // neighbour | side << 31, 0xFFFFFFFF if no face
    std::vector<double> nx, ny, le, g;    // edge normal, length, Green-Gauss weight
    std::vector<double> dsx, dsy;         // x_f - x_self
    std::vector<double> dnx, dny;         // x_f - x_neighbour
    std::vector<int32_t> ghost_group, ghost_cell;
    std::vector<uint8_t> ghost_slot;
    std::vector<double> g_nx, g_ny, g_le, g_dx, g_dy;   // per ghost: face normal, length, x_f - x_interior
    std::vector<double> area;             // [n_total] device numbering
    int32_t cell0 = 0;                    // device index of reference cell 0
};
void build_face_arrays(const HostMesh& m, FaceArrays& fa);

// Tiles of `tile_cells` consecutive device-numbered real cells.  Each tile
// lists the edges touching its cells (an edge cut by a tile boundary is
// listed by both tiles) with tile-local cell indices: owned cell c ->
// c - tile_start, halo cell h -> tile_cells + h.  Edges keep the reference
// orientation (first index = edge_cells(e, 0)).
struct TileArrays {
    int tile_cells = 0, n_tiles = 0;
    int max_halo = 0, max_edges = 0;
    std::vector<int32_t> info;        // [n_tiles][4]: edge_off, n_edges, halo_off, n_halo
    std::vector<int32_t> halo;        // device cell index of each halo slot
    std::vector<uint32_t> edge_ij;    // local i | local j << 16
    std::vector<int32_t> edge_ref;    // reference edge index of each tile edge
    std::vector<double> enx, eny, ele, exf, eyf, eg;  // per tile edge
    std::vector<uint16_t> face;       // [MAXF][n_real]: local edge | side << 15, 0xFFFF = none
    std::vector<double> ccx, ccy;     // [n_total] device numbering
};
void build_tiles(const HostMesh& m, const FaceArrays& fa, int tile_cells, TileArrays& ta);

// Two-ring tiles of the fused stage kernel, which computes the gradients and
// limiters of its own cells and of their face neighbours (ring 1) before the
// fluxes of its edges, so it stages the states of ring 2 as well.  Local
// slots: owned cells [0, T), ring 1 [T, T + n1) (face neighbours of owned
// cells, real or ghost), ring 2 [T + n1, T + n1 + n2) (face neighbours of
// ring-1 real cells not already local).  Local edges: the flux edges (those
// touching an owned cell, in first-visit order over the owned cells' faces)
// first, then the edges of ring-1 real cells not yet listed.  Every
// gradient slot (owned and ring 1) has four face words (local edge | ghost
// neighbour << 14 | side << 15, 0xFFFF = none) in increasing reference edge
// order; ring-1 ghosts and the unused owned slots of a last, partial tile
// have none.
struct Tile2Arrays {
    int tile_cells = 0, n_tiles = 0;
    int max_slots = 0, max_grad = 0, max_edges = 0, max_flux = 0;  // max_edges: a multiple of 4
    std::vector<int32_t> info;        // [n_tiles][8]: edge_off, n_edges, n_flux, halo_off, n1, n2, face_off, owned cells
    std::vector<int32_t> halo;        // device cell index of each ring-1, then ring-2 slot
    std::vector<uint32_t> edge_ij;    // local i | local j << 16, reference orientation; each
                                      // tile's run padded to a multiple of 4 entries
    std::vector<double> enx, eny, ele, exf, eyf, eg;  // per local edge
    std::vector<uint16_t> face;       // [sum over tiles of (T + n1)][4]
};
void build_tiles2(const HostMesh& m, const FaceArrays& fa, int tile_cells, Tile2Arrays& ta);

// One part of a decomposition of a single mesh into n_parts parts.  Part p
// owns device real cells [own_off[p], own_off[p+1]) (contiguous ranges of the
// Hilbert order) and the boundary ghosts of those cells; its local mesh adds
// ring 1 (face neighbours of owned cells), ring 2 (face neighbours of ring-1
// cells) and the boundary ghosts of ring 1, with every edge of an owned or
// ring-1 cell in reference edge order, so that each owned and ring-1 cell
// keeps all its faces in the order of the whole mesh.  Local numbering (also
// the part's device numbering): owned cells (those in other parts' halos, the
// band, first), halo real cells, owned ghosts, halo ghosts; each group in
// device order, so the halo groups are grouped by owner.
struct PartPlan {
    int n_parts = 1, part = 0;
    std::vector<int64_t> own_off;     // [n_parts + 1] device real cells of each part
    std::vector<int64_t> ghost_off;   // [n_parts + 1] device ghosts (offsets from n_real) of each part
    std::vector<int32_t> local2ref;   // reference index of each local cell
    std::vector<int32_t> local_edges; // reference index of each local edge, ascending
    int64_t n_own = 0, n_own_ghost = 0;
    int64_t n_band = 0;               // owned cells [0, n_band) are in other parts' halos
    int32_t cell0 = -1;               // local index of reference cell 0, -1 if another part owns it
    int32_t owner0 = 0;               // the part that owns reference cell 0
    // halo states from part r land in local cells recv_idx[recv_off[r] .. recv_off[r+1])
    std::vector<int64_t> recv_off;
    std::vector<int32_t> recv_idx;
    // states for part r: local cells send_idx[send_off[r] .. send_off[r+1]), in r's receive order
    std::vector<int64_t> send_off;
    std::vector<int32_t> send_idx;
};
// Returns "" on success, else an error message.  g: a single mesh with its
// device numbering.
std::string build_part(const HostMesh& g, int n_parts, int part, HostMesh& local, PartPlan& plan);

// Builds the reference geometry from an element mesh (mesh.cpp:130-260,
// 623-669).  Returns "" on success, else an error message.
std::string build_geometry(HostMesh& m);
// Hilbert renumbering of real cells + ghost order + face lists.
void build_device_numbering(HostMesh& m);
// Gmsh MSH 4.1 ASCII reader (the subset fvhyper's reader accepts,
// mesh.cpp:264-570).  Fills the element-mesh part of m.
std::string read_msh41(const std::string& path, HostMesh& m);
// SU2 native ASCII mesh, 2D (triangles, quadrilaterals, segment markers).
std::string read_su2(const std::string& path, HostMesh& m);

}  // namespace fvgpu
