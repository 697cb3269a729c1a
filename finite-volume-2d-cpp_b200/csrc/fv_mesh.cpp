// Host mesh construction: reference-equivalent geometry, MSH 4.1 reader,
// Hilbert renumbering and per-cell face lists.
#include "fv_mesh.h"

#include <algorithm>
#include <charconv>
#include <thread>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <numeric>
#include <sstream>

namespace fvgpu {

namespace {

// Open-addressing map from an undirected node pair to an edge index.
struct EdgeMap {
    std::vector<uint64_t> key;
    std::vector<int64_t> val;
    uint64_t mask = 0;
    explicit EdgeMap(size_t expected) {
        size_t cap = 16;
        while (cap < 2 * expected + 16) cap <<= 1;
        key.assign(cap, UINT64_MAX);
        val.assign(cap, -1);
        mask = cap - 1;
    }
    static uint64_t mix(uint64_t x) {
        x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
        return x;
    }
    static uint64_t make(uint32_t a, uint32_t b) {
        uint32_t lo = std::min(a, b), hi = std::max(a, b);
        return (uint64_t(lo) << 32) | hi;
    }
    // returns slot value pointer; *found tells whether the key existed
    int64_t* slot(uint64_t k, bool* found) {
        uint64_t h = mix(k) & mask;
        while (key[h] != UINT64_MAX) {
            if (key[h] == k) { *found = true; return &val[h]; }
            h = (h + 1) & mask;
        }
        *found = false;
        key[h] = k;
        return &val[h];
    }
    int64_t find(uint64_t k) const {
        uint64_t h = mix(k) & mask;
        while (key[h] != UINT64_MAX) {
            if (key[h] == k) return val[h];
            h = (h + 1) & mask;
        }
        return -1;
    }
};

// Hilbert index of (x, y) on a 2^order grid (the classic rotate-and-reflect walk).
uint64_t hilbert_d(uint32_t x, uint32_t y, int order) {
    uint64_t d = 0;
    for (uint32_t s = 1u << (order - 1); s > 0; s >>= 1) {
        uint32_t rx = (x & s) > 0, ry = (y & s) > 0;
        d += uint64_t(s) * s * ((3 * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) { x = s - 1 - x; y = s - 1 - y; }
            std::swap(x, y);
        }
    }
    return d;
}

}  // namespace

// mesh::read_file's geometry passes: add_cell_edges (mesh.cpp:130-154),
// convert_node_face_info (157-187), compute_mesh (190-260) and
// add_boundary_cells (623-669).  Same arithmetic, same order, so every
// array is bit-identical to the reference's.
std::string build_geometry(HostMesh& m) {
    const int64_t nc = (int64_t)m.cells4.size() / 4;
    const int64_t nb = (int64_t)m.bnd_group.size();
    const double* X = m.nodes_x.data();
    const double* Y = m.nodes_y.data();
    const int64_t nn = (int64_t)m.nodes_x.size();
    for (int64_t c = 0; c < nc; ++c)
        for (int k = 0; k < 4; ++k) {
            int32_t v = m.cells4[4 * c + k];
            if ((k < 3 && v < 0) || v >= nn) return "cell " + std::to_string(c) + " has an invalid node";
        }
    EdgeMap em((size_t)(2 * nc + 4));
    m.edge_cells.clear(); m.edge_nodes.clear();
    m.edge_cells.reserve(3 * nc); m.edge_nodes.reserve(3 * nc);
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t* cn = &m.cells4[4 * c];
        const int sz = cn[3] < 0 ? 3 : 4;
        for (int i = 0; i < sz; ++i) {
            const int j = (i < sz - 1) ? i + 1 : 0;
            bool found;
            int64_t* v = em.slot(EdgeMap::make(cn[i], cn[j]), &found);
            if (!found) {
                *v = (int64_t)m.edge_cells.size() / 2;
                m.edge_cells.push_back((uint32_t)c); m.edge_cells.push_back(0);
                m.edge_nodes.push_back(cn[i]); m.edge_nodes.push_back(cn[j]);
            }
        }
    }
    const int64_t E = (int64_t)m.edge_cells.size() / 2;
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t* cn = &m.cells4[4 * c];
        const int sz = cn[3] < 0 ? 3 : 4;
        for (int i = 0; i < sz; ++i) {
            const int j = (i < sz - 1) ? i + 1 : 0;
            int64_t e = em.find(EdgeMap::make(cn[i], cn[j]));
            if ((uint32_t)c != m.edge_cells[2 * e]) {
                if (m.edge_cells[2 * e + 1] != 0 && m.edge_cells[2 * e + 1] != (uint32_t)c)
                    return "edge shared by more than two cells (non-manifold mesh)";
                m.edge_cells[2 * e + 1] = (uint32_t)c;
            }
        }
    }
    const int64_t nt = nc + nb;
    m.n_real = nc; m.n_total = nt; m.n_edges = E; m.n_bound = nb;
    m.enx.assign(E, 0.); m.eny.assign(E, 0.); m.elen.assign(E, 0.);
    m.ecx.assign(E, 0.); m.ecy.assign(E, 0.);
    m.area.assign(nt, 0.); m.ccx.assign(nt, 0.); m.ccy.assign(nt, 0.);
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t* cn = &m.cells4[4 * c];
        const int sz = cn[3] < 0 ? 3 : 4;
        double cx = 0., cy = 0.;
        for (int j = 0; j < sz; ++j) {
            cx += X[cn[j]] / ((double)sz);
            cy += Y[cn[j]] / ((double)sz);
        }
        m.ccx[c] = cx; m.ccy[c] = cy;
    }
    for (int64_t e = 0; e < E; ++e) {
        const uint32_t a = m.edge_nodes[2 * e], b = m.edge_nodes[2 * e + 1];
        m.ecx[e] = (X[b] + X[a]) * 0.5;
        m.ecy[e] = (Y[b] + Y[a]) * 0.5;
        double dex = X[b] - X[a], dey = Y[b] - Y[a];
        double l = std::sqrt(dex * dex + dey * dey);
        m.elen[e] = l;
        m.enx[e] = -dey / l;
        m.eny[e] = dex / l;
        const uint32_t c0 = m.edge_cells[2 * e];
        double dot = m.enx[e] * (m.ecx[e] - m.ccx[c0]) + m.eny[e] * (m.ecy[e] - m.ccy[c0]);
        if (dot < 0) { m.enx[e] *= -1.; m.eny[e] *= -1.; }
    }
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t* cn = &m.cells4[4 * c];
        double x1 = X[cn[0]], x2 = X[cn[1]], x3 = X[cn[2]];
        double y1 = Y[cn[0]], y2 = Y[cn[1]], y3 = Y[cn[2]];
        if (cn[3] < 0) {
            m.area[c] = 0.5 * std::fabs(x1 * (y2 - y3) + x2 * (y3 - y1) + x3 * (y1 - y2));
        } else {
            double x4 = X[cn[3]], y4 = Y[cn[3]];
            m.area[c] = 0.5 * std::fabs(x1 * (y2 - y3) + x2 * (y3 - y1) + x3 * (y1 - y2)) +
                        0.5 * std::fabs(x1 * (y3 - y4) + x3 * (y4 - y1) + x4 * (y1 - y3));
        }
        if (!(m.area[c] >= 1e-300)) return "cell " + std::to_string(c) + " has zero area";
    }
    m.bound_edges.assign(nb, 0);
    std::vector<uint8_t> is_bnd(E, 0);
    for (int64_t b = 0; b < nb; ++b) {
        int64_t e = em.find(EdgeMap::make(m.bnd_nodes[2 * b], m.bnd_nodes[2 * b + 1]));
        if (e < 0)
            return "invalid edge ref (" + std::to_string(std::min(m.bnd_nodes[2 * b], m.bnd_nodes[2 * b + 1])) +
                   ", " + std::to_string(std::max(m.bnd_nodes[2 * b], m.bnd_nodes[2 * b + 1])) + ")";
        if (is_bnd[e]) return "boundary segment listed twice";
        if (m.edge_cells[2 * e + 1] != 0) return "boundary segment on an interior edge";
        is_bnd[e] = 1;
        const uint32_t cell = m.edge_cells[2 * e];
        double dx = m.ecx[e] - m.ccx[cell], dy = m.ecy[e] - m.ccy[cell];
        double dist = std::sqrt(dx * dx + dy * dy);
        const int64_t g = nc + b;
        m.area[g] = m.area[cell];
        m.ccx[g] = m.ecx[e] + dist * m.enx[e];
        m.ccy[g] = m.ecy[e] + dist * m.eny[e];
        m.edge_cells[2 * e + 1] = (uint32_t)g;
        m.bound_edges[b] = (uint32_t)e;
    }
    // Every edge must now have a second cell: an edge seen by one cell only
    // and not declared as a boundary would point at cell 0 in the reference.
    std::vector<uint8_t> deg(nc, 0);
    for (int64_t e = 0; e < E; ++e) {
        uint32_t i = m.edge_cells[2 * e], j = m.edge_cells[2 * e + 1];
        if (i == j) return "edge " + std::to_string(e) + " has one cell and is not a boundary segment";
        if (i < (uint32_t)nc) deg[i]++;
        if (j < (uint32_t)nc) deg[j]++;
    }
    for (int64_t c = 0; c < nc; ++c) {
        const int sz = m.cells4[4 * c + 3] < 0 ? 3 : 4;
        if (deg[c] != sz) return "cell " + std::to_string(c) + " has an open face (undeclared boundary)";
    }
    return "";
}

// Rank coordinate of every cell of [c0, c1) along one axis: its position in
// the sorted centroid coordinates (equal coordinates share their mean
// position), scaled to [0, 1].  In rank coordinates the cells are evenly
// spread along each axis, so a Hilbert tile is compact in cell counts even
// where cells are strongly graded (boundary layers), not only in space.
static void axis_ranks(const std::vector<double>& x, int64_t c0, int64_t c1, std::vector<double>& r) {
    const int64_t n = c1 - c0;
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return x[c0 + a] < x[c0 + b]; });
    const double scale = n > 1 ? 1.0 / (double)(n - 1) : 0.0;
    for (int64_t i = 0; i < n;) {
        int64_t j = i;
        while (j + 1 < n && x[c0 + idx[j + 1]] == x[c0 + idx[i]]) ++j;
        const double mean = 0.5 * (double)(i + j) * scale;
        for (int64_t k = i; k <= j; ++k) r[c0 + idx[k]] = mean;
        i = j + 1;
    }
}

// Hilbert order of the real cells, case by case (the case index above the
// key keeps the cases of a batch contiguous; a single mesh is one case), on
// the centroids (rank = false: each case's bounding square) or on their rank
// coordinates.  Returns new2ref of the real cells.
static std::vector<int32_t> hilbert_order(const HostMesh& m, const std::vector<int64_t>& offs, bool rank) {
    const int64_t nc = m.n_real;
    const int order = 16;
    const double top = (double)((1u << order) - 1);
    std::vector<uint64_t> key(nc);
    std::vector<double> rx, ry;
    if (rank) { rx.resize(nc); ry.resize(nc); }
    for (size_t k = 0; k + 1 < offs.size(); ++k) {
        double x0 = 0, y0 = 0, scale = top;
        if (rank) {
            axis_ranks(m.ccx, offs[k], offs[k + 1], rx);
            axis_ranks(m.ccy, offs[k], offs[k + 1], ry);
        } else {
            double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
            for (int64_t c = offs[k]; c < offs[k + 1]; ++c) {
                xmin = std::min(xmin, m.ccx[c]); xmax = std::max(xmax, m.ccx[c]);
                ymin = std::min(ymin, m.ccy[c]); ymax = std::max(ymax, m.ccy[c]);
            }
            x0 = xmin; y0 = ymin;
            scale = top / std::max(std::max(xmax - xmin, ymax - ymin), 1e-300);
        }
        for (int64_t c = offs[k]; c < offs[k + 1]; ++c) {
            const double fx = rank ? rx[c] * top : (m.ccx[c] - x0) * scale;
            const double fy = rank ? ry[c] * top : (m.ccy[c] - y0) * scale;
            key[c] = ((uint64_t)k << 32) | hilbert_d((uint32_t)fx, (uint32_t)fy, order);
        }
    }
    std::vector<int32_t> n2r(nc);
    std::iota(n2r.begin(), n2r.end(), 0);
    std::stable_sort(n2r.begin(), n2r.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
    return n2r;
}

// Halo cells of tiles of 128 consecutive cells in an order: mean + max / 4
// (the mean sets the re-read traffic, the max the shared memory per tile).
static double halo_score(const HostMesh& m, const std::vector<int32_t>& n2r) {
    const int64_t nc = m.n_real;
    const int T = 128;
    std::vector<int32_t> r2n(nc);
    for (int64_t n = 0; n < nc; ++n) r2n[n2r[n]] = (int32_t)n;
    std::vector<uint64_t> pairs;  // tile << 32 | halo cell (ghosts keep their reference index)
    pairs.reserve(2 * (size_t)m.n_edges);
    for (int64_t e = 0; e < m.n_edges; ++e) {
        const uint32_t i = m.edge_cells[2 * e], j = m.edge_cells[2 * e + 1];
        const uint64_t ti = (uint64_t)(r2n[i] / T);
        if (j >= (uint32_t)nc) { pairs.push_back(ti << 32 | j); continue; }
        const uint64_t tj = (uint64_t)(r2n[j] / T);
        if (ti != tj) { pairs.push_back(ti << 32 | j); pairs.push_back(tj << 32 | i); }
    }
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    const int64_t nt = (nc + T - 1) / T;
    std::vector<int32_t> cnt((size_t)nt, 0);
    for (uint64_t p : pairs) cnt[(size_t)(p >> 32)]++;
    int32_t mx = 0;
    for (int32_t v : cnt) mx = std::max(mx, v);
    return (double)pairs.size() / (double)std::max<int64_t>(nt, 1) + 0.25 * mx;
}

// Faces of each device-numbered real cell in increasing reference edge order.
static void build_face_lists(HostMesh& m) {
    const int64_t nc = m.n_real, E = m.n_edges;
    m.face_edge.assign(nc * HostMesh::MAXF, -1);
    m.face_side.assign(nc * HostMesh::MAXF, 0);
    m.n_faces.assign(nc, 0);
    for (int64_t e = 0; e < E; ++e) {
        for (int s = 0; s < 2; ++s) {
            const uint32_t rc = m.edge_cells[2 * e + s];
            if (rc >= (uint32_t)nc) continue;
            const int32_t c = m.ref2new[rc];
            const int k = m.n_faces[c]++;
            m.face_edge[c * HostMesh::MAXF + k] = (int32_t)e;
            m.face_side[c * HostMesh::MAXF + k] = (uint8_t)s;
        }
    }
}

void build_device_numbering(HostMesh& m) {
    const int64_t nc = m.n_real, nt = m.n_total;
    std::vector<int64_t> offs = m.case_real_off;
    if (offs.size() < 2) offs = {0, nc};
    // Hilbert order on the centroids keeps isotropic meshes (and O-grids,
    // strips) compact; on rank coordinates it keeps strongly graded cells
    // (boundary layers) compact in cell counts.  The order with the smaller
    // tile halos is kept.
    // the two candidate orders are built and scored on two threads
    std::vector<int32_t> geo, rnk;
    double s_geo = 0., s_rnk = 0.;
    std::thread tr([&] { rnk = hilbert_order(m, offs, true); s_rnk = halo_score(m, rnk); });
    geo = hilbert_order(m, offs, false);
    s_geo = halo_score(m, geo);
    tr.join();
    const bool use_rank = s_rnk < s_geo;
    m.new2ref.resize(nt);
    std::copy(use_rank ? rnk.begin() : geo.begin(), use_rank ? rnk.end() : geo.end(), m.new2ref.begin());
    m.ref2new.assign(nt, -1);
    for (int64_t n = 0; n < nc; ++n) m.ref2new[m.new2ref[n]] = (int32_t)n;
    // ghosts follow their interior cell's new index (stable in reference order)
    std::vector<int32_t> gorder(m.n_bound);
    std::iota(gorder.begin(), gorder.end(), 0);
    std::stable_sort(gorder.begin(), gorder.end(), [&](int32_t a, int32_t b) {
        return m.ref2new[m.edge_cells[2 * m.bound_edges[a]]] < m.ref2new[m.edge_cells[2 * m.bound_edges[b]]];
    });
    for (int64_t k = 0; k < m.n_bound; ++k) {
        const int32_t ref = (int32_t)(nc + gorder[k]);
        m.new2ref[nc + k] = ref;
        m.ref2new[ref] = (int32_t)(nc + k);
    }
    build_face_lists(m);
}

// The per-face quantities use the reference's arithmetic: the Green-Gauss
// weight of calc_gradients (explicit.cpp:132-140) and the face-centre offsets
// of calc_limiters / calc_time_derivatives (explicit.cpp:216-217, 297-301).
void build_face_arrays(const HostMesh& m, FaceArrays& fa) {
    const int64_t N = m.n_real, NT = m.n_total, F = HostMesh::MAXF;
    fa.nbr.assign(F * N, 0xFFFFFFFFu);
    for (auto* v : {&fa.nx, &fa.ny, &fa.le, &fa.g, &fa.dsx, &fa.dsy, &fa.dnx, &fa.dny}) v->assign(F * N, 0.);
    for (int64_t c = 0; c < N; ++c) {
        const int32_t self_ref = m.new2ref[c];
        for (int k = 0; k < m.n_faces[c]; ++k) {
            const int32_t e = m.face_edge[c * F + k];
            const int side = m.face_side[c * F + k];
            const uint32_t i = m.edge_cells[2 * e], j = m.edge_cells[2 * e + 1];
            const uint32_t nb_ref = side == 0 ? j : i;
            const size_t s = (size_t)k * N + c;
            fa.nbr[s] = (uint32_t)m.ref2new[nb_ref] | ((uint32_t)side << 31);
            fa.nx[s] = m.enx[e]; fa.ny[s] = m.eny[e]; fa.le[s] = m.elen[e];
            const double dxif = m.ecx[e] - m.ccx[i], dyif = m.ecy[e] - m.ccy[i];
            const double dif = std::sqrt(dxif * dxif + dyif * dyif);
            const double dxij = m.ccx[i] - m.ccx[j], dyij = m.ccy[i] - m.ccy[j];
            const double dij = std::sqrt(dxij * dxij + dyij * dyij);
            fa.g[s] = dif / dij;
            fa.dsx[s] = m.ecx[e] - m.ccx[self_ref]; fa.dsy[s] = m.ecy[e] - m.ccy[self_ref];
            fa.dnx[s] = m.ecx[e] - m.ccx[nb_ref]; fa.dny[s] = m.ecy[e] - m.ccy[nb_ref];
        }
    }
    const int64_t G = m.n_bound;
    fa.ghost_group.assign(G, 0); fa.ghost_cell.assign(G, 0); fa.ghost_slot.assign(G, 0);
    for (auto* v : {&fa.g_nx, &fa.g_ny, &fa.g_le, &fa.g_dx, &fa.g_dy}) v->assign(G, 0.);
    for (int64_t b = 0; b < G; ++b) {
        const int32_t ref = m.new2ref[N + b];          // reference ghost index
        const int64_t rb = ref - N;                    // its boundary segment
        const uint32_t e = m.bound_edges[rb];
        const int32_t c = m.ref2new[m.edge_cells[2 * e]];
        fa.ghost_group[b] = m.bnd_group[rb];
        fa.ghost_cell[b] = c;
        for (int k = 0; k < m.n_faces[c]; ++k)
            if (m.face_edge[c * F + k] == (int32_t)e) fa.ghost_slot[b] = (uint8_t)k;
        const uint32_t ci = m.edge_cells[2 * e];  // reference index of the interior cell
        fa.g_nx[b] = m.enx[e]; fa.g_ny[b] = m.eny[e]; fa.g_le[b] = m.elen[e];
        fa.g_dx[b] = m.ecx[e] - m.ccx[ci];
        fa.g_dy[b] = m.ecy[e] - m.ccy[ci];
    }
    fa.area.assign(NT, 0.);
    for (int64_t n = 0; n < NT; ++n) fa.area[n] = m.area[m.new2ref[n]];
    fa.cell0 = m.ref2new[0];
}

void build_tiles(const HostMesh& m, const FaceArrays& fa, int T, TileArrays& ta) {
    const int64_t N = m.n_real, NT = m.n_total, F = HostMesh::MAXF;
    const int64_t NO = m.owned_real();
    ta.tile_cells = T;
    ta.n_tiles = (int)((NO + T - 1) / T);
    ta.info.assign((size_t)ta.n_tiles * 4, 0);
    ta.halo.clear(); ta.edge_ij.clear(); ta.edge_ref.clear();
    for (auto* v : {&ta.enx, &ta.eny, &ta.ele, &ta.exf, &ta.eyf, &ta.eg}) v->clear();
    ta.face.assign((size_t)F * N, 0xFFFF);
    ta.max_halo = 0; ta.max_edges = 0;
    std::vector<int32_t> local(NT, -1);          // device cell -> local index in the current tile
    std::vector<int32_t> edge_stamp(m.n_edges, -1), edge_local(m.n_edges, 0);
    std::vector<int32_t> touched;
    for (int t = 0; t < ta.n_tiles; ++t) {
        const int64_t c0 = (int64_t)t * T, c1 = std::min<int64_t>(c0 + T, NO);
        const int edge_off = (int)ta.edge_ij.size(), halo_off = (int)ta.halo.size();
        int n_halo = 0, n_edges = 0;
        touched.clear();
        for (int64_t c = c0; c < c1; ++c) { local[c] = (int32_t)(c - c0); touched.push_back((int32_t)c); }
        auto loc = [&](int32_t dev) {
            if (local[dev] < 0) {
                local[dev] = T + n_halo++;
                ta.halo.push_back(dev);
                touched.push_back(dev);
            }
            return local[dev];
        };
        for (int64_t c = c0; c < c1; ++c) {
            for (int k = 0; k < m.n_faces[c]; ++k) {
                const int32_t e = m.face_edge[c * F + k];
                const int side = m.face_side[c * F + k];
                if (edge_stamp[e] != t) {
                    edge_stamp[e] = t;
                    edge_local[e] = n_edges++;
                    const int32_t di = m.ref2new[m.edge_cells[2 * e]], dj = m.ref2new[m.edge_cells[2 * e + 1]];
                    const uint32_t li = (uint32_t)loc(di), lj = (uint32_t)loc(dj);
                    ta.edge_ij.push_back(li | (lj << 16));
                    ta.edge_ref.push_back(e);
                    ta.enx.push_back(m.enx[e]); ta.eny.push_back(m.eny[e]); ta.ele.push_back(m.elen[e]);
                    ta.exf.push_back(m.ecx[e]); ta.eyf.push_back(m.ecy[e]);
                    const size_t s = (size_t)k * N + c;
                    ta.eg.push_back(fa.g[s]);
                }
                const uint32_t other = m.edge_cells[2 * e + (side ? 0 : 1)];
                const int ghost = other >= (uint32_t)N ? 1 : 0;
                ta.face[(size_t)k * N + c] = (uint16_t)(edge_local[e] | (ghost << 14) | (side << 15));
            }
        }
        ta.info[4 * t + 0] = edge_off; ta.info[4 * t + 1] = n_edges;
        ta.info[4 * t + 2] = halo_off; ta.info[4 * t + 3] = n_halo;
        ta.max_halo = std::max(ta.max_halo, n_halo);
        ta.max_edges = std::max(ta.max_edges, n_edges);
        for (int32_t d : touched) local[d] = -1;
    }
    ta.ccx.assign(NT, 0.); ta.ccy.assign(NT, 0.);
    for (int64_t n = 0; n < NT; ++n) { ta.ccx[n] = m.ccx[m.new2ref[n]]; ta.ccy[n] = m.ccy[m.new2ref[n]]; }
}

void build_tiles2(const HostMesh& m, const FaceArrays& fa, int T, Tile2Arrays& ta) {
    const int64_t N = m.n_real, NT = m.n_total, F = HostMesh::MAXF;
    const int64_t NO = m.owned_real();
    ta = Tile2Arrays();
    ta.tile_cells = T;
    ta.n_tiles = (int)((NO + T - 1) / T);
    ta.info.assign((size_t)ta.n_tiles * 8, 0);
    std::vector<int32_t> local(NT, -1);          // device cell -> local slot in the current tile
    std::vector<int32_t> edge_stamp(m.n_edges, -1), edge_local(m.n_edges, 0);
    std::vector<int32_t> touched, ring1;
    for (int t = 0; t < ta.n_tiles; ++t) {
        const int64_t c0 = (int64_t)t * T, c1 = std::min<int64_t>(c0 + T, NO);
        const int edge_off = (int)ta.edge_ij.size(), halo_off = (int)ta.halo.size();
        const int face_off = (int)(ta.face.size() / 4);
        int n_halo = 0, n_edges = 0;
        touched.clear();
        ring1.clear();
        for (int64_t c = c0; c < c1; ++c) { local[c] = (int32_t)(c - c0); touched.push_back((int32_t)c); }
        auto loc = [&](int32_t dev) {
            if (local[dev] < 0) {
                local[dev] = T + n_halo++;
                ta.halo.push_back(dev);
                touched.push_back(dev);
            }
            return local[dev];
        };
        // faces of one gradient cell (device index c < N); new edges get the next local index
        auto add_faces = [&](int64_t c, uint16_t* w) {
            for (int k = 0; k < m.n_faces[c]; ++k) {
                const int32_t e = m.face_edge[c * F + k];
                const int side = m.face_side[c * F + k];
                if (edge_stamp[e] != t) {
                    edge_stamp[e] = t;
                    edge_local[e] = n_edges++;
                    const int32_t di = m.ref2new[m.edge_cells[2 * e]], dj = m.ref2new[m.edge_cells[2 * e + 1]];
                    const uint32_t li = (uint32_t)loc(di), lj = (uint32_t)loc(dj);
                    ta.edge_ij.push_back(li | (lj << 16));
                    ta.enx.push_back(m.enx[e]); ta.eny.push_back(m.eny[e]); ta.ele.push_back(m.elen[e]);
                    ta.exf.push_back(m.ecx[e]); ta.eyf.push_back(m.ecy[e]);
                    ta.eg.push_back(fa.g[(size_t)k * N + c]);
                }
                const uint32_t other = m.edge_cells[2 * e + (side ? 0 : 1)];
                const int ghost = other >= (uint32_t)N ? 1 : 0;
                w[k] = (uint16_t)(edge_local[e] | (ghost << 14) | (side << 15));
            }
        };
        // owned cells: the flux edges and ring 1
        std::vector<uint16_t> words((size_t)T * 4, 0xFFFF);
        for (int64_t c = c0; c < c1; ++c) add_faces(c, &words[(size_t)(c - c0) * 4]);
        const int n_flux = n_edges, n1 = n_halo;
        for (int h = 0; h < n1; ++h) ring1.push_back(ta.halo[halo_off + h]);
        // ring-1 real cells: their remaining edges and ring 2
        words.resize((size_t)(T + n1) * 4, 0xFFFF);
        for (int h = 0; h < n1; ++h)
            if (ring1[h] < N) add_faces(ring1[h], &words[(size_t)(T + h) * 4]);
        const int n2 = n_halo - n1;
        ta.face.insert(ta.face.end(), words.begin(), words.end());
        // each tile's edge run starts on a multiple of 4 entries, so that it
        // is copied in 16-byte chunks
        while (ta.edge_ij.size() % 4) {
            ta.edge_ij.push_back(0);
            for (auto* v : {&ta.enx, &ta.eny, &ta.ele, &ta.exf, &ta.eyf, &ta.eg}) v->push_back(0.);
        }
        int32_t* inf = &ta.info[(size_t)8 * t];
        inf[0] = edge_off; inf[1] = n_edges; inf[2] = n_flux; inf[3] = halo_off;
        inf[4] = n1; inf[5] = n2; inf[6] = face_off; inf[7] = (int32_t)(c1 - c0);
        ta.max_slots = std::max(ta.max_slots, T + n1 + n2);
        ta.max_grad = std::max(ta.max_grad, T + n1);
        ta.max_edges = std::max(ta.max_edges, (n_edges + 3) / 4 * 4);
        ta.max_flux = std::max(ta.max_flux, n_flux);
        for (int32_t d : touched) local[d] = -1;
    }
}

// ----------------------------------------------------------------------------
// Domain decomposition.  The reference decomposes with gmsh partitions and
// exchanges q, gx, gy, limiters and dt of one ring of ghost elements per
// stage (mesh.cpp:673-799, explicit.cpp:420-477, 636-648, 729-746).  Here a
// part owns a contiguous range of the device numbering (Hilbert order, so
// parts are compact) and holds two rings of halo cells plus the boundary
// ghosts of ring 1, so that the fused stage kernel recomputes the ring-1
// gradients and limiters it needs and only the stage state crosses between
// parts, once per stage.
// ----------------------------------------------------------------------------
namespace {
struct Halo {
    std::vector<int32_t> real;   // device indices of ring-1 and ring-2 real cells, ascending
    std::vector<int32_t> ghost;  // device ghost offsets (from n_real) of ring-1 ghosts, ascending
    std::vector<int32_t> ring1;  // device indices of ring-1 real cells
};
}  // namespace

std::string build_part(const HostMesh& g, int n_parts, int part, HostMesh& L, PartPlan& plan) {
    const int64_t N = g.n_real, NB = g.n_bound, F = HostMesh::MAXF;
    if (g.case_real_off.size() > 2) return "a batch of cases cannot be decomposed";
    if (n_parts < 1 || part < 0 || part >= n_parts) return "part index out of range";
    if (n_parts > N) return "more parts than cells";
    plan = PartPlan();
    plan.n_parts = n_parts;
    plan.part = part;
    plan.own_off.resize(n_parts + 1);
    for (int p = 0; p <= n_parts; ++p) plan.own_off[p] = N * p / n_parts;
    auto owner = [&](int64_t d) {
        return (int)(std::upper_bound(plan.own_off.begin(), plan.own_off.end(), d) - plan.own_off.begin() - 1);
    };
    // device interior cell of each device ghost; ghosts are ordered by it, so
    // each part's ghosts form a contiguous range
    std::vector<int32_t> ghost_in(NB);
    for (int64_t k = 0; k < NB; ++k)
        ghost_in[k] = g.ref2new[g.edge_cells[2 * g.bound_edges[g.new2ref[N + k] - N]]];
    plan.ghost_off.assign(n_parts + 1, NB);
    for (int64_t k = NB - 1; k >= 0; --k) plan.ghost_off[owner(ghost_in[k])] = k;
    for (int p = n_parts - 1; p >= 0; --p) plan.ghost_off[p] = std::min(plan.ghost_off[p], plan.ghost_off[p + 1]);
    auto nbr = [&](int64_t c, int k) {  // device index of the other cell of face k of device cell c
        const int32_t e = g.face_edge[c * F + k];
        return g.ref2new[g.edge_cells[2 * e + (g.face_side[c * F + k] ? 0 : 1)]];
    };
    std::vector<int32_t> mark(N + NB, -1);
    auto halo_of = [&](int p, Halo& h) {
        const int64_t a = plan.own_off[p], b = plan.own_off[p + 1];
        h = Halo();
        for (int64_t c = a; c < b; ++c)
            for (int k = 0; k < g.n_faces[c]; ++k) {
                const int32_t d = nbr(c, k);
                if (d < N && (d < a || d >= b) && mark[d] != p) { mark[d] = p; h.ring1.push_back(d); }
            }
        h.real = h.ring1;
        for (int32_t c : h.ring1)
            for (int k = 0; k < g.n_faces[c]; ++k) {
                const int32_t d = nbr(c, k);
                if (mark[d] == p) continue;
                if (d < N && d >= a && d < b) continue;
                mark[d] = p;
                if (d < N) h.real.push_back(d);
                else h.ghost.push_back(d - (int32_t)N);
            }
        std::sort(h.real.begin(), h.real.end());
        std::sort(h.ghost.begin(), h.ghost.end());
    };
    std::vector<Halo> halos(n_parts);
    for (int p = 0; p < n_parts; ++p) halo_of(p, halos[p]);
    const Halo& H = halos[part];
    const int64_t a = plan.own_off[part], b = plan.own_off[part + 1];
    const int64_t ga = plan.ghost_off[part], gb = plan.ghost_off[part + 1];
    plan.n_own = b - a;
    // owned cells in other parts' halos (the band) first, so that the first
    // tiles compute every state this part sends; each group in device order
    std::vector<uint8_t> band(b - a, 0);
    for (int r = 0; r < n_parts; ++r)
        if (r != part)
            for (int32_t d : halos[r].real)
                if (d >= a && d < b) band[d - a] = 1;
    std::vector<int32_t> own_order;
    own_order.reserve(b - a);
    for (int pass = 1; pass >= 0; --pass)
        for (int64_t i = 0; i < b - a; ++i)
            if (band[i] == pass) own_order.push_back((int32_t)(a + i));
    plan.n_band = (int64_t)std::count(band.begin(), band.end(), (uint8_t)1);
    plan.n_own_ghost = gb - ga;
    const int64_t nr = plan.n_own + (int64_t)H.real.size();
    const int64_t nbl = plan.n_own_ghost + (int64_t)H.ghost.size();
    // local numbering: owned cells, halo cells (grouped by owner), owned
    // ghosts, halo ghosts (grouped by owner); each group in device order
    std::vector<int32_t> dev_of(nr + nbl);   // device index (ghosts: N + offset) of each local cell
    for (int64_t i = 0; i < plan.n_own; ++i) dev_of[i] = own_order[i];
    for (size_t i = 0; i < H.real.size(); ++i) dev_of[plan.n_own + i] = H.real[i];
    for (int64_t i = 0; i < plan.n_own_ghost; ++i) dev_of[nr + i] = (int32_t)(N + ga + i);
    for (size_t i = 0; i < H.ghost.size(); ++i) dev_of[nr + plan.n_own_ghost + i] = (int32_t)(N + H.ghost[i]);
    std::vector<int32_t> loc(N + NB, -1);    // device index -> local index
    for (size_t i = 0; i < dev_of.size(); ++i) loc[dev_of[i]] = (int32_t)i;
    plan.local2ref.resize(dev_of.size());
    for (size_t i = 0; i < dev_of.size(); ++i) plan.local2ref[i] = g.new2ref[dev_of[i]];
    // receive lists: from each owner, its real halo cells, then its ghosts
    plan.recv_off.assign(n_parts + 1, 0);
    plan.recv_idx.clear();
    for (int r = 0; r < n_parts; ++r) {
        plan.recv_off[r] = (int64_t)plan.recv_idx.size();
        if (r == part) continue;
        for (size_t i = 0; i < H.real.size(); ++i)
            if (owner(H.real[i]) == r) plan.recv_idx.push_back((int32_t)(plan.n_own + i));
        for (size_t i = 0; i < H.ghost.size(); ++i)
            if (owner(ghost_in[H.ghost[i]]) == r) plan.recv_idx.push_back((int32_t)(nr + plan.n_own_ghost + i));
    }
    plan.recv_off[n_parts] = (int64_t)plan.recv_idx.size();
    // send lists: to each part, the cells and ghosts of this part in its halo, in its receive order
    plan.send_off.assign(n_parts + 1, 0);
    plan.send_idx.clear();
    for (int r = 0; r < n_parts; ++r) {
        plan.send_off[r] = (int64_t)plan.send_idx.size();
        if (r == part) continue;
        for (int32_t d : halos[r].real)
            if (d >= a && d < b) plan.send_idx.push_back(loc[d]);
        for (int32_t o : halos[r].ghost)
            if (o >= ga && o < gb) plan.send_idx.push_back((int32_t)(nr + (o - ga)));
    }
    plan.send_off[n_parts] = (int64_t)plan.send_idx.size();
    const int32_t d0 = g.ref2new[0];
    plan.owner0 = owner(d0);
    plan.cell0 = plan.owner0 == part ? loc[d0] : -1;

    // local edges: every edge of an owned or ring-1 cell, in reference edge order
    std::vector<int32_t> edges;
    std::vector<uint8_t> seen(g.n_edges, 0);
    auto take = [&](int64_t c) {
        for (int k = 0; k < g.n_faces[c]; ++k) {
            const int32_t e = g.face_edge[c * F + k];
            if (!seen[e]) { seen[e] = 1; edges.push_back(e); }
        }
    };
    for (int64_t c = a; c < b; ++c) take(c);
    for (int32_t c : H.ring1) take(c);
    std::sort(edges.begin(), edges.end());
    plan.local_edges = edges;
    std::vector<int32_t> eloc(g.n_edges, -1);
    for (size_t i = 0; i < edges.size(); ++i) eloc[edges[i]] = (int32_t)i;

    L = HostMesh();
    L.group_names = g.group_names;
    L.n_real = nr; L.n_total = nr + nbl; L.n_bound = nbl; L.n_edges = (int64_t)edges.size();
    L.n_own = plan.n_own;
    L.edge_cells.resize(2 * edges.size()); L.edge_nodes.resize(2 * edges.size());
    for (auto* v : {&L.enx, &L.eny, &L.elen, &L.ecx, &L.ecy}) v->resize(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) {
        const int32_t e = edges[i];
        for (int s = 0; s < 2; ++s) {
            const int32_t l = loc[g.ref2new[g.edge_cells[2 * e + s]]];
            if (l < 0) return "internal error: an edge of the part reaches outside its halo";
            L.edge_cells[2 * i + s] = (uint32_t)l;
            L.edge_nodes[2 * i + s] = g.edge_nodes[2 * e + s];
        }
        L.enx[i] = g.enx[e]; L.eny[i] = g.eny[e]; L.elen[i] = g.elen[e];
        L.ecx[i] = g.ecx[e]; L.ecy[i] = g.ecy[e];
    }
    L.area.resize(L.n_total); L.ccx.resize(L.n_total); L.ccy.resize(L.n_total);
    for (int64_t i = 0; i < L.n_total; ++i) {
        const int32_t r = plan.local2ref[i];
        L.area[i] = g.area[r]; L.ccx[i] = g.ccx[r]; L.ccy[i] = g.ccy[r];
    }
    L.bound_edges.resize(nbl); L.bnd_group.resize(nbl);
    for (int64_t k = 0; k < nbl; ++k) {
        const int64_t rb = plan.local2ref[nr + k] - N;
        const int32_t le = eloc[g.bound_edges[rb]];
        if (le < 0) return "internal error: a ghost's boundary edge is not in the part";
        L.bound_edges[k] = (uint32_t)le;
        L.bnd_group[k] = g.bnd_group[rb];
    }
    // the local numbering is the device numbering
    L.ref2new.resize(L.n_total);
    std::iota(L.ref2new.begin(), L.ref2new.end(), 0);
    L.new2ref = L.ref2new;
    build_face_lists(L);
    return "";
}

// ----------------------------------------------------------------------------
// MSH 4.1 ASCII reader.  Accepts what fvhyper's reader accepts for a single
// partition: $PhysicalNames, $Entities (curve -> physical tag, token 8 of a
// curve line, mesh.cpp:308-311), $Nodes (node index = order of appearance,
// mesh.cpp:392-401), $Elements (dim-1 two-node elements are boundary
// segments, mesh.cpp:460-473; dim-2 three/four-node elements are cells in
// file order, mesh.cpp:528-559).
// ----------------------------------------------------------------------------
std::string read_msh41(const std::string& path, HostMesh& m) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::string buf((size_t)sz, '\0');
    if (sz > 0 && std::fread(&buf[0], 1, (size_t)sz, f) != (size_t)sz) { std::fclose(f); return "read error"; }
    std::fclose(f);
    const char* p = buf.c_str();
    const char* end = p + buf.size();
    auto next_line = [&](std::string& line) -> bool {
        if (p >= end) return false;
        const char* q = (const char*)std::memchr(p, '\n', end - p);
        if (!q) q = end;
        line.assign(p, q);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        p = (q < end) ? q + 1 : end;
        return true;
    };
    // the node and element lines are parsed in place: integers and doubles
    // with std::from_chars (correctly rounded, as strtod), no line copies
    auto skip_ws = [&]() { while (p < end && (*p == ' ' || *p == '\t')) ++p; };
    auto eol = [&]() {
        const char* q = (const char*)std::memchr(p, '\n', end - p);
        p = q ? q + 1 : end;
    };
    auto read_long = [&](long& v) -> bool {
        skip_ws();
        auto r = std::from_chars(p, end, v);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
        return true;
    };
    auto read_double = [&](double& v) -> bool {
        skip_ws();
        auto r = std::from_chars(p, end, v);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
        return true;
    };
    std::map<long, std::string> phys_names;
    std::map<long, long> curve_phys;
    // MSH node tag -> index: dense over [tag_min, tag_max] when the tags are
    // (nearly) contiguous, as gmsh writes them; a hash map otherwise
    long tag_min = 0;
    std::vector<int64_t> node_dense;
    std::unordered_map<long, int64_t> node_sparse;
    bool dense = true;
    auto node_of = [&](long tag) -> int64_t {
        if (dense) {
            const long i = tag - tag_min;
            return (i >= 0 && i < (long)node_dense.size()) ? node_dense[(size_t)i] : -1;
        }
        auto it = node_sparse.find(tag);
        return it == node_sparse.end() ? -1 : it->second;
    };
    std::map<long, int32_t> tag_group;
    m.nodes_x.clear(); m.nodes_y.clear(); m.cells4.clear();
    m.bnd_nodes.clear(); m.bnd_group.clear(); m.group_names.clear();
    std::string line;
    bool have_nodes = false, have_elements = false;
    try {
        while (next_line(line)) {
            if (line.empty() || line[0] != '$') continue;
            const std::string sec = line.substr(1);
            if (sec == "PhysicalNames") {
                next_line(line);
                long n = std::stol(line);
                for (long i = 0; i < n; ++i) {
                    next_line(line);
                    std::istringstream ss(line);
                    long dim, tag; std::string name;
                    ss >> dim >> tag;
                    std::getline(ss, name);
                    name.erase(std::remove(name.begin(), name.end(), '"'), name.end());
                    name.erase(0, name.find_first_not_of(' '));
                    phys_names[tag] = name;
                }
            } else if (sec == "Entities") {
                next_line(line);
                long np, ncv, ns, nv;
                if (std::sscanf(line.c_str(), "%ld %ld %ld %ld", &np, &ncv, &ns, &nv) != 4) return "bad $Entities header";
                for (long i = 0; i < np; ++i) next_line(line);
                for (long i = 0; i < ncv; ++i) {
                    next_line(line);
                    std::istringstream ss(line);
                    std::vector<std::string> tok; std::string t;
                    while (ss >> t) tok.push_back(t);
                    if (tok.size() < 9) return "bad curve entity line";
                    curve_phys[std::stol(tok[0])] = (long)std::stod(tok[8]);
                }
            } else if (sec == "PartitionedEntities" || sec == "GhostElements") {
                return "partitioned meshes are not supported on the single-GPU path";
            } else if (sec == "Nodes") {
                next_line(line);
                long nblocks, nnodes, mn, mx;
                if (std::sscanf(line.c_str(), "%ld %ld %ld %ld", &nblocks, &nnodes, &mn, &mx) != 4) return "bad $Nodes header";
                m.nodes_x.reserve(nnodes); m.nodes_y.reserve(nnodes);
                tag_min = mn;
                dense = mx >= mn && mx - mn < 4 * std::max(nnodes, 1L) + 16;
                if (dense) node_dense.assign((size_t)(mx - mn + 1), -1);
                for (long b = 0; b < nblocks; ++b) {
                    next_line(line);
                    long edim, etag, param, nin;
                    if (std::sscanf(line.c_str(), "%ld %ld %ld %ld", &edim, &etag, &param, &nin) != 4) return "bad node block";
                    std::vector<long> tags(nin);
                    for (long i = 0; i < nin; ++i) {
                        if (!read_long(tags[i])) return "bad node tag";
                        eol();
                    }
                    for (long i = 0; i < nin; ++i) {
                        double x, y;
                        if (!read_double(x) || !read_double(y)) return "bad node coordinates";
                        eol();
                        const long t = tags[i];
                        if (dense) {
                            if (t < mn || t > mx) return "node tag outside the $Nodes range";
                            node_dense[(size_t)(t - mn)] = (int64_t)m.nodes_x.size();
                        } else {
                            node_sparse[t] = (int64_t)m.nodes_x.size();
                        }
                        m.nodes_x.push_back(x); m.nodes_y.push_back(y);
                    }
                }
                have_nodes = true;
            } else if (sec == "Elements") {
                if (!have_nodes) return "$Elements before $Nodes";
                next_line(line);
                long nblocks, nel, mn, mx;
                if (std::sscanf(line.c_str(), "%ld %ld %ld %ld", &nblocks, &nel, &mn, &mx) != 4) return "bad $Elements header";
                for (long b = 0; b < nblocks; ++b) {
                    next_line(line);
                    long edim, etag, etype, nin;
                    if (std::sscanf(line.c_str(), "%ld %ld %ld %ld", &edim, &etag, &etype, &nin) != 4) return "bad element block";
                    int32_t group = -1;
                    if (edim == 1) {
                        auto it = curve_phys.find(etag);
                        if (it == curve_phys.end()) return "curve entity " + std::to_string(etag) + " has no physical tag";
                        auto g = tag_group.find(it->second);
                        if (g == tag_group.end()) {
                            group = (int32_t)m.group_names.size();
                            tag_group[it->second] = group;
                            auto nm = phys_names.find(it->second);
                            m.group_names.push_back(nm == phys_names.end() ? std::string() : nm->second);
                        } else {
                            group = g->second;
                        }
                    }
                    if (edim == 2) m.cells4.reserve(m.cells4.size() + 4 * (size_t)nin);
                    for (long i = 0; i < nin; ++i) {
                        long v[16]; int nv = 0;
                        const char* le = (const char*)std::memchr(p, '\n', end - p);
                        if (!le) le = end;
                        while (nv < 16) {
                            while (p < le && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
                            auto r = std::from_chars(p, le, v[nv]);
                            if (r.ec != std::errc()) break;
                            p = r.ptr;
                            ++nv;
                        }
                        p = le < end ? le + 1 : end;
                        const int nnode = nv - 1;
                        int64_t idx[4] = {-1, -1, -1, -1};
                        for (int k = 0; k < nnode && k < 4; ++k) {
                            idx[k] = node_of(v[1 + k]);
                            if (idx[k] < 0) return "element " + std::to_string(v[0]) + " names an unknown node";
                        }
                        if (edim == 1 && nnode == 2) {
                            m.bnd_nodes.push_back((int32_t)idx[0]);
                            m.bnd_nodes.push_back((int32_t)idx[1]);
                            m.bnd_group.push_back(group);
                        } else if (edim == 2) {
                            if (nnode != 3 && nnode != 4) return "only 3- and 4-node cells are supported";
                            for (int k = 0; k < 4; ++k) m.cells4.push_back(k < nnode ? (int32_t)idx[k] : -1);
                        }
                    }
                }
                have_elements = true;
            }
        }
    } catch (const std::exception& ex) {
        return std::string("malformed MSH file: ") + ex.what();
    }
    if (!have_nodes || !have_elements) return "missing $Nodes or $Elements";
    return "";
}

// SU2 native mesh (ASCII, 2D): NDIME= 2; NELEM= n with one element per line
// (VTK type 5 = triangle, 9 = quadrilateral, node indices, optional element
// index); NPOIN= n with "x y [index]" lines; NMARK= n, each MARKER_TAG= name
// with MARKER_ELEMS= n lines of type 3 (segment) and two node indices.
// Nodes, cells and boundary segments keep file order; boundary groups are the
// marker tags in file order.  The reference reads Gmsh files only: its
// examples/naca ships SU2 meshes to be converted with gmsh first
// (examples/naca/naca.geo:1-7).
std::string read_su2(const std::string& path, HostMesh& m) {
    std::ifstream in(path);
    if (!in) return "cannot open " + path;
    m.nodes_x.clear(); m.nodes_y.clear(); m.cells4.clear();
    m.bnd_nodes.clear(); m.bnd_group.clear(); m.group_names.clear();
    std::string line;
    auto value_of = [](const std::string& l, const char* key, long* v) -> bool {
        const size_t k = l.find(key);
        if (k == std::string::npos) return false;
        *v = std::strtol(l.c_str() + k + std::strlen(key), nullptr, 10);
        return true;
    };
    long ndime = 0, nelem = -1, npoin = -1;
    std::vector<int32_t> cells;
    try {
        while (std::getline(in, line)) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            const size_t c = line.find('%');
            if (c != std::string::npos) line.erase(c);
            long v;
            if (value_of(line, "NDIME=", &v)) {
                ndime = v;
                if (ndime != 2) return "SU2 mesh is not two-dimensional (NDIME= " + std::to_string(ndime) + ")";
            } else if (value_of(line, "NELEM=", &v)) {
                nelem = v;
                cells.reserve((size_t)nelem * 4);
                for (long e = 0; e < nelem; ++e) {
                    if (!std::getline(in, line)) return "SU2: NELEM section ends early";
                    std::istringstream ss(line);
                    long type;
                    ss >> type;
                    const int nn = type == 5 ? 3 : type == 9 ? 4 : 0;
                    if (!nn) return "SU2: element type " + std::to_string(type) + " is not a triangle or quadrilateral";
                    int32_t id[4] = {-1, -1, -1, -1};
                    for (int k = 0; k < nn; ++k) {
                        long x;
                        if (!(ss >> x)) return "SU2: short element line";
                        id[k] = (int32_t)x;
                    }
                    cells.insert(cells.end(), id, id + 4);
                }
            } else if (value_of(line, "NPOIN=", &v)) {
                npoin = v;
                m.nodes_x.reserve((size_t)npoin); m.nodes_y.reserve((size_t)npoin);
                for (long i = 0; i < npoin; ++i) {
                    if (!std::getline(in, line)) return "SU2: NPOIN section ends early";
                    char* e1;
                    char* e2;
                    const double x = std::strtod(line.c_str(), &e1);
                    const double y = std::strtod(e1, &e2);
                    if (e1 == line.c_str() || e2 == e1) return "SU2: bad point line";
                    m.nodes_x.push_back(x); m.nodes_y.push_back(y);
                }
            } else if (line.find("MARKER_TAG=") != std::string::npos) {
                std::string name = line.substr(line.find("MARKER_TAG=") + 11);
                name.erase(0, name.find_first_not_of(" \t"));
                name.erase(name.find_last_not_of(" \t") + 1);
                long ne = 0;
                while (std::getline(in, line) && !value_of(line, "MARKER_ELEMS=", &ne)) {}
                const int32_t g = (int32_t)m.group_names.size();
                m.group_names.push_back(name);
                for (long e = 0; e < ne; ++e) {
                    if (!std::getline(in, line)) return "SU2: MARKER_ELEMS section ends early";
                    std::istringstream ss(line);
                    long type, a, b;
                    if (!(ss >> type >> a >> b) || type != 3) return "SU2: boundary element of marker " + name + " is not a segment";
                    m.bnd_nodes.push_back((int32_t)a); m.bnd_nodes.push_back((int32_t)b);
                    m.bnd_group.push_back(g);
                }
            }
        }
    } catch (const std::exception& e) {
        return std::string("SU2 parse error: ") + e.what();
    }
    if (ndime != 2 || nelem < 0 || npoin < 0) return "SU2 mesh without NDIME= 2, NELEM= or NPOIN=";
    for (int32_t id : cells)
        if (id >= npoin) return "SU2: element node index out of range";
    for (int32_t id : m.bnd_nodes)
        if (id < 0 || id >= npoin) return "SU2: marker node index out of range";
    m.cells4.swap(cells);
    return "";
}

}  // namespace fvgpu
