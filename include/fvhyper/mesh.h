/*
 * fvhyper/mesh.h — mesh class of the fvhyper API, B200 build.
 *
 * Declares what user code of the reference touches (fvhyper/mesh.h:36-39,
 * 61-190): the boundaries::bounds table the user defines, the meshArray row
 * container, and class mesh with the reference's public geometry arrays in
 * the reference's numbering and layout (edges in first-visit order, ghost
 * cells appended after the real cells, one per boundary edge), filled by
 * read_file(name, pool).  User callbacks such as calc_dt and
 * generate_initial_solution read these arrays exactly as with the reference.
 *
 * The geometry is built by libfvgpu (fv_mesh_read_msh, include/fvgpu.h) and
 * the device handle stays attached to the mesh for run().
 */
#pragma once

#include <math.h>
#include <sys/types.h>

#include <algorithm>
#include <iostream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <fvhyper/parallel.h>

struct fv_mesh;  // include/fvgpu.h

namespace fvhyper {

extern const int vars;

namespace boundaries {
// user-defined: physical name -> b = bc(q_interior, n)
extern std::map<std::string, void (*)(double*, double*, double*)> bounds;
}  // namespace boundaries

// Row-major table of N unsigned ints per row (fvhyper/mesh.h:61-120).
template <uint N>
class meshArray {
private:
    std::vector<uint> nodes;

public:
    uint& operator()(const uint& i, const uint& j) { return nodes[(size_t)i * N + j]; }
    const uint& operator()(const uint& i, const uint& j) const { return nodes[(size_t)i * N + j]; }
    void push_back(const std::vector<uint> v) {
        if (v.size() != N)
            throw std::invalid_argument("size of input array " + std::to_string(v.size()) + " not equal to " +
                                        std::to_string(N));
        nodes.insert(nodes.end(), v.begin(), v.end());
    }
    uint cols() const { return (uint)(nodes.size() / N); }
    uint rows() const { return N; }
    void dump() {
        for (uint i = 0; i < cols(); ++i) {
            for (uint j = 0; j < N; ++j) std::cout << (*this)(i, j) << " ";
            std::cout << "\n";
        }
    }
    void swap(const uint& i, const uint& j) {
        for (uint k = 0; k < N; ++k) std::swap(nodes[(size_t)i * N + k], nodes[(size_t)j * N + k]);
    }
    void move_to_end(const uint& i) {
        std::rotate(nodes.begin() + (size_t)N * i, nodes.begin() + (size_t)N * i + N, nodes.end());
    }
    const std::vector<uint>& get_vector() { return nodes; }
    // B200 build: bulk fill
    std::vector<uint>& data() { return nodes; }
};

class mesh {
public:
    std::string filename;

    std::map<uint, std::string> physicalNames;  // boundary group index -> physical name

    std::vector<double> nodesX;
    std::vector<double> nodesY;

    meshArray<2> edgesNodes;
    meshArray<2> edgesCells;
    std::vector<double> edgesLengths;
    std::vector<double> edgesNormalsX;
    std::vector<double> edgesNormalsY;
    std::vector<double> edgesCentersX;
    std::vector<double> edgesCentersY;

    std::vector<uint> boundaryEdges;        // edge index of each boundary ghost, in ghost order
    std::vector<uint> boundaryEdgesIntTag;  // boundary group of each ghost
    std::vector<void (*)(double*, double*, double*)> boundaryFuncs;

    meshArray<4> cellsNodes;  // real cells: 3 or 4 node indices (0 in column 3 for triangles)
    std::vector<bool> cellsIsTriangle;
    std::vector<double> cellsAreas;     // [real + ghost]
    std::vector<double> cellsCentersX;  // [real + ghost]
    std::vector<double> cellsCentersY;  // [real + ghost]
    std::vector<bool> cellsIsGhost;     // [real]: MPI ghosts, all false on one GPU

    uint nRealCells = 0;

    // Reads "<name>.msh" (Gmsh MSH 4.1 ASCII, fvhyper/src/mesh.cpp:800-855),
    // or "<name>.su2" (SU2 native ASCII) when there is no .msh file, and
    // binds each boundary edge to boundaries::bounds[physical name / marker tag].
    void read_file(std::string filename, mpi_wrapper& pool);

    // B200 build: the device-side mesh this object was read into (owned).
    const ::fv_mesh* device_mesh() const { return dev_.get(); }
    // B200 build: fill this object from a mesh built by libfvgpu and take
    // ownership of it; bind_bounds looks each boundary group up in
    // boundaries::bounds as read_file does.
    void attach(::fv_mesh* dm, bool bind_bounds);

private:
    std::shared_ptr<::fv_mesh> dev_;
};

std::vector<std::string> cut_str(const std::string s, const char c);
std::vector<uint> str_to_ints(std::string s);

}  // namespace fvhyper
