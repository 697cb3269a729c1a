/*
 * fvhyper/post.h — VTK output of fvhyper, B200 build.
 *
 * Same declarations as the reference (fvhyper/post.h:22-42).  writeVtk
 * writes <name>[_<time>].vtu (under times/ when time is given) and, when
 * world_size > 1, the rank-0 <name>_parallel[_<time>].pvtu index, with the
 * reference's file names.  Cell data: rank, the vars named in var_names, and
 * the user's post::extra_scalars / extra_vectors evaluated per real cell.
 *
 * Two encodings, chosen by the FVGPU_VTK_FORMAT environment variable:
 *   "binary" (default): VTK XML with raw appended little-endian data, Float64
 *                       cell values (lossless), one write per file;
 *   "ascii":            the reference's exact text layout (6-digit fixed
 *                       values), byte-identical to fvhyper/src/post.cpp:21-200
 *                       for the same mesh and state.
 */
#pragma once

#include <map>
#include <string>
#include <vector>

#include <fvhyper/mesh.h>

namespace fvhyper {

namespace post {
extern std::map<std::string, void (*)(double*, double*)> extra_scalars;
extern std::map<std::string, void (*)(double*, double*)> extra_vectors;
}  // namespace post

extern const std::vector<std::string> var_names;

void writeVtk(const std::string name, std::vector<double>& q, mesh& m, int rank, int world_size,
              const std::string time = "");

}  // namespace fvhyper
