// Tile kernels with the exact (reference evaluation order) FP64 policy.
// Compiled with -fmad=false so that no multiply-add is contracted.
#include "fv_tile.cuh"

namespace fvgpu {
namespace tile {
cudaError_t prepare_exact(const TileParams& TP) { return TileLaunch<MExact>::prepare(TP); }
void launch_dt_exact(const TileParams& TP, const TileIO& io, cudaStream_t st) { TileLaunch<MExact>::dt(TP, io, st); }
void launch_gradlim_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool with_dt) {
    TileLaunch<MExact>::gradlim(TP, io, st, with_dt);
}
void launch_stage_exact(const TileParams& TP, const TileIO& io, cudaStream_t st) {
    TileLaunch<MExact>::stage(TP, io, st);
}
}  // namespace tile
}  // namespace fvgpu
