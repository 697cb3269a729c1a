// Tile kernels with the exact (reference evaluation order) FP64 policy.
// Compiled with -fmad=false so that no multiply-add is contracted.
#include "fv_tile.cuh"
#include "fv_fused.cuh"

namespace fvgpu {
namespace tile {
cudaError_t prepare_exact(const TileParams& TP) { return TileLaunch<MExact>::prepare(TP); }
void launch_dt_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl) {
    TileLaunch<MExact>::dt(TP, io, st, pdl);
}
void launch_gradlim_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool with_dt, bool pdl) {
    TileLaunch<MExact>::gradlim(TP, io, st, with_dt, pdl);
}
void launch_stage_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl, int phase) {
    TileLaunch<MExact>::stage(TP, io, st, pdl, phase);
}
cudaError_t prepare_fused_exact(const FusedParams& FP) { return FusedLaunch<MExact>::prepare(FP); }
size_t smem_fused_exact(const FusedParams& FP) { return FusedLaunch<MExact>::smem(FP); }
int work_grid_fused_exact(const FusedParams& FP, int n_tiles) { return FusedLaunch<MExact>::work_grid(FP, n_tiles); }
void launch_fused_exact(const FusedParams& FP, const TileIO& io, cudaStream_t st, bool pdl, int n_tiles, int grid,
                        const PartIO* part) {
    FusedLaunch<MExact>::stage(FP, io, st, pdl, n_tiles, grid, part);
}
}  // namespace tile
}  // namespace fvgpu
