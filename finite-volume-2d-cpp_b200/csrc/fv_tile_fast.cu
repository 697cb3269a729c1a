// Tile kernels with the FP64 and FP32-bulk fast policies, and the
// per-precision dispatch.
#include "fv_tile.cuh"
#include "fv_fused.cuh"

namespace fvgpu {
namespace tile {
cudaError_t prepare_exact(const TileParams& TP);
void launch_dt_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl);
void launch_gradlim_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool with_dt, bool pdl);
void launch_stage_exact(const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl, int phase);
cudaError_t prepare_fused_exact(const FusedParams& FP);
size_t smem_fused_exact(const FusedParams& FP);
int work_grid_fused_exact(const FusedParams& FP, int n_tiles);
void launch_fused_exact(const FusedParams& FP, const TileIO& io, cudaStream_t st, bool pdl, int n_tiles, int grid,
                        const PartIO* part);

cudaError_t prepare(int precision, const TileParams& TP) {
    if (precision == 0) return prepare_exact(TP);
    if (precision == 1) return TileLaunch<MF64>::prepare(TP);
    return TileLaunch<MF32>::prepare(TP);
}
void launch_dt(int precision, const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl) {
    if (precision == 0) launch_dt_exact(TP, io, st, pdl);
    else if (precision == 1) TileLaunch<MF64>::dt(TP, io, st, pdl);
    else TileLaunch<MF32>::dt(TP, io, st, pdl);
}
void launch_gradlim(int precision, const TileParams& TP, const TileIO& io, cudaStream_t st, bool with_dt, bool pdl) {
    if (precision == 0) launch_gradlim_exact(TP, io, st, with_dt, pdl);
    else if (precision == 1) TileLaunch<MF64>::gradlim(TP, io, st, with_dt, pdl);
    else TileLaunch<MF32>::gradlim(TP, io, st, with_dt, pdl);
}
void launch_stage(int precision, const TileParams& TP, const TileIO& io, cudaStream_t st, bool pdl, int phase) {
    if (precision == 0) launch_stage_exact(TP, io, st, pdl, phase);
    else if (precision == 1) TileLaunch<MF64>::stage(TP, io, st, pdl, phase);
    else TileLaunch<MF32>::stage(TP, io, st, pdl, phase);
}
cudaError_t prepare_fused(int precision, const FusedParams& FP) {
    if (precision == 0) return prepare_fused_exact(FP);
    if (precision == 1) return FusedLaunch<MF64>::prepare(FP);
    return FusedLaunch<MF32>::prepare(FP);
}
size_t smem_fused(int precision, const FusedParams& FP) {
    if (precision == 0) return smem_fused_exact(FP);
    if (precision == 1) return FusedLaunch<MF64>::smem(FP);
    return FusedLaunch<MF32>::smem(FP);
}
int work_grid_fused(int precision, const FusedParams& FP, int n_tiles) {
    if (precision == 0) return work_grid_fused_exact(FP, n_tiles);
    if (precision == 1) return FusedLaunch<MF64>::work_grid(FP, n_tiles);
    return FusedLaunch<MF32>::work_grid(FP, n_tiles);
}
void launch_fused(int precision, const FusedParams& FP, const TileIO& io, cudaStream_t st, bool pdl, int n_tiles,
                  int grid, const PartIO* part) {
    if (precision == 0) launch_fused_exact(FP, io, st, pdl, n_tiles, grid, part);
    else if (precision == 1) FusedLaunch<MF64>::stage(FP, io, st, pdl, n_tiles, grid, part);
    else FusedLaunch<MF32>::stage(FP, io, st, pdl, n_tiles, grid, part);
}
}  // namespace tile
}  // namespace fvgpu
