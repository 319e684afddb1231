// cgfd_bulk_tma.cu -- dispatch of the TMA-pipelined bulk RK-stage kernel by medium and tile
// shape (the kernel: cgfd_bulk_tma.cuh; its instantiations: cgfd_bulk_tma_{iso,vti,aniso}.cu).
#include "cgfd_bulk_tma.cuh"

namespace cgfd {

extern template int launch_bulk_tma_med<MED_ISO>(int, int, int, const StageP &, const TmaP &, const BulkTiles &,
                                                 cudaStream_t);
extern template int launch_bulk_tma_med<MED_VTI>(int, int, int, const StageP &, const TmaP &, const BulkTiles &,
                                                 cudaStream_t);
extern template int launch_bulk_tma_med<MED_ANISO>(int, int, int, const StageP &, const TmaP &, const BulkTiles &,
                                                 cudaStream_t);
extern template cudaError_t prepare_bulk_tma_med<MED_ISO>(int, int, int);
extern template cudaError_t prepare_bulk_tma_med<MED_VTI>(int, int, int);
extern template cudaError_t prepare_bulk_tma_med<MED_ANISO>(int, int, int);

int tma_tile_y(int med, int shape) {
  if (med == MED_ISO) return shape ? TileShape<MED_ISO, 1>::TYT : TileShape<MED_ISO, 0>::TYT;
  if (med == MED_VTI) return shape ? TileShape<MED_VTI, 1>::TYT : TileShape<MED_VTI, 0>::TYT;
  return shape ? TileShape<MED_ANISO, 1>::TYT : TileShape<MED_ANISO, 0>::TYT;
}

int tma_blocks_per_sm(int med, int shape) {
  if (med == MED_ISO) return shape ? TileShape<MED_ISO, 1>::MINB : TileShape<MED_ISO, 0>::MINB;
  if (med == MED_VTI) return shape ? TileShape<MED_VTI, 1>::MINB : TileShape<MED_VTI, 0>::MINB;
  return shape ? TileShape<MED_ANISO, 1>::MINB : TileShape<MED_ANISO, 0>::MINB;
}

cudaError_t tma_prepare(int med, int coef_type, int wave16, int shape) {
  if (med == MED_ISO) return prepare_bulk_tma_med<MED_ISO>(coef_type, wave16, shape);
  if (med == MED_VTI) return prepare_bulk_tma_med<MED_VTI>(coef_type, wave16, shape);
  return prepare_bulk_tma_med<MED_ANISO>(coef_type, wave16, shape);
}

int launch_stage_bulk_tma(int med, int coef_type, int wave16, int shape, const StageP &p, const TmaP &tm,
                          const BulkTiles &t, cudaStream_t st) {
  if (p.nbulk <= 0) return 0;
  if (med == MED_ISO) return launch_bulk_tma_med<MED_ISO>(coef_type, wave16, shape, p, tm, t, st);
  if (med == MED_VTI) return launch_bulk_tma_med<MED_VTI>(coef_type, wave16, shape, p, tm, t, st);
  return launch_bulk_tma_med<MED_ANISO>(coef_type, wave16, shape, p, tm, t, st);
}

}  // namespace cgfd
