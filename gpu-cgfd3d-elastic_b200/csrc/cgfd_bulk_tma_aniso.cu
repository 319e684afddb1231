// cgfd_bulk_tma_aniso.cu -- the bulk RK-stage kernel's instantiations for the aniso medium (every
// operator direction, coefficient storage, wave policy, PML / interior variant and tile shape).
#include "cgfd_bulk_tma.cuh"

namespace cgfd {
template int launch_bulk_tma_med<MED_ANISO>(int, int, int, const StageP &, const TmaP &, const BulkTiles &,
                                         cudaStream_t);
template cudaError_t prepare_bulk_tma_med<MED_ANISO>(int, int, int);
}  // namespace cgfd
