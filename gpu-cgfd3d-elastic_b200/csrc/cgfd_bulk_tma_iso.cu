// cgfd_bulk_tma_iso.cu -- the bulk RK-stage kernel's instantiations for the iso medium (every
// operator direction, coefficient storage, wave policy, PML / interior variant and tile shape).
#include "cgfd_bulk_tma.cuh"

namespace cgfd {
template int launch_bulk_tma_med<MED_ISO>(int, int, int, const StageP &, const TmaP &, const BulkTiles &,
                                         cudaStream_t);
template cudaError_t prepare_bulk_tma_med<MED_ISO>(int, int, int);
}  // namespace cgfd
