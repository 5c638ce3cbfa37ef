// scan_mma.cu -- tensor-core (tcgen05) form of the pair scan. Not built yet: reports
// itself unavailable so that EPI_FORM_AUTO selects the popcount form.
#include "epi_internal.cuh"

namespace epi {
bool mma_available() { return false; }
int mma_tile_i() { return 1; }
int mma_tile_j() { return 1; }
int mma_min_nid() { return 1 << 30; }
cudaError_t launch_mma(const ScanArgs &, int, cudaStream_t) { return cudaErrorNotSupported; }
}  // namespace epi
