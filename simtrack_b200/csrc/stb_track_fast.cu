// The tracking kernel with FMA contraction allowed (this unit is compiled
// with -fmad=true; stb_track.cu, the strict kernel, with -fmad=false).
//
// Same maps, same launch variants, same loss bookkeeping.  Where a map
// multiplies and then adds, the compiler may issue one fused multiply-add
// with a single rounding, so results differ from the reference's in the last
// bits and chaotic trajectories drift apart over many turns; the strict
// kernel remains the one compared with the reference element by element.
// Selected per table with stb_table_set_contraction.
#include <cuda_runtime.h>

#include "stb_track_launch.cuh"

namespace stb {

cudaError_t launch_track_fast(const TrackArgs &a, int num_sms, int variant, cudaStream_t stream) {
  return launch_track_variants(a, num_sms, variant, stream);
}

}  // namespace stb
