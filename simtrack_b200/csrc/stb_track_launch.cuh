// Launch code of the tracking kernel, shared by the strict translation unit
// (stb_track.cu, compiled with -fmad=false: every FP64 add and multiply
// rounds separately, as in the reference) and the fast one
// (stb_track_fast.cu, compiled with -fmad=true: the compiler may contract a
// multiply and an add into one FMA).  Internal linkage: each unit gets its
// own kernel instantiations.
#pragma once
#include <cuda_runtime.h>

#include "stb_track_impl.cuh"

namespace stb {
namespace {

// Persistent grid: as many CTAs as fit on the device at once (never more
// than the particles need); each CTA strides over the particle range.
template <bool kSmem, int kBlock, int kMinBlocks, int kPPT, bool kDump, bool kPF = false, bool kSeg = false,
          bool kRad = false>
cudaError_t launch_variant(const TrackArgs &a, int num_sms, size_t smem, cudaStream_t stream) {
  auto kern = track_kernel<kSmem, kBlock, kMinBlocks, kPPT, kDump, kPF, kSeg, kRad>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const long chunk = (long)kBlock * kPPT;
  long need = (a.n + chunk - 1) / chunk;
  long grid = (long)num_sms * per_sm;
  if (grid > need) grid = need;
  kern<<<(unsigned)grid, kBlock, smem, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_track_variants(const TrackArgs &a, int num_sms, int variant, cudaStream_t stream) {
  const size_t sm = track_smem_bytes(a.nelem, a.npool_padded);
  const size_t sg = 2 * (size_t)a.seg_bytes;  // two segment buffers
  const bool seg_ok = a.segs != nullptr && a.nseg > 0 && a.seg_bytes > 0;
  if (kVariants[variant < 0 || variant >= kNumTrackVariants ? 0 : variant].seg && !seg_ok)
    return cudaErrorInvalidValue;
  if (a.dump) {
    // Per-element probe (diagnostics and parity tests): small particle counts
    // only; through the segment buffers when the table is tracked that way.
    if (seg_ok && kVariants[variant].seg)
      return launch_variant<true, 256, 1, 1, true, false, true, true>(a, num_sms, sg, stream);
    return launch_variant<false, 256, 1, 1, true, false, false, true>(a, num_sms, 0, stream);
  }
  // Tables with radiating elements run the one instantiation that carries the
  // radiating maps (the shape of l1_b256_r128), whatever the variant.
  if (a.radiate) return launch_variant<false, 256, 2, 1, false, false, false, true>(a, num_sms, 0, stream);
  switch (variant) {
    case 0: return launch_variant<true, 512, 1, 1, false>(a, num_sms, sm, stream);
    case 1: return launch_variant<true, 1024, 1, 1, false>(a, num_sms, sm, stream);
    case 2: return launch_variant<true, 768, 1, 1, false>(a, num_sms, sm, stream);
    case 3: return launch_variant<false, 256, 2, 1, false>(a, num_sms, 0, stream);
    case 4: return launch_variant<false, 256, 3, 1, false>(a, num_sms, 0, stream);
    case 5: return launch_variant<false, 256, 4, 1, false>(a, num_sms, 0, stream);
    case 6: return launch_variant<false, 384, 2, 1, false>(a, num_sms, 0, stream);
    case 7: return launch_variant<true, 512, 1, 2, false>(a, num_sms, sm, stream);
    case 8: return launch_variant<false, 128, 3, 2, false>(a, num_sms, 0, stream);
    case 9: return launch_variant<true, 1024, 1, 1, false, true>(a, num_sms, sm, stream);
    case 10: return launch_variant<true, 768, 1, 1, false, true>(a, num_sms, sm, stream);
    case 11: return launch_variant<true, 1024, 1, 1, false, false, true>(a, num_sms, sg, stream);
    case 12: return launch_variant<true, 768, 1, 1, false, false, true>(a, num_sms, sg, stream);
    case 13: return launch_variant<true, 512, 1, 1, false, false, true>(a, num_sms, sg, stream);
    case 14: return launch_variant<true, 256, 1, 1, false>(a, num_sms, sm, stream);
    case 15: return launch_variant<true, 128, 1, 1, false>(a, num_sms, sm, stream);
    case 16: return launch_variant<true, 896, 1, 1, false>(a, num_sms, sm, stream);
    case 17: return launch_variant<true, 640, 1, 1, false>(a, num_sms, sm, stream);
    default: return cudaErrorInvalidValue;
  }
}


}  // namespace
}  // namespace stb
