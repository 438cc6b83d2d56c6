// FP64 element-by-element tracking kernel for sm_100a.
//
// One thread carries one particle through a block of turns with its six
// coordinates and pt-only cache in registers; particles are stored as SoA
// FP64 arrays so every load/store of a warp is one coalesced 256-byte
// transaction per coordinate.  All lanes of a warp walk the same element
// sequence, so element dispatch is warp-uniform; a lane whose particle is
// lost leaves the loops and idles until the compaction pass (stb_compact.cu)
// removes it between turn blocks.
//
// The element table (headers + parameter pool, built by stb_flatten.cpp) is
// staged into shared memory once per CTA with bulk TMA copies
// (cp.async.bulk, completion on an mbarrier, bounded wait) when it fits the
// shared-memory budget; otherwise the kernel reads it through the read-only
// data cache.  The Track() loss convention (simtrack.cpp:20791-20814) is
// applied after every element: |x| > APx, |y| > APy, isnan(x), isnan(y),
// plus an optional circular aperture.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "stb_track_launch.cuh"

namespace stb {

size_t track_smem_bytes(int nelem, int npool_padded) {
  return (size_t)nelem * sizeof(ElemHeader) + (size_t)npool_padded * 8;
}

int track_smem_limit(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return 0;
  return v - 1024;  // static shared memory and the mbarrier
}

// Launch variants the autotuner chooses from: element table in shared
// memory or read through L1, CTA size, minimum resident CTAs per SM (which
// caps registers per thread at 65536 / (block * min_blocks)) and particles
// per thread.
const TrackVariant kVariants[kNumTrackVariants] = {
    {true, false, 512, 1, 1, "smem_b512_r128", false},      {true, false, 1024, 1, 1, "smem_b1024_r64", false},
    {true, false, 768, 1, 1, "smem_b768_r85", false},       {false, false, 256, 2, 1, "l1_b256_r128", false},
    {false, false, 256, 3, 1, "l1_b256_r80", false},        {false, false, 256, 4, 1, "l1_b256_r64", false},
    {false, false, 384, 2, 1, "l1_b384_r85", false},        {true, false, 512, 1, 2, "smem_b512_r128_ppt2", false},
    {false, false, 128, 3, 2, "l1_b128_r168_ppt2", false},  {true, false, 1024, 1, 1, "smem_b1024_r64_pf", true},
    {true, false, 768, 1, 1, "smem_b768_r85_pf", true},     {true, true, 1024, 1, 1, "seg_b1024_r64", false},
    {true, true, 768, 1, 1, "seg_b768_r85", false},         {true, true, 512, 1, 1, "seg_b512_r128", false},
    {true, false, 256, 1, 1, "smem_b256_r255", false},      {true, false, 128, 1, 1, "smem_b128_r255", false},
    {true, false, 896, 1, 1, "smem_b896_r72", false},       {true, false, 640, 1, 1, "smem_b640_r96", false},
};

// Segments of at most `budget` bytes each (headers plus the 16-byte aligned
// pool slice), in element order; empty when one element alone exceeds it.
std::vector<SegDesc> plan_segments(const ElemHeader *hdr, int nelem, int npool_padded, size_t budget) {
  std::vector<SegDesc> out;
  int e0 = 0;
  auto pool_end = [&](int e) { return e + 1 < nelem ? hdr[e + 1].poff : npool_padded; };
  while (e0 < nelem) {
    const int lo = hdr[e0].poff & ~1;
    int e1 = e0;
    while (e1 < nelem) {
      const int hi = (pool_end(e1) + 1) & ~1;
      const size_t b = (size_t)(e1 - e0 + 1) * sizeof(ElemHeader) + (size_t)(hi - lo) * 8;
      if (b > budget) break;
      e1++;
    }
    if (e1 == e0) return {};
    const int hi = (pool_end(e1 - 1) + 1) & ~1;
    out.push_back(SegDesc{e0, e1 - e0, lo, hi - lo});
    e0 = e1;
  }
  return out;
}

cudaError_t launch_track(const TrackArgs &a, int num_sms, int variant, cudaStream_t stream) {
  return launch_track_variants(a, num_sms, variant, stream);
}

namespace {

__global__ void aos_to_soa_kernel(const double *__restrict__ aos, const int32_t *__restrict__ stable, long n,
                                  int nc, double *__restrict__ soa, int32_t *__restrict__ lost_turn,
                                  int32_t *__restrict__ lost_elem) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double *q = aos + (size_t)nc * i;
    for (int k = 0; k < nc; k++) soa[(size_t)k * n + i] = q[k];
    // Track()'s entry quick check, simtrack.cpp:20795-20796
    lost_turn[i] = (stable[i] == 0 || fabs(q[0]) > 0.1 || fabs(q[2]) > 0.1) ? 0 : -1;
    lost_elem[i] = 0;
  }
}

__global__ void soa_to_aos_kernel(const double *__restrict__ soa, const int32_t *__restrict__ lost_turn,
                                  const int32_t *__restrict__ lost_elem, long n, int nc, double *__restrict__ aos,
                                  int32_t *__restrict__ stable, int32_t *__restrict__ lost_turn_out,
                                  int32_t *__restrict__ lost_post) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double *q = aos + (size_t)nc * i;
    for (int k = 0; k < nc; k++) q[k] = soa[(size_t)k * n + i];
    const int32_t t = lost_turn[i];
    stable[i] = t < 0 ? 1 : 0;
    lost_turn_out[i] = t < 0 ? 0 : t;
    lost_post[i] = t < 0 ? 0 : lost_elem[i];
  }
}

unsigned io_grid(long n) {
  long g = (n + 255) / 256;
  return (unsigned)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

cudaError_t launch_aos_to_soa(const double *aos, const int32_t *stable, long n, int nc, double *soa,
                              int32_t *lost_turn, int32_t *lost_elem, cudaStream_t s) {
  aos_to_soa_kernel<<<io_grid(n), 256, 0, s>>>(aos, stable, n, nc, soa, lost_turn, lost_elem);
  return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const double *soa, const int32_t *lost_turn, const int32_t *lost_elem, long n, int nc,
                              double *aos, int32_t *stable, int32_t *lost_turn_out, int32_t *lost_post,
                              cudaStream_t s) {
  soa_to_aos_kernel<<<io_grid(n), 256, 0, s>>>(soa, lost_turn, lost_elem, n, nc, aos, stable, lost_turn_out,
                                               lost_post);
  return cudaGetLastError();
}

}  // namespace stb
