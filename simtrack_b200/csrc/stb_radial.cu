// Track_Radial (simtrack.cpp:21641-21680) on the GPU.
//
// Track_Radial tracks like Track() but, after every element j, subtracts
// from z the path-length change x04[j] of the on-momentum reference particle
// through that element, so that z measures the offset from the on-momentum
// closed path.  x04 comes from one pass of a particle that starts at zero and
// has z and pt reset to zero before every element (simtrack.cpp:21652-21657):
// radial_ref_kernel computes it with one thread, then radial_track_kernel
// tracks the particles (one per thread) through the same element maps as
// the plain tracker.
#include <cuda_runtime.h>

#include <cstdint>

#include "stb_track_impl.cuh"

namespace stb {
namespace {

__global__ void radial_ref_kernel(const __grid_constant__ TrackArgs a, double *zsub) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const RefConsts &R = a.ref;
  Particle p[1] = {Particle{0., 0., 0., 0., 0., 0.}};
  PtCache c[1];
  for (int j = 0; j < a.nelem; j++) {
    p[0].z = 0.;
    p[0].pt = 0.;
    pt_refresh(R, 0.0, c[0]);
    const ElemHeader h = a.hdr[j];
    apply_element<1>(h, a.pool + h.poff, p, c, R);
    zsub[j] = p[0].z;
  }
}

// Cal_dz0_OnMomentumPart (simtrack.cpp:20929-20940): the particle x0 (six
// coordinates, in/out) passes every element with z and pt reset to zero
// before it; dz0[j] = its z after element j.  One device thread.
__global__ void onmom_dz0_kernel(const __grid_constant__ TrackArgs a, double *x0, double *dz0) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const RefConsts &R = a.ref;
  Particle p[1] = {Particle{x0[0], x0[1], x0[2], x0[3], x0[4], x0[5]}};
  PtCache c[1];
  for (int j = 0; j < a.nelem; j++) {
    p[0].z = 0.;
    p[0].pt = 0.;
    pt_refresh(R, 0.0, c[0]);
    const ElemHeader h = a.hdr[j];
    apply_element<1>(h, a.pool + h.poff, p, c, R);
    dz0[j] = p[0].z;
  }
  x0[0] = p[0].x; x0[1] = p[0].px; x0[2] = p[0].y; x0[3] = p[0].py; x0[4] = p[0].z; x0[5] = p[0].pt;
}

template <bool kSmem, int kBlock, bool kDump>
__global__ void __launch_bounds__(kBlock, 1) radial_track_kernel(const __grid_constant__ TrackArgs a,
                                                                  const double *zsub) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  const ElemHeader *hdr = a.hdr;
  const double *pool = a.pool;
  if (kSmem) {
    if (!stage_table(a, smem, &bar)) {
      if (threadIdx.x == 0) atomicExch(a.status, STB_ETIMEOUT);
      return;
    }
    hdr = reinterpret_cast<const ElemHeader *>(smem);
    pool = reinterpret_cast<const double *>(smem + (size_t)a.nelem * sizeof(ElemHeader));
  }
  const RefConsts &R = a.ref;
  for (long i = (long)blockIdx.x * kBlock + threadIdx.x; i < a.n; i += (long)gridDim.x * kBlock) {
    if (a.lost_turn[i] >= 0) continue;
    Particle p[1];
    PtCache c[1];
    p[0] = Particle{a.x[i], a.px[i], a.y[i], a.py[i], a.z[i], a.pt[i]};
    // Track_Radial()'s entry quick check, simtrack.cpp:21647-21649
    if (a.turn0 == 0 && (fabs(p[0].x) > 0.1 || fabs(p[0].y) > 0.1)) {
      a.lost_turn[i] = 0;
      a.lost_elem[i] = 0;
      continue;
    }
    pt_refresh(R, p[0].pt, c[0]);
    int lt = -1, le = 0;
    for (int t = 0; t < a.nturn && lt < 0; t++) {
      for (int e = 0; e < a.nelem; e++) {
        const ElemHeader h = hdr[e];
        apply_element<1>(h, pool + h.poff, p, c, R);
        p[0].z = p[0].z - zsub[e];
        if (kDump) {
          double *d = a.dump + (((size_t)i * a.nturn + t) * a.nelem + e) * 6;
          d[0] = p[0].x; d[1] = p[0].px; d[2] = p[0].y; d[3] = p[0].py; d[4] = p[0].z; d[5] = p[0].pt;
        }
        if (needs_loss_check(h) && is_lost(p[0], h.apx, h.apy, a.r2, a.loss_mode)) {
          lt = a.turn0 + t;
          le = e;
          break;
        }
      }
    }
    a.x[i] = p[0].x;
    a.px[i] = p[0].px;
    a.y[i] = p[0].y;
    a.py[i] = p[0].py;
    a.z[i] = p[0].z;
    a.pt[i] = p[0].pt;
    if (lt >= 0) {
      a.lost_turn[i] = lt;
      a.lost_elem[i] = le;
    }
  }
}

template <bool kSmem, int kBlock, bool kDump>
cudaError_t launch_radial_variant(const TrackArgs &a, const double *zsub, int num_sms, size_t smem,
                                  cudaStream_t stream) {
  auto kern = radial_track_kernel<kSmem, kBlock, kDump>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  long need = (a.n + kBlock - 1) / kBlock;
  long grid = (long)num_sms * per_sm;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, kBlock, smem, stream>>>(a, zsub);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_radial_reference(const TrackArgs &a, double *zsub, cudaStream_t stream) {
  radial_ref_kernel<<<1, 32, 0, stream>>>(a, zsub);
  return cudaGetLastError();
}

cudaError_t launch_onmom_dz0(const TrackArgs &a, double *x0, double *dz0, cudaStream_t stream) {
  onmom_dz0_kernel<<<1, 32, 0, stream>>>(a, x0, dz0);
  return cudaGetLastError();
}

cudaError_t launch_radial(const TrackArgs &a, const double *zsub, int num_sms, bool use_smem, cudaStream_t stream) {
  if (a.n <= 0 || a.nturn <= 0) return cudaSuccess;
  if (a.dump) return launch_radial_variant<false, 256, true>(a, zsub, num_sms, 0, stream);
  if (use_smem)
    return launch_radial_variant<true, 1024, false>(a, zsub, num_sms, track_smem_bytes(a.nelem, a.npool_padded),
                                                    stream);
  return launch_radial_variant<false, 256, false>(a, zsub, num_sms, 0, stream);
}

}  // namespace stb
