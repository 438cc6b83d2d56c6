// Internal runtime pieces shared by the C ABI translation units: the table
// object, status-code plumbing and CUDA error handling.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "simtrack_b200.hpp"
#include "stb_flatten.hpp"
#include "stb_kernels.hpp"
#include "stb_status.hpp"

struct stb_table {
  int device = 0;
  stb::HostTable host;
  stb::ElemHeader *d_hdr = nullptr;
  double *d_pool = nullptr;
  int npool_padded = 0;
  bool use_smem = false;  // the table fits the shared-memory variants
  int variant = 2;        // launch variant (stb::kVariants), set by the autotuner
  bool fast = false;      // FMA-contracted kernel (stb_table_set_contraction) instead of the strict one
  double min_ap2 = 0.;    // min over loss-checked elements of RN(APx^2), RN(APy^2) (loss_mode_for)
  // Segment plan for tables that do not fit shared memory whole (seg_*
  // launch variants): segments of at most seg_bytes bytes each.
  stb::SegDesc *d_segs = nullptr;
  int nseg = 0;
  int seg_bytes = 0;
  int *d_status = nullptr;
  int num_sms = 0;
  double *d_zsub = nullptr;  // Track_Radial's per-element on-momentum z (computed on first use)
  // Host-buffer entry points (stb_track_host): device staging grown on
  // demand and kept with the table, and the stream their copies and kernels
  // run on (created on first use).
  void *d_io = nullptr;
  size_t io_cap = 0;  // particles d_io holds
  cudaStream_t io_stream = nullptr;
};

namespace stb {

// Runs f(), mapping exceptions onto status codes and the thread's message.
template <class F>
int guarded(F &&f) {
  try {
    int rc = f();
    if (rc == STB_OK) set_last_error("");
    return rc;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return STB_ENOMEM;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return STB_EINVAL;
  }
}

inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? STB_ENOMEM : STB_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// One launch of nturn turns from turn0 on the probe variant of the tracking
// kernel, which writes dump[((i*nturn + turn)*nelem + j)*6 + k] after every
// element j (no circular aperture); default stream, asynchronous.
void track_device_dump(stb_table *t, double *const c[6], long n, int turn0, int nturn, int32_t *lost_turn,
                       int32_t *lost_elem, double *dump);
// The same for spin tracking (a spin table, nine arrays, dump[...*9 + k]).
void spin_device_dump(stb_table *t, double *const c[9], long n, int turn0, int nturn, int32_t *lost_turn,
                      int32_t *lost_elem, double *dump);

// Track()'s entry quick check (simtrack.cpp:20795-20796; the same in
// Track_Radial and Track_Spin): a particle whose input flag is 0 or whose
// |x| or |y| exceeds 0.1 m is lost at turn 0, element 0, whatever nturn is.
inline bool entry_rejected(const double *x, int stable) {
  return stable == 0 || std::fabs(x[0]) > 0.1 || std::fabs(x[2]) > 0.1;
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cuda_check(cudaGetDevice(&prev), "cudaGetDevice");
    if (prev != dev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
  }
};

// cudaFree on scope exit.
struct DevFree {
  void *p;
  ~DevFree() {
    if (p) cudaFree(p);
  }
};

}  // namespace stb
