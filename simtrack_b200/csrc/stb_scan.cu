// Batched dynamic-aperture scan: many lattices (one per field-error seed) x
// per-seed particle grids, tracked turn block by turn block on one GPU.
//
// Per turn block (all device-side, so a block of them is captured once in a
// CUDA graph and replayed):
//   1. scan_worklist_kernel  builds the work list: for every seed, its live
//      particles (always the first live[s] slots of the seed's range) are cut
//      into chunks of `chunk` particles; items are (seed, first slot).
//   2. scan_track_kernel     persistent CTAs pull items from an atomic
//      counter, stage that seed's element table into shared memory when it
//      differs from the one already staged (bulk TMA copies), and track the
//      item's particles for `nturn` turns starting at the device turn counter.
//   3. scan_compact_kernel   one CTA per seed stably compacts the seed's live
//      particles to the front of its range (warp ballots + a block prefix
//      sum), writes the final state of every particle lost in this block to
//      the outputs (indexed by original particle id) and advances the turn
//      counter.
// Dead lanes therefore stop costing cycles at the next turn-block boundary,
// and the work list shrinks with the uneven survival of the seeds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "stb_scan.hpp"
#include "stb_track_impl.cuh"

namespace stb {

namespace {

constexpr int kCompactBlock = 1024;

// Work-item size adapts to the live population: with few survivors the items
// shrink (down to one warp) so that they still spread over every resident
// CTA; with many they grow up to the configured chunk.  In packed mode the
// items keep the full chunk, so a small population occupies few SMs with many
// warps each: latency-bound tails run faster that way when warps that walk
// the same element sequence share their SM's instruction fetches.
__global__ void scan_worklist_kernel(ScanArgs a) {
  __shared__ int pre[kMaxScanSeeds + 1];
  __shared__ int chunk_s;
  __shared__ int abort_s;
  const int s = threadIdx.x;
  // The caller's abort flag is read once per turn block: a set flag empties
  // the work list, so the block tracks nothing and (through block_skipped)
  // leaves the turn counter where it is; the state stays resumable.
  if (s == 0) {
    abort_s = (a.abort && *a.abort != 0) ? 1 : 0;
    *a.block_skipped = abort_s;
    if (abort_s) {
      *a.n_items = 0;
      *a.next_item = 0;
    }
  }
  __syncthreads();
  if (abort_s) return;
  const int lv = s < a.nseed ? a.live[s] : 0;
  // total live particles (block reduction through the prefix array)
  pre[s + 1] = lv;
  if (s == 0) pre[0] = 0;
  __syncthreads();
  for (int off = 1; off <= a.nseed; off <<= 1) {
    int v = 0;
    if (s + 1 > off && s < a.nseed) v = pre[s + 1 - off];
    __syncthreads();
    if (s < a.nseed) pre[s + 1] += v;
    __syncthreads();
  }
  if (s == 0) {
    const long total = pre[a.nseed];
    long c = (total + a.grid - 1) / (a.grid > 0 ? a.grid : 1);
    c = ((c + 31) / 32) * 32;
    if (c < 32) c = 32;
    if (c > a.chunk || a.pack) c = a.chunk;
    chunk_s = (int)c;
  }
  __syncthreads();
  const int chunk = chunk_s;
  const int n = s < a.nseed ? (lv + chunk - 1) / chunk : 0;
  __syncthreads();
  pre[s + 1] = n;
  __syncthreads();
  for (int off = 1; off <= a.nseed; off <<= 1) {
    int v = 0;
    if (s + 1 > off && s < a.nseed) v = pre[s + 1 - off];
    __syncthreads();
    if (s < a.nseed) pre[s + 1] += v;
    __syncthreads();
  }
  if (s < a.nseed) {
    const int base = pre[s + 1] - n;
    for (int k = 0; k < n; k++) {
      a.items[2 * (base + k)] = s;
      a.items[2 * (base + k) + 1] = k * chunk;
    }
  }
  if (s == 0) {
    *a.n_items = pre[a.nseed];
    *a.next_item = 0;
    *a.item_chunk = chunk;
  }
}

template <bool kSmem, int kBlock, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks) scan_track_kernel(const __grid_constant__ ScanArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int item_s;
  const RefConsts &R = a.ref;
  const int turn0 = *a.turn0;
  const int n_items = *a.n_items;
  const int chunk = *a.item_chunk;
  int staged = -1;
  uint32_t phase = 0;
  for (;;) {
    if (threadIdx.x == 0) item_s = atomicAdd(a.next_item, 1);
    __syncthreads();
    const int item = item_s;
    __syncthreads();
    if (item >= n_items) break;
    const int s = a.items[2 * item];
    const int first = a.items[2 * item + 1];
    const ScanSeed sd = a.seeds[s];
    const ElemHeader *hdr = sd.hdr;
    const double *pool = sd.pool;
    if (kSmem) {
      if (s != staged) {
        if (!stage_table_ptr(sd.hdr, sd.nelem, sd.pool, sd.npool_padded, smem, &bar, phase, staged < 0)) {
          if (threadIdx.x == 0) atomicExch(a.status, STB_ETIMEOUT);
          return;
        }
        phase ^= 1u;
        staged = s;
      }
      hdr = reinterpret_cast<const ElemHeader *>(smem);
      pool = reinterpret_cast<const double *>(smem + (size_t)sd.nelem * sizeof(ElemHeader));
    }
    const int live = a.live[s];
    for (int j = threadIdx.x; j < chunk; j += kBlock) {
      const int slot_in_seed = first + j;
      if (slot_in_seed >= live) continue;
      const long i = sd.off + slot_in_seed;
      if (a.lost_turn[i] >= 0) continue;
      Particle p[1];
      PtCache c[1];
      p[0].x = a.x[i];
      p[0].px = a.px[i];
      p[0].y = a.y[i];
      p[0].py = a.py[i];
      p[0].z = a.z[i];
      p[0].pt = a.pt[i];
      // Track()'s entry quick check, simtrack.cpp:20795-20796
      if (turn0 == 0 && (fabs(p[0].x) > 0.1 || fabs(p[0].y) > 0.1)) {
        a.lost_turn[i] = 0;
        a.lost_elem[i] = 0;
        continue;
      }
      pt_refresh(R, p[0].pt, c[0]);
      int lt = -1, le = 0;
      const long id = a.tbt ? (long)a.id[i] : 0;
      for (int t = 0; t < a.nturn && lt < 0; t++) {
        for (int e = 0; e < sd.nelem; e++) {
          const ElemHeader h = hdr[e];
          apply_element<1, (kBlock >= 512)>(h, pool + h.poff, p, c, R);
          if (needs_loss_check(h) && is_lost(p[0], h.apx, h.apy, a.r2, a.loss_mode)) {
            lt = turn0 + t;
            le = e;
            break;
          }
        }
        const int tg = turn0 + t;
        if (a.tbt && lt < 0 && tg < a.tbt_turns) {
          double *d = a.tbt + (size_t)tg * 4 * a.ntot + id;
          d[0] = p[0].x;
          d[a.ntot] = p[0].px;
          d[2 * a.ntot] = p[0].y;
          d[3 * a.ntot] = p[0].py;
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
    __syncthreads();
  }
}

__device__ __forceinline__ void write_output(const ScanArgs &a, long slot, int lt, int le) {
  const long o = a.id[slot];
  a.out_lost_turn[o] = lt;
  a.out_lost_elem[o] = le;
  double *x = a.out_x + 6 * o;
  x[0] = a.x[slot];
  x[1] = a.px[slot];
  x[2] = a.y[slot];
  x[3] = a.py[slot];
  x[4] = a.z[slot];
  x[5] = a.pt[slot];
}

// Stable compaction of every seed's live slots [off, off + live) in three
// passes over windows of kCompactWindow slots, one CTA per (window, seed), so
// that it runs on every SM whatever the number of seeds:
//   1. count:   the survivors of each window (a block-wide count); particles
//               lost in this block get their outputs (indexed by original id);
//   2. gather:  each window's survivors, ranked by warp ballots and a block
//               prefix over warps, go to the staging arrays at the seed offset
//               plus the survivors of the windows before it;
//   3. back:    the seed's first `survivors` slots are copied back from the
//               staging arrays and marked alive; the live count and the turn
//               counter are updated.
// Order within a seed is kept, so results equal those of tracking each seed
// alone.
__global__ void __launch_bounds__(kCompactBlock) compact_count_kernel(ScanArgs a) {
  const int s = blockIdx.y, w = blockIdx.x;
  const ScanSeed sd = a.seeds[s];
  const int live = a.live[s];
  const int j = w * kCompactWindow + threadIdx.x;
  bool keep = false;
  if (j < live) {
    const long src = sd.off + j;
    const int lt = a.lost_turn[src];
    if (lt >= 0) write_output(a, src, lt, a.lost_elem[src]);
    keep = lt < 0;
  }
  const int c = __syncthreads_count(keep);
  if (threadIdx.x == 0) a.win_count[s * a.nwin + w] = w * kCompactWindow < live ? c : 0;
}

// Sum of win_count[s][0, upto) by the whole block.
__device__ __forceinline__ int windows_before(const ScanArgs &a, int s, int upto, int *red) {
  int acc = 0;
  for (int k = threadIdx.x; k < upto; k += kCompactBlock) acc += a.win_count[s * a.nwin + k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  int tot = 0;
  for (int k = 0; k < kCompactBlock / 32; k++) tot += red[k];
  __syncthreads();
  return tot;
}

__global__ void __launch_bounds__(kCompactBlock) compact_gather_kernel(ScanArgs a) {
  constexpr int kWarps = kCompactBlock / 32;
  __shared__ int red[kWarps];
  __shared__ int warp_off[kWarps];
  const int s = blockIdx.y, w = blockIdx.x;
  const ScanSeed sd = a.seeds[s];
  const int live = a.live[s];
  if (w * kCompactWindow >= live) return;
  const int base = windows_before(a, s, w, red);
  const int j = w * kCompactWindow + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long src = sd.off + j;
  const bool keep = j < live && a.lost_turn[src] < 0;
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) warp_off[warp] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int k = 0; k < kWarps; k++) {
      const int c = warp_off[k];
      warp_off[k] = acc;
      acc += c;
    }
  }
  __syncthreads();
  if (keep) {
    const long dst = sd.off + base + warp_off[warp] + __popc(m & ((1u << lane) - 1u));
    const long n = a.ntot;
    a.stage[dst] = a.x[src];
    a.stage[n + dst] = a.px[src];
    a.stage[2 * n + dst] = a.y[src];
    a.stage[3 * n + dst] = a.py[src];
    a.stage[4 * n + dst] = a.z[src];
    a.stage[5 * n + dst] = a.pt[src];
    a.stage_id[dst] = a.id[src];
  }
}

__global__ void __launch_bounds__(kCompactBlock) compact_back_kernel(ScanArgs a) {
  __shared__ int red[kCompactBlock / 32];
  const int s = blockIdx.y, w = blockIdx.x;
  const ScanSeed sd = a.seeds[s];
  const int live = a.live[s];
  if (w * kCompactWindow >= live) return;  // every block of this seed sees the old live count
  const int total = windows_before(a, s, a.nwin, red);
  const int j = w * kCompactWindow + threadIdx.x;
  if (j < total) {
    const long i = sd.off + j;
    const long n = a.ntot;
    a.x[i] = a.stage[i];
    a.px[i] = a.stage[n + i];
    a.y[i] = a.stage[2 * n + i];
    a.py[i] = a.stage[3 * n + i];
    a.z[i] = a.stage[4 * n + i];
    a.pt[i] = a.stage[5 * n + i];
    a.id[i] = a.stage_id[i];
    a.lost_turn[i] = -1;
    a.lost_elem[i] = 0;
  }
}

// Live counts and the turn counter, after every window of every seed is back.
__global__ void compact_finish_kernel(ScanArgs a) {
  __shared__ int red[kCompactBlock / 32];
  const int s = blockIdx.x;
  const int total = windows_before(a, s, a.nwin, red);
  if (threadIdx.x == 0) {
    a.live[s] = total;
    if (s == 0 && *a.block_skipped == 0) *a.turn0 += a.nturn;
  }
}

cudaError_t launch_compaction(const ScanArgs &a, cudaStream_t st) {
  const dim3 grid((unsigned)a.nwin, (unsigned)a.nseed);
  compact_count_kernel<<<grid, kCompactBlock, 0, st>>>(a);
  compact_gather_kernel<<<grid, kCompactBlock, 0, st>>>(a);
  compact_back_kernel<<<grid, kCompactBlock, 0, st>>>(a);
  compact_finish_kernel<<<a.nseed, kCompactBlock, 0, st>>>(a);
  return cudaGetLastError();
}

__global__ void scan_retire_kernel(ScanArgs a, const uint8_t *mask) {
  const int s = blockIdx.y;
  const ScanSeed sd = a.seeds[s];
  const int live = a.live[s];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < live; j += gridDim.x * blockDim.x) {
    const long i = sd.off + j;
    if (a.lost_turn[i] < 0 && mask[a.id[i]]) {
      a.lost_turn[i] = kRetiredCode;
      a.lost_elem[i] = 0;
    }
  }
}

// Particles still alive at the end of the run: outputs with lost_turn = -1.
__global__ void scan_finalize_kernel(ScanArgs a) {
  const int s = blockIdx.y;
  const ScanSeed sd = a.seeds[s];
  const int live = a.live[s];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < live; j += gridDim.x * blockDim.x)
    write_output(a, sd.off + j, -1, 0);
}

template <bool kSmem, int kBlock, int kMinBlocks>
cudaError_t prepare_scan_variant(int num_sms, size_t smem, int *grid) {
  auto kern = scan_track_kernel<kSmem, kBlock, kMinBlocks>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  *grid = num_sms * per_sm;
  return cudaSuccess;
}

}  // namespace

const ScanVariant kScanVariants[kNumScanVariants] = {
    {true, 1024, 1, "smem_b1024_r64"}, {true, 512, 1, "smem_b512_r128"}, {false, 256, 4, "l1_b256_r64"},
    {false, 256, 3, "l1_b256_r80"},    {false, 128, 8, "l1_b128_r64"},    {false, 256, 2, "l1_b256_r128"},
    {false, 128, 2, "l1_b128_r255"},   {true, 256, 1, "smem_b256_r255"},  {true, 128, 1, "smem_b128_r255"},
};

cudaError_t prepare_scan(int variant, int num_sms, size_t smem, int *grid) {
  switch (variant) {
    case 0: return prepare_scan_variant<true, 1024, 1>(num_sms, smem, grid);
    case 1: return prepare_scan_variant<true, 512, 1>(num_sms, smem, grid);
    case 2: return prepare_scan_variant<false, 256, 4>(num_sms, 0, grid);
    case 3: return prepare_scan_variant<false, 256, 3>(num_sms, 0, grid);
    case 4: return prepare_scan_variant<false, 128, 8>(num_sms, 0, grid);
    case 5: return prepare_scan_variant<false, 256, 2>(num_sms, 0, grid);
    case 6: return prepare_scan_variant<false, 128, 2>(num_sms, 0, grid);
    case 7: return prepare_scan_variant<true, 256, 1>(num_sms, smem, grid);
    case 8: return prepare_scan_variant<true, 128, 1>(num_sms, smem, grid);
    default: return cudaErrorInvalidValue;
  }
}

// Only kernel launches: safe inside stream capture (prepare_scan ran before).
cudaError_t launch_scan_block(const ScanArgs &a, int variant, int grid, size_t smem, cudaStream_t st) {
  scan_worklist_kernel<<<1, 1024, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  switch (variant) {
    case 0: scan_track_kernel<true, 1024, 1><<<grid, 1024, smem, st>>>(a); break;
    case 1: scan_track_kernel<true, 512, 1><<<grid, 512, smem, st>>>(a); break;
    case 2: scan_track_kernel<false, 256, 4><<<grid, 256, 0, st>>>(a); break;
    case 3: scan_track_kernel<false, 256, 3><<<grid, 256, 0, st>>>(a); break;
    case 4: scan_track_kernel<false, 128, 8><<<grid, 128, 0, st>>>(a); break;
    case 5: scan_track_kernel<false, 256, 2><<<grid, 256, 0, st>>>(a); break;
    case 6: scan_track_kernel<false, 128, 2><<<grid, 128, 0, st>>>(a); break;
    case 7: scan_track_kernel<true, 256, 1><<<grid, 256, smem, st>>>(a); break;
    case 8: scan_track_kernel<true, 128, 1><<<grid, 128, smem, st>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_compaction(a, st);
}

cudaError_t launch_scan_compact_only(const ScanArgs &a, cudaStream_t st) { return launch_compaction(a, st); }

cudaError_t launch_scan_track_only(const ScanArgs &a, int variant, int grid, size_t smem, cudaStream_t st) {
  scan_worklist_kernel<<<1, 1024, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  switch (variant) {
    case 0: scan_track_kernel<true, 1024, 1><<<grid, 1024, smem, st>>>(a); break;
    case 2: scan_track_kernel<false, 256, 4><<<grid, 256, 0, st>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_scan_retire(const ScanArgs &a, const uint8_t *mask, long max_per_seed, cudaStream_t st) {
  dim3 grid((unsigned)std::max<long>(1, std::min<long>((max_per_seed + 255) / 256, 64)), (unsigned)a.nseed);
  scan_retire_kernel<<<grid, 256, 0, st>>>(a, mask);
  return cudaGetLastError();
}

cudaError_t launch_scan_finalize(const ScanArgs &a, long max_per_seed, cudaStream_t st) {
  dim3 grid((unsigned)std::max<long>(1, std::min<long>((max_per_seed + 255) / 256, 64)), (unsigned)a.nseed);
  scan_finalize_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace stb
