// stb_track_seeds_static: seed-batched tracking whose scratch lives in a
// fixed-size static device array instead of memory allocated per call.
//
// Callers that cannot allocate device memory while tracking (a process whose
// device memory is entirely handed to another allocator's pool, or code that
// must not hit the implicit synchronisation of cudaMalloc/cudaFree between
// kernels) get the work-list tracking of the batched scan here: the seed
// table, per-seed particle counts, the work list, its counters and the status
// word sit in g_static_scratch; the particles stay in the caller's buffers.
//
// Every call looks up the scratch address (cudaGetSymbolAddress, which
// allocates nothing), so the entry point stays valid after a
// cudaDeviceReset reloads the module.  The scratch is shared by all
// calls on a device, so calls that overlap in time on one device (several
// host threads, or several streams without ordering between them) race on it.
// Each call waits for its stream before returning, so sequential calls from
// one thread are safe.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include "stb_runtime.hpp"
#include "stb_scan.hpp"

namespace stb {
namespace {

constexpr int kStaticMaxSeeds = STB_STATIC_MAX_SEEDS;
constexpr long kStaticMaxParticles = STB_STATIC_MAX_PARTICLES;
// A work item holds at least one warp of particles, so a seed of n particles
// yields at most ceil(n / 32) items.
constexpr long kStaticMaxItems = kStaticMaxParticles / 32 + kStaticMaxSeeds;
constexpr int kMaxDevices = 64;

struct StaticScratch {
  ScanSeed seeds[kStaticMaxSeeds];
  int32_t live[kStaticMaxSeeds];
  int32_t ctr[4];  // n_items, next_item, turn0, item_chunk
  int32_t status;
  int32_t block_skipped;  // written by the work-list kernel
  int32_t pad[2];
  int32_t items[2 * kStaticMaxItems];
};

static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

// Everything the init kernel writes, passed by value.
struct StaticInit {
  ScanSeed seeds[kStaticMaxSeeds];
  int nseed;
  int turn0;
};

// Fills the parts of the scratch that must hold defined values before the
// work-list kernel runs: the seed table, live counts (= all slots, lost
// particles are skipped by their lost_turn), the turn counter and the status
// word (zero).  The work-list kernel itself resets n_items and next_item.
__global__ void static_init_kernel(const __grid_constant__ StaticInit in, StaticScratch *sc) {
  const int s = threadIdx.x;
  if (s < in.nseed) {
    sc->seeds[s] = in.seeds[s];
    sc->live[s] = in.seeds[s].cap;
  }
  if (s == 0) {
    sc->ctr[0] = 0;
    sc->ctr[1] = 0;
    sc->ctr[2] = in.turn0;
    sc->ctr[3] = 0;
    sc->status = 0;
  }
}

// The scratch of the current device.
StaticScratch *scratch_for() {
  void *p = nullptr;
  cuda_check(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress(scratch)");
  return static_cast<StaticScratch *>(p);
}

int track_seeds_static(stb_table *const *tables, int nseed, const long *n_per_seed, double *x, double *px,
                       double *y, double *py, double *z, double *pt, int32_t *lost_turn, int32_t *lost_elem,
                       int turn0, int nturn, double radius, cudaStream_t stream) {
  if (!tables || !n_per_seed) throw Error(STB_EINVAL, "NULL argument");
  if (nseed < 1 || nseed > kStaticMaxSeeds)
    throw Error(STB_EINVAL, "seed count out of range (1.." + std::to_string(kStaticMaxSeeds) + ")");
  long total = 0;
  for (int i = 0; i < nseed; i++) {
    if (n_per_seed[i] < 0) throw Error(STB_EINVAL, "negative particle count");
    total += n_per_seed[i];
    if (total > kStaticMaxParticles)
      throw Error(STB_EINVAL, "more than " + std::to_string(kStaticMaxParticles) +
                                  " particles: the static scratch is sized for that many");
  }
  if (nturn < 0 || turn0 < 0) throw Error(STB_EINVAL, "negative turn count");
  if (total == 0 || nturn == 0) return STB_OK;
  if (!x || !px || !y || !py || !z || !pt || !lost_turn || !lost_elem) throw Error(STB_EINVAL, "NULL buffer");
  const int device = tables[0] ? tables[0]->device : -1;
  if (device < 0 || device >= kMaxDevices) throw Error(STB_EINVAL, "bad device");
  StaticInit in;
  std::memset(&in, 0, sizeof(in));
  size_t smem = 0;
  bool smem_ok = true;
  long off = 0;
  for (int i = 0; i < nseed; i++) {
    stb_table *t = tables[i];
    if (!t) throw Error(STB_EINVAL, "NULL table");
    if (t->device != device) throw Error(STB_EINVAL, "all tables must live on one device");
    if (t->host.spin) throw Error(STB_EINVAL, "spin tables need the stb_track_spin_* entry points");
    if (t->host.radiate)
      throw Error(STB_EUNSUPPORTED, "tables flattened with GP.radiate need the stb_track_* entry points");
    if (std::memcmp(&t->host.ref, &tables[0]->host.ref, sizeof(RefConsts)) != 0)
      throw Error(STB_EINVAL, "all tables must be flattened for the same reference particle");
    in.seeds[i] = ScanSeed{t->d_hdr, t->d_pool, (int)t->host.hdr.size(), t->npool_padded, off, (int)n_per_seed[i], 0};
    off += n_per_seed[i];
    smem = std::max(smem, track_smem_bytes((int)t->host.hdr.size(), t->npool_padded));
    smem_ok = smem_ok && t->use_smem;
  }
  in.nseed = nseed;
  in.turn0 = turn0;
  DeviceGuard g(device);
  StaticScratch *sc = scratch_for();
  const int variant = smem_ok ? 0 : 2;
  // Raise (never lower) the kernel's shared-memory limit to the device maximum,
  // so that handles prepared with other table sizes keep working.
  int grid = 0;
  cuda_check(prepare_scan(variant, tables[0]->num_sms, smem_ok ? (size_t)track_smem_limit(device) : 0, &grid),
             "kernel setup");
  ScanArgs a;
  std::memset(&a, 0, sizeof(a));
  a.seeds = sc->seeds;
  a.nseed = nseed;
  a.chunk = kScanVariants[variant].block;
  a.grid = grid;
  a.ref = tables[0]->host.ref;
  a.x = x;
  a.px = px;
  a.y = y;
  a.py = py;
  a.z = z;
  a.pt = pt;
  a.lost_turn = lost_turn;
  a.lost_elem = lost_elem;
  a.live = sc->live;
  a.items = sc->items;
  a.n_items = sc->ctr;
  a.next_item = sc->ctr + 1;
  a.turn0 = sc->ctr + 2;
  a.item_chunk = sc->ctr + 3;
  a.nturn = nturn;
  a.r2 = radius > 0.0 ? radius * radius : INFINITY;
  double min_ap2 = INFINITY;
  for (int i = 0; i < nseed; i++) min_ap2 = std::fmin(min_ap2, tables[i]->min_ap2);
  a.loss_mode = loss_mode_for(a.r2, min_ap2);
  a.status = &sc->status;
  a.ntot = total;
  a.abort = nullptr;
  a.block_skipped = &sc->block_skipped;
  static_init_kernel<<<1, kStaticMaxSeeds, 0, stream>>>(in, sc);
  cuda_check(cudaGetLastError(), "init launch");
  cuda_check(launch_scan_track_only(a, variant, grid, smem_ok ? smem : 0, stream), "tracking launch");
  int status = 0;
  cuda_check(cudaMemcpyAsync(&status, &sc->status, sizeof(int), cudaMemcpyDeviceToHost, stream), "read status");
  cuda_check(cudaStreamSynchronize(stream), "tracking");
  if (status != 0) throw Error(status, "tracking kernel reported status " + std::to_string(status));
  return STB_OK;
}

}  // namespace
}  // namespace stb

extern "C" int stb_track_seeds_static(stb_table *const *tables, int nseed, const long *n_per_seed, double *x,
                                      double *px, double *y, double *py, double *z, double *pt, int32_t *lost_turn,
                                      int32_t *lost_elem, int turn0, int nturn, double aperture_radius,
                                      void *stream) {
  return stb::guarded([&] {
    return stb::track_seeds_static(tables, nseed, n_per_seed, x, px, y, py, z, pt, lost_turn, lost_elem, turn0,
                                   nturn, aperture_radius, (cudaStream_t)stream);
  });
}
