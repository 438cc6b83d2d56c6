// Host side of the batched dynamic-aperture scan (C ABI stb_scan_*).
//
// The scan owns the flat particle state of all seeds on one device and
// drives turn blocks of (work list, tracking, compaction).  Turn blocks are
// captured into a CUDA graph once and replayed; the device turn counter makes
// every replay identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "simtrack_b200.h"
#include "stb_runtime.hpp"
#include "stb_scan.hpp"

struct stb_scan {
  int device = 0;
  int num_sms = 0;
  int nseed = 0;
  long ntot = 0;
  long max_per_seed = 0;
  std::vector<long> n_per_seed;
  bool smem_ok = false;
  size_t smem = 0;
  int variant = 2;
  int grid = 0;  // persistent grid of the current variant
  int chunk = 1024;
  int pack = 0;  // packed work items (see scan_worklist_kernel), chosen by the autotuner
  stb::ScanArgs args{};
  // device buffers
  stb::ScanSeed *d_seeds = nullptr;
  double *d_coords = nullptr;
  int32_t *d_i32 = nullptr;  // id, lost_turn, lost_elem, out_lost_turn, out_lost_elem
  int32_t *d_live = nullptr, *d_items = nullptr, *d_ctr = nullptr;
  double *d_out_x = nullptr;
  int *d_status = nullptr;
  long max_items = 0;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_blocks = 0, graph_tpb = 0, graph_variant = -1, graph_chunk = -1, graph_pack = -1;
  int turns_done = 0;
  double device_ms = 0.0;
  long blocks_run = 0;
  int32_t *h_abort = nullptr;  // mapped host flag read by every turn block (stb_scan_set_abort)
  int32_t *d_win = nullptr;    // compaction: survivors per window
  double *d_stage = nullptr;   // compaction: staging copy of the slots (6 coordinates + ids)
  double budget_s = 0.0;       // wall-clock budget of one stb_scan_run call (0: none)
};

namespace stb {
namespace {

// Device counters: n_items, next_item, turn counter, item_chunk, block_skipped.
constexpr int kScanCounters = 5;

void scan_destroy(stb_scan *s) {
  if (!s) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->h_abort) cudaFreeHost(s->h_abort);
  for (void *p : {(void *)s->d_seeds, (void *)s->d_coords, (void *)s->d_i32, (void *)s->d_live, (void *)s->d_items,
                  (void *)s->d_ctr, (void *)s->d_out_x, (void *)s->d_status, (void *)s->d_win, (void *)s->d_stage})
    if (p) cudaFree(p);
  if (prev >= 0) cudaSetDevice(prev);
  delete s;
}

void set_chunk(stb_scan *s, int chunk) {
  s->chunk = chunk;
  long items = 0;
  for (long n : s->n_per_seed) items += (n + chunk - 1) / chunk;
  if (items > s->max_items) throw Error(STB_EINVAL, "work list capacity exceeded (chunk too small)");
  s->args.chunk = chunk;
}

stb_scan *scan_build(stb_table **tables, int nseed, const double *x0, const long *n_per_seed, double radius,
                     int device) {
  if (!tables || !x0 || !n_per_seed) throw Error(STB_EINVAL, "NULL argument");
  if (nseed < 1 || nseed > kMaxScanSeeds) throw Error(STB_EINVAL, "seed count out of range");
  std::unique_ptr<stb_scan, void (*)(stb_scan *)> s(new stb_scan(), scan_destroy);
  s->device = device;
  s->nseed = nseed;
  DeviceGuard g(device);
  cuda_check(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  std::vector<ScanSeed> seeds(nseed);
  long off = 0;
  s->smem_ok = true;
  for (int i = 0; i < nseed; i++) {
    stb_table *t = tables[i];
    if (!t) throw Error(STB_EINVAL, "NULL table");
    if (t->device != device) throw Error(STB_EINVAL, "all tables must live on the scan's device");
    if (t->host.spin) throw Error(STB_EINVAL, "spin tables cannot be scanned");
    if (t->host.radiate)
      throw Error(STB_EUNSUPPORTED, "tables flattened with GP.radiate cannot be scanned (Track() entry points only)");
    if (std::memcmp(&t->host.ref, &tables[0]->host.ref, sizeof(RefConsts)) != 0)
      throw Error(STB_EINVAL, "all tables must be flattened for the same reference particle");
    if (n_per_seed[i] < 0 || n_per_seed[i] > (1L << 30)) throw Error(STB_EINVAL, "bad particle count");
    seeds[i] = ScanSeed{t->d_hdr, t->d_pool, (int)t->host.hdr.size(), t->npool_padded, off, (int)n_per_seed[i], 0};
    s->n_per_seed.push_back(n_per_seed[i]);
    off += n_per_seed[i];
    s->max_per_seed = std::max(s->max_per_seed, n_per_seed[i]);
    s->smem = std::max(s->smem, track_smem_bytes((int)t->host.hdr.size(), t->npool_padded));
    s->smem_ok = s->smem_ok && t->use_smem;
  }
  s->ntot = off;
  if (s->ntot == 0) throw Error(STB_EINVAL, "no particles");
  if (s->ntot > (1L << 31) - 1) throw Error(STB_EINVAL, "too many particles for 32-bit ids");
  const long n = s->ntot;
  s->max_items = 0;
  for (long v : s->n_per_seed) s->max_items += (v + 31) / 32;  // smallest work item: one warp
  cuda_check(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
  cuda_check(cudaMalloc(&s->d_seeds, sizeof(ScanSeed) * nseed), "cudaMalloc(seeds)");
  cuda_check(cudaMalloc(&s->d_coords, sizeof(double) * 6 * n), "cudaMalloc(coordinates)");
  cuda_check(cudaMalloc(&s->d_i32, sizeof(int32_t) * 5 * n), "cudaMalloc(particle state)");
  cuda_check(cudaMalloc(&s->d_live, sizeof(int32_t) * nseed), "cudaMalloc(live)");
  cuda_check(cudaMalloc(&s->d_items, sizeof(int32_t) * 2 * std::max<long>(1, s->max_items)), "cudaMalloc(items)");
  cuda_check(cudaMalloc(&s->d_ctr, sizeof(int32_t) * kScanCounters), "cudaMalloc(counters)");
  cuda_check(cudaHostAlloc(&s->h_abort, sizeof(int32_t), cudaHostAllocMapped), "cudaHostAlloc(abort flag)");
  *(volatile int32_t *)s->h_abort = 0;
  int32_t *d_abort = nullptr;
  cuda_check(cudaHostGetDevicePointer((void **)&d_abort, s->h_abort, 0), "abort flag mapping");
  cuda_check(cudaMalloc(&s->d_out_x, sizeof(double) * 6 * n), "cudaMalloc(outputs)");
  cuda_check(cudaMalloc(&s->d_status, sizeof(int)), "cudaMalloc(status)");
  const int nwin = (int)std::max<long>(1, (s->max_per_seed + kCompactWindow - 1) / kCompactWindow);
  cuda_check(cudaMalloc(&s->d_win, sizeof(int32_t) * (size_t)nseed * nwin), "cudaMalloc(compaction windows)");
  cuda_check(cudaMalloc(&s->d_stage, (sizeof(double) * 6 + sizeof(int32_t)) * (size_t)n), "cudaMalloc(compaction staging)");
  // initial state: AoS host -> SoA device; id = original index; all alive
  std::vector<double> soa((size_t)6 * n);
  for (long i = 0; i < n; i++)
    for (int k = 0; k < 6; k++) soa[(size_t)k * n + i] = x0[6 * i + k];
  std::vector<int32_t> i32((size_t)5 * n);
  for (long i = 0; i < n; i++) {
    i32[i] = (int32_t)i;
    i32[n + i] = -1;
    i32[2 * n + i] = 0;
    i32[3 * n + i] = -1;
    i32[4 * n + i] = 0;
  }
  std::vector<int32_t> live(nseed);
  for (int i = 0; i < nseed; i++) live[i] = (int32_t)s->n_per_seed[i];
  cuda_check(cudaMemcpy(s->d_seeds, seeds.data(), sizeof(ScanSeed) * nseed, cudaMemcpyHostToDevice), "upload");
  cuda_check(cudaMemcpy(s->d_coords, soa.data(), sizeof(double) * 6 * n, cudaMemcpyHostToDevice), "upload");
  cuda_check(cudaMemcpy(s->d_i32, i32.data(), sizeof(int32_t) * 5 * n, cudaMemcpyHostToDevice), "upload");
  cuda_check(cudaMemcpy(s->d_live, live.data(), sizeof(int32_t) * nseed, cudaMemcpyHostToDevice), "upload");
  cuda_check(cudaMemset(s->d_ctr, 0, sizeof(int32_t) * kScanCounters), "reset counters");
  cuda_check(cudaMemset(s->d_status, 0, sizeof(int)), "reset status");
  cuda_check(cudaMemcpy(s->d_out_x, x0, sizeof(double) * 6 * n, cudaMemcpyHostToDevice), "upload");
  ScanArgs &a = s->args;
  a.seeds = s->d_seeds;
  a.nseed = nseed;
  a.ref = tables[0]->host.ref;
  a.x = s->d_coords;
  a.px = a.x + n;
  a.y = a.x + 2 * n;
  a.py = a.x + 3 * n;
  a.z = a.x + 4 * n;
  a.pt = a.x + 5 * n;
  a.id = s->d_i32;
  a.lost_turn = s->d_i32 + n;
  a.lost_elem = s->d_i32 + 2 * n;
  a.out_lost_turn = s->d_i32 + 3 * n;
  a.out_lost_elem = s->d_i32 + 4 * n;
  a.out_x = s->d_out_x;
  a.live = s->d_live;
  a.items = s->d_items;
  a.n_items = s->d_ctr;
  a.next_item = s->d_ctr + 1;
  a.turn0 = s->d_ctr + 2;
  a.item_chunk = s->d_ctr + 3;
  a.block_skipped = s->d_ctr + 4;
  a.abort = d_abort;
  a.nwin = nwin;
  a.win_count = s->d_win;
  a.stage = s->d_stage;
  a.stage_id = reinterpret_cast<int32_t *>(s->d_stage + 6 * n);
  a.r2 = radius > 0.0 ? radius * radius : INFINITY;
  double min_ap2 = INFINITY;
  for (int i = 0; i < nseed; i++) min_ap2 = std::fmin(min_ap2, tables[i]->min_ap2);
  a.loss_mode = loss_mode_for(a.r2, min_ap2);
  a.status = s->d_status;
  a.tbt = nullptr;
  a.tbt_turns = 0;
  a.ntot = n;
  s->variant = s->smem_ok ? 0 : 2;
  cuda_check(prepare_scan(s->variant, s->num_sms, s->smem, &s->grid), "scan kernel setup");
  a.grid = s->grid;
  set_chunk(s.get(), kScanVariants[s->variant].block);
  return s.release();
}

long total_live(stb_scan *s) {
  std::vector<int32_t> live(s->nseed);
  cuda_check(cudaMemcpyAsync(live.data(), s->d_live, sizeof(int32_t) * s->nseed, cudaMemcpyDeviceToHost, s->stream),
             "read live counts");
  cuda_check(cudaStreamSynchronize(s->stream), "scan");
  long t = 0;
  for (int v : live) t += v;
  return t;
}

void check_status(stb_scan *s) {
  int st = 0;
  cuda_check(cudaMemcpy(&st, s->d_status, sizeof(int), cudaMemcpyDeviceToHost), "read status");
  if (st != 0) throw Error(st, "scan kernel reported status " + std::to_string(st));
}

void run_blocks_direct(stb_scan *s, int nblocks, int tpb) {
  ScanArgs a = s->args;
  a.nturn = tpb;
  for (int b = 0; b < nblocks; b++)
    cuda_check(launch_scan_block(a, s->variant, s->grid, s->smem, s->stream), "scan block launch");
}

void ensure_graph(stb_scan *s, int blocks, int tpb) {
  if (s->graph && s->graph_blocks == blocks && s->graph_tpb == tpb && s->graph_variant == s->variant &&
      s->graph_chunk == s->chunk && s->graph_pack == s->pack)
    return;
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  cudaGraph_t graph = nullptr;
  cuda_check(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  ScanArgs a = s->args;
  a.nturn = tpb;
  cudaError_t le = cudaSuccess;
  for (int b = 0; b < blocks && le == cudaSuccess; b++) le = launch_scan_block(a, s->variant, s->grid, s->smem, s->stream);
  cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
  cuda_check(le, "scan block capture");
  cuda_check(ce, "end capture");
  cudaError_t ie = cudaGraphInstantiate(&s->graph, graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(ie, "graph instantiate");
  s->graph_blocks = blocks;
  s->graph_tpb = tpb;
  s->graph_variant = s->variant;
  s->graph_chunk = s->chunk;
  s->graph_pack = s->pack;
}

int32_t device_turn(stb_scan *s) {
  int32_t t = 0;
  cuda_check(cudaMemcpyAsync(&t, s->d_ctr + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream), "read turn");
  cuda_check(cudaStreamSynchronize(s->stream), "scan");
  return t;
}

bool abort_requested(const stb_scan *s) { return *(const volatile int32_t *)s->h_abort != 0; }

// Advances every live particle by nturn turns (fewer if all are lost).  Stops
// early, with the state consistent at a turn-block boundary (resumable by
// another stb_scan_run or from a checkpoint), when the caller's abort flag is
// set (STB_EABORTED; blocks still queued track nothing) or when the run's
// wall-clock budget is spent (STB_ETIMEOUT); both are checked between groups
// of turn blocks, the abort flag also by every block on the device.
void scan_run(stb_scan *s, int nturn, int tpb, int use_graph) {
  if (nturn < 0 || tpb <= 0) throw Error(STB_EINVAL, "bad turn counts");
  DeviceGuard g(s->device);
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  struct Events {
    cudaEvent_t a, b;
    ~Events() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } ev{e0, e1};
  const auto t_start = std::chrono::steady_clock::now();
  const int nblocks = nturn / tpb, rem = nturn % tpb;
  const int per_graph = std::max(1, std::min(nblocks, 16));
  int done_blocks = 0;
  float ms_total = 0.f;
  auto timed = [&](auto &&fn) {
    cuda_check(cudaEventRecord(e0, s->stream), "event");
    fn();
    cuda_check(cudaEventRecord(e1, s->stream), "event");
    cuda_check(cudaEventSynchronize(e1), "scan");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
    ms_total += ms;
  };
  auto stop_check = [&]() {
    s->turns_done = device_turn(s);
    int code = 0;
    const char *why = nullptr;
    if (abort_requested(s)) {
      code = STB_EABORTED;
      why = "scan stopped by the caller's abort flag";
    } else if (s->budget_s > 0.0 &&
               std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count() > s->budget_s) {
      code = STB_ETIMEOUT;
      why = "scan stopped: its wall-clock budget is spent";
    }
    if (!code) return;
    cuda_check(launch_scan_finalize(s->args, s->max_per_seed, s->stream), "finalize");
    cuda_check(cudaStreamSynchronize(s->stream), "finalize");
    s->device_ms += ms_total;
    throw Error(code, std::string(why) + " at turn " + std::to_string(s->turns_done));
  };
  stop_check();
  while (done_blocks < nblocks) {
    const int todo = std::min(per_graph, nblocks - done_blocks);
    if (use_graph && todo == per_graph) {
      ensure_graph(s, per_graph, tpb);
      timed([&] { cuda_check(cudaGraphLaunch(s->graph, s->stream), "graph launch"); });
    } else {
      timed([&] { run_blocks_direct(s, todo, tpb); });
    }
    done_blocks += todo;
    s->blocks_run += todo;
    check_status(s);
    stop_check();
    if (total_live(s) == 0) break;
  }
  if (rem > 0 && total_live(s) > 0) {
    timed([&] { run_blocks_direct(s, 1, rem); });
    s->blocks_run += 1;
    check_status(s);
    stop_check();
  }
  s->turns_done = device_turn(s);
  cuda_check(launch_scan_finalize(s->args, s->max_per_seed, s->stream), "finalize");
  cuda_check(cudaStreamSynchronize(s->stream), "finalize");
  s->device_ms += ms_total;
}

// Checkpoint file: a header (magic, version, seed count, particle count,
// particles per seed, turn counter, bookkeeping) and the device state (SoA
// slots, ids and loss state, live counts, counters, outputs).
constexpr char kCkptMagic[8] = {'S', 'T', 'B', 'S', 'C', 'A', 'N', '1'};

void scan_checkpoint(stb_scan *s, const char *path) {
  if (!path) throw Error(STB_EINVAL, "NULL path");
  DeviceGuard g(s->device);
  const long n = s->ntot;
  std::vector<double> coords((size_t)6 * n), out_x((size_t)6 * n);
  std::vector<int32_t> i32((size_t)5 * n), live(s->nseed), ctr(kScanCounters);
  cuda_check(cudaStreamSynchronize(s->stream), "scan");
  cuda_check(cudaMemcpy(coords.data(), s->d_coords, sizeof(double) * coords.size(), cudaMemcpyDeviceToHost), "save");
  cuda_check(cudaMemcpy(out_x.data(), s->d_out_x, sizeof(double) * out_x.size(), cudaMemcpyDeviceToHost), "save");
  cuda_check(cudaMemcpy(i32.data(), s->d_i32, sizeof(int32_t) * i32.size(), cudaMemcpyDeviceToHost), "save");
  cuda_check(cudaMemcpy(live.data(), s->d_live, sizeof(int32_t) * live.size(), cudaMemcpyDeviceToHost), "save");
  cuda_check(cudaMemcpy(ctr.data(), s->d_ctr, sizeof(int32_t) * ctr.size(), cudaMemcpyDeviceToHost), "save");
  const std::string tmp = std::string(path) + ".tmp";
  std::FILE *f = std::fopen(tmp.c_str(), "wb");
  if (!f) throw Error(STB_EINVAL, std::string("cannot write ") + tmp);
  bool ok = true;
  auto put = [&](const void *p, size_t bytes) { ok = ok && std::fwrite(p, 1, bytes, f) == bytes; };
  const int32_t version = 1, nseed = s->nseed;
  const int64_t ntot = n, blocks = s->blocks_run;
  put(kCkptMagic, sizeof(kCkptMagic));
  put(&version, sizeof(version));
  put(&nseed, sizeof(nseed));
  put(&ntot, sizeof(ntot));
  for (long v : s->n_per_seed) {
    const int64_t w = v;
    put(&w, sizeof(w));
  }
  put(&blocks, sizeof(blocks));
  put(&s->device_ms, sizeof(s->device_ms));
  put(ctr.data(), sizeof(int32_t) * ctr.size());
  put(live.data(), sizeof(int32_t) * live.size());
  put(coords.data(), sizeof(double) * coords.size());
  put(i32.data(), sizeof(int32_t) * i32.size());
  put(out_x.data(), sizeof(double) * out_x.size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    throw Error(STB_EINVAL, std::string("cannot write checkpoint ") + path);
  }
}

void scan_restore(stb_scan *s, const char *path) {
  if (!path) throw Error(STB_EINVAL, "NULL path");
  std::FILE *f = std::fopen(path, "rb");
  if (!f) throw Error(STB_EINVAL, std::string("cannot read ") + path);
  struct Close {
    std::FILE *f;
    ~Close() { std::fclose(f); }
  } c{f};
  bool ok = true;
  auto get = [&](void *p, size_t bytes) { ok = ok && std::fread(p, 1, bytes, f) == bytes; };
  char magic[8];
  int32_t version = 0, nseed = 0;
  int64_t ntot = 0, blocks = 0;
  double dev_ms = 0.0;
  get(magic, sizeof(magic));
  get(&version, sizeof(version));
  get(&nseed, sizeof(nseed));
  get(&ntot, sizeof(ntot));
  if (!ok || std::memcmp(magic, kCkptMagic, sizeof(magic)) != 0 || version != 1)
    throw Error(STB_EINVAL, std::string("not a scan checkpoint: ") + path);
  if (nseed != s->nseed || ntot != s->ntot) throw Error(STB_EINVAL, "checkpoint was written by a different scan");
  for (int i = 0; i < nseed; i++) {
    int64_t w = 0;
    get(&w, sizeof(w));
    if (!ok || w != s->n_per_seed[i]) throw Error(STB_EINVAL, "checkpoint was written by a different scan");
  }
  const long n = s->ntot;
  std::vector<double> coords((size_t)6 * n), out_x((size_t)6 * n);
  std::vector<int32_t> i32((size_t)5 * n), live(nseed), ctr(kScanCounters);
  get(&blocks, sizeof(blocks));
  get(&dev_ms, sizeof(dev_ms));
  get(ctr.data(), sizeof(int32_t) * ctr.size());
  get(live.data(), sizeof(int32_t) * live.size());
  get(coords.data(), sizeof(double) * coords.size());
  get(i32.data(), sizeof(int32_t) * i32.size());
  get(out_x.data(), sizeof(double) * out_x.size());
  if (!ok || std::fgetc(f) != EOF) throw Error(STB_EINVAL, std::string("truncated or oversized checkpoint ") + path);
  DeviceGuard g(s->device);
  cuda_check(cudaStreamSynchronize(s->stream), "scan");
  cuda_check(cudaMemcpy(s->d_coords, coords.data(), sizeof(double) * coords.size(), cudaMemcpyHostToDevice), "load");
  cuda_check(cudaMemcpy(s->d_out_x, out_x.data(), sizeof(double) * out_x.size(), cudaMemcpyHostToDevice), "load");
  cuda_check(cudaMemcpy(s->d_i32, i32.data(), sizeof(int32_t) * i32.size(), cudaMemcpyHostToDevice), "load");
  cuda_check(cudaMemcpy(s->d_live, live.data(), sizeof(int32_t) * live.size(), cudaMemcpyHostToDevice), "load");
  cuda_check(cudaMemcpy(s->d_ctr, ctr.data(), sizeof(int32_t) * ctr.size(), cudaMemcpyHostToDevice), "load");
  s->turns_done = ctr[2];
  s->blocks_run = blocks;
  s->device_ms = dev_ms;
}

// Times one turn block of `nturn` turns per launch variant on a snapshot of
// the current state (restored after every trial) and keeps the fastest.
int scan_autotune(stb_scan *s, int nturn, double *timings, int ntimings) {
  DeviceGuard g(s->device);
  const long n = s->ntot;
  const size_t bc = sizeof(double) * 6 * n, bi = sizeof(int32_t) * 5 * n, bl = sizeof(int32_t) * s->nseed,
               bk = sizeof(int32_t) * kScanCounters;
  char *snap = nullptr;
  cuda_check(cudaMalloc(&snap, bc + bi + bl + bk), "cudaMalloc(autotune snapshot)");
  DevFree f{snap};
  auto save = [&](bool restore) {
    void *dst[4] = {snap, snap + bc, snap + bc + bi, snap + bc + bi + bl};
    void *src[4] = {s->d_coords, s->d_i32, s->d_live, s->d_ctr};
    size_t sz[4] = {bc, bi, bl, bk};
    for (int k = 0; k < 4; k++)
      cuda_check(cudaMemcpyAsync(restore ? src[k] : dst[k], restore ? dst[k] : src[k], sz[k], cudaMemcpyDeviceToDevice,
                                 s->stream), "autotune snapshot");
  };
  save(false);
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  const int saved_v = s->variant, saved_grid = s->grid;
  int best = -1, best_pack = 0;
  float best_ms = 0.f;
  for (int vv = 0; vv < 2 * kNumScanVariants; vv++) {
    // every variant with spread and with packed work items
    const int v = vv >> 1, pack = vv & 1;
    float ms = -1.f;
    int grid = 0;
    if ((!kScanVariants[v].smem || s->smem_ok) && prepare_scan(v, s->num_sms, s->smem, &grid) == cudaSuccess) {
      ScanArgs a = s->args;
      a.nturn = nturn;
      a.grid = grid;
      a.chunk = kScanVariants[v].block;
      a.pack = pack;
      cuda_check(cudaEventRecord(e0, s->stream), "event");
      cudaError_t le = launch_scan_block(a, v, grid, s->smem, s->stream);
      cuda_check(cudaEventRecord(e1, s->stream), "event");
      cuda_check(cudaEventSynchronize(e1), "autotune trial");
      if (le == cudaSuccess) cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
      else cudaGetLastError();
      save(true);
      cuda_check(cudaStreamSynchronize(s->stream), "autotune restore");
    } else {
      cudaGetLastError();
    }
    if (timings && v < ntimings && ms > 0.f && (timings[v] <= 0.0 || pack == 0 || ms < timings[v])) timings[v] = ms;
    if (timings && v < ntimings && pack == 0 && ms <= 0.f) timings[v] = ms;
    if (ms > 0.f && (best < 0 || ms < best_ms)) {
      best = v;
      best_pack = pack;
      best_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best < 0) {
    s->variant = saved_v;
    s->grid = saved_grid;
  } else {
    s->variant = best;
    cuda_check(prepare_scan(best, s->num_sms, s->smem, &s->grid), "scan kernel setup");
    set_chunk(s, kScanVariants[best].block);
    s->pack = best_pack;
    s->args.pack = best_pack;
  }
  s->args.grid = s->grid;
  return s->variant;
}

}  // namespace
}  // namespace stb

using namespace stb;

extern "C" {

int stb_scan_create(stb_table **tables, int nseed, const double *x0, const long *n_per_seed, double aperture_radius,
                    int device, stb_scan **out) {
  return guarded([&] {
    if (!out) throw Error(STB_EINVAL, "NULL output");
    *out = scan_build(tables, nseed, x0, n_per_seed, aperture_radius, device);
    return STB_OK;
  });
}

int stb_scan_free(stb_scan *s) {
  return guarded([&] {
    scan_destroy(s);
    return STB_OK;
  });
}

int stb_scan_configure(stb_scan *s, int variant, int chunk) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    if (variant >= 0) {
      if (variant >= kNumScanVariants) throw Error(STB_EINVAL, "variant out of range");
      if (kScanVariants[variant].smem && !s->smem_ok) throw Error(STB_EINVAL, "tables do not fit shared memory");
      DeviceGuard g(s->device);
      int grid = 0;
      cuda_check(prepare_scan(variant, s->num_sms, s->smem, &grid), "scan kernel setup");
      s->variant = variant;
      s->grid = grid;
      s->args.grid = grid;
    }
    if (chunk > 0) {
      if (chunk < 32 || chunk % 32) throw Error(STB_EINVAL, "chunk must be a positive multiple of 32");
      set_chunk(s, chunk);
    }
    return STB_OK;
  });
}

int stb_scan_run(stb_scan *s, int nturn, int turns_per_block, int use_graph) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    scan_run(s, nturn, turns_per_block, use_graph);
    return STB_OK;
  });
}

int stb_scan_results(stb_scan *s, int32_t *lost_turn, int32_t *lost_elem, double *x_aos) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    DeviceGuard g(s->device);
    const long n = s->ntot;
    if (lost_turn)
      cuda_check(cudaMemcpy(lost_turn, s->args.out_lost_turn, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "download");
    if (lost_elem)
      cuda_check(cudaMemcpy(lost_elem, s->args.out_lost_elem, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "download");
    if (x_aos) cuda_check(cudaMemcpy(x_aos, s->d_out_x, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost), "download");
    return STB_OK;
  });
}

int stb_scan_autotune(stb_scan *s, int nturn, int *chosen, double *timings_ms, int ntimings) {
  return guarded([&] {
    if (!s || nturn <= 0) throw Error(STB_EINVAL, "bad arguments");
    const int v = scan_autotune(s, nturn, timings_ms, ntimings);
    if (chosen) *chosen = v;
    return STB_OK;
  });
}

int stb_scan_set_tbt(stb_scan *s, double *tbt, int nturns) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    if (nturns < 0 || (nturns > 0 && !tbt)) throw Error(STB_EINVAL, "bad turn-by-turn buffer");
    s->args.tbt = nturns > 0 ? tbt : nullptr;
    s->args.tbt_turns = nturns;
    if (s->graph) {  // captured launches embed the old arguments
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
    return STB_OK;
  });
}

int stb_scan_retire(stb_scan *s, const uint8_t *mask) {
  return guarded([&] {
    if (!s || !mask) throw Error(STB_EINVAL, "NULL argument");
    DeviceGuard g(s->device);
    uint8_t *d = nullptr;
    cuda_check(cudaMalloc(&d, (size_t)s->ntot), "cudaMalloc(retire mask)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, mask, (size_t)s->ntot, cudaMemcpyHostToDevice), "upload mask");
    cuda_check(launch_scan_retire(s->args, d, s->max_per_seed, s->stream), "retire");
    // compact now so the retired particles leave the work list immediately
    ScanArgs a = s->args;
    a.nturn = 0;
    cuda_check(stb::launch_scan_compact_only(a, s->stream), "compaction");
    cuda_check(launch_scan_finalize(s->args, s->max_per_seed, s->stream), "finalize");
    cuda_check(cudaStreamSynchronize(s->stream), "retire");
    return STB_OK;
  });
}

int stb_scan_set_packing(stb_scan *s, int pack) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    s->pack = pack != 0;
    s->args.pack = s->pack;
    if (s->graph) {  // captured launches embed the old arguments
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
    return STB_OK;
  });
}

int stb_scan_packing(const stb_scan *s, int *pack) {
  return guarded([&] {
    if (!s || !pack) throw Error(STB_EINVAL, "NULL argument");
    *pack = s->pack;
    return STB_OK;
  });
}

int stb_scan_set_abort(stb_scan *s, int value) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    *(volatile int32_t *)s->h_abort = value ? 1 : 0;
    return STB_OK;
  });
}

int stb_scan_set_budget(stb_scan *s, double max_seconds) {
  return guarded([&] {
    if (!s || !(max_seconds >= 0.0)) throw Error(STB_EINVAL, "bad arguments");
    s->budget_s = max_seconds;
    return STB_OK;
  });
}

int stb_scan_checkpoint(stb_scan *s, const char *path) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    scan_checkpoint(s, path);
    return STB_OK;
  });
}

int stb_scan_restore(stb_scan *s, const char *path) {
  return guarded([&] {
    if (!s) throw Error(STB_EINVAL, "NULL scan");
    scan_restore(s, path);
    return STB_OK;
  });
}

int stb_scan_stats(const stb_scan *s, double *st) {
  return guarded([&] {
    if (!s || !st) throw Error(STB_EINVAL, "NULL argument");
    st[0] = (double)s->turns_done;
    st[1] = s->device_ms;
    st[2] = (double)s->blocks_run;
    st[3] = (double)s->variant;
    st[4] = (double)s->chunk;
    st[5] = (double)s->ntot;
    return STB_OK;
  });
}

}  // extern "C"
