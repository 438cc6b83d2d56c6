// C ABI and C++ Track entry points over the element classes, the flattener
// and the CUDA kernels.  Exceptions never cross the C boundary: every entry
// point converts them into a status code plus a thread-local message.
#include "simtrack_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "simtrack_b200.hpp"
#include "stb_flatten.hpp"
#include "stb_kernels.hpp"
#include "stb_runtime.hpp"
#include "stb_status.hpp"

namespace stb {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

namespace {

Element *make_element(const char *type, const char *name, const double *a, int n) {
  if (!type) throw Error(STB_EINVAL, "element type is NULL");
  const std::string t(type), nm(name ? name : "");
  auto need = [&](int k) {
    if (n < k || (k > 0 && !a))
      throw Error(STB_EINVAL, t + " needs " + std::to_string(k) + " constructor arguments, got " + std::to_string(n));
  };
  if (t == "DRIFT") { need(1); return new DRIFT(nm, a[0]); }
  if (t == "MARKER") { need(1); return new MARKER(nm, a[0]); }
  if (t == "BPM") { need(1); return new BPM(nm, a[0]); }
  if (t == "HBPM") { need(1); return new HBPM(nm, a[0]); }
  if (t == "VBPM") { need(1); return new VBPM(nm, a[0]); }
  if (t == "SBEND") { need(4); return new SBEND(nm, a[0], a[1], a[2], a[3]); }
  if (t == "GSBEND") { need(5); return new GSBEND(nm, a[0], a[1], a[2], a[3], a[4]); }
  if (t == "QUAD") { need(3); return new QUAD(nm, a[0], a[1], a[2]); }
  if (t == "SKEWQ") { need(2); return new SKEWQ(nm, a[0], a[1]); }
  if (t == "SEXT") { need(3); return new SEXT(nm, a[0], a[1], a[2]); }
  if (t == "OCT") { need(3); return new OCT(nm, a[0], a[1], a[2]); }
  if (t == "MULT") { need(23); return new MULT(nm, a[0], a + 1, a + 12); }
  if (t == "GMULT") { need(26); return new GMULT(nm, a[0], a[1], a[2], a[3], a + 4, a + 15); }
  if (t == "SBENDMULT") { need(26); return new SBENDMULT(nm, a[0], a[1], a[2], a[3], a + 4, a + 15); }
  if (t == "KICKER") { need(3); return new KICKER(nm, a[0], a[1], a[2]); }
  if (t == "HKICKER") { need(2); return new HKICKER(nm, a[0], a[1]); }
  if (t == "VKICKER") { need(2); return new VKICKER(nm, a[0], a[1]); }
  if (t == "SOLEN") { need(2); return new SOLEN(nm, a[0], a[1]); }
  if (t == "PATCH") { need(4); return new PATCH(nm, a[0], a[1], a[2], a[3]); }
  if (t == "RFCAV") { need(4); return new RFCAV(nm, a[0], a[1], a[2], a[3]); }
  if (t == "CRABRF") { need(4); return new CRABRF(nm, a[0], a[1], a[2], a[3]); }
  if (t == "CCMULT") {
    need(12);
    return new CCMULT(nm, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
  }
  if (t == "LBT") { need(1); return new LBT(nm, a[0]); }
  if (t == "ILBT") { need(1); return new ILBT(nm, a[0]); }
  if (t == "BEAMBEAM") {
    need(11);
    const int treatment = (int)a[0];
    if (treatment != 4 && treatment != 6) throw Error(STB_EINVAL, "Error: beambeam treatment only can be 4 or 6");
    return new BEAMBEAM(nm, treatment, a[1], a[2], a[3], (int)a[4], a[5], a[6], a[7], a[8], a[9], a[10]);
  }
  throw Error(STB_EUNSUPPORTED, "element type " + t + " is not supported");
}

Element *E(stb_element *e) { return reinterpret_cast<Element *>(e); }
const Element *E(const stb_element *e) { return reinterpret_cast<const Element *>(e); }
Line *Lp(stb_line *l) { return reinterpret_cast<Line *>(l); }
const Line *Lp(const stb_line *l) { return reinterpret_cast<const Line *>(l); }

void table_destroy(stb_table *t) {
  if (!t) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(t->device);
  if (t->d_hdr) cudaFree(t->d_hdr);
  if (t->d_pool) cudaFree(t->d_pool);
  if (t->d_status) cudaFree(t->d_status);
  if (t->d_zsub) cudaFree(t->d_zsub);
  if (t->d_io) cudaFree(t->d_io);
  if (t->d_segs) cudaFree(t->d_segs);
  if (t->io_stream) cudaStreamDestroy(t->io_stream);
  if (prev >= 0) cudaSetDevice(prev);
  delete t;
}

// Plans the table's segments for buffers of `budget` bytes and uploads the
// plan (nseg = 0 when an element alone exceeds the budget).
void set_segments(stb_table *t, size_t budget) {
  const std::vector<SegDesc> segs =
      plan_segments(t->host.hdr.data(), (int)t->host.hdr.size(), t->npool_padded, budget);
  if (t->d_segs) {
    cudaFree(t->d_segs);
    t->d_segs = nullptr;
  }
  t->nseg = 0;
  t->seg_bytes = 0;
  if (segs.empty()) return;
  cuda_check(cudaMalloc(&t->d_segs, sizeof(SegDesc) * segs.size()), "cudaMalloc(segments)");
  cuda_check(cudaMemcpy(t->d_segs, segs.data(), sizeof(SegDesc) * segs.size(), cudaMemcpyHostToDevice),
             "upload segments");
  t->nseg = (int)segs.size();
  t->seg_bytes = (int)budget;
}

bool variant_allowed(const stb_table *t, int v) {
  if (t->host.spin) return !kSpinVariants[v].smem || t->use_smem;
  if (kVariants[v].seg) return !t->use_smem && t->nseg > 1;
  return !kVariants[v].smem || t->use_smem;
}

stb_table *table_build_from(HostTable host, int device, bool spin) {
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(new stb_table(), table_destroy);
  t->device = device;
  t->host = std::move(host);
  t->min_ap2 = INFINITY;
  for (const ElemHeader &h : t->host.hdr)
    if ((h.flags & EF_NO_LOSS_CHECK) == 0) t->min_ap2 = std::fmin(t->min_ap2, std::fmin(h.apx * h.apx, h.apy * h.apy));
  if (t->host.hdr.empty()) throw Error(STB_EINVAL, "line has no elements");
  DeviceGuard g(device);
  std::vector<double> pool = t->host.pool;
  pool.resize((pool.size() + 1) & ~size_t(1), 0.0);  // 16-byte multiple for the bulk copy
  if (pool.empty()) pool.assign(2, 0.0);
  t->npool_padded = (int)pool.size();
  const size_t hb = t->host.hdr.size() * sizeof(ElemHeader), pb = pool.size() * sizeof(double);
  cuda_check(cudaMalloc(&t->d_hdr, hb), "cudaMalloc(element headers)");
  cuda_check(cudaMalloc(&t->d_pool, pb), "cudaMalloc(parameter pool)");
  cuda_check(cudaMalloc(&t->d_status, sizeof(int)), "cudaMalloc(status)");
  cuda_check(cudaMemcpy(t->d_hdr, t->host.hdr.data(), hb, cudaMemcpyHostToDevice), "upload headers");
  cuda_check(cudaMemcpy(t->d_pool, pool.data(), pb, cudaMemcpyHostToDevice), "upload pool");
  cuda_check(cudaMemset(t->d_status, 0, sizeof(int)), "clear status");
  cuda_check(cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  const size_t need = track_smem_bytes((int)t->host.hdr.size(), t->npool_padded);
  t->use_smem = (long)need <= (long)track_smem_limit(device);
  // default launch variant: the first shared-memory one when the table fits,
  // else the first L1 one (stb_track.cu kVariants, stb_spin.cu kSpinVariants)
  t->variant = t->use_smem ? 0 : 3;
  // tables too large for one shared-memory copy are also staged segment by
  // segment (two buffers of half the shared memory each) by the seg_* variants
  if (!t->use_smem && !spin) set_segments(t.get(), (size_t)track_smem_limit(device) / 2 & ~size_t(15));
  return t.release();
}

stb_table *table_build(const Line &line, int device, bool spin = false) {
  return table_build_from(spin ? flatten_spin(line) : flatten(line), device, spin);
}

TrackArgs make_args(stb_table *t) {
  TrackArgs a{};
  a.hdr = t->d_hdr;
  a.pool = t->d_pool;
  a.nelem = (int)t->host.hdr.size();
  a.npool_padded = t->npool_padded;
  a.ref = t->host.ref;
  a.status = t->d_status;
  a.segs = t->d_segs;
  a.nseg = t->nseg;
  a.seg_bytes = t->seg_bytes;
  a.radiate = (t->host.radiate && !t->host.spin) ? 1 : 0;
  return a;
}

int track_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt, long n,
                 int turn0, int nturn, double radius, int32_t *lost_turn, int32_t *lost_elem, cudaStream_t s,
                 double *dump = nullptr) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (t->host.spin) throw Error(STB_EINVAL, "table is flattened for spin tracking (use stb_track_spin_*)");
  if (n < 0 || nturn < 0 || turn0 < 0) throw Error(STB_EINVAL, "negative particle count or turn");
  if (n == 0 || nturn == 0) return STB_OK;
  if (!x || !px || !y || !py || !z || !pt || !lost_turn || !lost_elem)
    throw Error(STB_EINVAL, "coordinate or loss array is NULL");
  DeviceGuard g(t->device);
  TrackArgs a = make_args(t);
  a.x = x; a.px = px; a.y = y; a.py = py; a.z = z; a.pt = pt;
  a.n = n;
  a.turn0 = turn0;
  a.nturn = nturn;
  a.r2 = radius > 0.0 ? radius * radius : INFINITY;
  a.loss_mode = loss_mode_for(a.r2, t->min_ap2);
  a.lost_turn = lost_turn;
  a.lost_elem = lost_elem;
  a.dump = dump;
  cuda_check((t->fast ? launch_track_fast : launch_track)(a, t->num_sms, t->variant, s), "track kernel launch");
  return STB_OK;
}

// Times every launch variant (the orbit kernel's, or the spin kernel's for a
// spin table) on a device-side copy of the n given particles (nc = 6 or 9
// coordinate arrays, not modified) and keeps the fastest for this table.
int autotune(stb_table *t, const double *const *in, int nc, long n, int nturn, double radius, int *chosen,
             double *timings, int ntimings) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (nc != (t->host.spin ? 9 : 6))
    throw Error(STB_EINVAL, t->host.spin ? "a spin table is tuned on nine coordinate arrays"
                                         : "table is flattened for orbit tracking: six coordinate arrays");
  for (int k = 0; k < nc; k++)
    if (!in[k]) throw Error(STB_EINVAL, "NULL coordinate array");
  if (n <= 0 || nturn <= 0) throw Error(STB_EINVAL, "autotune needs particles and turns");
  DeviceGuard g(t->device);
  const long m = n;
  double *buf = nullptr;
  int32_t *lost = nullptr;
  cuda_check(cudaMalloc(&buf, sizeof(double) * nc * m), "cudaMalloc(autotune)");
  DevFree f1{buf};
  cuda_check(cudaMalloc(&lost, sizeof(int32_t) * 2 * m), "cudaMalloc(autotune)");
  DevFree f2{lost};
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  const int saved = t->variant;
  const int nvar = t->host.spin ? kNumSpinVariants : kNumTrackVariants;
  int best = -1;
  float best_ms = 0.f;
  // segment length: the largest buffers (half the shared memory each) and
  // buffers half that size; the faster plan stays with the seg_* variants
  const size_t seg_full = (size_t)track_smem_limit(t->device) / 2 & ~size_t(15);
  const size_t seg_budgets[2] = {seg_full, seg_full / 2 & ~size_t(15)};
  size_t best_seg = (size_t)t->seg_bytes;
  int seg_list[kNumTrackVariants], nseg_v = 0;
  if (!t->host.spin && t->nseg > 0)
    for (int v = 0; v < kNumTrackVariants; v++)
      if (kVariants[v].seg) seg_list[nseg_v++] = v;
  for (int vv = 0; vv < nvar + nseg_v; vv++) {
    // vv >= nvar: the seg_* variants again with the smaller segment budget
    const int v = vv < nvar ? vv : seg_list[vv - nvar];
    const bool seg_v = !t->host.spin && kVariants[v].seg;
    if (seg_v) set_segments(t, seg_budgets[vv < nvar ? 0 : 1]);
    float ms = -1.f;
    if (variant_allowed(t, v)) {
      float runs[2] = {0.f, 0.f};
      bool ok = true;
      for (int r = 0; r < 2 && ok; r++) {
        for (int k = 0; k < nc; k++)
          cuda_check(cudaMemcpy(buf + k * m, in[k], sizeof(double) * m, cudaMemcpyDeviceToDevice), "copy");
        cuda_check(cudaMemset(lost, 0xff, sizeof(int32_t) * m), "reset");
        cuda_check(cudaMemset(lost + m, 0, sizeof(int32_t) * m), "reset");
        TrackArgs a = make_args(t);
        a.x = buf; a.px = buf + m; a.y = buf + 2 * m; a.py = buf + 3 * m; a.z = buf + 4 * m; a.pt = buf + 5 * m;
        a.n = m; a.turn0 = 1; a.nturn = nturn; a.r2 = radius > 0 ? radius * radius : INFINITY;
        a.loss_mode = loss_mode_for(a.r2, t->min_ap2);
        a.lost_turn = lost; a.lost_elem = lost + m; a.dump = nullptr;
        cuda_check(cudaEventRecord(e0), "event");
        cudaError_t le;
        if (t->host.spin) {
          SpinArgs sa{};
          sa.t = a;
          sa.sx = buf + 6 * m; sa.sy = buf + 7 * m; sa.sz = buf + 8 * m;
          sa.dump = nullptr;
          sa.radiate = t->host.radiate ? 1 : 0;
          le = launch_spin(sa, t->num_sms, v, 0);
        } else {
          le = (t->fast ? launch_track_fast : launch_track)(a, t->num_sms, v, 0);
        }
        if (le != cudaSuccess) {
          cudaGetLastError();
          ok = false;
          break;
        }
        cuda_check(cudaEventRecord(e1), "event");
        cuda_check(cudaEventSynchronize(e1), "autotune run");
        cuda_check(cudaEventElapsedTime(&runs[r], e0, e1), "event time");
      }
      if (ok) ms = runs[1];
    }
    if (timings && v < ntimings && (vv < nvar || (ms > 0.f && (timings[v] <= 0.0 || ms < timings[v]))))
      timings[v] = ms;
    if (ms > 0.f && (best < 0 || ms < best_ms)) {
      best = v;
      best_ms = ms;
      if (seg_v) best_seg = (size_t)t->seg_bytes;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (t->nseg > 0 || best_seg > 0) set_segments(t, best_seg > 0 ? best_seg : seg_full);
  t->variant = best >= 0 ? best : saved;
  if (chosen) *chosen = t->variant;
  return STB_OK;
}

// Device staging of the host-buffer entry points, kept with the table and
// grown on demand: AoS and SoA copies of up to nine coordinates per particle
// plus five int32 arrays (input flag / stable, internal loss turn and
// element, Track()'s lost_turn and lost_post).
struct IoBufs {
  double *aos, *soa;
  int32_t *st, *lt, *le, *lt_out, *lp_out;
};
constexpr size_t kIoBytesPerParticle = 18 * sizeof(double) + 5 * sizeof(int32_t);

IoBufs io_buffers(stb_table *t, long n) {
  if (!t->io_stream) cuda_check(cudaStreamCreateWithFlags(&t->io_stream, cudaStreamNonBlocking), "create stream");
  if ((size_t)n > t->io_cap) {
    if (t->d_io) {
      cuda_check(cudaStreamSynchronize(t->io_stream), "staging stream");
      cudaFree(t->d_io);
      t->d_io = nullptr;
      t->io_cap = 0;
    }
    cuda_check(cudaMalloc(&t->d_io, (size_t)n * kIoBytesPerParticle), "cudaMalloc(host-buffer staging)");
    t->io_cap = (size_t)n;
  }
  const size_t cap = t->io_cap;
  IoBufs b;
  b.aos = static_cast<double *>(t->d_io);
  b.soa = b.aos + 9 * cap;
  int32_t *ip = reinterpret_cast<int32_t *>(b.soa + 9 * cap);
  b.st = ip;
  b.lt = ip + cap;
  b.le = ip + 2 * cap;
  b.lt_out = ip + 3 * cap;
  b.lp_out = ip + 4 * cap;
  return b;
}

// Host AoS -> device SoA, track, back; Track()'s stable/lost_turn/lost_post
// outputs.  The caller's arrays are copied as they are (pinned memory gives
// full-speed DMA); the transposes, Track()'s entry check and the output
// flags are computed on the device; everything runs on the table's own
// stream, which the call waits for before returning.
int track_host(stb_table *t, double *xa, long n, int nturn, double radius, int *stable, int *lost_turn,
               int *lost_post, double *dump_host = nullptr) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (t->host.spin) throw Error(STB_EINVAL, "table is flattened for spin tracking (use stb_track_spin_*)");
  if (n < 0 || nturn < 0) throw Error(STB_EINVAL, "negative particle count or turn count");
  if (n == 0) return STB_OK;
  if (!xa || !stable || !lost_turn || !lost_post) throw Error(STB_EINVAL, "NULL host buffer");
  DeviceGuard g(t->device);
  const IoBufs b = io_buffers(t, n);
  cudaStream_t s = t->io_stream;
  cuda_check(cudaMemcpyAsync(b.aos, xa, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s), "upload coordinates");
  cuda_check(cudaMemcpyAsync(b.st, stable, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s), "upload input flags");
  cuda_check(launch_aos_to_soa(b.aos, b.st, n, 6, b.soa, b.lt, b.le, s), "AoS to SoA");
  cuda_check(cudaMemsetAsync(t->d_status, 0, sizeof(int), s), "clear status");
  double *dd = nullptr;
  const size_t dump_n = dump_host ? (size_t)n * nturn * t->host.hdr.size() * 6 : 0;
  if (dump_host) {
    cuda_check(cudaMalloc(&dd, sizeof(double) * dump_n), "cudaMalloc(probe)");
    // Entries after a loss keep their previous content, as in the oracle probe.
    cuda_check(cudaMemcpyAsync(dd, dump_host, sizeof(double) * dump_n, cudaMemcpyHostToDevice, s), "upload probe");
  }
  DevFree f3{dd};
  double *c = b.soa;
  if (nturn > 0)
    track_device(t, c, c + n, c + 2 * n, c + 3 * n, c + 4 * n, c + 5 * n, n, 0, nturn, radius, b.lt, b.le, s, dd);
  cuda_check(launch_soa_to_aos(c, b.lt, b.le, n, 6, b.aos, b.st, b.lt_out, b.lp_out, s), "SoA to AoS");
  int st = 0;
  cuda_check(cudaMemcpyAsync(&st, t->d_status, sizeof(int), cudaMemcpyDeviceToHost, s), "read status");
  cuda_check(cudaStreamSynchronize(s), "track kernel");
  if (st != 0) throw Error(st, "tracking kernel reported status " + std::to_string(st));
  if (dump_host)
    cuda_check(cudaMemcpyAsync(dump_host, dd, sizeof(double) * dump_n, cudaMemcpyDeviceToHost, s), "download probe");
  cuda_check(cudaMemcpyAsync(xa, b.aos, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s), "download coordinates");
  cuda_check(cudaMemcpyAsync(stable, b.st, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s), "download outputs");
  cuda_check(cudaMemcpyAsync(lost_turn, b.lt_out, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s),
             "download outputs");
  cuda_check(cudaMemcpyAsync(lost_post, b.lp_out, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s),
             "download outputs");
  cuda_check(cudaStreamSynchronize(s), "download");
  return STB_OK;
}

// Track_Radial on device SoA arrays, asynchronous after the first call on a
// table (which computes the reference particle's per-element z).
int radial_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt, long n,
                  int turn0, int nturn, double radius, int32_t *lost_turn, int32_t *lost_elem, cudaStream_t s,
                  double *dump = nullptr) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (t->host.spin) throw Error(STB_EINVAL, "table is flattened for spin tracking");
  if (t->host.radiate)
    throw Error(STB_EUNSUPPORTED, "Track_Radial of a table flattened with GP.radiate is not implemented");
  if (n < 0 || nturn < 0 || turn0 < 0) throw Error(STB_EINVAL, "negative particle count or turn");
  if (n == 0 || nturn == 0) return STB_OK;
  if (!x || !px || !y || !py || !z || !pt || !lost_turn || !lost_elem)
    throw Error(STB_EINVAL, "coordinate or loss array is NULL");
  DeviceGuard g(t->device);
  TrackArgs a = make_args(t);
  if (!t->d_zsub) {
    double *zs = nullptr;
    cuda_check(cudaMalloc(&zs, sizeof(double) * t->host.hdr.size()), "cudaMalloc(radial reference)");
    cudaError_t e = launch_radial_reference(a, zs, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      cudaFree(zs);
      cuda_check(e, "radial reference pass");
    }
    t->d_zsub = zs;
  }
  a.x = x; a.px = px; a.y = y; a.py = py; a.z = z; a.pt = pt;
  a.n = n;
  a.turn0 = turn0;
  a.nturn = nturn;
  a.r2 = radius > 0.0 ? radius * radius : INFINITY;
  a.loss_mode = loss_mode_for(a.r2, t->min_ap2);
  a.lost_turn = lost_turn;
  a.lost_elem = lost_elem;
  a.dump = dump;
  cuda_check(launch_radial(a, t->d_zsub, t->num_sms, t->use_smem, s), "radial kernel launch");
  return STB_OK;
}

int radial_host(stb_table *t, double *xa, long n, int nturn, double radius, int *stable, int *lost_turn,
                int *lost_post, double *dump_host = nullptr) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (n < 0 || nturn < 0) throw Error(STB_EINVAL, "negative particle count or turn count");
  if (n == 0) return STB_OK;
  if (!xa || !stable || !lost_turn || !lost_post) throw Error(STB_EINVAL, "NULL host buffer");
  DeviceGuard g(t->device);
  std::vector<double> soa((size_t)n * 6);
  std::vector<int32_t> lt((size_t)n), le((size_t)n, 0);
  for (long i = 0; i < n; i++) {
    for (int k = 0; k < 6; k++) soa[(size_t)k * n + i] = xa[6 * i + k];
    lt[i] = entry_rejected(xa + 6 * i, stable[i]) ? 0 : -1;  // Track_Radial's entry check, 21647-21649
  }
  double *d = nullptr;
  int32_t *dl = nullptr;
  cuda_check(cudaMalloc(&d, sizeof(double) * 6 * n), "cudaMalloc(coordinates)");
  DevFree f1{d};
  cuda_check(cudaMalloc(&dl, sizeof(int32_t) * 2 * n), "cudaMalloc(loss arrays)");
  DevFree f2{dl};
  cuda_check(cudaMemcpy(d, soa.data(), sizeof(double) * 6 * n, cudaMemcpyHostToDevice), "upload coordinates");
  cuda_check(cudaMemcpy(dl, lt.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice), "upload loss state");
  cuda_check(cudaMemcpy(dl + n, le.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice), "upload loss state");
  cuda_check(cudaMemset(t->d_status, 0, sizeof(int)), "clear status");
  double *dd = nullptr;
  const size_t dump_n = dump_host ? (size_t)n * nturn * t->host.hdr.size() * 6 : 0;
  if (dump_host) {
    cuda_check(cudaMalloc(&dd, sizeof(double) * dump_n), "cudaMalloc(probe)");
    cuda_check(cudaMemcpy(dd, dump_host, sizeof(double) * dump_n, cudaMemcpyHostToDevice), "upload probe");
  }
  DevFree f3{dd};
  if (nturn > 0)
    radial_device(t, d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, n, 0, nturn, radius, dl, dl + n, 0, dd);
  cuda_check(cudaDeviceSynchronize(), "radial kernel");
  if (dump_host)
    cuda_check(cudaMemcpy(dump_host, dd, sizeof(double) * dump_n, cudaMemcpyDeviceToHost), "download probe");
  int st = 0;
  cuda_check(cudaMemcpy(&st, t->d_status, sizeof(int), cudaMemcpyDeviceToHost), "read status");
  if (st != 0) throw Error(st, "radial kernel reported status " + std::to_string(st));
  cuda_check(cudaMemcpy(soa.data(), d, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost), "download coordinates");
  cuda_check(cudaMemcpy(lt.data(), dl, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "download loss state");
  cuda_check(cudaMemcpy(le.data(), dl + n, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "download loss state");
  for (long i = 0; i < n; i++) {
    for (int k = 0; k < 6; k++) xa[6 * i + k] = soa[(size_t)k * n + i];
    if (lt[i] < 0) {
      stable[i] = 1; lost_turn[i] = 0; lost_post[i] = 0;
    } else {
      stable[i] = 0; lost_turn[i] = lt[i]; lost_post[i] = le[i];
    }
  }
  return STB_OK;
}

// Track_Spin on device SoA arrays (orbit + spin unit vector), asynchronous.
int spin_device(stb_table *t, double *const xs[9], long n, int turn0, int nturn, double radius, int32_t *lost_turn,
                int32_t *lost_elem, cudaStream_t s, double *dump = nullptr) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (!t->host.spin) throw Error(STB_EINVAL, "table is not flattened for spin tracking (use stb_table_create_spin)");
  if (n < 0 || nturn < 0 || turn0 < 0) throw Error(STB_EINVAL, "negative particle count or turn");
  if (n == 0 || nturn == 0) return STB_OK;
  for (int k = 0; k < 9; k++)
    if (!xs[k]) throw Error(STB_EINVAL, "coordinate or spin array is NULL");
  if (!lost_turn || !lost_elem) throw Error(STB_EINVAL, "loss array is NULL");
  DeviceGuard g(t->device);
  SpinArgs a{};
  a.t = make_args(t);
  a.t.x = xs[0]; a.t.px = xs[1]; a.t.y = xs[2]; a.t.py = xs[3]; a.t.z = xs[4]; a.t.pt = xs[5];
  a.sx = xs[6]; a.sy = xs[7]; a.sz = xs[8];
  a.radiate = t->host.radiate ? 1 : 0;
  a.t.n = n;
  a.t.turn0 = turn0;
  a.t.nturn = nturn;
  a.t.r2 = radius > 0.0 ? radius * radius : INFINITY;
  a.t.loss_mode = loss_mode_for(a.t.r2, t->min_ap2);
  a.t.lost_turn = lost_turn;
  a.t.lost_elem = lost_elem;
  a.dump = dump;
  cuda_check(launch_spin(a, t->num_sms, t->variant, s), "spin kernel launch");
  return STB_OK;
}

// Host AoS x[n*9] -> device SoA, Track_Spin, back; optional per-element probe.
int spin_host(stb_table *t, double *xa, long n, int nturn, double radius, int *stable, int *lost_turn,
              int *lost_post, double *dump_host = nullptr) {
  if (!t) throw Error(STB_EINVAL, "table is NULL");
  if (n < 0 || nturn < 0) throw Error(STB_EINVAL, "negative particle count or turn count");
  if (n == 0) return STB_OK;
  if (!xa || !stable || !lost_turn || !lost_post) throw Error(STB_EINVAL, "NULL host buffer");
  if (!t->host.spin) throw Error(STB_EINVAL, "table is not flattened for spin tracking (use stb_table_create_spin)");
  DeviceGuard g(t->device);
  std::vector<double> soa((size_t)n * 9);
  std::vector<int32_t> lt((size_t)n), le((size_t)n, 0);
  for (long i = 0; i < n; i++) {
    for (int k = 0; k < 9; k++) soa[(size_t)k * n + i] = xa[9 * i + k];
    lt[i] = entry_rejected(xa + 9 * i, stable[i]) ? 0 : -1;  // Track_Spin's entry check, 21769-21771
  }
  double *d = nullptr;
  int32_t *dl = nullptr;
  cuda_check(cudaMalloc(&d, sizeof(double) * 9 * n), "cudaMalloc(coordinates)");
  DevFree f1{d};
  cuda_check(cudaMalloc(&dl, sizeof(int32_t) * 2 * n), "cudaMalloc(loss arrays)");
  DevFree f2{dl};
  cuda_check(cudaMemcpy(d, soa.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice), "upload coordinates");
  cuda_check(cudaMemcpy(dl, lt.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice), "upload loss state");
  cuda_check(cudaMemcpy(dl + n, le.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice), "upload loss state");
  cuda_check(cudaMemset(t->d_status, 0, sizeof(int)), "clear status");
  double *dd = nullptr;
  const size_t dump_n = dump_host ? (size_t)n * nturn * t->host.hdr.size() * 9 : 0;
  if (dump_host) {
    cuda_check(cudaMalloc(&dd, sizeof(double) * dump_n), "cudaMalloc(probe)");
    cuda_check(cudaMemcpy(dd, dump_host, sizeof(double) * dump_n, cudaMemcpyHostToDevice), "upload probe");
  }
  DevFree f3{dd};
  double *xs[9];
  for (int k = 0; k < 9; k++) xs[k] = d + (size_t)k * n;
  if (nturn > 0) spin_device(t, xs, n, 0, nturn, radius, dl, dl + n, 0, dd);
  cuda_check(cudaDeviceSynchronize(), "spin kernel");
  if (dump_host)
    cuda_check(cudaMemcpy(dump_host, dd, sizeof(double) * dump_n, cudaMemcpyDeviceToHost), "download probe");
  int st = 0;
  cuda_check(cudaMemcpy(&st, t->d_status, sizeof(int), cudaMemcpyDeviceToHost), "read status");
  if (st != 0) throw Error(st, "spin kernel reported status " + std::to_string(st));
  cuda_check(cudaMemcpy(soa.data(), d, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost), "download coordinates");
  cuda_check(cudaMemcpy(lt.data(), dl, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "download loss state");
  cuda_check(cudaMemcpy(le.data(), dl + n, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "download loss state");
  for (long i = 0; i < n; i++) {
    for (int k = 0; k < 9; k++) xa[9 * i + k] = soa[(size_t)k * n + i];
    if (lt[i] < 0) {
      stable[i] = 1; lost_turn[i] = 0; lost_post[i] = 0;
    } else {
      stable[i] = 0; lost_turn[i] = lt[i]; lost_post[i] = le[i];
    }
  }
  return STB_OK;
}

}  // namespace

// The same for spin tracking: dump[((i*nturn + turn)*nelem + j)*9 + k].
void spin_device_dump(stb_table *t, double *const c[9], long n, int turn0, int nturn, int32_t *lost_turn,
                      int32_t *lost_elem, double *dump) {
  spin_device(t, c, n, turn0, nturn, 0.0, lost_turn, lost_elem, 0, dump);
}

// One-turn-block launch with the per-element record (the probe variant of the
// tracking kernel): dump[((i*nturn + turn)*nelem + j)*6 + k] after element j.
void track_device_dump(stb_table *t, double *const c[6], long n, int turn0, int nturn, int32_t *lost_turn,
                       int32_t *lost_elem, double *dump) {
  track_device(t, c[0], c[1], c[2], c[3], c[4], c[5], n, turn0, nturn, 0.0, lost_turn, lost_elem, 0, dump);
}

// ---- C++ Track entry points ----
void Track_Batch(Line &line, double *x, long n, int nturn, int *stable, int *lost_turn, int *lost_post,
                 const TrackOptions &opt) {
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(table_build(line, opt.device), table_destroy);
  int rc = track_host(t.get(), x, n, nturn, opt.aperture_radius, stable, lost_turn, lost_post);
  if (rc != STB_OK) throw Error(rc, last_error());
}

void Track(Line &line, double x[], int nturn, int &stable, int &lost_turn, int &lost_post) {
  Track_Batch(line, x, 1, nturn, &stable, &lost_turn, &lost_post);
}

// Cal_SRLoss_Particle (simtrack.cpp:20768-20781): one pass of x through
// every element but the RF cavities, loss = (pt - pt0) GP.beta GP.energy.
// The reference passes without loss tests; a particle that Track()'s tests
// would stop (|x| or |y| > 0.1 at entry, outside an aperture, NaN) is
// rejected here instead of tracked on.
void Cal_SRLoss_Particle(Line &line, double x[], double &loss, int device) {
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(table_build_from(flatten(line, true), device, false),
                                                      table_destroy);
  const double pt0 = x[5];
  double y[6];
  for (int i = 0; i < 6; i++) y[i] = x[i];
  int stable = 1, lost_turn = 0, lost_post = 0;
  int rc = track_host(t.get(), y, 1, 1, 0.0, &stable, &lost_turn, &lost_post);
  if (rc != STB_OK) throw Error(rc, last_error());
  if (!stable)
    throw Error(STB_EINVAL, "the particle fails Track()'s loss test (entry check or element " +
                                std::to_string(lost_post) + "'s aperture); the reference's pass has none");
  for (int i = 0; i < 6; i++) x[i] = y[i];
  loss = (x[5] - pt0) * GP.beta * GP.energy;
}

void Track_Radial(Line &line, double x[], int nturn, int &stable, int &lost_turn, int &lost_post) {
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(table_build(line, 0), table_destroy);
  int rc = radial_host(t.get(), x, 1, nturn, 0.0, &stable, &lost_turn, &lost_post);
  if (rc != STB_OK) throw Error(rc, last_error());
}

void Cal_dz0_OnMomentumPart_dev(Line &line, double x0[], double dz0[], int device) {
  if (!x0 || !dz0) throw Error(STB_EINVAL, "NULL buffer");
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(table_build(line, device), table_destroy);
  DeviceGuard g(device);
  const size_t ne = t->host.hdr.size();
  double *d = nullptr;
  cuda_check(cudaMalloc(&d, sizeof(double) * (6 + ne)), "cudaMalloc(on-momentum pass)");
  std::unique_ptr<double, cudaError_t (*)(void *)> hold(d, cudaFree);
  cuda_check(cudaMemcpy(d, x0, sizeof(double) * 6, cudaMemcpyHostToDevice), "upload x0");
  cuda_check(launch_onmom_dz0(make_args(t.get()), d, d + 6, 0), "on-momentum pass launch");
  cuda_check(cudaDeviceSynchronize(), "on-momentum pass");
  cuda_check(cudaMemcpy(x0, d, sizeof(double) * 6, cudaMemcpyDeviceToHost), "download x0");
  cuda_check(cudaMemcpy(dz0, d + 6, sizeof(double) * ne, cudaMemcpyDeviceToHost), "download dz0");
}

void Cal_dz0_OnMomentumPart(Line &line, double x0[], double dz0[]) { Cal_dz0_OnMomentumPart_dev(line, x0, dz0, 0); }

void Track_wrt_OnMomentumPart_Batch(Line &line, double *x, long n, const double *dz0, int nturn, int *stable,
                                    int *lost_turn, int *lost_post, int device) {
  if (!dz0) throw Error(STB_EINVAL, "NULL dz0");
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(table_build(line, device), table_destroy);
  DeviceGuard g(device);
  const size_t ne = t->host.hdr.size();
  double *zs = nullptr;
  cuda_check(cudaMalloc(&zs, sizeof(double) * ne), "cudaMalloc(dz0)");
  t->d_zsub = zs;  // owned by the table from here on
  cuda_check(cudaMemcpy(zs, dz0, sizeof(double) * ne, cudaMemcpyHostToDevice), "upload dz0");
  const int rc = radial_host(t.get(), x, n, nturn, 0.0, stable, lost_turn, lost_post);
  if (rc != STB_OK) throw Error(rc, last_error());
}

void Track_wrt_OnMomentumPart(Line &line, double x[], double dz0[], int nturn, int &stable, int &lost_turn,
                              int &lost_post) {
  Track_wrt_OnMomentumPart_Batch(line, x, 1, dz0, nturn, &stable, &lost_turn, &lost_post, 0);
}

void Track_Spin(Line &line, double x[], int nturn, int &stable, int &lost_turn, int &lost_post) {
  std::unique_ptr<stb_table, void (*)(stb_table *)> t(table_build(line, 0, true), table_destroy);
  int rc = spin_host(t.get(), x, 1, nturn, 0.0, &stable, &lost_turn, &lost_post);
  if (rc != STB_OK) throw Error(rc, last_error());
}

}  // namespace stb

using namespace stb;

namespace stb {
namespace {
// Runs f with FineTuneFinder's window set to [lo, hi), restoring it
// afterwards.  The window is the process-wide tune_low / tune_high pair (a
// global in the reference too, simtrack.cpp:27), so C-ABI calls that set it
// are serialised: two host threads never see each other's window.
std::mutex g_tune_window_mu;
template <class F>
void with_tune_window(double lo, double hi, F f) {
  std::lock_guard<std::mutex> lk(g_tune_window_mu);
  const double lo0 = tune_low, hi0 = tune_high;
  tune_low = lo;
  tune_high = hi;
  struct Restore {
    double lo, hi;
    ~Restore() { tune_low = lo; tune_high = hi; }
  } restore{lo0, hi0};
  f();
}
}  // namespace
}  // namespace stb

extern "C" {

const char *stb_last_error(void) { return stb::last_error(); }
int stb_version(void) { return 100; }

int stb_set_ref_energy(double gamma, double E0, double Q, double A) {
  return guarded([&] {
    if (!(gamma >= 1.0)) throw Error(STB_EINVAL, "gamma must be >= 1");
    Set_RefPartEnergy(gamma, E0, Q, A);
    return STB_OK;
  });
}
int stb_set_spin_g(double g) {
  return guarded([&] { Set_Spin_G(g); return STB_OK; });
}
int stb_set_flags(int h_expand, int quad_fringe) {
  return guarded([&] {
    GP.H_expand = h_expand != 0;
    GP.quad_fringe = quad_fringe != 0;
    return STB_OK;
  });
}
int stb_set_radiation(int radiate, unsigned long long seed) {
  return guarded([&] {
    GP.radiate = radiate != 0;
    set_radiation_seed(seed);
    return STB_OK;
  });
}
int stb_get_ref(double *o) {
  return guarded([&] {
    if (!o) throw Error(STB_EINVAL, "NULL output");
    o[0] = GP.gamma; o[1] = GP.beta; o[2] = GP.energy; o[3] = GP.brho;
    o[4] = GP.Q; o[5] = GP.energy0; o[6] = GP.G; o[7] = GP.p;
    return STB_OK;
  });
}

int stb_element_new(const char *type, const char *name, const double *args, int nargs, stb_element **out) {
  return guarded([&] {
    if (!out) throw Error(STB_EINVAL, "NULL output");
    *out = reinterpret_cast<stb_element *>(make_element(type, name, args, nargs));
    return STB_OK;
  });
}
int stb_element_free(stb_element *e) {
  return guarded([&] { delete E(e); return STB_OK; });
}
int stb_element_setp(stb_element *e, const char *pname, double value) {
  return guarded([&] {
    if (!e || !pname) throw Error(STB_EINVAL, "NULL element or name");
    E(e)->SetP(pname, value);
    return STB_OK;
  });
}
int stb_element_getp(const stb_element *e, const char *pname, double *value) {
  return guarded([&] {
    if (!e || !pname || !value) throw Error(STB_EINVAL, "NULL argument");
    *value = E(e)->GetP(pname);
    return STB_OK;
  });
}
int stb_element_set_misalign(stb_element *e, double dx, double dy, double ds, double dtheta, double dphi,
                             double dpsi) {
  return guarded([&] {
    if (!e) throw Error(STB_EINVAL, "NULL element");
    Element *p = E(e);
    p->DX = dx; p->DY = dy; p->DS = ds; p->DTHETA = dtheta; p->DPHI = dphi; p->DPSI = dpsi;
    return STB_OK;
  });
}
int stb_element_set_aperture(stb_element *e, double apx, double apy) {
  return guarded([&] {
    if (!e) throw Error(STB_EINVAL, "NULL element");
    E(e)->APx = apx;
    E(e)->APy = apy;
    return STB_OK;
  });
}
int stb_element_name(const stb_element *e, char *buf, int cap) {
  return guarded([&] {
    if (!e || !buf || cap <= 0) throw Error(STB_EINVAL, "NULL argument");
    std::snprintf(buf, (size_t)cap, "%s", E(e)->NAME.c_str());
    return STB_OK;
  });
}
int stb_element_geometry(const stb_element *e, double *out10) {
  return guarded([&] {
    if (!e || !out10) throw Error(STB_EINVAL, "NULL argument");
    const Element *x = E(e);
    const double v[10] = {x->L, x->S, x->DX, x->DY, x->DS, x->DTHETA, x->DPHI, x->DPSI, x->APx, x->APy};
    for (int k = 0; k < 10; k++) out10[k] = v[k];
    return STB_OK;
  });
}
int stb_cal_srloss_u0rad(stb_line *l, int track_form, double *u0rad_mev) {
  return guarded([&] {
    if (!l || !u0rad_mev) throw Error(STB_EINVAL, "NULL argument");
    *u0rad_mev = Cal_SRLoss_U0rad(*Lp(l), track_form != 0);
    return STB_OK;
  });
}

int stb_cal_srloss_particle(stb_line *l, double *x6, double *loss_mev, int device) {
  return guarded([&] {
    if (!l || !x6 || !loss_mev) throw Error(STB_EINVAL, "NULL argument");
    Cal_SRLoss_Particle(*Lp(l), x6, *loss_mev, device);
    return STB_OK;
  });
}

int stb_cal_orbit(stb_line *l, double deltap, double *orbit6, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    Line &line = *Lp(l);
    Cal_Orbit_Num(line, deltap, device);
    if (orbit6)
      for (size_t j = 0; j < line.Cell.size(); j++)
        for (int i = 0; i < 6; i++) orbit6[j * 6 + i] = line.Cell[j]->X[i];
    return STB_OK;
  });
}
int stb_track_da(stb_line *l, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
                 double *angles10, double *sigma10, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    if (nturn < 0) throw Error(STB_EINVAL, "negative turn count");
    Track_DA(*Lp(l), nturn, deltap0, sigmax0, sigmay0, filename, angles10, sigma10, device);
    return STB_OK;
  });
}
int stb_track_da_driver(stb_line *l, int which, int nturn, double deltap0, double angle, double sigmax0,
                        double sigmay0, const char *filename, double *out_a, double *out_sigma, long *nout,
                        int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    Line &L = *Lp(l);
    long n = 0;
    switch (which) {
      case STB_DA1: Track_DA1(L, nturn, deltap0, sigmax0, sigmay0, filename, out_a, out_sigma, device); n = 5; break;
      case STB_DA2: Track_DA2(L, nturn, deltap0, sigmax0, sigmay0, filename, out_a, out_sigma, device); n = 10; break;
      case STB_DA3: Track_DA3(L, nturn, deltap0, sigmax0, sigmay0, filename, out_a, out_sigma, device); n = 5; break;
      case STB_DA_RADIAL:
        Track_DA_Radial(L, nturn, deltap0, sigmax0, sigmay0, filename, out_a, out_sigma, device);
        n = 10;
        break;
      case STB_DA_UNIFORM:
        n = Track_DA_Uniform(L, nturn, deltap0, angle, sigmax0, sigmay0, filename, out_sigma, out_a, device);
        break;
      case STB_DA_RADIAL_UNIFORM:
        n = Track_DA_Radial_Uniform(L, nturn, deltap0, angle, sigmax0, sigmay0, filename, out_sigma, out_a, device);
        break;
      default: throw Error(STB_EINVAL, "unknown DA driver");
    }
    if (nout) *nout = n;
    return STB_OK;
  });
}

int stb_cal_tunes_track(stb_line *l, double *x6, int nturn, double tune_lower, double tune_upper, double *tunes2,
                        int *stable, int device) {
  return guarded([&] {
    if (!l || !x6 || !tunes2) throw Error(STB_EINVAL, "NULL argument");
    double t1 = NAN, t2 = NAN;
    with_tune_window(tune_lower, tune_upper, [&] { Cal_Tunes_Track(*Lp(l), x6, nturn, t1, t2, device); });
    const bool ok = !std::isnan(t1);
    if (ok) {
      tunes2[0] = t1;
      tunes2[1] = t2;
    }
    if (stable) *stable = ok ? 1 : 0;
    return STB_OK;
  });
}

int stb_cal_chrom_track(stb_line *l, double tune_lower, double tune_upper, double *chroms4, int device) {
  return guarded([&] {
    if (!l || !chroms4) throw Error(STB_EINVAL, "NULL argument");
    with_tune_window(tune_lower, tune_upper, [&] { Cal_Chrom_Track(*Lp(l), device); });
    const Line &L = *Lp(l);
    chroms4[0] = L.Chromx1;
    chroms4[1] = L.Chromy1;
    chroms4[2] = L.Chromx2;
    chroms4[3] = L.Chromy2;
    return STB_OK;
  });
}

int stb_cal_tunes_track_orbit(stb_line *l, double deltap0, double tune_lower, double tune_upper, double *tunes2,
                              int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    with_tune_window(tune_lower, tune_upper, [&] { Cal_Tunes_Track(*Lp(l), deltap0, device); });
    if (tunes2) {
      tunes2[0] = Lp(l)->Tune1;
      tunes2[1] = Lp(l)->Tune2;
    }
    return STB_OK;
  });
}

int stb_line_read_madx(stb_line *l, const char *path) {
  return guarded([&] {
    if (!l || !path) throw Error(STB_EINVAL, "NULL argument");
    Read_MADX_Lattice(*Lp(l), path);
    return STB_OK;
  });
}

int stb_line_read_bmad(stb_line *l, const char *path) {
  return guarded([&] {
    if (!l || !path) throw Error(STB_EINVAL, "NULL argument");
    Read_BMAD_Lattice(*Lp(l), path);
    return STB_OK;
  });
}

int stb_track_tbt(stb_line *l, double *x, long n, int nturn, double *x_tbt, int *stable, int *lost_turn,
                  int *lost_post, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    Track_tbt_Batch(*Lp(l), x, n, nturn, x_tbt, stable, lost_turn, lost_post, device);
    return STB_OK;
  });
}

int stb_track_tbt_bpm(stb_line *l, double *x, long n, int nturn, double *x_tbt, int bpm_index, int *stable,
                      int *lost_turn, int *lost_post, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    Track_tbt_bpm_Batch(*Lp(l), x, n, nturn, x_tbt, bpm_index, stable, lost_turn, lost_post, device);
    return STB_OK;
  });
}

int stb_cal_dz0(stb_line *l, double *x0, double *dz0, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    Cal_dz0_OnMomentumPart_dev(*Lp(l), x0, dz0, device);
    return STB_OK;
  });
}

int stb_track_wrt_onmom(stb_line *l, double *x, long n, const double *dz0, int nturn, int *stable, int *lost_turn,
                        int *lost_post, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    Track_wrt_OnMomentumPart_Batch(*Lp(l), x, n, dz0, nturn, stable, lost_turn, lost_post, device);
    return STB_OK;
  });
}

int stb_track_tbt_spin_bpm(stb_line *l, double *x9, long n, int nturn, double *x_tbt9, int bpm_index, int *stable,
                           int *lost_turn, int *lost_post, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    Track_tbt_spin_bpm_Batch(*Lp(l), x9, n, nturn, x_tbt9, bpm_index, stable, lost_turn, lost_post, device);
    return STB_OK;
  });
}

int stb_track_tbt_spin(stb_line *l, double *x9, long n, int nturn, double *x_tbt9, int *stable, int *lost_turn,
                       int *lost_post, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    Track_tbt_spin_Batch(*Lp(l), x9, n, nturn, x_tbt9, stable, lost_turn, lost_post, device);
    return STB_OK;
  });
}

int stb_track_tbt_fma(stb_line *l, double deltap0, double sigmax0, double sigmay0, double tune_lower,
                      double tune_upper, const char *filename, long *rows, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    long r = 0;
    with_tune_window(tune_lower, tune_upper,
                     [&] { r = Track_tbt_FMA(*Lp(l), deltap0, sigmax0, sigmay0, filename, device); });
    if (rows) *rows = r;
    return STB_OK;
  });
}

int stb_track_tbt_lyapunov(stb_line *l, double deltap0, double sigmax0, double sigmay0, const char *filename,
                           long *rows, int device) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "line is NULL");
    const long r = Track_tbt_Lyapunov(*Lp(l), deltap0, sigmax0, sigmay0, filename, device);
    if (rows) *rows = r;
    return STB_OK;
  });
}
int stb_element_type(const stb_element *e, char *buf, int cap) {
  return guarded([&] {
    if (!e || !buf || cap <= 0) throw Error(STB_EINVAL, "NULL argument");
    std::strncpy(buf, E(e)->TYPE.c_str(), (size_t)cap - 1);
    buf[cap - 1] = 0;
    return STB_OK;
  });
}

int stb_line_new(stb_line **out) {
  return guarded([&] {
    if (!out) throw Error(STB_EINVAL, "NULL output");
    *out = reinterpret_cast<stb_line *>(new Line());
    return STB_OK;
  });
}
int stb_line_free(stb_line *l) {
  return guarded([&] { delete Lp(l); return STB_OK; });
}
int stb_line_append(stb_line *l, stb_element *e) {
  return guarded([&] {
    if (!l || !e) throw Error(STB_EINVAL, "NULL line or element");
    Lp(l)->Append(E(e));
    return STB_OK;
  });
}
int stb_line_insert(stb_line *l, long i, stb_element *e) {
  return guarded([&] {
    if (!l || !e) throw Error(STB_EINVAL, "NULL line or element");
    Lp(l)->Insert((int)i, E(e));
    return STB_OK;
  });
}
int stb_line_delete(stb_line *l, long i) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    Lp(l)->Delete((int)i);
    return STB_OK;
  });
}
int stb_line_replace(stb_line *l, long i, stb_element *e) {
  return guarded([&] {
    if (!l || !e) throw Error(STB_EINVAL, "NULL line or element");
    Lp(l)->Replace((int)i, E(e));
    return STB_OK;
  });
}
int stb_line_rewind(stb_line *l, long i) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    Lp(l)->Rewind((int)i);
    return STB_OK;
  });
}
int stb_line_invert(stb_line *l) {
  return guarded([&] {
    if (!l) throw Error(STB_EINVAL, "NULL line");
    Lp(l)->Invert();
    return STB_OK;
  });
}
long stb_line_ncell(const stb_line *l) { return l ? Lp(l)->Ncell : -1; }
double stb_line_length(const stb_line *l) { return l ? Lp(l)->Length : NAN; }
int stb_line_cell(stb_line *l, long i, stb_element **out) {
  return guarded([&] {
    if (!l || !out) throw Error(STB_EINVAL, "NULL argument");
    if (i < 0 || i >= (long)Lp(l)->Cell.size()) throw Error(STB_EINVAL, "cell index out of range");
    *out = reinterpret_cast<stb_element *>(Lp(l)->Cell[(size_t)i]);
    return STB_OK;
  });
}

int stb_table_create(const stb_line *l, int device, stb_table **out) {
  return guarded([&] {
    if (!l || !out) throw Error(STB_EINVAL, "NULL argument");
    *out = table_build(*Lp(l), device);
    return STB_OK;
  });
}
int stb_table_create_spin(const stb_line *l, int device, stb_table **out) {
  return guarded([&] {
    if (!l || !out) throw Error(STB_EINVAL, "NULL argument");
    *out = table_build(*Lp(l), device, true);
    return STB_OK;
  });
}
int stb_table_free(stb_table *t) {
  return guarded([&] { table_destroy(t); return STB_OK; });
}
int stb_table_info(const stb_table *t, double *info) {
  return guarded([&] {
    if (!t || !info) throw Error(STB_EINVAL, "NULL argument");
    info[0] = (double)t->host.hdr.size();
    info[1] = (double)t->host.pool.size();
    info[2] = t->host.flops_per_turn;
    info[3] = (t->host.spin ? stb::kSpinVariants[t->variant].smem : stb::kVariants[t->variant].smem) ? 1.0 : 0.0;
    info[4] = (double)track_smem_bytes((int)t->host.hdr.size(), t->npool_padded);
    info[5] = (double)t->variant;
    return STB_OK;
  });
}

int stb_track_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt, long n,
                     int turn0, int nturn, double aperture_radius, int32_t *lost_turn, int32_t *lost_elem,
                     void *stream) {
  return guarded([&] {
    return track_device(t, x, px, y, py, z, pt, n, turn0, nturn, aperture_radius, lost_turn, lost_elem,
                        (cudaStream_t)stream);
  });
}

int stb_track_host(stb_table *t, double *x, long n, int nturn, double aperture_radius, int *stable,
                   int *lost_turn, int *lost_post) {
  return guarded([&] { return track_host(t, x, n, nturn, aperture_radius, stable, lost_turn, lost_post); });
}

int stb_table_autotune(stb_table *t, const double *x, const double *px, const double *y, const double *py,
                       const double *z, const double *pt, long n, int nturn, double aperture_radius, int *chosen,
                       double *timings_ms, int ntimings) {
  return guarded([&] {
    const double *in[6] = {x, px, y, py, z, pt};
    return autotune(t, in, 6, n, nturn, aperture_radius, chosen, timings_ms, ntimings);
  });
}

int stb_table_autotune_spin(stb_table *t, const double *const *xs9, long n, int nturn, double aperture_radius,
                            int *chosen, double *timings_ms, int ntimings) {
  return guarded([&] {
    if (!xs9) throw Error(STB_EINVAL, "NULL coordinate array list");
    return autotune(t, xs9, 9, n, nturn, aperture_radius, chosen, timings_ms, ntimings);
  });
}

int stb_table_set_variant(stb_table *t, int variant) {
  return guarded([&] {
    if (!t) throw Error(STB_EINVAL, "table is NULL");
    const int nvar = t->host.spin ? kNumSpinVariants : kNumTrackVariants;
    if (variant < 0 || variant >= nvar) throw Error(STB_EINVAL, "variant out of range");
    if (!variant_allowed(t, variant))
      throw Error(STB_EINVAL, !t->host.spin && kVariants[variant].seg
                                  ? "segmented staging is for tables that do not fit shared memory whole"
                                  : "table does not fit shared memory");
    t->variant = variant;
    return STB_OK;
  });
}

int stb_spin_variant_info(int variant, char *name, int cap, int *block, int *smem) {
  return guarded([&] {
    if (variant < 0 || variant >= kNumSpinVariants) throw Error(STB_EINVAL, "variant out of range");
    if (name && cap > 0) {
      std::strncpy(name, kSpinVariants[variant].name, (size_t)cap - 1);
      name[cap - 1] = 0;
    }
    if (block) *block = kSpinVariants[variant].block;
    if (smem) *smem = kSpinVariants[variant].smem ? 1 : 0;
    return STB_OK;
  });
}

int stb_table_segments(const stb_table *t, int *nseg, int *seg_bytes) {
  return guarded([&] {
    if (!t) throw Error(STB_EINVAL, "table is NULL");
    if (nseg) *nseg = t->nseg;
    if (seg_bytes) *seg_bytes = t->seg_bytes;
    return STB_OK;
  });
}

int stb_table_set_segment_bytes(stb_table *t, long bytes) {
  return guarded([&] {
    if (!t) throw Error(STB_EINVAL, "table is NULL");
    if (t->host.spin || t->use_smem) throw Error(STB_EINVAL, "only orbit tables too large for shared memory are segmented");
    const long limit = track_smem_limit(t->device) / 2;
    if (bytes < 1024 || bytes > limit) throw Error(STB_EINVAL, "segment bytes out of range (1024..half the shared memory)");
    DeviceGuard g(t->device);
    set_segments(t, (size_t)bytes & ~size_t(15));
    if (t->nseg == 0) throw Error(STB_EINVAL, "an element's parameters alone exceed the segment size");
    return STB_OK;
  });
}

int stb_table_set_contraction(stb_table *t, int fast) {
  return guarded([&] {
    if (!t) throw Error(STB_EINVAL, "table is NULL");
    t->fast = fast != 0;
    return STB_OK;
  });
}

int stb_track_variant_info(int variant, char *name, int cap, int *block, int *smem) {
  return guarded([&] {
    if (variant < 0 || variant >= kNumTrackVariants) throw Error(STB_EINVAL, "variant out of range");
    if (name && cap > 0) {
      std::strncpy(name, kVariants[variant].name, (size_t)cap - 1);
      name[cap - 1] = 0;
    }
    if (block) *block = kVariants[variant].block;
    if (smem) *smem = kVariants[variant].smem ? 1 : 0;
    return STB_OK;
  });
}

int stb_fp64_peak(int device, double *tflops) {
  return guarded([&] {
    if (!tflops) throw Error(STB_EINVAL, "NULL output");
    DeviceGuard g(device);
    cuda_check(fp64_peak_probe(device, tflops), "fp64 peak probe");
    return STB_OK;
  });
}

int stb_check_drift_quotients(long n, unsigned long long seed, int device, unsigned long long *mismatch4) {
  return guarded([&] {
    if (!mismatch4 || n < 0) throw Error(STB_EINVAL, "bad arguments");
    if (device >= 0) {
      DeviceGuard g(device);
      cuda_check(drift_quotient_check(n, seed, device, mismatch4), "drift quotient check");
    } else {
      cuda_check(drift_quotient_check(n, seed, -1, mismatch4), "drift quotient check");
    }
    return STB_OK;
  });
}

int stb_check_sincos(long n, unsigned long long seed, int device, unsigned long long *count4) {
  return guarded([&] {
    if (!count4 || n < 0) throw Error(STB_EINVAL, "bad arguments");
    if (device >= 0) {
      DeviceGuard g(device);
      cuda_check(sincos_fast_check(n, seed, device, count4), "sin/cos check");
    } else {
      cuda_check(sincos_fast_check(n, seed, -1, count4), "sin/cos check");
    }
    return STB_OK;
  });
}

namespace {
// BeamBeam4D_SoftGaussian's arguments: BB4D's constant 2 N rp / gamma for
// each beam (kicked by the other beam's N), in the reference's order.
void soft_gaussian_args(double Np1, long n1, double Np2, long n2, double gamma1, double gamma2, double &c4_1,
                        double &c4_2) {
  if (n1 < 1 || n2 < 1) throw Error(STB_EINVAL, "each beam needs at least one macro-particle");
  if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
  const double rp = 1.53469826769e-18;  // BB4D, simtrack.cpp:6328
  c4_1 = 2 * Np2 * rp / gamma1;
  c4_2 = 2 * Np1 * rp / gamma2;
}
void pic_args(long n1, long n2, double gamma1, double gamma2) {
  // the reference keeps Mp in an int and the sort keys 9 Mp items in one
  if (n1 < 2 || n2 < 2) throw Error(STB_EINVAL, "each beam needs at least two macro-particles (an rms size)");
  if (n1 > INT32_MAX / 9 || n2 > INT32_MAX / 9) throw Error(STB_EINVAL, "too many macro-particles");
  if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
}

void pic_run(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1, double gamma2,
             double bbscale1, double bbscale2, int device, cudaStream_t s) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const cudaError_t e = pic_4d(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2, sms, s);
  if (e == cudaErrorInvalidValue)
    throw Error(STB_EINVAL, "a macro-particle maps outside the 64 x 64 grid (non-finite rms size or coordinates)");
  cuda_check(e, "particle-in-cell beam-beam");
}
}  // namespace

int stb_bb4d_pic_device(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1,
                        double gamma2, double bbscale1, double bbscale2, int device, void *stream) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL beam");
    pic_args(n1, n2, gamma1, gamma2);
    DeviceGuard g(device);
    pic_run(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2, device, (cudaStream_t)stream);
    return STB_OK;
  });
}

int stb_bb4d_pic_host(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1, double gamma2,
                      double bbscale1, double bbscale2, int device) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL beam");
    pic_args(n1, n2, gamma1, gamma2);
    DeviceGuard g(device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)n1, b2 = sizeof(double) * 6 * (size_t)n2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(beams)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload beam 1");
    cuda_check(cudaMemcpy(d + 6 * n1, x2, b2, cudaMemcpyHostToDevice), "upload beam 2");
    pic_run(Np1, n1, d, Np2, n2, d + 6 * n1, gamma1, gamma2, bbscale1, bbscale2, device, 0);
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download beam 1");
    cuda_check(cudaMemcpy(x2, d + 6 * n1, b2, cudaMemcpyDeviceToHost), "download beam 2");
    return STB_OK;
  });
}

int stb_pic_green_function(double xoffset, double yoffset, int Nx, int Ny, double hx, double hy, double *grn_c_r,
                           double *grn_c_i, int device) {
  return guarded([&] {
    if (!grn_c_r || !grn_c_i) throw Error(STB_EINVAL, "NULL argument");
    if (!pic_grid_valid(Nx, Ny)) throw Error(STB_EINVAL, "the grid must be square, Nx a power of two from 8 to 512");
    DeviceGuard g(device);
    cuda_check(pic_green_function(xoffset, yoffset, Nx, hx, hy, grn_c_r, grn_c_i, 0), "Green function");
    return STB_OK;
  });
}

int stb_bb4d_pic_nonoffset_device(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                  double gamma2, double bbscale1, double bbscale2, int Nx, int Ny, double hx,
                                  double hy, const double *grn_c_r, const double *grn_c_i, int device,
                                  void *stream) {
  return guarded([&] {
    if (!x1 || !x2 || !grn_c_r || !grn_c_i) throw Error(STB_EINVAL, "NULL argument");
    if (!pic_grid_valid(Nx, Ny)) throw Error(STB_EINVAL, "the grid must be square, Nx a power of two from 8 to 512");
    if (Mp1 < 1 || Mp2 < 1 || Mp1 > INT32_MAX / 9 || Mp2 > INT32_MAX / 9)
      throw Error(STB_EINVAL, "macro-particle counts must be 1 .. INT32_MAX / 9");
    if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const cudaError_t e = pic_4d_nonoffset(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, Nx, hx,
                                           hy, grn_c_r, grn_c_i, sms, (cudaStream_t)stream);
    if (e == cudaErrorInvalidValue) throw Error(STB_EINVAL, "a macro-particle maps outside the grid");
    cuda_check(e, "particle-in-cell beam-beam");
    return STB_OK;
  });
}

int stb_bb4d_pic_nonoffset_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int Nx, int Ny, double hx, double hy,
                                const double *grn_c_r, const double *grn_c_i, int device) {
  return guarded([&] {
    if (!x1 || !x2 || !grn_c_r || !grn_c_i) throw Error(STB_EINVAL, "NULL argument");
    if (!pic_grid_valid(Nx, Ny)) throw Error(STB_EINVAL, "the grid must be square, Nx a power of two from 8 to 512");
    if (Mp1 < 1 || Mp2 < 1 || Mp1 > INT32_MAX / 9 || Mp2 > INT32_MAX / 9)
      throw Error(STB_EINVAL, "macro-particle counts must be 1 .. INT32_MAX / 9");
    DeviceGuard g(device);
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    const size_t bg = sizeof(double) * 4 * (size_t)Nx * Ny;
    double *d = nullptr;
    cuda_check(cudaMalloc(&d, b1 + b2 + 2 * bg), "cudaMalloc(beams)");
    DevFree f{d};
    double *d2 = d + 6 * Mp1, *gr = d2 + 6 * Mp2, *gi = gr + 4 * (size_t)Nx * Ny;
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload beam 1");
    cuda_check(cudaMemcpy(d2, x2, b2, cudaMemcpyHostToDevice), "upload beam 2");
    cuda_check(cudaMemcpy(gr, grn_c_r, bg, cudaMemcpyHostToDevice), "upload Green function");
    cuda_check(cudaMemcpy(gi, grn_c_i, bg, cudaMemcpyHostToDevice), "upload Green function");
    int rc = stb_bb4d_pic_nonoffset_device(Np1, Mp1, d, Np2, Mp2, d2, gamma1, gamma2, bbscale1, bbscale2, Nx, Ny,
                                           hx, hy, gr, gi, device, nullptr);
    if (rc != STB_OK) throw Error(rc, last_error());
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download beam 1");
    cuda_check(cudaMemcpy(x2, d2, b2, cudaMemcpyDeviceToHost), "download beam 2");
    return STB_OK;
  });
}

int stb_lumi_pic_4d_device(double Np1, long Mp1, double Np2, long Mp2, const double *x1, const double *x2, int Ncoll,
                           double freq, int device, void *stream, double *lumi) {
  return guarded([&] {
    if (!x1 || !x2 || !lumi) throw Error(STB_EINVAL, "NULL argument");
    if (Mp1 < 1 || Mp2 < 1 || Mp1 > INT32_MAX / 9 || Mp2 > INT32_MAX / 9)
      throw Error(STB_EINVAL, "macro-particle counts must be 1 .. INT32_MAX / 9");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const cudaError_t e = lumi_pic_4d(Np1, Mp1, Np2, Mp2, x1, x2, Ncoll, freq, sms, (cudaStream_t)stream, lumi);
    if (e == cudaErrorInvalidValue)
      throw Error(STB_EINVAL, "the beams span no area (zero or non-finite extent) or hold non-finite coordinates");
    cuda_check(e, "PIC luminosity");
    return STB_OK;
  });
}

int stb_lumi_pic_4d_host(double Np1, long Mp1, double Np2, long Mp2, const double *x1, const double *x2, int Ncoll,
                         double freq, int device, double *lumi) {
  return guarded([&] {
    if (!x1 || !x2 || !lumi) throw Error(STB_EINVAL, "NULL argument");
    if (Mp1 < 1 || Mp2 < 1 || Mp1 > INT32_MAX / 9 || Mp2 > INT32_MAX / 9)
      throw Error(STB_EINVAL, "macro-particle counts must be 1 .. INT32_MAX / 9");
    DeviceGuard g(device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(beams)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload beam 1");
    cuda_check(cudaMemcpy(d + 6 * Mp1, x2, b2, cudaMemcpyHostToDevice), "upload beam 2");
    int rc = stb_lumi_pic_4d_device(Np1, Mp1, Np2, Mp2, d, d + 6 * Mp1, Ncoll, freq, device, nullptr, lumi);
    if (rc != STB_OK) throw Error(rc, last_error());
    return STB_OK;
  });
}

int stb_bb4d_soft_gaussian_device(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1,
                                  double gamma2, double bbscale1, double bbscale2, int device, void *stream) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL beam");
    double c4_1, c4_2;
    soft_gaussian_args(Np1, n1, Np2, n2, gamma1, gamma2, c4_1, c4_2);
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cuda_check(soft_gaussian_4d(x1, n1, x2, n2, c4_1, c4_2, bbscale1, bbscale2, sms, (cudaStream_t)stream),
               "soft-Gaussian beam-beam");
    return STB_OK;
  });
}

int stb_bb4d_soft_gaussian_host(double Np1, long n1, double *x1, double Np2, long n2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int device) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL beam");
    double c4_1, c4_2;
    soft_gaussian_args(Np1, n1, Np2, n2, gamma1, gamma2, c4_1, c4_2);
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)n1, b2 = sizeof(double) * 6 * (size_t)n2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(beams)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload beam 1");
    cuda_check(cudaMemcpy(d + 6 * n1, x2, b2, cudaMemcpyHostToDevice), "upload beam 2");
    cuda_check(soft_gaussian_4d(d, n1, d + 6 * n1, n2, c4_1, c4_2, bbscale1, bbscale2, sms, 0),
               "soft-Gaussian beam-beam");
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download beam 1");
    cuda_check(cudaMemcpy(x2, d + 6 * n1, b2, cudaMemcpyDeviceToHost), "download beam 2");
    return STB_OK;
  });
}

namespace {
void soft_gaussian_6d_args(long Mp1, long Mp2, double gamma1, double gamma2, int ns1, int ns2) {
  if (ns1 < 1 || ns2 < 1 || (long)ns1 * ns2 > 4096) throw Error(STB_EINVAL, "slice counts must be 1..4096 pairs");
  if (Mp1 / ns1 < 2 || Mp2 / ns2 < 2) throw Error(STB_EINVAL, "every slice needs at least two macro-particles");
  if (Mp1 > 0x7fffffffL || Mp2 > 0x7fffffffL) throw Error(STB_EINVAL, "too many macro-particles");
  if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
}
}  // namespace

int stb_bb6d_soft_gaussian_device(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                  double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                  int device, void *stream) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL bunch");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cuda_check(soft_gaussian_6d(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, nslice1, nslice2,
                                sms, (cudaStream_t)stream),
               "sliced soft-Gaussian beam-beam");
    return STB_OK;
  });
}

int stb_bb6d_soft_gaussian_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                int device) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL bunch");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(bunches)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d + 6 * Mp1, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    cuda_check(soft_gaussian_6d(Np1, Mp1, d, Np2, Mp2, d + 6 * Mp1, gamma1, gamma2, bbscale1, bbscale2, nslice1,
                                nslice2, sms, 0),
               "sliced soft-Gaussian beam-beam");
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d + 6 * Mp1, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_bb6d_pic_device(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                        double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2, int device,
                        void *stream) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL bunch");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    if (Mp1 / nslice1 > INT32_MAX / 9 || Mp2 / nslice2 > INT32_MAX / 9) throw Error(STB_EINVAL, "slices too large");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const cudaError_t e = pic_6d(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, nslice1, nslice2,
                                 sms, (cudaStream_t)stream);
    if (e == cudaErrorInvalidValue) throw Error(STB_EINVAL, "a macro-particle maps outside a slice pair's grid");
    cuda_check(e, "sliced particle-in-cell beam-beam");
    return STB_OK;
  });
}

int stb_bb6d_pic_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                      double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2, int device) {
  return guarded([&] {
    if (!x1 || !x2) throw Error(STB_EINVAL, "NULL bunch");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    DeviceGuard g(device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(bunches)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d + 6 * Mp1, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    int rc = stb_bb6d_pic_device(Np1, Mp1, d, Np2, Mp2, d + 6 * Mp1, gamma1, gamma2, bbscale1, bbscale2, nslice1,
                                 nslice2, device, nullptr);
    if (rc != STB_OK) throw Error(rc, last_error());
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d + 6 * Mp1, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_lumi_pic_6d_device(double Np1, long Mp1, double Np2, long Mp2, int nslice1, int nslice2, double *x1,
                           double *x2, double gamma1, double gamma2, double bbscale1, double bbscale2, int Ncoll,
                           double freq, int device, void *stream, double *lumi) {
  return guarded([&] {
    if (!x1 || !x2 || !lumi) throw Error(STB_EINVAL, "NULL argument");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    if (Mp1 / nslice1 > INT32_MAX / 9 || Mp2 / nslice2 > INT32_MAX / 9) throw Error(STB_EINVAL, "slices too large");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const cudaError_t e = lumi_pic_6d(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, nslice1,
                                      nslice2, Ncoll, freq, sms, (cudaStream_t)stream, lumi);
    if (e == cudaErrorInvalidValue)
      throw Error(STB_EINVAL, "a slice pair spans no area (zero or non-finite extent) or holds non-finite coordinates");
    cuda_check(e, "sliced PIC luminosity");
    return STB_OK;
  });
}

int stb_lumi_pic_6d_host(double Np1, long Mp1, double Np2, long Mp2, int nslice1, int nslice2, double *x1,
                         double *x2, double gamma1, double gamma2, double bbscale1, double bbscale2, int Ncoll,
                         double freq, int device, double *lumi) {
  return guarded([&] {
    if (!x1 || !x2 || !lumi) throw Error(STB_EINVAL, "NULL argument");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    DeviceGuard g(device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(bunches)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d + 6 * Mp1, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    int rc = stb_lumi_pic_6d_device(Np1, Mp1, Np2, Mp2, nslice1, nslice2, d, d + 6 * Mp1, gamma1, gamma2, bbscale1,
                                    bbscale2, Ncoll, freq, device, nullptr, lumi);
    if (rc != STB_OK) throw Error(rc, last_error());
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d + 6 * Mp1, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_lumi_pic_6d_angle_host(double Np1, long Mp1, double Np2, long Mp2, double theta, int nslice1, int nslice2,
                               double *x1, double *x2, double gamma1, double gamma2, double bbscale1,
                               double bbscale2, int Ncoll, double freq, int device, double *lumi) {
  return guarded([&] {
    if (!x1 || !x2 || !lumi) throw Error(STB_EINVAL, "NULL argument");
    soft_gaussian_6d_args(Mp1, Mp2, gamma1, gamma2, nslice1, nslice2);
    if (Mp1 / nslice1 > INT32_MAX / 9 || Mp2 / nslice2 > INT32_MAX / 9) throw Error(STB_EINVAL, "slices too large");
    if (!(std::fabs(theta) < 1.5)) throw Error(STB_EINVAL, "half crossing angle out of range");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(bunches)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d + 6 * Mp1, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    const cudaError_t e = lumi_pic_6d_angle(Np1, Mp1, d, Np2, Mp2, d + 6 * Mp1, theta, gamma1, gamma2, bbscale1,
                                            bbscale2, nslice1, nslice2, Ncoll, freq, sms, 0, lumi);
    if (e == cudaErrorInvalidValue)
      throw Error(STB_EINVAL, "a slice pair spans no area (zero or non-finite extent) or holds non-finite coordinates");
    cuda_check(e, "sliced PIC luminosity with crossing angle");
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d + 6 * Mp1, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_bb6d_soft_gaussian_zb_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2,
                                   double gamma1, double gamma2, double bbscale1, double bbscale2, int nslice1,
                                   int nslice2, const double *zb1, const double *zb2, int device) {
  return guarded([&] {
    if (!x1 || !x2 || !zb1 || !zb2) throw Error(STB_EINVAL, "NULL argument");
    if (nslice1 != nslice2)
      throw Error(STB_EINVAL, "the reference's slice-boundary form is defined for equal slice counts only");
    if (nslice1 < 1 || nslice1 > 64) throw Error(STB_EINVAL, "slice count must be 1..64");
    if (Mp1 < 2 || Mp2 < 2 || Mp1 > 0x7fffffffL || Mp2 > 0x7fffffffL) throw Error(STB_EINVAL, "bad bunch size");
    if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *d = nullptr;
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    cuda_check(cudaMalloc(&d, b1 + b2), "cudaMalloc(bunches)");
    DevFree f{d};
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d + 6 * Mp1, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    const cudaError_t e = soft_gaussian_6d_zb(Np1, Mp1, d, Np2, Mp2, d + 6 * Mp1, gamma1, gamma2, bbscale1, bbscale2,
                                              nslice1, zb1, zb2, sms, 0);
    if (e == cudaErrorInvalidValue)
      throw Error(STB_EINVAL, "a slice holds fewer than 2 or more than 2*Mp/Nslice particles");
    cuda_check(e, "sliced soft-Gaussian beam-beam (slice boundaries)");
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d + 6 * Mp1, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_bb6d_pic_nonoffset_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                const double *zb1, const double *zb2, int Nx, int Ny, double hx, double hy,
                                const double *grn_c_r, const double *grn_c_i, int device) {
  return guarded([&] {
    if (!x1 || !x2 || !zb1 || !zb2 || !grn_c_r || !grn_c_i) throw Error(STB_EINVAL, "NULL argument");
    if (nslice1 != nslice2)
      throw Error(STB_EINVAL, "the reference's slice-boundary form is defined for equal slice counts only");
    if (nslice1 < 1 || nslice1 > 64) throw Error(STB_EINVAL, "slice count must be 1..64");
    if (Mp1 < 2 || Mp2 < 2 || Mp1 > INT32_MAX / 9 || Mp2 > INT32_MAX / 9) throw Error(STB_EINVAL, "bad bunch size");
    if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
    if (!pic_grid_valid(Nx, Ny)) throw Error(STB_EINVAL, "the grid must be square, Nx a power of two from 8 to 512");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    const size_t bg = sizeof(double) * 4 * (size_t)Nx * Ny;
    double *d = nullptr;
    cuda_check(cudaMalloc(&d, b1 + b2 + 2 * bg), "cudaMalloc(bunches)");
    DevFree f{d};
    double *d2 = d + 6 * Mp1, *gr = d2 + 6 * Mp2, *gi = gr + 4 * (size_t)Nx * Ny;
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d2, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    cuda_check(cudaMemcpy(gr, grn_c_r, bg, cudaMemcpyHostToDevice), "upload Green function");
    cuda_check(cudaMemcpy(gi, grn_c_i, bg, cudaMemcpyHostToDevice), "upload Green function");
    const cudaError_t e = pic_6d_nonoffset(Np1, Mp1, d, Np2, Mp2, d2, gamma1, gamma2, bbscale1, bbscale2, nslice1,
                                           zb1, zb2, Nx, hx, hy, gr, gi, sms, 0);
    if (e == cudaErrorInvalidValue)
      throw Error(STB_EINVAL,
                  "a slice holds fewer than 2 or more than 2*Mp/Nslice particles, or a particle maps outside the grid");
    cuda_check(e, "sliced particle-in-cell beam-beam (slice boundaries)");
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d2, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_bb6d_pic_interpolation_host(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice1, int nslice2,
                                const double *zb1, const double *zb2, int Nx, int Ny, double hx, double hy,
                                const double *grn_c_r, const double *grn_c_i, int device) {
  return guarded([&] {
    if (!x1 || !x2 || !zb1 || !zb2 || !grn_c_r || !grn_c_i) throw Error(STB_EINVAL, "NULL argument");
    if (nslice1 != nslice2)
      throw Error(STB_EINVAL, "the reference's slice-boundary form is defined for equal slice counts only");
    if (nslice1 < 1 || nslice1 > 64) throw Error(STB_EINVAL, "slice count must be 1..64");
    if (Mp1 < 2 || Mp2 < 2 || Mp1 > INT32_MAX / 9 || Mp2 > INT32_MAX / 9) throw Error(STB_EINVAL, "bad bunch size");
    if (!(gamma1 > 0) || !(gamma2 > 0)) throw Error(STB_EINVAL, "gamma must be positive");
    if (!pic_grid_valid(Nx, Ny)) throw Error(STB_EINVAL, "the grid must be square, Nx a power of two from 8 to 512");
    DeviceGuard g(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t b1 = sizeof(double) * 6 * (size_t)Mp1, b2 = sizeof(double) * 6 * (size_t)Mp2;
    const size_t bg = sizeof(double) * 4 * (size_t)Nx * Ny;
    double *d = nullptr;
    cuda_check(cudaMalloc(&d, b1 + b2 + 2 * bg), "cudaMalloc(bunches)");
    DevFree f{d};
    double *d2 = d + 6 * Mp1, *gr = d2 + 6 * Mp2, *gi = gr + 4 * (size_t)Nx * Ny;
    cuda_check(cudaMemcpy(d, x1, b1, cudaMemcpyHostToDevice), "upload bunch 1");
    cuda_check(cudaMemcpy(d2, x2, b2, cudaMemcpyHostToDevice), "upload bunch 2");
    cuda_check(cudaMemcpy(gr, grn_c_r, bg, cudaMemcpyHostToDevice), "upload Green function");
    cuda_check(cudaMemcpy(gi, grn_c_i, bg, cudaMemcpyHostToDevice), "upload Green function");
    const cudaError_t e = pic_6d_interpolation(Np1, Mp1, d, Np2, Mp2, d2, gamma1, gamma2, bbscale1, bbscale2,
                                               nslice1, zb1, zb2, Nx, hx, hy, gr, gi, sms, 0);
    if (e == cudaErrorInvalidValue)
      throw Error(STB_EINVAL,
                  "a slice holds fewer than 2 or more than 2*Mp/Nslice particles, or a particle maps outside the grid");
    cuda_check(e, "sliced particle-in-cell beam-beam (interpolated potentials)");
    cuda_check(cudaMemcpy(x1, d, b1, cudaMemcpyDeviceToHost), "download bunch 1");
    cuda_check(cudaMemcpy(x2, d2, b2, cudaMemcpyDeviceToHost), "download bunch 2");
    return STB_OK;
  });
}

int stb_rad_normals(unsigned long long seed, unsigned long long id, unsigned long long k0, long n, double *out,
                    int device) {
  return guarded([&] {
    if (n < 0 || (n > 0 && !out)) throw Error(STB_EINVAL, "bad buffers");
    if (device >= 0) {
      DeviceGuard g(device);
      double *d = nullptr;
      cuda_check(cudaMalloc(&d, sizeof(double) * (size_t)(n > 0 ? n : 1)), "cudaMalloc(deviates)");
      DevFree f{d};
      cuda_check(rad_normals(seed, id, k0, n, d, device), "deviate kernel");
      cuda_check(cudaMemcpy(out, d, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost), "download deviates");
    } else {
      cuda_check(rad_normals(seed, id, k0, n, out, -1), "deviates");
    }
    return STB_OK;
  });
}

int stb_philox4x32_10(const unsigned int ctr[4], const unsigned int key[2], unsigned int out[4]) {
  return guarded([&] {
    if (!ctr || !key || !out) throw Error(STB_EINVAL, "NULL argument");
    philox_block(ctr, key, out);
    return STB_OK;
  });
}

int stb_math_eval(int fn, const double *in, double *out, long n, int device) {
  return guarded([&] {
    if (!math_fn_valid(fn)) throw Error(STB_EINVAL, "unknown function code");
    if (n < 0 || (n > 0 && (!in || !out))) throw Error(STB_EINVAL, "bad buffers");
    if (n == 0) return STB_OK;
    const long nin = n * math_input_arity(fn);
    if (device < 0) {
      math_eval_host(fn, in, out, n);
      return STB_OK;
    }
    DeviceGuard g(device);
    double *d = nullptr;
    cuda_check(cudaMalloc(&d, sizeof(double) * (nin + n)), "cudaMalloc(math eval)");
    struct Free {
      void *p;
      ~Free() { if (p) cudaFree(p); }
    } f{d};
    cuda_check(cudaMemcpy(d, in, sizeof(double) * nin, cudaMemcpyHostToDevice), "upload");
    cuda_check(math_eval_device(fn, d, d + nin, n, 0), "math eval launch");
    cuda_check(cudaDeviceSynchronize(), "math eval");
    cuda_check(cudaMemcpy(out, d + nin, sizeof(double) * n, cudaMemcpyDeviceToHost), "download");
    return STB_OK;
  });
}

int stb_track_probe(stb_table *t, double *x, long n, int nturn, double aperture_radius, double *dump, int *stable,
                    int *lost_turn, int *lost_post) {
  return guarded([&] {
    if (!dump) throw Error(STB_EINVAL, "NULL probe buffer");
    return track_host(t, x, n, nturn, aperture_radius, stable, lost_turn, lost_post, dump);
  });
}

int stb_track_radial_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt,
                            long n, int turn0, int nturn, double aperture_radius, int32_t *lost_turn,
                            int32_t *lost_elem, void *stream) {
  return guarded([&] {
    return radial_device(t, x, px, y, py, z, pt, n, turn0, nturn, aperture_radius, lost_turn, lost_elem,
                         (cudaStream_t)stream);
  });
}

int stb_track_radial_host(stb_table *t, double *x, long n, int nturn, double aperture_radius, int *stable,
                          int *lost_turn, int *lost_post) {
  return guarded([&] { return radial_host(t, x, n, nturn, aperture_radius, stable, lost_turn, lost_post); });
}

int stb_track_radial_probe(stb_table *t, double *x, long n, int nturn, double aperture_radius, double *dump,
                           int *stable, int *lost_turn, int *lost_post) {
  return guarded([&] {
    if (!dump) throw Error(STB_EINVAL, "NULL probe buffer");
    return radial_host(t, x, n, nturn, aperture_radius, stable, lost_turn, lost_post, dump);
  });
}

int stb_track_spin_device(stb_table *t, double *x, double *px, double *y, double *py, double *z, double *pt,
                          double *sx, double *sy, double *sz, long n, int turn0, int nturn, double aperture_radius,
                          int32_t *lost_turn, int32_t *lost_elem, void *stream) {
  return guarded([&] {
    double *xs[9] = {x, px, y, py, z, pt, sx, sy, sz};
    return spin_device(t, xs, n, turn0, nturn, aperture_radius, lost_turn, lost_elem, (cudaStream_t)stream);
  });
}

int stb_track_spin_host(stb_table *t, double *x9, long n, int nturn, double aperture_radius, int *stable,
                        int *lost_turn, int *lost_post) {
  return guarded([&] { return spin_host(t, x9, n, nturn, aperture_radius, stable, lost_turn, lost_post); });
}

int stb_track_spin_probe(stb_table *t, double *x9, long n, int nturn, double aperture_radius, double *dump9,
                         int *stable, int *lost_turn, int *lost_post) {
  return guarded([&] {
    if (!dump9) throw Error(STB_EINVAL, "NULL probe buffer");
    return spin_host(t, x9, n, nturn, aperture_radius, stable, lost_turn, lost_post, dump9);
  });
}

}  // extern "C"
