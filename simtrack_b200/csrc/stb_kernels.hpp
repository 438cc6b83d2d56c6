// Kernel launch interfaces shared by the host runtime and the .cu files.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "stb_status.hpp"
#include "stb_table.hpp"

namespace stb {

// One compiled launch configuration of the tracking kernel.
struct TrackVariant {
  bool smem;       // element table staged in shared memory (else read through L1)
  bool seg;        // staged segment by segment, double-buffered (tables too large for shared memory)
  int block;       // threads per CTA
  int min_blocks;  // __launch_bounds__ minimum resident CTAs per SM
  int ppt;         // particles per thread
  const char *name;
  bool prefetch;   // next element header loaded while the current element runs
};
constexpr int kNumTrackVariants = 18;
extern const TrackVariant kVariants[kNumTrackVariants];

struct TrackArgs {
  const ElemHeader *hdr;  // device
  const double *pool;     // device, padded to a multiple of 2 doubles
  int nelem;
  int npool_padded;
  RefConsts ref;
  double *x, *px, *y, *py, *z, *pt;  // SoA, n entries
  long n;
  int turn0;   // global index of the first turn of this block
  int nturn;   // turns in this block
  double r2;   // circular aperture radius squared; +inf when there is none
  int loss_mode;  // which terms of the loss test can fire (is_lost), set by loss_mode_for
  int32_t *lost_turn;  // < 0 while alive
  int32_t *lost_elem;
  int *status;  // device status word (STB_OK or an error code)
  // Optional per-element probe: when non-NULL, coordinates after every element
  // are written to dump[((i * nturn + t) * nelem + e) * 6 + k].
  double *dump;
  // Segmented staging (launch variants with seg set): nseg segments, each
  // staged into one of two shared-memory buffers of seg_bytes bytes.
  const SegDesc *segs;
  int nseg;
  int seg_bytes;
  // The table has radiating elements (GP.radiate): launched on the one
  // kernel instantiation that carries the radiating maps.
  int radiate;
};

// Spin tracking (stb_spin.cu): the orbit arguments plus the spin unit vector
// (x[6..8] of the reference's x[9]) as three SoA arrays, updated in place.
struct SpinArgs {
  TrackArgs t;  // t.dump is unused
  double *sx, *sy, *sz;
  int radiate;  // the table was flattened with GP.radiate
  // Optional per-element probe: dump[((i * nturn + t) * nelem + e) * 9 + k].
  double *dump;
};
struct SpinVariant {
  bool smem;
  int block;
  int min_blocks;
  const char *name;
};
constexpr int kNumSpinVariants = 12;
extern const SpinVariant kSpinVariants[kNumSpinVariants];
cudaError_t launch_spin(const SpinArgs &a, int num_sms, int variant, cudaStream_t stream);

// Track_Radial (stb_radial.cu): zsub[j] = z of the on-momentum reference
// particle after element j (one device thread), then the tracking kernel
// that subtracts it after every element.
cudaError_t launch_radial_reference(const TrackArgs &a, double *zsub, cudaStream_t stream);
cudaError_t launch_radial(const TrackArgs &a, const double *zsub, int num_sms, bool use_smem, cudaStream_t stream);
// Cal_dz0_OnMomentumPart (stb_radial.cu): x0[6] (device, in/out) through every
// element with z and pt reset before each, dz0[j] = z after element j.
cudaError_t launch_onmom_dz0(const TrackArgs &a, double *x0, double *dz0, cudaStream_t stream);

// Elementary-function diagnostics (stb_diag.cu).
int math_input_arity(int fn);
bool math_fn_valid(int fn);
cudaError_t math_eval_device(int fn, const double *d_in, double *d_out, long n, cudaStream_t s);
void math_eval_host(int fn, const double *in, double *out, long n);
cudaError_t fp64_peak_probe(int device, double *tflops);
cudaError_t drift_quotient_check(long n, unsigned long long seed, int device, unsigned long long *bad4);
cudaError_t sincos_fast_check(long n, unsigned long long seed, int device, unsigned long long *cnt4);
cudaError_t rad_normals(unsigned long long seed, unsigned long long id, unsigned long long k0, long n, double *out,
                        int device);
void philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
// BeamBeam4D_SoftGaussian on device AoS beams (stb_ssbb.cu); c4_k = 2 N_other rp / gamma_k.
cudaError_t soft_gaussian_4d(double *x1, long n1, double *x2, long n2, double c4_1, double c4_2, double bbscale1,
                             double bbscale2, int num_sms, cudaStream_t s);
cudaError_t sort_bunch_by_z(double *x, long n, double *scratch, int32_t *order, cudaStream_t s);
cudaError_t slice_mean_z(const double *x, int nslice, long m, double *z, cudaStream_t s);
cudaError_t slice_pair_collision(double *x1, long m1, double *x2, long m2, double S, double c4_1, double c4_2,
                                 double bbscale1, double bbscale2, int num_sms, cudaStream_t s);
// BeamBeam6D_SoftGaussian with slice boundaries zb1, zb2 (host arrays of
// nslice + 1, decreasing), on device AoS bunches (synchronises `s`).
cudaError_t soft_gaussian_6d_zb(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice, const double *zb1,
                                const double *zb2, int num_sms, cudaStream_t s);
// BeamBeam6D_SoftGaussian on device AoS bunches (synchronises `s`).
cudaError_t soft_gaussian_6d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                             double gamma2, double bbscale1, double bbscale2, int Nslice1, int Nslice2, int num_sms,
                             cudaStream_t s);

// Cal_Mean_RMS of x and y (simtrack.cpp:724-743) of two device AoS beams,
// out8 = mean x, mean y, rms x, rms y of beam 1, then of beam 2, the
// reference's running sums.
cudaError_t beam_pair_mean_rms(const double *x1, long n1, const double *x2, long n2, double *out8, cudaStream_t s);
// BeamBeam4D_PIC (simtrack.cpp:23286-23378) on device AoS beams
// (stb_pic.cu; synchronises `s`).  cudaErrorInvalidValue if a particle maps
// outside the 64 x 64 grid.
cudaError_t pic_4d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1, double gamma2,
                   double bbscale1, double bbscale2, int num_sms, cudaStream_t s);

// A grid the PIC functions take: nx == ny, a power of two from 8 to 512.
bool pic_grid_valid(int nx, int ny);
// BeamBeam4D_PIC_NonOffset (simtrack.cpp:24226-24280) on device AoS beams
// with the caller's nx x nx grid (nx a power of two, 8 .. 512), spacing and
// Green spectrum (device arrays of 4 nx^2); synchronises `s`.
cudaError_t pic_4d_nonoffset(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                             double gamma2, double bbscale1, double bbscale2, int nx, double hx, double hy,
                             const double *grn_re, const double *grn_im, int num_sms, cudaStream_t s);
// Cal_Effective_Green_Function (simtrack.cpp:2881-2921) into host arrays of
// 4 nx^2 (nx a power of two, 8 .. 512); synchronises `s`.
cudaError_t pic_green_function(double xoffset, double yoffset, int nx, double hx, double hy, double *grn_re,
                               double *grn_im, cudaStream_t s);
// Lumi_Cal_PIC_4D (simtrack.cpp:23617-23701) of two device AoS beams
// (synchronises `s`).  cudaErrorInvalidValue for a grid of zero or
// non-finite width.
cudaError_t lumi_pic_4d(double Np1, long Mp1, double Np2, long Mp2, const double *x1, const double *x2, int Ncoll,
                        double freq, int num_sms, cudaStream_t s, double *lumi_out);

// BeamBeam6D_PIC on device AoS bunches (stb_ssbb.cu; synchronises `s`).
cudaError_t pic_6d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1, double gamma2,
                   double bbscale1, double bbscale2, int Nslice1, int Nslice2, int num_sms, cudaStream_t s);

// BeamBeam6D_PIC_NonOffset with slice boundaries zb1, zb2 (host arrays of
// nslice + 1) and the caller's grid and Green spectrum (device arrays), on
// device AoS bunches (stb_ssbb.cu; synchronises `s`).
cudaError_t pic_6d_nonoffset(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                             double gamma2, double bbscale1, double bbscale2, int nslice, const double *zb1,
                             const double *zb2, int nx, double hx, double hy, const double *grn_re,
                             const double *grn_im, int num_sms, cudaStream_t s);
// One slice pair of BeamBeam6D_PIC_Interpolation (stb_pic.cu; synchronises
// `s`): slice centres z1c, z2c, kick factors Np/Mp of the whole bunches.
cudaError_t pic_interpolation_pair(double *x1, long m1, double *x2, long m2, double z1c, double z2c,
                                   double np1_per_mp1, double np2_per_mp2, double gamma1, double gamma2,
                                   double bbscale1, double bbscale2, int nx, double hx, double hy,
                                   const double *grn_re, const double *grn_im, int num_sms, cudaStream_t s);
// BeamBeam6D_PIC_Interpolation with slice boundaries zb1, zb2 (host arrays)
// and the caller's grid and Green spectrum (device arrays); stb_ssbb.cu.
cudaError_t pic_6d_interpolation(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                 double gamma2, double bbscale1, double bbscale2, int nslice, const double *zb1,
                                 const double *zb2, int nx, double hx, double hy, const double *grn_re,
                                 const double *grn_im, int num_sms, cudaStream_t s);
// Lumi_Cal_PIC_6D_Angle: the bunches boosted by half crossing angle theta,
// then Lumi_Cal_PIC_6D (stb_ssbb.cu; synchronises `s`).
cudaError_t lumi_pic_6d_angle(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double theta,
                              double gamma1, double gamma2, double bbscale1, double bbscale2, int Nslice1,
                              int Nslice2, int Ncoll, double freq, int num_sms, cudaStream_t s, double *lumi_out);
// Lumi_Cal_PIC_6D on device AoS bunches (stb_ssbb.cu; synchronises `s`).
cudaError_t lumi_pic_6d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                        double gamma2, double bbscale1, double bbscale2, int Nslice1, int Nslice2, int Ncoll,
                        double freq, int num_sms, cudaStream_t s, double *lumi_out);

size_t track_smem_bytes(int nelem, int npool_padded);
// The loss-test mode of a launch with circular aperture r2 (+inf: none) on a
// table whose loss-checked elements have min(RN(APx^2), RN(APy^2)) >= min_ap2.
inline int loss_mode_for(double r2, double min_ap2) {
  if (!(r2 < 1e300)) return 2;      // no circle
  return r2 < min_ap2 ? 1 : 0;      // circle strictly inside every rectangle
}
// Consecutive segments of at most `budget` bytes of staged table (headers plus
// 16-byte aligned pool slice); empty if one element alone exceeds the budget.
std::vector<SegDesc> plan_segments(const ElemHeader *hdr, int nelem, int npool_padded, size_t budget);
int track_smem_limit(int device);
cudaError_t launch_track(const TrackArgs &a, int num_sms, int variant, cudaStream_t stream);
// The same kernel compiled with FMA contraction allowed (stb_track_fast.cu).
cudaError_t launch_track_fast(const TrackArgs &a, int num_sms, int variant, cudaStream_t stream);

// Host-buffer staging of Track()'s AoS interface (stb_track.cu).  aos[n*nc]
// (nc = 6, or 9 with the spin vector) -> SoA soa[k*n + i]; lost_turn = 0 for
// particles Track()'s entry check rejects (input flag 0, |x| or |y| > 0.1),
// else -1; lost_elem = 0.
cudaError_t launch_aos_to_soa(const double *aos, const int32_t *stable, long n, int nc, double *soa,
                              int32_t *lost_turn, int32_t *lost_elem, cudaStream_t s);
// SoA -> AoS and Track()'s outputs: stable = lost_turn < 0; lost_turn_out /
// lost_post = the loss turn and element of lost particles, 0 for survivors.
cudaError_t launch_soa_to_aos(const double *soa, const int32_t *lost_turn, const int32_t *lost_elem, long n, int nc,
                              double *aos, int32_t *stable, int32_t *lost_turn_out, int32_t *lost_post,
                              cudaStream_t s);

}  // namespace stb
