// C ABI of the turn-by-turn diagnostics (tune finder, surrogate features).
#include <cmath>

#include "stb_runtime.hpp"
#include "stb_tune.hpp"

using namespace stb;

extern "C" {

int stb_fine_tune(const double *x, const double *px, int n, long nsig, long stride, double tune_lower,
                  double tune_upper, double *tune, int device, void *stream) {
  return guarded([&] {
    if (!x || !tune) throw Error(STB_EINVAL, "NULL argument");
    if (n < 1 || n > kMaxTuneSamples) throw Error(STB_EINVAL, "samples per signal out of range (1..4096)");
    if (nsig < 0 || stride < 1 || (nsig > 1 && stride < nsig))
      throw Error(STB_EINVAL, "bad signal count or stride");
    if (!(tune_lower < tune_upper) || !(tune_upper - tune_lower <= 1.0))
      throw Error(STB_EINVAL, "tune window must satisfy lower < upper <= lower + 1");
    if (nsig == 0) return STB_OK;
    DeviceGuard g(device);
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    FineTuneArgs a{x, px, n, nsig, stride, tune_lower, tune_upper, tune};
    cuda_check(launch_fine_tune(a, sms, (cudaStream_t)stream), "tune finder launch");
    return STB_OK;
  });
}

int stb_tbt_features(const double *tbt, long ntot, int nturn, const double *x0, const double *tunes,
                     const double *twiss6, float *features, int device, void *stream) {
  return guarded([&] {
    if (!tbt || !x0 || !tunes || !twiss6 || !features) throw Error(STB_EINVAL, "NULL argument");
    if (ntot < 0 || nturn < 1) throw Error(STB_EINVAL, "bad sizes");
    for (int k = 0; k < 6; k++)
      if (!std::isfinite(twiss6[k])) throw Error(STB_EINVAL, "non-finite optics");
    if (!(twiss6[0] > 0 && twiss6[2] > 0 && twiss6[4] > 0 && twiss6[5] > 0))
      throw Error(STB_EINVAL, "beta functions and emittances must be positive");
    if (ntot == 0) return STB_OK;
    DeviceGuard g(device);
    FeatureArgs a{};
    a.tbt = tbt;
    a.x0 = x0;
    a.tunes = tunes;
    a.ntot = ntot;
    a.nturn = nturn;
    for (int k = 0; k < 6; k++) a.twiss[k] = twiss6[k];
    a.out = features;
    cuda_check(launch_features(a, (cudaStream_t)stream), "feature launch");
    return STB_OK;
  });
}

}  // extern "C"
