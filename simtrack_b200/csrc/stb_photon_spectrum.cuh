// Photon energies of radiate2's Monte Carlo emission (simtrack.cpp:4305-4318):
// the reference's 43-point table of the synchrotron-radiation spectrum's
// inverse cumulative distribution, u -> E/Ec (kPhotonU -> kPhotonE), read by
// linear interpolation (splint, simtrack.cpp:333-358) for u >= 0.26.  The
// values are the reference's own: the sampled photon energies, and so the
// tracked momenta, must be the same.
#pragma once

namespace stb {

constexpr int kPhotonTable = 43;

__device__ const double kPhotonU[kPhotonTable] = {
    .00123e0, .0123e0,  .0265e0,  .0571e0,  .1228e0,  .1544e0, 0.194e0, .221e0,  .2619e0,   .2893e0,    .327e0,
    .36914e0, .4074e0,  .4417e0,  .47273e0, .5209e0,  .5791e0, .62385e0, .6517e0, .6905e0,  .7165e0,    .7494e0,
    .7726e0,  .8104e0,  .8401e0,  .85954e0, .8835e0,  .892e0,  .89665e0, .8997e0, .90397e0, .9067e0,    .9132e0,
    .93444e0, .9561e0,  .9661e0,  .9768e0,  .98734e0, .9930e0, .99776e0, .999574e0, .9999156e0, 1.e0};

__device__ const double kPhotonE[kPhotonTable] = {
    1.e-9,  1.e-6, 1.e-5, 1.e-4, 1.e-3, 2.e-3, 4.e-3, 6.e-3, .01e0, .0136e0, .02e0,  .0292e0, .04e0, .052e0, .065e0,
    .09e0,  .13e0, .17e0, .2e0,  .25e0, .29e0, .35e0, .4e0,  .5e0,  .6e0,    .68e0,  .8e0,    .85e0, .88e0,  .9e0,
    .93e0,  .95e0, 1.e0,  1.2e0, 1.5e0, 1.7e0, 2.e0,  2.5e0, 3.e0,  4.e0,    5.5e0,  7.e0,    1.e1};

}  // namespace stb
