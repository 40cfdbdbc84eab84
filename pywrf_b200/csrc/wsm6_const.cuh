// WSM6 single-moment 6-class microphysics: the scheme's constants
// (pywrf/config_params.py:163-253 and pywrf/wrf_physics.py), shared by the
// scheme's kernels and its tangent.
#pragma once

namespace wrf {
namespace mp {
constexpr double CPD = 1004.5, CPV = 1846.4, RV = 461.6, QMIN = 1.0e-15;
constexpr double XLS = 2850000.0, XLV0 = 2500000.0, XLF0 = 350000.0, DEN0 = 1.28, DENR = 1000.0;
constexpr double CLIQ = 4190.0, CICE = 2106.0, PSAT = 610.78, RCP = 0.2857143;
constexpr double T0C = 273.149993896484375, EP2 = 0.621750414371490479;
constexpr double DTCLDCR = 120.0, N0R = 8.0e6, AVTR = 841.9, QCRMIN = 1.0e-9, N0SMAX = 1.0e11, N0S = 2.0e6;
constexpr double ALPHA = 0.12, PFRZ1 = 100.0, PFRZ2 = 0.66, XNCR = 3.0e8, DICON = 11.9, DIMAX = 500.0e-6;
constexpr double DENS = 100.0, QS0 = 6.0e-4, QC0 = 5.0265482e-04, QCK1 = 6.773895, BVTR = 0.8, G6PBR = 495.4590;
constexpr double PVTR = 2500.064, PACRR = 2.4813369e10, PRECR1 = 3.9207076e07, PRECR2 = 8.2585357e08;
constexpr double ROQIMAX = 8.1250037e-05, BVTS = 0.41, N0G = 4000000.0, BVTG = 0.8, PVTS = 20.05161;
constexpr double PRECS1 = 5200000.0, PRECS2 = 1.8681944e07, PIDN0R = 2.5132743e10, PIDN0S = 6.2831853e08;
constexpr double XLV1 = 2343.6, PACRC = 5.5442112e07, PI = 3.141593, PVTG = 979.9514;
constexpr double PRECG1 = 1.9603538e07, PRECG2 = 2.5852333e08, PIDN0G = 6.2831857e09;
constexpr double RSLOPERMAX = 1.2500000e-05, RSLOPERBMAX = 1.1954404e-04, RSLOPER2MAX = 1.5624999e-10;
constexpr double RSLOPER3MAX = 1.9531248e-15;
}  // namespace mp
}  // namespace wrf

#define F(x) ((float)(x))
