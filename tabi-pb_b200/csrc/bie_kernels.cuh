// bie_kernels.cuh -- the four boundary-integral kernels of one (target, source)
// pair, as COMPP_DIRECT_PB (treecode3d_pb.f:969-1001) and LEAFMATVECpara
// (treecode3d_pb.f:1459-1487) write them:
//   rs = |r - s|, G0 = 1/(4 pi rs), Gk = exp(-kappa rs) G0,
//   c = v.(r-s)/rs, c0 = v0.(r-s)/rs, tp1 = G0/rs, tp2 = (1+kappa rs) e^{-kappa rs},
//   G1 = c tp1, G2 = tp2 G1, G10 = c0 tp1, G20 = tp2 G10,
//   G3 = (v0.v - 3 c0 c)/rs tp1, G4 = tp2 G3 - kappa^2 c0 c Gk,
//   K1 = G1 - eps G2, K2 = G0 - Gk, K3 = G4 - G3, K4 = G10 - G20/eps
// with s, v0 the target position / normal and r, v the source's.  Here in
// factored form with one reciprocal square root and one exp.
#pragma once

namespace tabi {

template <typename T>
__device__ __forceinline__ void bie4(T dx, T dy, T dz,          // r - s
                                     T vx, T vy, T vz,          // target normal v0
                                     T sx, T sy, T sz,          // source normal v
                                     T kappa, T eps, T inv_eps, T& K1, T& K2, T& K3,
                                     T& K4) {
  const T one_over_4pi = T(0.079577471545947667884441881686257181);
  T r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  T inv = rsqrt(r2);
  T rs = r2 * inv;
  T G0 = one_over_4pi * inv;
  T kr = kappa * rs;
  T e = exp(-kr);
  T vd = fma(sx, dx, fma(sy, dy, sz * dz));
  T v0d = fma(vx, dx, fma(vy, dy, vz * dz));
  T c = vd * inv, c0 = v0d * inv;
  T tp1 = G0 * inv;
  T tp2 = (T(1) + kr) * e;
  T vv = fma(vx, sx, fma(vy, sy, vz * sz));
  T G3 = fma(T(-3) * c0, c, vv) * inv * tp1;
  K1 = (c * tp1) * fma(-eps, tp2, T(1));
  K2 = G0 * (T(1) - e);
  K3 = fma(G3, tp2 - T(1), -(kappa * kappa) * c0 * c * e * G0);
  K4 = (c0 * tp1) * fma(-tp2, inv_eps, T(1));
}

}  // namespace tabi
