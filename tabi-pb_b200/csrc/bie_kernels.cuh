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

// e^x: the library exp in FP64; in FP32 __expf (the hardware exp2 path, a few
// ulp for the |x| < 10 that near pairs reach).
__device__ __forceinline__ double bie_exp(double v) { return exp(v); }
__device__ __forceinline__ float bie_exp(float v) { return __expf(v); }

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
  T e = bie_exp(-kr);
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

// FP32 form (mixed precision).  K2 needs g(u) = 1 - e^-u and K3 needs
// f(u) = 1 - (1+u) e^-u, u = kappa rs; formed directly, they lose ~1/u and
// ~2/u^2 ulps to cancellation, which at the u ~ 0.01-0.1 of adjacent panels
// leaves FP32 K3 with no correct digits.  Below u = 0.5 both come from their
// Maclaurin series (through u^8 for g, u^9 for f: truncation < 3e-8
// relative), above it from e^-u directly (cancellation < 12x there).
// K3 = G3 (tp2 - 1) - kappa^2 c0 c Gk is then -G3 f - kappa^2 c0 c e G0.
__device__ __forceinline__ void bie4(float dx, float dy, float dz, float vx, float vy, float vz,
                                     float sx, float sy, float sz, float kappa, float eps,
                                     float inv_eps, float& K1, float& K2, float& K3,
                                     float& K4) {
  const float one_over_4pi = 0.0795774715459476679f;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float inv = rsqrtf(r2);
  const float rs = r2 * inv;
  const float G0 = one_over_4pi * inv;
  const float u = kappa * rs;
  const float e = __expf(-u);
  const float gs =
      u * (1.f - u * (1.f / 2 - u * (1.f / 6 - u * (1.f / 24 - u * (1.f / 120 -
          u * (1.f / 720 - u * (1.f / 5040 - u * (1.f / 40320))))))));
  const float fs =
      u * u * (1.f / 2 - u * (1.f / 3 - u * (1.f / 8 - u * (1.f / 30 - u * (1.f / 144 -
          u * (1.f / 840 - u * (1.f / 5760 - u * (1.f / 45360))))))));
  const bool small = u < 0.5f;
  const float tp2 = (1.f + u) * e;
  const float g = small ? gs : 1.f - e;
  const float f = small ? fs : 1.f - tp2;
  const float vd = fmaf(sx, dx, fmaf(sy, dy, sz * dz));
  const float v0d = fmaf(vx, dx, fmaf(vy, dy, vz * dz));
  const float c = vd * inv, c0 = v0d * inv;
  const float tp1 = G0 * inv;
  const float vv = fmaf(vx, sx, fmaf(vy, sy, vz * sz));
  const float G3 = fmaf(-3.f * c0, c, vv) * inv * tp1;
  K1 = (c * tp1) * fmaf(-eps, tp2, 1.f);
  K2 = G0 * g;
  K3 = fmaf(-G3, f, -(kappa * kappa) * c0 * c * e * G0);
  K4 = (c0 * tp1) * fmaf(-tp2, inv_eps, 1.f);
}

}  // namespace tabi
