// Device physics of the OpenCFD-EC hot path: reconstruction schemes (sub_scheme.f90), 1-D
// fluxes (sub_flux_split.f90) and the LU-SGS flux difference (sub_LU_SGS.f90:135-157).
//
// Templated on the arithmetic type T: double for the FP64 path (compiled with --fmad=false so
// every a*b+c rounds twice, as the Fortran reference evaluates it), float for the mixed path.
// The order of every operation follows the reference source (left-to-right evaluation, x**n as
// the powi multiplication chain, default-real literals such as 1.e-8 rounded to float first).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace ocfd {

constexpr int LAP = 4;
enum { S_UD1 = 0, S_NND2 = 1, S_UD3 = 2, S_MUSCL2U = 3, S_MUSCL2C = 4, S_MUSCL3 = 5, S_OMUSCL2 = 6,
       S_WENO5 = 7, S_UD5 = 8, S_WENO7 = 9, S_CD2 = 20 };
enum { F_SW = 1, F_HLL = 2, F_HLLC = 3, F_ROE = 4, F_VL = 5, F_AUSM = 6 };

template <class T> __device__ __forceinline__ T sq(T x) { return x * x; }
template <class T> __device__ __forceinline__ T cube(T x) { return (x * x) * x; }
template <class T> __device__ __forceinline__ T pow4(T x) { T t = x * x; return t * t; }
template <class T> __device__ __forceinline__ T pow6(T x) { T t = (x * x) * x; return t * t; }
template <class T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }
template <class T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }
// max/min(a, b) with the comparison order of std::max / std::min (the CPU restatement uses those)
template <class T> __device__ __forceinline__ T fmax_(T a, T b) { return (a < b) ? b : a; }
template <class T> __device__ __forceinline__ T fmin_(T a, T b) { return (b < a) ? b : a; }

__device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double dabs(double x) { return fabs(x); }
__device__ __forceinline__ float dabs(float x) { return fabsf(x); }
__device__ __forceinline__ double dexp(double x) { return exp(x); }
__device__ __forceinline__ float dexp(float x) { return expf(x); }
__device__ __forceinline__ double dpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float dpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double dtanh(double x) { return tanh(x); }
__device__ __forceinline__ float dtanh(float x) { return tanhf(x); }

template <class T> __device__ __forceinline__ T minmod(T a, T b) {  // sub_scheme.f90:281-292
  if (a * b <= T(0)) return T(0);
  if (dabs(a) <= dabs(b)) return a;
  return b;
}

// u[0..7] = u(-3..4): u(0) is the cell left of the face, u(1) the cell right of it.
#define UU(k) u[(k) + 3]
template <class T> __device__ __forceinline__ T weno5_L(const T* u) {  // sub_scheme.f90:101-119
  const T ep = T(1.e-6), C03 = T(3.0 / 10.0), C13 = T(3.0 / 5.0), C23 = T(1.0 / 10.0);
  const T c1312 = T(13.0 / 12.0), c14 = T(1.0 / 4.0), c13 = T(1.0 / 3.0), c56 = T(5.0 / 6.0), c16 = T(1.0 / 6.0), c76 = T(7.0 / 6.0), c116 = T(11.0 / 6.0);
  T S0 = c1312 * sq(UU(0) - T(2) * UU(1) + UU(2)) + c14 * sq(T(3) * UU(0) - T(4) * UU(1) + UU(2));
  T S1 = c1312 * sq(UU(-1) - T(2) * UU(0) + UU(1)) + c14 * sq(UU(-1) - UU(1));
  T S2 = c1312 * sq(UU(-2) - T(2) * UU(-1) + UU(0)) + c14 * sq(UU(-2) - T(4) * UU(-1) + T(3) * UU(0));
  T a0 = C03 / sq(ep + S0), a1 = C13 / sq(ep + S1), a2 = C23 / sq(ep + S2);
  T am = a0 + a1 + a2;
  T q03 = c13 * UU(0) + c56 * UU(1) - c16 * UU(2);
  T q13 = -c16 * UU(-1) + c56 * UU(0) + c13 * UU(1);
  T q23 = c13 * UU(-2) - c76 * UU(-1) + c116 * UU(0);
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
template <class T> __device__ __forceinline__ T weno5_R(const T* u) {  // sub_scheme.f90:122-140
  const T ep = T(1.e-6), C03 = T(3.0 / 10.0), C13 = T(3.0 / 5.0), C23 = T(1.0 / 10.0);
  const T c1312 = T(13.0 / 12.0), c14 = T(1.0 / 4.0), c13 = T(1.0 / 3.0), c56 = T(5.0 / 6.0), c16 = T(1.0 / 6.0), c76 = T(7.0 / 6.0), c116 = T(11.0 / 6.0);
  T S0 = c1312 * sq(UU(1) - T(2) * UU(0) + UU(-1)) + c14 * sq(T(3) * UU(1) - T(4) * UU(0) + UU(-1));
  T S1 = c1312 * sq(UU(2) - T(2) * UU(1) + UU(0)) + c14 * sq(UU(2) - UU(0));
  T S2 = c1312 * sq(UU(3) - T(2) * UU(2) + UU(1)) + c14 * sq(UU(3) - T(4) * UU(2) + T(3) * UU(1));
  T a0 = C03 / sq(ep + S0), a1 = C13 / sq(ep + S1), a2 = C23 / sq(ep + S2);
  T am = a0 + a1 + a2;
  T q03 = c13 * UU(1) + c56 * UU(0) - c16 * UU(-1);
  T q13 = -c16 * UU(2) + c56 * UU(1) + c13 * UU(0);
  T q23 = c13 * UU(3) - c76 * UU(2) + c116 * UU(1);
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
// WENO7 (sub_scheme.f90:144-277): weno7_R is weno7_L with the stencil mirrored.
template <class T> __device__ __forceinline__ T weno7_core(T vm3, T vm2, T vm1, T v0, T v1, T v2, T v3) {
  const T C0 = T(1.0 / 35.0), C1 = T(12.0 / 35.0), C2 = T(18.0 / 35.0), C3 = T(4.0 / 35.0);
  const T a11 = T(-2.0 / 6.0), a12 = T(9.0 / 6.0), a13 = T(-18.0 / 6.0), a14 = T(11.0 / 6.0);
  const T a21 = T(1.0 / 6.0), a23 = T(3.0 / 6.0), a24 = T(2.0 / 6.0);
  const T a31 = T(-2.0 / 6.0), a32 = T(-3.0 / 6.0), a34 = T(-1.0 / 6.0);
  const T a41 = T(-11.0 / 6.0), a42 = T(18.0 / 6.0), a43 = T(-9.0 / 6.0), a44 = T(2.0 / 6.0);
  const T b12 = T(4), b13 = T(-5), b14 = T(2), b22 = T(-2), b41 = T(2), b42 = T(-5), b43 = T(4), c12 = T(3);
  const T d12 = T(13.0 / 12.0), d13 = T(1043.0 / 960.0), d14 = T(1.0 / 12.0);
  const T e11 = T(-3.0 / 12.0), e12 = T(13.0 / 12.0), e13 = T(-23.0 / 12.0), e14 = T(25.0 / 12.0);
  const T e21 = T(1.0 / 12.0), e22 = T(-5.0 / 12.0), e23 = T(13.0 / 12.0), e24 = T(3.0 / 12.0);
  const T e31 = T(-1.0 / 12.0), e32 = T(7.0 / 12.0), e33 = T(7.0 / 12.0), e34 = T(-1.0 / 12.0);
  const T e41 = T(3.0 / 12.0), e42 = T(13.0 / 12.0), e43 = T(-5.0 / 12.0), e44 = T(1.0 / 12.0);
  const T ep = T(1.e-8);
  T S10 = a11 * vm3 + a12 * vm2 + a13 * vm1 + a14 * v0;
  T S11 = a21 * vm2 - vm1 + a23 * v0 + a24 * v1;
  T S12 = a31 * vm1 + a32 * v0 + v1 + a34 * v2;
  T S13 = a41 * v0 + a42 * v1 + a43 * v2 + a44 * v3;
  T S20 = -vm3 + b12 * vm2 + b13 * vm1 + b14 * v0;
  T S21 = vm1 + b22 * v0 + v1;
  T S22 = v0 + b22 * v1 + v2;
  T S23 = b41 * v0 + b42 * v1 + b43 * v2 - v3;
  T S30 = -vm3 + c12 * (vm2 - vm1) + v0;
  T S31 = -vm2 + c12 * (vm1 - v0) + v1;
  T S32 = -vm1 + c12 * (v0 - v1) + v2;
  T S33 = -v0 + c12 * (v1 - v2) + v3;
  T S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  T S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  T S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  T S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  T a0 = C0 / sq(ep + S0), a1 = C1 / sq(ep + S1), a2 = C2 / sq(ep + S2), a3 = C3 / sq(ep + S3);
  T am = a0 + a1 + a2 + a3;
  T q0 = e11 * vm3 + e12 * vm2 + e13 * vm1 + e14 * v0;
  T q1 = e21 * vm2 + e22 * vm1 + e23 * v0 + e24 * v1;
  T q2 = e31 * vm1 + e32 * v0 + e33 * v1 + e34 * v2;
  T q3 = e41 * v0 + e42 * v1 + e43 * v2 + e44 * v3;
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}

template <class T> __device__ __forceinline__ void scheme_LR(const T* u, int s, T& L, T& R) {  // scheme_fP / scheme_fm
  const T k2c = T(1), k2u = T(-1), b2 = T(2), k3 = T(1.0 / 3.0), sep = T(1.e-6);
  const T eta = T((double)0.05f);  // OMUSCL2 `eta=0.05` is a default-real literal
  switch (s) {
    case S_CD2: L = T(0.5) * (UU(0) + UU(1)); R = L; return;
    case S_UD1: L = UU(0); R = UU(1); return;
    case S_UD3: L = (-UU(-1) + T(5) * UU(0) + T(2) * UU(1)) / T(6); R = (T(2) * UU(0) + T(5) * UU(1) - UU(2)) / T(6); return;
    case S_NND2:
      L = UU(0) + T(0.5) * minmod(UU(0) - UU(-1), UU(1) - UU(0));
      R = UU(1) - T(0.5) * minmod(UU(1) - UU(0), UU(2) - UU(1));
      return;
    case S_MUSCL2U:
    case S_MUSCL2C: {
      T kk = s == S_MUSCL2U ? k2u : k2c;
      L = UU(0) + T(0.25) * ((T(1) - kk) * minmod(UU(0) - UU(-1), b2 * (UU(1) - UU(0))) + (T(1) + kk) * minmod(UU(1) - UU(0), b2 * (UU(0) - UU(-1))));
      R = UU(1) - T(0.25) * ((T(1) - kk) * minmod(UU(2) - UU(1), b2 * (UU(1) - UU(0))) + (T(1) + kk) * minmod(UU(1) - UU(0), b2 * (UU(2) - UU(1))));
      return;
    }
    case S_MUSCL3: {
      T up = UU(1) - UU(0), um = UU(0) - UU(-1);
      T s_ = (T(2) * up * um + sep) / (up * up + um * um + sep);
      L = UU(0) + T(0.25) * s_ * ((T(1) - k3 * s_) * um + (T(1) + k3 * s_) * up);
      up = UU(2) - UU(1); um = UU(1) - UU(0);
      s_ = (T(2) * up * um + sep) / (up * up + um * um + sep);
      R = UU(1) - T(0.25) * s_ * ((T(1) - k3 * s_) * up + (T(1) + k3 * s_) * um);
      return;
    }
    case S_OMUSCL2: {
      T r1 = (UU(0) - UU(-1) + sep) / (UU(1) - UU(0) + sep), r2 = (UU(1) - UU(0) + sep) / (UU(2) - UU(1) + sep);
      T f1 = (T(1) - eta) + (eta - T(0.55)) * T(0.5) / r2 + (eta + T(0.55)) * T(0.5) * r1;
      T f = fmax_(T(0), fmin_(fmin_(T(2), f1), T(2) * r1));
      L = UU(0) + T(0.5) * f * (UU(1) - UU(0));
      r1 = (UU(2) - UU(1) + sep) / (UU(1) - UU(0) + sep); r2 = (UU(1) - UU(0) + sep) / (UU(0) - UU(-1) + sep);
      f1 = (T(1) - eta) + (eta - T(0.55)) * T(0.5) / r2 + (eta + T(0.55)) * T(0.5) * r1;
      f = fmax_(T(0), fmin_(fmin_(T(2), f1), T(2) * r1));
      R = UU(1) - T(0.5) * f * (UU(1) - UU(0));
      return;
    }
    case S_WENO5: L = weno5_L(u); R = weno5_R(u); return;
    case S_WENO7:
      L = weno7_core(UU(-3), UU(-2), UU(-1), UU(0), UU(1), UU(2), UU(3));
      R = weno7_core(UU(4), UU(3), UU(2), UU(1), UU(0), UU(-1), UU(-2));
      return;
    case S_UD5:
      L = (T(2) * UU(-2) - T(13) * UU(-1) + T(47) * UU(0) + T(27) * UU(1) - T(3) * UU(2)) / T(60);
      R = (T(-3) * UU(-1) + T(27) * UU(0) + T(47) * UU(1) - T(13) * UU(2) + T(2) * UU(3)) / T(60);
      return;
  }
  L = T(0); R = T(0);
}
#undef UU

// ---------------- 1-D fluxes, sub_flux_split.f90 ----------------------------------------------
template <class T> __device__ __forceinline__ void flux_hll_hllc(const T* QL, const T* QR, T* F, T gamma, int iflux) {  // 13-95
  T dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  T dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  T UL[5], UR[5], Fl[5], Fr[5];
  UL[0] = dl; UL[1] = dl * uul; UL[2] = dl * vvl; UL[3] = dl * wwl; UL[4] = pl / (gamma - T(1)) + dl * (uul * uul + vvl * vvl + wwl * wwl) * T(0.5);
  UR[0] = dr; UR[1] = dr * uur; UR[2] = dr * vvr; UR[3] = dr * wwr; UR[4] = pr / (gamma - T(1)) + dr * (uur * uur + vvr * vvr + wwr * wwr) * T(0.5);
  T al = dsqrt(gamma * pl / dl), ar = dsqrt(gamma * pr / dr);
  T p_pvrs = T(0.5) * (pl + pr) - (uur - uul) * (dl + dr) * (al + ar) * T(0.125);
  T p_star = fmax_(T(0), p_pvrs);
  T qql, qqr;
  if (p_star <= pl) qql = T(1); else qql = dsqrt(T(1) + ((gamma + T(1)) / (T(2) * gamma)) * (p_star / pl - T(1)));
  if (p_star <= pr) qqr = T(1); else qqr = dsqrt(T(1) + ((gamma + T(1)) / (T(2) * gamma)) * (p_star / pr - T(1)));
  T Sl = uul - al * qql, Sr = uur + ar * qqr;
  Fl[0] = UL[1]; Fl[1] = UL[1] * uul + pl; Fl[2] = UL[2] * uul; Fl[3] = UL[3] * uul; Fl[4] = uul * (UL[4] + pl);
  Fr[0] = UR[1]; Fr[1] = UR[1] * uur + pr; Fr[2] = UR[2] * uur; Fr[3] = UR[3] * uur; Fr[4] = uur * (UR[4] + pr);
  if (iflux == F_HLL) {
    if (Sl >= T(0)) { for (int m = 0; m < 5; m++) F[m] = Fl[m]; }
    else if (Sr <= T(0)) { for (int m = 0; m < 5; m++) F[m] = Fr[m]; }
    else { for (int m = 0; m < 5; m++) F[m] = (Sr * Fl[m] - Sl * Fr[m] + Sl * Sr * (UR[m] - UL[m])) / (Sr - Sl); }
    return;
  }
  T S_star = (pr - pl + dl * uul * (Sl - uul) - dr * uur * (Sr - uur)) / (dl * (Sl - uul) - dr * (Sr - uur));
  if (Sl >= T(0)) { for (int m = 0; m < 5; m++) F[m] = Fl[m]; return; }
  if (Sr <= T(0)) { for (int m = 0; m < 5; m++) F[m] = Fr[m]; return; }
  if (S_star >= T(0)) {
    T tmpl = dl * (Sl - uul) / (Sl - S_star);
    F[0] = Fl[0] + Sl * (tmpl - UL[0]);
    F[1] = Fl[1] + Sl * (tmpl * S_star - UL[1]);
    F[2] = Fl[2] + Sl * (tmpl * vvl - UL[2]);
    F[3] = Fl[3] + Sl * (tmpl * wwl - UL[3]);
    T tmp = UL[4] / dl + (S_star - uul) * (S_star + pl / (dl * (Sl - uul)));
    F[4] = Fl[4] + Sl * (tmpl * tmp - UL[4]);
  } else {
    T tmpr = dr * (Sr - uur) / (Sr - S_star);
    F[0] = Fr[0] + Sr * (tmpr - UR[0]);
    F[1] = Fr[1] + Sr * (tmpr * S_star - UR[1]);
    F[2] = Fr[2] + Sr * (tmpr * vvr - UR[2]);
    F[3] = Fr[3] + Sr * (tmpr * vvr - UR[3]);  // vvr, as the reference (sub_flux_split.f90:67)
    T tmp = UR[4] / dr + (S_star - uur) * (S_star + pr / (dr * (Sr - uur)));
    F[4] = Fr[4] + Sr * (tmpr * tmp - UR[4]);
  }
}

template <class T> __device__ __forceinline__ void flux_sw(const T* QL, const T* QR, T* F, T gamma) {  // 102-141
  T dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  T dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  T al = dsqrt(gamma * pl / dl), ar = dsqrt(gamma * pr / dr);
  T tmp1 = T(2) * (gamma - T(1)), tmp3 = (T(3) - gamma) / (T(2) * (gamma - T(1)));
  T E1P = (uul + dabs(uul)) * T(0.5), E2P = (uul - al + dabs(uul - al)) * T(0.5), E3P = (uul + al + dabs(uul + al)) * T(0.5);
  T tmp0 = dl / (T(2) * gamma);
  T fp0 = tmp0 * (tmp1 * E1P + E2P + E3P);
  T fp1 = tmp0 * (tmp1 * E1P * uul + E2P * (uul - al) + E3P * (uul + al));
  T fp2 = tmp0 * (tmp1 * E1P * vvl + E2P * vvl + E3P * vvl);
  T fp3 = tmp0 * (tmp1 * E1P * wwl + E2P * wwl + E3P * wwl);
  T fp4 = tmp0 * (E1P * (gamma - T(1)) * (uul * uul + vvl * vvl + wwl * wwl) + E2P * (sq(uul - al) + vvl * vvl + wwl * wwl) * T(0.5) +
                  E3P * (sq(uul + al) + vvl * vvl + wwl * wwl) * T(0.5) + tmp3 * al * al * (E2P + E3P));
  T E1M = (uur - dabs(uur)) * T(0.5), E2M = (uur - ar - dabs(uur - ar)) * T(0.5), E3M = (uur + ar - dabs(uur + ar)) * T(0.5);
  tmp0 = dr / (T(2) * gamma);
  T fm0 = tmp0 * (tmp1 * E1M + E2M + E3M);
  T fm1 = tmp0 * (tmp1 * E1M * uur + E2M * (uur - ar) + E3M * (uur + ar));
  T fm2 = tmp0 * (tmp1 * E1M * vvr + E2M * vvr + E3M * vvr);
  T fm3 = tmp0 * (tmp1 * E1M * wwr + E2M * wwr + E3M * wwr);
  T fm4 = tmp0 * (E1M * (gamma - T(1)) * (uur * uur + vvr * vvr + wwr * wwr) + E2M * (sq(uur - ar) + vvr * vvr + wwr * wwr) * T(0.5) +
                  E3M * (sq(uur + ar) + vvr * vvr + wwr * wwr) * T(0.5) + tmp3 * ar * ar * (E2M + E3M));
  F[0] = fp0 + fm0; F[1] = fp1 + fm1; F[2] = fp2 + fm2; F[3] = fp3 + fm3; F[4] = fp4 + fm4;
}

template <class T> __device__ __forceinline__ void flux_roe(const T* QL, const T* QR, T* F, T gamma) {  // 148-210
  const T delt = T(0.1);
  const T e8 = T((double)1.e-8f);  // `1.e-8` default-real literal (lines 195, 197)
  T dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  T dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  T hl = gamma * pl / ((gamma - T(1)) * dl) + T(0.5) * (uul * uul + vvl * vvl + wwl * wwl);
  T hr = gamma * pr / ((gamma - T(1)) * dr) + T(0.5) * (uur * uur + vvr * vvr + wwr * wwr);
  T UL1 = dl * uul, UL2 = dl * vvl, UL3 = dl * wwl, UL4 = pl / (gamma - T(1)) + dl * (uul * uul + vvl * vvl + wwl * wwl) * T(0.5);
  T UR1 = dr * uur, UR2 = dr * vvr, UR3 = dr * wwr, UR4 = pr / (gamma - T(1)) + dr * (uur * uur + vvr * vvr + wwr * wwr) * T(0.5);
  T Fl0 = UL1, Fl1 = UL1 * uul + pl, Fl2 = UL2 * uul, Fl3 = UL3 * uul, Fl4 = uul * (UL4 + pl);
  T Fr0 = UR1, Fr1 = UR1 * uur + pr, Fr2 = UR2 * uur, Fr3 = UR3 * uur, Fr4 = uur * (UR4 + pr);
  T tmpp = dsqrt(dr / dl);
  T avu = (uul + tmpp * uur) / (T(1) + tmpp);
  T avv = (vvl + tmpp * vvr) / (T(1) + tmpp);
  T avw = (wwl + tmpp * wwr) / (T(1) + tmpp);
  T avh = (hl + tmpp * hr) / (T(1) + tmpp);
  T ava = dsqrt((gamma - T(1)) * (avh - T(0.5) * (avu * avu + avv * avv + avw * avw)));
  T l1 = dabs(avu - ava), l2 = dabs(avu), l3 = dabs(avu + ava);
  if (l1 < delt) l1 = (sq(l1) + delt * delt) / (T(2) * delt);
  if (l2 < delt) l2 = (sq(l2) + delt * delt) / (T(2) * delt);
  if (l3 < delt) l3 = (sq(l3) + delt * delt) / (T(2) * delt);
  T arr2 = (UR2 - UL2) / (avv + e8) - (dr - dl);
  T arr3 = (UR3 - UL3) / (avw + e8) - (dr - dl);
  T arr4 = (gamma - T(1)) * ((dr - dl) * (avh - avu * avu - avv * avv - avw * avw) + avu * (UR1 - UL1) + avv * (UR2 - UL2) + avw * (UR3 - UL3) - (UR4 - UL4)) / (ava * ava);
  T arr1 = ((avu + ava) * (dr - dl) - UR1 + UL1 - ava * arr4) / (T(2) * ava);
  T arr5 = dr - dl - (arr1 + arr4);
  F[0] = T(0.5) * (Fl0 + Fr0) - T(0.5) * (l1 * arr1 + l2 * arr4 + l3 * arr5);
  F[1] = T(0.5) * (Fl1 + Fr1) - T(0.5) * (l1 * arr1 * (avu - ava) + l2 * arr4 * avu + l3 * arr5 * (avu + ava));
  F[2] = T(0.5) * (Fl2 + Fr2) - T(0.5) * (l1 * arr1 * avv + l2 * arr2 * avv + l2 * arr4 * avv + l3 * arr5 * avv);
  F[3] = T(0.5) * (Fl3 + Fr3) - T(0.5) * (l1 * arr1 * avw + l2 * arr3 * avw + l2 * arr4 * avw + l3 * arr5 * avw);
  F[4] = T(0.5) * (Fl4 + Fr4) - T(0.5) * (l1 * arr1 * (avh - avu * ava) + l2 * arr2 * avv * avv + l2 * arr3 * avw * avw +
                                          l2 * arr4 * T(0.5) * (avu * avu + avv * avv + avw * avw) + l3 * arr5 * (avh + avu * ava));
}

template <class T> __device__ __forceinline__ void flux_vl(const T* QL, const T* QR, T* F, T gamma) {  // 217-275
  T dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  T dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  T al = dsqrt(gamma * pl / dl), ar = dsqrt(gamma * pr / dr);
  T Ml = uul / al, Mr = uur / ar;
  T fp[5] = {T(0), T(0), T(0), T(0), T(0)}, fm[5] = {T(0), T(0), T(0), T(0), T(0)};
  if (Ml >= T(1)) {
    fp[0] = dl * uul; fp[1] = dl * uul * uul + pl; fp[2] = dl * uul * vvl; fp[3] = dl * uul * wwl;
    fp[4] = uul * (gamma * pl / (gamma - T(1)) + T(0.5) * dl * (uul * uul + vvl * vvl + wwl * wwl));
  } else if (dabs(Ml) < T(1)) {
    T Mp = T(0.25) * (T(1) + Ml) * (T(1) + Ml), tmp0 = dl * al * Mp;
    fp[0] = tmp0; fp[1] = tmp0 * ((gamma - T(1)) * uul + T(2) * al) / gamma; fp[2] = tmp0 * vvl; fp[3] = tmp0 * wwl;
    fp[4] = tmp0 * (((gamma - T(1)) * uul + T(2) * al) * ((gamma - T(1)) * uul + T(2) * al) * T(0.5) / (gamma * gamma - T(1)) + T(0.5) * (vvl * vvl + wwl * wwl));
  }
  if (Mr >= T(1)) {
  } else if (dabs(Mr) < T(1)) {
    T Mm = T(-0.25) * (Mr - T(1)) * (Mr - T(1)), tmp0 = dr * ar * Mm;
    fm[0] = tmp0; fm[1] = tmp0 * ((gamma - T(1)) * uur - T(2) * ar) / gamma; fm[2] = tmp0 * vvr; fm[3] = tmp0 * wwr;
    fm[4] = tmp0 * (((gamma - T(1)) * uur - T(2) * ar) * ((gamma - T(1)) * uur - T(2) * ar) * T(0.5) / (gamma * gamma - T(1)) + T(0.5) * (vvr * vvr + wwr * wwr));
  } else if (Mr <= T(-1)) {
    fm[0] = dr * uur; fm[1] = dr * uur * uur + pr; fm[2] = dr * uur * vvr; fm[3] = dr * uur * wwr;
    fm[4] = uur * (gamma * pr / (gamma - T(1)) + T(0.5) * dr * (uur * uur + vvr * vvr + wwr * wwr));
  }
  for (int m = 0; m < 5; m++) F[m] = fp[m] + fm[m];
}

template <class T> __device__ __forceinline__ void flux_ausmpw(const T* QL, const T* QR, T* F, T gamma) {  // 356-442
  T dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  T dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  T hl = gamma * pl / ((gamma - T(1)) * dl) + T(0.5) * (uul * uul + vvl * vvl + wwl * wwl);
  T hr = gamma * pr / ((gamma - T(1)) * dr) + T(0.5) * (uur * uur + vvr * vvr + wwr * wwr);
  T al = dsqrt(gamma * pl / dl), ar = dsqrt(gamma * pr / dr);
  T a = T(0.5) * (al + ar), Ml = uul / a, Mr = uur / a;
  T rmin = fmin_(pl / pr, pr / pl);
  T wpl = T(1) - dpow(rmin, T(3));
  T plpl = ((T(0.75) <= rmin) && (T(1) > rmin)) ? T(4) * rmin - T(3) : T(0);
  T rmin2 = fmin_(pr / pl, pl / pr);
  T plpr = ((T(0.75) <= rmin2) && (T(1) > rmin2)) ? T(4) * rmin2 - T(3) : T(0);
  T Pp5, Pm5;
  if (dabs(Ml) >= T(1)) Pp5 = T(0.5) * (Ml + dabs(Ml)) / Ml;
  else Pp5 = T(0.25) * (Ml + T(1)) * (Ml + T(1)) * (T(2) - Ml) + T(3) * Ml * (Ml * Ml - T(1)) * (Ml * Ml - T(1)) / T(16);
  if (dabs(Mr) >= T(1)) Pm5 = T(0.5) * (Mr - dabs(Mr)) / Mr;
  else Pm5 = T(0.25) * (Mr - T(1)) * (Mr - T(1)) * (T(2) + Mr) - T(3) * Mr * (Mr * Mr - T(1)) * (Mr * Mr - T(1)) / T(16);
  T p = pl * Pp5 + pr * Pm5;
  T Mp4, Mm4, fL, fR;
  if (dabs(Ml) >= T(1)) { Mp4 = T(0.5) * (Ml + dabs(Ml)); fL = T(0); }
  else {
    Mp4 = T(0.25) * (Ml + T(1)) * (Ml + T(1)) + T(0.125) * (Ml * Ml - T(1)) * (Ml * Ml - T(1));
    fL = (pl / p - T(1)) * plpl * dabs(T(0.25) * (Ml + T(1)) * (Ml + T(1))) * fmin_(T(1), dpow(dsqrt(uul * uul + vvl * vvl + wwl * wwl) / a, T(0.25)));
  }
  if (dabs(Mr) >= T(1)) { Mm4 = T(0.5) * (Mr - dabs(Mr)); fR = T(0); }
  else {
    Mm4 = T(-0.25) * (Mr - T(1)) * (Mr - T(1)) - T(0.125) * (Mr * Mr - T(1)) * (Mr * Mr - T(1));
    fR = (pr / p - T(1)) * plpr * dabs(T(-0.25) * (Mr - T(1)) * (Mr - T(1))) * fmin_(T(1), dpow(dsqrt(uur * uur + vvr * vvr + wwr * wwr) / a, T(0.25)));
  }
  T M = Mp4 + Mm4, MLp, MRm;
  if (M >= T(0)) MLp = Mp4 + Mm4 - Mm4 * wpl * (T(1) + fR) + (fL * Mp4 + fR * Mm4); else MLp = Mp4 * wpl * (T(1) + fL);
  if (M < T(0)) MRm = Mp4 + Mm4 - Mp4 * wpl * (T(1) + fL) + (fL * Mp4 + fR * Mm4); else MRm = Mm4 * wpl * (T(1) + fR);
  F[0] = MLp * a * dl + MRm * a * dr;
  F[1] = MLp * a * (dl * uul) + MRm * a * (dr * uur) + p;
  F[2] = MLp * a * (dl * vvl) + MRm * a * (dr * vvr);
  F[3] = MLp * a * (dl * wwl) + MRm * a * (dr * wwr);
  F[4] = MLp * a * (dl * hl) + MRm * a * (dr * hr);
}

template <class T> __device__ __forceinline__ void flux_1d(const T* QL, const T* QR, T* F, T gamma, int iflux) {
  if (iflux == F_ROE) flux_roe(QL, QR, F, gamma);
  else if (iflux == F_SW) flux_sw(QL, QR, F, gamma);
  else if (iflux == F_VL) flux_vl(QL, QR, F, gamma);
  else if (iflux == F_AUSM) flux_ausmpw(QL, QR, F, gamma);
  else flux_hll_hllc(QL, QR, F, gamma, iflux);
}

}  // namespace ocfd
