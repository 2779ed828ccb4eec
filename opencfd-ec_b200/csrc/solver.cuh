// Solver kernels of the per-iteration hot path (one NS_Time_advance, sub_time_advance.f90:6-23).
// Templated on T, the precision of reconstruction / fluxes / sources / metrics / Res / dt / Lc /
// Lv: double for the FP64 path, float for the mixed path.  State U, DU, the LU-SGS diagonal and
// divide, the limiter test, norms and forces are FP64 in both.
//
// U6/U7 clamp: limit_vt (sub_time_advance.f90:410-443) sets U6/U7 < 0 to 0 on the 0..n box before
// the residual, while the LU-SGS update uses Un saved before that clamp (Set_Un, 635-656).  Here U
// is never clamped in place; every read of U6/U7 during the residual, LU-SGS and RK3 stage update
// applies the clamp instead ("clamp on read"), which gives the same values and keeps the
// unclamped interior for U = Un + DU.  The clamped ghost values of the reference are always
// rewritten by BC + halo + corner averaging before the step ends.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.h"
#include "physics.cuh"

// residual kernels bound by memory latency: at most 64 registers, four 256-thread CTAs per SM
#ifndef OCFD_MEM_MINB
#define OCFD_MEM_MINB 4
#endif

namespace ocfd {

#define OCFD_GRID_STRIDE(g, n) for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < (n); g += (long long)gridDim.x * blockDim.x)

__device__ __forceinline__ int find_blk(const long long* pre, int n, long long g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(pre + mid) <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}
// the same block as find_blk, from the chunk's hint: one table load and (usually) one check of
// the next block's start instead of log2(nblk) dependent loads
__device__ __forceinline__ int find_blk_h(const long long* pre, const int* hint, int n, long long g) {
  int b = __ldg(hint + (g >> HINT_SHIFT));
  while (b + 1 < n && __ldg(pre + b + 1) <= g) b++;
  return b;
}
__device__ __forceinline__ long long bix(const BlkD& B, int i, int j, int k) {
  return B.obox + (long long)(i + 3) + (long long)B.NX * ((long long)(j + 3) + (long long)B.NY * (long long)(k + 3));
}
__device__ __forceinline__ long long fix_(const BlkD& B, int i, int j, int k) {
  return B.oface + (long long)(i - 1) + (long long)B.nx * ((long long)(j - 1) + (long long)B.ny * (long long)(k - 1));
}
__device__ __forceinline__ long long cix(const BlkD& B, int i, int j, int k) {
  return B.ocell + (long long)(i - 1) + (long long)(B.nx - 1) * ((long long)(j - 1) + (long long)(B.ny - 1) * (long long)(k - 1));
}
__device__ __forceinline__ long long nix(const BlkD& B, int i, int j, int k) {
  return B.onode + (long long)i + (long long)B.NXn * ((long long)j + (long long)B.NYn * (long long)k);
}
__device__ __forceinline__ double clamp0(double v) { return v < 0.0 ? 0.0 : v; }
template <class T> __device__ __forceinline__ T ld(const T* p, long long i) { return p[i]; }

// decode helpers: index within a block -> (i,j,k).  A block's ghost box holds fewer than 2^31
// cells (ocfd_create checks it), so the decode divides in 32 bits instead of 64.
__device__ __forceinline__ void dec_cell(const BlkD& B, long long l, int& i, int& j, int& k) {
  const unsigned u = (unsigned)l, nxm = (unsigned)(B.nx - 1), nym = (unsigned)(B.ny - 1);
  const unsigned t = u / nxm;
  i = (int)(u - t * nxm) + 1; j = (int)(t % nym) + 1; k = (int)(t / nym) + 1;
}
__device__ __forceinline__ void dec_face(const BlkD& B, long long l, int& i, int& j, int& k) {
  const unsigned u = (unsigned)l, nx = (unsigned)B.nx, ny = (unsigned)B.ny;
  const unsigned t = u / nx;
  i = (int)(u - t * nx) + 1; j = (int)(t % ny) + 1; k = (int)(t / ny) + 1;
}
__device__ __forceinline__ void dec_box(const BlkD& B, long long l, int& i, int& j, int& k) {
  const unsigned u = (unsigned)l, NX = (unsigned)B.NX, NY = (unsigned)B.NY;
  const unsigned t = u / NX;
  i = (int)(u - t * NX) - 3; j = (int)(t % NY) - 3; k = (int)(t / NY) - 3;
}

// a block's primitive region (cells 1-glo .. n-1+ghi) and its 0..n layer
__device__ __forceinline__ void dec_reg(const BlkD& B, long long l, int& i, int& j, int& k) {
  const unsigned u = (unsigned)l, RX = (unsigned)B.RX, RY = (unsigned)B.RY;
  const unsigned t = u / RX;
  i = (int)(u - t * RX) + 1 - B.glo[0]; j = (int)(t % RY) + 1 - B.glo[1]; k = (int)(t / RY) + 1 - B.glo[2];
}
__device__ __forceinline__ void dec_r1(const BlkD& B, long long l, int& i, int& j, int& k) {
  const unsigned u = (unsigned)l, X = (unsigned)(B.nx + 1), Y = (unsigned)(B.ny + 1);
  const unsigned t = u / X;
  i = (int)(u - t * X); j = (int)(t % Y); k = (int)(t / Y);
}

// ============================================================================================
// primitives (comput_duvtpc, sub_Residual.f90:1417-1456) on the cells a residual reads: the
// reference fills the whole ghost box, of which the stencils across a physical face read only
// the layers their boundary scheme reaches (BlkD::glo/ghi); the cells left out are never read
// ============================================================================================
template <class T>
__global__ void k_prim(Arena<T> A) {
  const long long tb = A.tot_box, tr = __ldg(A.pre_reg + A.nblk);
  OCFD_GRID_STRIDE(r, tr) {
    const int b = find_blk_h(A.pre_reg, A.hint_reg, A.nblk, r);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_reg(B, r - __ldg(A.pre_reg + b), i, j, k);
    const long long g = bix(B, i, j, k);
    const SolveP& s = A.sp[B.solve];
    double d = A.U[g], u1 = A.U[tb + g], u2 = A.U[2 * tb + g], u3 = A.U[3 * tb + g], u4 = A.U[4 * tb + g];
    double uu = u1 / d, v = u2 / d, w = u3 / d;
    double Tt = (u4 - 0.5 * d * (uu * uu + v * v + w * w)) / (s.cv * d);
    A.P[P_D * tb + g] = T(d);
    A.P[P_U * tb + g] = T(uu);
    A.P[P_V * tb + g] = T(v);
    A.P[P_W * tb + g] = T(w);
    A.P[P_T * tb + g] = T(Tt);
    A.P[P_P * tb + g] = T(s.p00 * d * Tt);
    A.P[P_C * tb + g] = T(sqrt(Tt) / s.ma);
  }
}

// get_viscous (sub_Residual.f90:1355-1383): Sutherland mu on the interior + the 6 face ghost
// layers (edge/corner ghosts keep their previous values, as in the reference)
template <class T>
__global__ void k_mu(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, A.tot_cell) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    double Tt = (double)A.P[P_T * tb + bix(B, i, j, k)];
    T mu = T(1.0 / s.re * (1.0 + s.tsb) * sqrt(cube(Tt)) / (s.tsb + Tt));
    A.mu[bix(B, i, j, k)] = mu;
    if (i == 1) A.mu[bix(B, 0, j, k)] = mu;
    if (i == B.nx - 1) A.mu[bix(B, B.nx, j, k)] = mu;
    if (j == 1) A.mu[bix(B, i, 0, k)] = mu;
    if (j == B.ny - 1) A.mu[bix(B, i, B.ny, k)] = mu;
    if (k == 1) A.mu[bix(B, i, j, 0)] = mu;
    if (k == B.nz - 1) A.mu[bix(B, i, j, B.nz)] = mu;
  }
}

// ============================================================================================
// turbulence: SA (sub_turbulence_SA.f90) and SST (sub_turbulence_SST.f90)
// ============================================================================================
namespace sa {
constexpr double sigma = 2.0 / 3.0, Cb1 = 0.1355, Cb2 = 0.622, kap = 0.41;
constexpr double Cw2 = 0.3, Ct3 = 1.2, Ct4 = 0.5;
constexpr double Cv1_3 = 357.91099999999994;  // Cv1**3 (7.1d0**3), constant-folded by the compiler
constexpr double Cw3_6 = 64.0;
__device__ __forceinline__ double Cw1() { return Cb1 / (kap * kap) + (1.0 + Cb2) / sigma; }
}  // namespace sa

// mu *= Re, mu_t = fv1 rho vt, first limit_mut (SA.f90:37-64), on the 0..n box
template <class T>
__global__ void k_sa_pre(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(r, A.tot_r1) {
    const int b = find_blk_h(A.pre_r1, A.hint_r1, A.nblk, r);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_r1(B, r - B.or1, i, j, k);
    const long long g = bix(B, i, j, k);
    const SolveP& s = A.sp[B.solve];
    T mu = T((double)A.mu[g] * s.re);
    T vt = T(clamp0(A.U[5 * tb + g]));
    T d = A.P[P_D * tb + g];
    A.mu[g] = mu;  // after the loads: a store before them would hold them back
    T X = d * vt / mu;
    T fv1 = cube(X) / (cube(X) + T(sa::Cv1_3));
    T mut = fv1 * d * vt;
    if (mut < T(0)) mut = T(0);
    if (s.mut_max >= 0.0 && mut > T(s.mut_max) * mu) mut = T(s.mut_max) * mu;
    A.mut[g] = mut;
  }
}

// SA face fluxes Fluxv / Fluxv2 (SA.f90:74-96, 110-131, 145-167) for direction DIR
template <class T, int DIR, class VT>
__device__ __forceinline__ void sa_face_vt(const Arena<T>& A, const BlkD& B, const SolveP& s, int i, int j, int k, long long g, T& Fo,
                                           T& Go, VT vt);
// one face of direction DIR: the SA convection + diffusion flux F and the gradient flux G (the
// face's two Ft plane entries)
template <class T, int DIR>
__device__ __forceinline__ void sa_face(const Arena<T>& A, const BlkD& B, const SolveP& s, int i, int j, int k, long long g, T& Fo,
                                        T& Go) {
  const long long tb = A.tot_box;
  sa_face_vt<T, DIR>(A, B, s, i, j, k, g, Fo, Go, [&](int a, int c, int e) -> T { return T(clamp0(A.U[5 * tb + bix(B, a, c, e)])); });
}
// the same, the SA variable's values (clamped at 0) from vt(i, j, k)
template <class T, int DIR, class VT>
__device__ __forceinline__ void sa_face_vt(const Arena<T>& A, const BlkD& B, const SolveP& s, int i, int j, int k, long long g, T& Fo,
                                           T& Go, VT vt) {
  const long long tb = A.tot_box, tf = A.tot_face;
  const int di = DIR == 0, dj = DIR == 1, dk = DIR == 2;
  const int im = i - di, jm = j - dj, km = k - dk;  // the other cell of the face
  T s1x = A.M[(M_NI1 + 3 * DIR) * tf + g], s1y = A.M[(M_NI2 + 3 * DIR) * tf + g], s1z = A.M[(M_NI3 + 3 * DIR) * tf + g];
  T S = A.M[(M_SI + DIR) * tf + g];
  T vti, vtj, vtk;
  if (DIR == 0) {
    vti = vt(i, j, k) - vt(i - 1, j, k);
    vtj = T(0.25) * (vt(i, j + 1, k) - vt(i, j - 1, k) + vt(i - 1, j + 1, k) - vt(i - 1, j - 1, k));
    vtk = T(0.25) * (vt(i, j, k + 1) - vt(i, j, k - 1) + vt(i - 1, j, k + 1) - vt(i - 1, j, k - 1));
  } else if (DIR == 1) {
    vti = T(0.25) * (vt(i + 1, j, k) - vt(i - 1, j, k) + vt(i + 1, j - 1, k) - vt(i - 1, j - 1, k));
    vtj = vt(i, j, k) - vt(i, j - 1, k);
    vtk = T(0.25) * (vt(i, j, k + 1) - vt(i, j, k - 1) + vt(i, j - 1, k + 1) - vt(i, j - 1, k - 1));
  } else {
    vti = T(0.25) * (vt(i + 1, j, k) - vt(i - 1, j, k) + vt(i + 1, j, k - 1) - vt(i - 1, j, k - 1));
    vtj = T(0.25) * (vt(i, j + 1, k) - vt(i, j - 1, k) + vt(i, j + 1, k - 1) - vt(i, j - 1, k - 1));
    vtk = vt(i, j, k) - vt(i, j, k - 1);
  }
  const int J = DIR == 0 ? M_J1 : (DIR == 1 ? M_J2 : M_J3);
  T ix = A.M[(J + 0) * tf + g], iy = A.M[(J + 1) * tf + g], iz = A.M[(J + 2) * tf + g];
  T jx = A.M[(J + 3) * tf + g], jy = A.M[(J + 4) * tf + g], jz = A.M[(J + 5) * tf + g];
  T kx = A.M[(J + 6) * tf + g], ky = A.M[(J + 7) * tf + g], kz = A.M[(J + 8) * tf + g];
  T vtx = vti * ix + vtj * jx + vtk * kx, vty = vti * iy + vtj * jy + vtk * ky, vtz = vti * iz + vtj * jz + vtk * kz;
  long long c0 = bix(B, i, j, k), c1 = bix(B, im, jm, km);
  T d0 = A.P[P_D * tb + c0], d1 = A.P[P_D * tb + c1];
  const T cc = T(0.5 * (1.0 + sa::Cb2) / sa::sigma);
  T v0 = cc * (vt(i, j, k) + A.mu[c0] / d0 + vt(im, jm, km) + A.mu[c1] / d1);
  T vn1 = A.P[P_U * tb + c1] * s1x + A.P[P_V * tb + c1] * s1y + A.P[P_W * tb + c1] * s1z;
  T vn2 = A.P[P_U * tb + c0] * s1x + A.P[P_V * tb + c0] * s1y + A.P[P_W * tb + c0] * s1z;
  T vfi = T(0.5) * ((vn1 + dabs(vn1)) * vt(im, jm, km) + (vn2 - dabs(vn2)) * vt(i, j, k));
  T gn = vtx * s1x + vty * s1y + vtz * s1z;
  Fo = (-vfi + v0 / T(s.re) * gn) * S;
  Go = gn * S;
}

template <class T, int DIR>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_sa_flux(Arena<T> A) {
  const long long tf = A.tot_face;
  OCFD_GRID_STRIDE(g, tf) {
    int b = find_blk_h(A.pre_face, A.hint_face, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_face(B, g - B.oface, i, j, k);
    if (DIR == 0 && (j == B.ny || k == B.nz)) continue;
    if (DIR == 1 && (i == B.nx || k == B.nz)) continue;
    if (DIR == 2 && (i == B.nx || j == B.ny)) continue;
    T F, G;
    sa_face<T, DIR>(A, B, A.sp[B.solve], i, j, k, g, F, G);
    A.Ft[(DIR * 2 + 0) * tf + g] = F;
    A.Ft[(DIR * 2 + 1) * tf + g] = G;
  }
}

// Res(6): flux sums in the i, j, k order of SA.f90:99-178 plus the source (180-254)
// Res(6) of one cell: the SA source (CFL3D form, SA.f90:188-249) added to the flux sum R, stored
template <class T>
__device__ __forceinline__ void sa_finish(const Arena<T>& A, const BlkD& B, const SolveP& s, int i, int j, int k, long long g, long long c,
                                          long long f, T vt0, T mu0, T d0, T R) {
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  const T Re = T(s.re);
  const T* Pu = A.P + P_U * tb;
  const T* Pv = A.P + P_V * tb;
  const T* Pw = A.P + P_W * tb;
  long long cip = bix(B, i + 1, j, k), cim = bix(B, i - 1, j, k), cjp = bix(B, i, j + 1, k), cjm = bix(B, i, j - 1, k);
  long long ckp = bix(B, i, j, k + 1), ckm = bix(B, i, j, k - 1);
  T ui = Pu[cip] - Pu[cim], vi = Pv[cip] - Pv[cim], wi = Pw[cip] - Pw[cim];
  T uj = Pu[cjp] - Pu[cjm], vj = Pv[cjp] - Pv[cjm], wj = Pw[cjp] - Pw[cjm];
  T uk = Pu[ckp] - Pu[ckm], vk = Pv[ckp] - Pv[ckm], wk = Pw[ckp] - Pw[ckm];
  T ix = A.M[(M_J0 + 0) * tf + f], iy = A.M[(M_J0 + 1) * tf + f], iz = A.M[(M_J0 + 2) * tf + f];
  T jx = A.M[(M_J0 + 3) * tf + f], jy = A.M[(M_J0 + 4) * tf + f], jz = A.M[(M_J0 + 5) * tf + f];
  T kx = A.M[(M_J0 + 6) * tf + f], ky = A.M[(M_J0 + 7) * tf + f], kz = A.M[(M_J0 + 8) * tf + f];
  T ux = ui * ix + uj * jx + uk * kx, vx = vi * ix + vj * jx + vk * kx, wx = wi * ix + wj * jx + wk * kx;
  T uy = ui * iy + uj * jy + uk * ky, vy = vi * iy + vj * jy + vk * ky, wy = wi * iy + wj * jy + wk * ky;
  T uz = ui * iz + uj * jz + uk * kz, vz = vi * iz + vj * jz + vk * kz, wz = wi * iz + wj * jz + wk * kz;
  (void)ux; (void)vy; (void)wz;
  T Sv = dsqrt(sq(wy - vz) + sq(uz - wx) + sq(vx - uy));
  T dw = A.dw[g];
  T X = d0 * vt0 / mu0;
  T fv1 = cube(X) / (cube(X) + T(sa::Cv1_3));
  T fv2 = T(1) - X / (T(1) + X * fv1);
  T ft2 = T(sa::Ct3) * dexp(-(T(sa::Ct4) * X * X));
  const T kap = T(sa::kap);
  T S1 = fmax_(Sv + fv2 * vt0 / (Re * sq(kap * dw)), T(0));
  T r = fmin_(vt0 / (Re * S1 * kap * kap * dw * dw), T(10));
  T gg = r + T(sa::Cw2) * (pow6(r) - r);
  T fw = gg * dpow((T(1) + T(sa::Cw3_6)) / (pow6(gg) + T(sa::Cw3_6)), T(1.0 / 6.0));
  T Q3 = T(sa::Cb1) * ((T(1) - ft2) * fv2 + ft2) / (kap * kap) - T(sa::Cw1()) * fw;
  T Q = T(sa::Cb1) * (T(1) - ft2) * S1 * vt0 + Q3 * sq(vt0 / dw) / Re;
  R = R + Q * A.vol[g];
  A.Res[5 * tc + g] = R;
}

template <class T>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_sa_res(Arena<T> A) {
  const long long tb = A.tot_box, tf = A.tot_face;
  OCFD_GRID_STRIDE(g, A.tot_cell) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    long long c = bix(B, i, j, k);
    T vt0 = T(clamp0(A.U[5 * tb + c])), mu0 = A.mu[c], d0 = A.P[P_D * tb + c];
    T Re = T(s.re);
    T v0 = (vt0 + mu0 / d0) * T(sa::Cb2) / T(sa::sigma);
    long long f = fix_(B, i, j, k);
    const T *F0 = A.Ft, *G0 = A.Ft + tf, *F1 = A.Ft + 2 * tf, *G1 = A.Ft + 3 * tf, *F2 = A.Ft + 4 * tf, *G2 = A.Ft + 5 * tf;
    long long fi1 = fix_(B, i + 1, j, k), fj1 = fix_(B, i, j + 1, k), fk1 = fix_(B, i, j, k + 1);
    T R = F0[fi1] - F0[f] - v0 / Re * (G0[fi1] - G0[f]);
    R = R + F1[fj1] - F1[f] - v0 / Re * (G1[fj1] - G1[f]);
    R = R + F2[fk1] - F2[f] - v0 / Re * (G2[fk1] - G2[f]);
    sa_finish(A, B, s, i, j, k, g, c, f, vt0, mu0, d0, R);
  }
}

// Res(6) of a tile of cells in one pass: the SA face fluxes F, G of direction i, then j, then k, in
// shared memory, each cell adding its two faces' terms in the order of k_sa_res, then the source;
// bit-equal to k_sa_flux + k_sa_res without the Ft planes (faces on a tile border are computed by
// both tiles that share them).  The SA variable of the tile and one layer around it, which every
// face's gradient stencil reads about ten times, is staged in shared memory first.
template <class T, int DIR>
__device__ __forceinline__ void tile_sa_dir(const Arena<T>& A, const BlkD& B, const SolveP& s, int i0, int j0, int k0, int ni, int nj,
                                            int nk, T* Fs, T* Rs, const T* Vs, const T* Vt) {
  const int fa = ni + (DIR == 0), fb = nj + (DIR == 1), fc = nk + (DIR == 2);
  const int nf = fa * fb * fc, MF = A.tile_maxf;
  // the tile's SA values with one layer around it, staged in shared memory (box ni+2 x nj+2 x nk+2)
  const int bx = ni + 2, by = nj + 2;
  auto vt = [&](int a, int c, int e) -> T { return Vt[(a - i0 + 1) + bx * ((c - j0 + 1) + by * (e - k0 + 1))]; };
  for (int q = threadIdx.x; q < nf; q += blockDim.x) {
    const int a = q % fa, r = q / fa, bb = r % fb, c = r / fb;
    T F, G;
    sa_face_vt<T, DIR>(A, B, s, i0 + a, j0 + bb, k0 + c, fix_(B, i0 + a, j0 + bb, k0 + c), F, G, vt);
    Fs[q] = F;
    Fs[MF + q] = G;
  }
  __syncthreads();
  const int nc = ni * nj * nk, step = DIR == 0 ? 1 : (DIR == 1 ? fa : fa * fb);
  const T Re = T(s.re);
  for (int q = threadIdx.x; q < nc; q += blockDim.x) {
    const int a = q % ni, r = q / ni, bb = r % nj, c = r / nj;
    const int lo = a + fa * (bb + fb * c), hi = lo + step;
    const T* F = Fs;
    const T* G = Fs + MF;
    const T v0 = Vs[q];
    if (DIR == 0) Rs[q] = F[hi] - F[lo] - v0 / Re * (G[hi] - G[lo]);
    else Rs[q] = Rs[q] + F[hi] - F[lo] - v0 / Re * (G[hi] - G[lo]);
  }
  __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_sa_tile(Arena<T> A) {
  extern __shared__ __align__(16) unsigned char sa_smem[];
  T* Fs = reinterpret_cast<T*>(sa_smem);
  T* Rs = Fs + 2 * A.tile_maxf;
  T* Vs = Rs + A.tile_maxc;
  T* Vt = Vs + A.tile_maxc;  // (tile + 1 layer) box of the SA variable, at most tile_maxb values
  const long long tb = A.tot_box;
  for (int t = blockIdx.x; t < A.ntile; t += gridDim.x) {
    const int4 tl = A.tiles[t];
    const int b = tl.x, i0 = tl.y, j0 = tl.z, k0 = tl.w;
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    const int ni = min(B.tdim[0], B.nx - i0), nj = min(B.tdim[1], B.ny - j0), nk = min(B.tdim[2], B.nz - k0);
    const int nc = ni * nj * nk;
    for (int q = threadIdx.x; q < nc; q += blockDim.x) {
      const int i = i0 + q % ni, r = q / ni, j = j0 + r % nj, k = k0 + r / nj;
      const long long c = bix(B, i, j, k);
      T vt0 = T(clamp0(A.U[5 * tb + c])), mu0 = A.mu[c], d0 = A.P[P_D * tb + c];
      Vs[q] = (vt0 + mu0 / d0) * T(sa::Cb2) / T(sa::sigma);
    }
    const int bx = ni + 2, by = nj + 2, nb = bx * by * (nk + 2);
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
      const int a = q % bx, r = q / bx;
      Vt[q] = T(clamp0(A.U[5 * tb + bix(B, i0 - 1 + a, j0 - 1 + r % by, k0 - 1 + r / by)]));
    }
    __syncthreads();  // the faces of direction i read the staged box
    tile_sa_dir<T, 0>(A, B, s, i0, j0, k0, ni, nj, nk, Fs, Rs, Vs, Vt);
    tile_sa_dir<T, 1>(A, B, s, i0, j0, k0, ni, nj, nk, Fs, Rs, Vs, Vt);
    tile_sa_dir<T, 2>(A, B, s, i0, j0, k0, ni, nj, nk, Fs, Rs, Vs, Vt);
    for (int q = threadIdx.x; q < nc; q += blockDim.x) {
      const int i = i0 + q % ni, r = q / ni, j = j0 + r % nj, k = k0 + r / nj;
      const long long c = bix(B, i, j, k);
      T vt0 = T(clamp0(A.U[5 * tb + c])), mu0 = A.mu[c], d0 = A.P[P_D * tb + c];
      sa_finish(A, B, s, i, j, k, cix(B, i, j, k), c, fix_(B, i, j, k), vt0, mu0, d0, Rs[q]);
    }
    __syncthreads();
  }
}

namespace sst {
constexpr double sigma_k1 = 0.85, sigma_w1 = 0.5, beta1 = 0.075, Cw1 = 0.533, sigma_k2 = 1.0, sigma_w2 = 0.856, beta2 = 0.0828, Cw2 = 0.440;
constexpr double a1 = 0.31, betas = 0.09;
}  // namespace sst

// mu *= Re, Kt = U6/U1, Wt = U7/U1 on the 0..n box (SST.f90:40-58)
template <class T>
__global__ void k_sst_pre(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(r, A.tot_r1) {
    const int b = find_blk_h(A.pre_r1, A.hint_r1, A.nblk, r);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_r1(B, r - B.or1, i, j, k);
    const long long g = bix(B, i, j, k);
    const SolveP& s = A.sp[B.solve];
    const T mu = T((double)A.mu[g] * s.re);
    const double d = A.U[g], u5 = A.U[5 * tb + g], u6 = A.U[6 * tb + g];  // loads before the stores
    A.mu[g] = mu;
    A.Kt[g] = T(clamp0(u5) / d);
    A.Wt[g] = T(clamp0(u6) / d);
  }
}

// SST sources, mu_t and f1 on the interior (SST.f90:62-162)
template <class T>
__global__ void k_sst_src(Arena<T> A) {
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    const T *Pu = A.P + P_U * tb, *Pv = A.P + P_V * tb, *Pw = A.P + P_W * tb;
    long long c = bix(B, i, j, k);
    long long cip = bix(B, i + 1, j, k), cim = bix(B, i - 1, j, k), cjp = bix(B, i, j + 1, k), cjm = bix(B, i, j - 1, k);
    long long ckp = bix(B, i, j, k + 1), ckm = bix(B, i, j, k - 1);
    T ui = Pu[cip] - Pu[cim], vi = Pv[cip] - Pv[cim], wi = Pw[cip] - Pw[cim], Kti = A.Kt[cip] - A.Kt[cim], wti = A.Wt[cip] - A.Wt[cim];
    T uj = Pu[cjp] - Pu[cjm], vj = Pv[cjp] - Pv[cjm], wj = Pw[cjp] - Pw[cjm], Ktj = A.Kt[cjp] - A.Kt[cjm], wtj = A.Wt[cjp] - A.Wt[cjm];
    T uk = Pu[ckp] - Pu[ckm], vk = Pv[ckp] - Pv[ckm], wk = Pw[ckp] - Pw[ckm], Ktk = A.Kt[ckp] - A.Kt[ckm], wtk = A.Wt[ckp] - A.Wt[ckm];
    long long f = fix_(B, i, j, k);
    T ix = A.M[(M_J0 + 0) * tf + f], iy = A.M[(M_J0 + 1) * tf + f], iz = A.M[(M_J0 + 2) * tf + f];
    T jx = A.M[(M_J0 + 3) * tf + f], jy = A.M[(M_J0 + 4) * tf + f], jz = A.M[(M_J0 + 5) * tf + f];
    T kx = A.M[(M_J0 + 6) * tf + f], ky = A.M[(M_J0 + 7) * tf + f], kz = A.M[(M_J0 + 8) * tf + f];
    T vx = vi * ix + vj * jx + vk * kx, wx = wi * ix + wj * jx + wk * kx;
    T Ktx = Kti * ix + Ktj * jx + Ktk * kx, wtx = wti * ix + wtj * jx + wtk * kx;
    T uy = ui * iy + uj * jy + uk * ky, wy = wi * iy + wj * jy + wk * ky;
    T Kty = Kti * iy + Ktj * jy + Ktk * ky, wty = wti * iy + wtj * jy + wtk * ky;
    T uz = ui * iz + uj * jz + uk * kz, vz = vi * iz + vj * jz + vk * kz;
    T Ktz = Kti * iz + Ktj * jz + Ktk * kz, wtz = wti * iz + wtj * jz + wtk * kz;
    T omega = dsqrt(sq(wy - vz) + sq(uz - wx) + sq(vx - uy));
    T Re = T(s.re), dw = A.dw[g], K = A.Kt[c], Wv = A.Wt[c], dd = A.P[P_D * tb + c], mu = A.mu[c];
    const T volg = A.vol[g];  // before the stores below
    const T c009 = T((double)0.09f);  // `0.09` default-real literal (SST.f90:108, 120)
    T arg2 = fmax_(T(2) * dsqrt(dabs(K)) / (c009 * Wv * dw * Re), T(500) * mu / (dd * Wv * sq(dw) * Re * Re));
    T f2 = dtanh(sq(arg2));
    T mut = T(sst::a1) * dd * K / fmax_(T(sst::a1) * Wv, f2 * dabs(omega) / Re);
    A.mut[c] = mut;
    T Kws = T(2) * (Ktx * wtx + Kty * wty + Ktz * wtz) * dd * T(sst::sigma_w2) / (Wv + T(1.e-20));
    T CD_kw = fmax_(Kws, T(1.e-20));
    T arg3 = fmax_(dsqrt(dabs(K)) / (c009 * Wv * dw * Re), T(500) * mu / (dd * Wv * sq(dw) * Re * Re));
    T arg1 = fmin_(arg3, T(4) * dd * T(sst::sigma_w2) * K / (CD_kw * sq(dw)));
    T f1 = dtanh(pow4(arg1));
    A.f1[f] = f1;
    T Pk = mut * omega * omega;
    T Qk = Pk / Re - Re * T(sst::betas) * dd * Wv * K;
    T Cw = f1 * T(sst::Cw1) + (T(1) - f1) * T(sst::Cw2);
    T beta = f1 * T(sst::beta1) + (T(1) - f1) * T(sst::beta2);
    T Qw = Cw * dd * omega * omega / Re - Re * beta * dd * sq(Wv) + (T(1) - f1) * Kws / Re;
    A.Res[5 * tc + g] = Qk * volg;
    A.Res[6 * tc + g] = Qw * volg;
  }
}

// SST mu_t ghost copies over the whole -1..n+1 extent (SST.f90:170-175), one pass per direction
template <class T, int DIR>
__global__ void k_sst_mut_ghost(Arena<T> A) {
  OCFD_GRID_STRIDE(g, A.tot_box) {
    int b = find_blk_h(A.pre_box, A.hint_box, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_box(B, g - B.obox, i, j, k);
    if (i < -1 || i > B.nx + 1 || j < -1 || j > B.ny + 1 || k < -1 || k > B.nz + 1) continue;
    if (DIR == 0) {
      if (i == 0) A.mut[g] = A.mut[bix(B, 1, j, k)];
      else if (i == B.nx) A.mut[g] = A.mut[bix(B, B.nx - 1, j, k)];
    } else if (DIR == 1) {
      if (j == 0) A.mut[g] = A.mut[bix(B, i, 1, k)];
      else if (j == B.ny) A.mut[g] = A.mut[bix(B, i, B.ny - 1, k)];
    } else {
      if (k == 0) A.mut[g] = A.mut[bix(B, i, j, 1)];
      else if (k == B.nz) A.mut[g] = A.mut[bix(B, i, j, B.nz - 1)];
    }
  }
}

// SST diffusion + first-order convection fluxes (SST.f90:182-318) for direction DIR
template <class T, int DIR>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_sst_flux(Arena<T> A) {
  const long long tb = A.tot_box, tf = A.tot_face;
  OCFD_GRID_STRIDE(g, tf) {
    int b = find_blk_h(A.pre_face, A.hint_face, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_face(B, g - B.oface, i, j, k);
    if (DIR == 0 && (j == B.ny || k == B.nz)) continue;
    if (DIR == 1 && (i == B.nx || k == B.nz)) continue;
    if (DIR == 2 && (i == B.nx || j == B.ny)) continue;
    const SolveP& s = A.sp[B.solve];
    const int di = DIR == 0, dj = DIR == 1, dk = DIR == 2;
    const int im = i - di, jm = j - dj, km = k - dk;
    // f1 is undefined at i=nx / j=ny / k=nz in the reference (uninitialised): nearest interior cell
    T f1 = A.f1[fix_(B, i < B.nx ? i : B.nx - 1, j < B.ny ? j : B.ny - 1, k < B.nz ? k : B.nz - 1)];
    T sk = f1 * T(sst::sigma_k1) + (T(1) - f1) * T(sst::sigma_k2);
    T sw = f1 * T(sst::sigma_w1) + (T(1) - f1) * T(sst::sigma_w2);
    long long c0 = bix(B, i, j, k), c1 = bix(B, im, jm, km);
    T Re = T(s.re);
    T muk = (A.mu[c1] + A.mu[c0] + sk * (A.mut[c1] + A.mut[c0])) * T(0.5) / Re;
    T muw = (A.mu[c1] + A.mu[c0] + sw * (A.mut[c1] + A.mut[c0])) * T(0.5) / Re;
    T s1x = A.M[(M_NI1 + 3 * DIR) * tf + g], s1y = A.M[(M_NI2 + 3 * DIR) * tf + g], s1z = A.M[(M_NI3 + 3 * DIR) * tf + g];
    T S = A.M[(M_SI + DIR) * tf + g];
    auto K = [&](int a, int c, int e) -> T { return A.Kt[bix(B, a, c, e)]; };
    auto W = [&](int a, int c, int e) -> T { return A.Wt[bix(B, a, c, e)]; };
    T kti, ktj, ktk, wti, wtj, wtk;
    if (DIR == 0) {
      kti = K(i, j, k) - K(i - 1, j, k); wti = W(i, j, k) - W(i - 1, j, k);
      ktj = T(0.25) * (K(i, j + 1, k) - K(i, j - 1, k) + K(i - 1, j + 1, k) - K(i - 1, j - 1, k));
      wtj = T(0.25) * (W(i, j + 1, k) - W(i, j - 1, k) + W(i - 1, j + 1, k) - W(i - 1, j - 1, k));
      ktk = T(0.25) * (K(i, j, k + 1) - K(i, j, k - 1) + K(i - 1, j, k + 1) - K(i - 1, j, k - 1));
      wtk = T(0.25) * (W(i, j, k + 1) - W(i, j, k - 1) + W(i - 1, j, k + 1) - W(i - 1, j, k - 1));
    } else if (DIR == 1) {
      kti = T(0.25) * (K(i + 1, j, k) - K(i - 1, j, k) + K(i + 1, j - 1, k) - K(i - 1, j - 1, k));
      ktj = K(i, j, k) - K(i, j - 1, k);
      ktk = T(0.25) * (K(i, j, k + 1) - K(i, j, k - 1) + K(i, j - 1, k + 1) - K(i, j - 1, k - 1));
      wti = T(0.25) * (W(i + 1, j, k) - W(i - 1, j, k) + W(i + 1, j - 1, k) - W(i - 1, j - 1, k));
      wtj = W(i, j, k) - W(i, j - 1, k);
      wtk = T(0.25) * (W(i, j, k + 1) - W(i, j, k - 1) + W(i, j - 1, k + 1) - W(i, j - 1, k - 1));
    } else {
      kti = T(0.25) * (K(i + 1, j, k) - K(i - 1, j, k) + K(i + 1, j, k - 1) - K(i - 1, j, k - 1));
      ktj = T(0.25) * (K(i, j + 1, k) - K(i, j - 1, k) + K(i, j + 1, k - 1) - K(i, j - 1, k - 1));
      ktk = K(i, j, k) - K(i, j, k - 1);
      wti = T(0.25) * (W(i + 1, j, k) - W(i - 1, j, k) + W(i + 1, j, k - 1) - W(i - 1, j, k - 1));
      wtj = T(0.25) * (W(i, j + 1, k) - W(i, j - 1, k) + W(i, j + 1, k - 1) - W(i, j - 1, k - 1));
      wtk = W(i, j, k) - W(i, j, k - 1);
    }
    const int J = DIR == 0 ? M_J1 : (DIR == 1 ? M_J2 : M_J3);
    T ix = A.M[(J + 0) * tf + g], iy = A.M[(J + 1) * tf + g], iz = A.M[(J + 2) * tf + g];
    T jx = A.M[(J + 3) * tf + g], jy = A.M[(J + 4) * tf + g], jz = A.M[(J + 5) * tf + g];
    T kx = A.M[(J + 6) * tf + g], ky = A.M[(J + 7) * tf + g], kz = A.M[(J + 8) * tf + g];
    T ktx = kti * ix + ktj * jx + ktk * kx, wtx = wti * ix + wtj * jx + wtk * kx;
    T kty = kti * iy + ktj * jy + ktk * ky, wty = wti * iy + wtj * jy + wtk * ky;
    T ktz = kti * iz + ktj * jz + ktk * kz, wtz = wti * iz + wtj * jz + wtk * kz;
    T vn1 = A.P[P_U * tb + c1] * s1x + A.P[P_V * tb + c1] * s1y + A.P[P_W * tb + c1] * s1z;
    T vn2 = A.P[P_U * tb + c0] * s1x + A.P[P_V * tb + c0] * s1y + A.P[P_W * tb + c0] * s1z;
    T kfi = T(0.5) * ((vn1 + dabs(vn1)) * A.Kt[c1] + (vn2 - dabs(vn2)) * A.Kt[c0]);
    T wfi = T(0.5) * ((vn1 + dabs(vn1)) * A.Wt[c1] + (vn2 - dabs(vn2)) * A.Wt[c0]);
    A.Ft[(DIR * 2 + 0) * tf + g] = (-kfi + muk * (ktx * s1x + kty * s1y + ktz * s1z)) * S;
    A.Ft[(DIR * 2 + 1) * tf + g] = (-wfi + muw * (wtx * s1x + wty * s1y + wtz * s1z)) * S;
  }
}

// Res(6,7) += flux differences in the i, j, k order (SST.f90:221-330)
template <class T>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_sst_res(Arena<T> A) {
  const long long tf = A.tot_face, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    long long f = fix_(B, i, j, k), fi1 = fix_(B, i + 1, j, k), fj1 = fix_(B, i, j + 1, k), fk1 = fix_(B, i, j, k + 1);
    T Rq[2];  // both values before the stores
#pragma unroll
    for (int q = 0; q < 2; q++) {
      T R = A.Res[(5 + q) * tc + g];
      R = R + A.Ft[(0 + q) * tf + fi1] - A.Ft[(0 + q) * tf + f];
      R = R + A.Ft[(2 + q) * tf + fj1] - A.Ft[(2 + q) * tf + f];
      R = R + A.Ft[(4 + q) * tf + fk1] - A.Ft[(4 + q) * tf + f];
      Rq[q] = R;
    }
    A.Res[5 * tc + g] = Rq[0];
    A.Res[6 * tc + g] = Rq[1];
  }
}

// mu /= Re, mu_t /= Re (end of SA/SST), then limit_mut (sub_Residual.f90:1387-1406) on 0..n.
// MODE 0: laminar (mu_t was zeroed); 1: turbulence model ran with mu scaled by Re.
template <class T, int MODE>
__global__ void k_mu_finish(Arena<T> A) {
  OCFD_GRID_STRIDE(r, A.tot_r1) {
    const int b = find_blk_h(A.pre_r1, A.hint_r1, A.nblk, r);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_r1(B, r - B.or1, i, j, k);
    const long long g = bix(B, i, j, k);
    const SolveP& s = A.sp[B.solve];
    T mu = A.mu[g], mut = A.mut[g];
    if (MODE == 1) { mu = T((double)mu / s.re); mut = T((double)mut / s.re); A.mu[g] = mu; }
    if (mut < T(0)) mut = T(0);
    if (s.mut_max >= 0.0 && mut > T(s.mut_max) * mu) mut = T(s.mut_max) * mu;
    A.mut[g] = mut;
  }
}

// decode a face cell of a subface (transverse ranges b..e-1)
__device__ __forceinline__ void subcell_ijk(const SubD& S, long long l, int& i, int& j, int& k) {
  int f = S.face;
  const unsigned u = (unsigned)l;  // a subface's cell count is below 2^31
  if (f == 1 || f == 4) { unsigned nj = (unsigned)(S.je - S.jb); j = S.jb + (int)(u % nj); k = S.kb + (int)(u / nj); i = f == 1 ? 1 : S.ie - 1; }
  else if (f == 2 || f == 5) { unsigned ni = (unsigned)(S.ie - S.ib); i = S.ib + (int)(u % ni); k = S.kb + (int)(u / ni); j = f == 2 ? 1 : S.je - 1; }
  else { unsigned ni = (unsigned)(S.ie - S.ib); i = S.ib + (int)(u % ni); j = S.jb + (int)(u / ni); k = f == 3 ? 1 : S.ke - 1; }
}
__device__ __forceinline__ void ghost_of(const SubD& S, int i, int j, int k, int& gi, int& gj, int& gk) {
  gi = i; gj = j; gk = k;
  switch (S.face) {
    case 1: gi = 0; break;
    case 4: gi = S.ie; break;
    case 2: gj = 0; break;
    case 5: gj = S.je; break;
    case 3: gk = 0; break;
    default: gk = S.ke; break;
  }
}

// Amut_boundary (sub_turbulence_SA.f90:282-368): wall ghost mu_t = -mu_t of the first cell
template <class T>
__global__ void k_amut(Arena<T> A) {
  OCFD_GRID_STRIDE(g, A.tot_subcell) {
    int s = find_blk(A.pre_subcell, A.nsub, g);
    const SubD S = A.sub[s];
    if (S.bc != 2) continue;
    const BlkD& B = A.blk[S.blk];
    int i, j, k, gi, gj, gk;
    subcell_ijk(S, g - A.pre_subcell[s], i, j, k);
    ghost_of(S, i, j, k, gi, gj, gk);
    A.mut[bix(B, gi, gj, gk)] = -A.mut[bix(B, i, j, k)];
  }
}

#ifndef INV_FLUX_MIXED_MINB
#define INV_FLUX_MIXED_MINB 4
#endif
// ============================================================================================
// inviscid fluxes (flux_inviscous_i/j/k, sub_Residual.f90:182-705)
// ============================================================================================
// FP64: three 256-thread CTAs per SM (at most 80 registers; a few hundred bytes of spills to L1),
// FP32: four (64 registers, no spills): the kernel is bound by arithmetic latency and more warps
// hide more of it (FP64 on config 2: 0.34 -> 0.29 ms per direction against two CTAs at 120
// registers; FP32: config 2 residual phase -0.07 ms, config 3 -0.26 ms against three CTAs)
template <class T>
struct InvFluxOcc { static constexpr int value = sizeof(T) == 8 ? 3 : INV_FLUX_MIXED_MINB; };
// PRIM: every solve of the handle reconstructs the primitive variables (IFlag_Reconstruction = 0),
// so the conservative / characteristic branches are compiled out.  ISCH / IFLUX (>= 0): every
// solve uses this interior scheme / flux, so the faces that use the interior scheme take a
// straight-line path (the five reconstructions without a switch between them, free to interleave)
// and the flux switch folds; boundary faces keep the general path.
// CTAs per SM: FP64 3 (80 registers); the FP64 MUSCL3 specialisation 2 (about 120 registers, no
// spills: config 1 residual phase 0.099 -> 0.094 ms; WENO5 is faster at 3, 1.85 against 2.00 ms)
template <class T, int ISCH>
struct InvFluxOccS { static constexpr int value = (sizeof(T) == 8 && ISCH == S_MUSCL3) ? 2 : InvFluxOcc<T>::value; };
// one face of direction DIR: its five inviscid flux components (the face's Fi plane entries)
template <class T, int DIR, bool PRIM, int ISCH, int IFLUX>
__device__ __forceinline__ void inv_face(const Arena<T>& A, const BlkD& B, const SolveP& s, int b, int i, int j, int k, long long g,
                                         T* Fo) {
  const long long tb = A.tot_box, tf = A.tot_face;
  int idx, nd;
  unsigned char bc;
  if (DIR == 0) { idx = i; nd = B.nx; bc = A.bci[B.obci + (j - 1) + (long long)(B.ny - 1) * (k - 1)]; }
  else if (DIR == 1) { idx = j; nd = B.ny; bc = A.bcj[B.obcj + (i - 1) + (long long)(B.nx - 1) * (k - 1)]; }
  else { idx = k; nd = B.nz; bc = A.bck[B.obck + (i - 1) + (long long)(B.nx - 1) * (j - 1)]; }
  int scheme = s.scheme;
  if (bc & 1) { if (idx == 1) scheme = S_CD2; else if (idx < LAP) scheme = s.bound_scheme; }
  if (bc & 2) { if (idx == nd) scheme = S_CD2; else if (idx > nd - LAP + 1) scheme = s.bound_scheme; }
  if (A.flags[b] == 1) scheme = S_UD1;
  const int di = DIR == 0, dj = DIR == 1, dk = DIR == 2;
  // stencil cells idx-4 .. idx+3 along DIR
  long long c0 = bix(B, i - 4 * di, j - 4 * dj, k - 4 * dk);
  const long long st = DIR == 0 ? 1 : (DIR == 1 ? (long long)B.NX : (long long)B.NX * B.NY);
  T UL[5], UR[5];
  if ((PRIM || s.recon == 0) && ISCH >= 0 && scheme == ISCH) {
#pragma unroll
    for (int m = 0; m < 5; m++) {
      const int pl = m == 4 ? P_P : m;
      T u[8];
#pragma unroll
      for (int q = 0; q < 8; q++) u[q] = A.P[pl * tb + c0 + q * st];
      scheme_LR(u, ISCH < 0 ? 0 : ISCH, UL[m], UR[m]);
    }
  } else if (PRIM || s.recon == 0) {
    T u[8];
#pragma unroll
    for (int m = 0; m < 5; m++) {
      const int pl = m == 4 ? P_P : m;
#pragma unroll
      for (int q = 0; q < 8; q++) u[q] = A.P[pl * tb + c0 + q * st];
      scheme_LR(u, scheme, UL[m], UR[m]);
    }
  } else {
    T gm = T(s.gamma);
    T U0[5][8];
    for (int m = 0; m < 5; m++)
      for (int q = 0; q < 8; q++) U0[m][q] = T(A.U[m * tb + c0 + q * st]);
    if (s.recon == 1) {
      T QL[5], QR[5];
      for (int m = 0; m < 5; m++) scheme_LR(U0[m], scheme, QL[m], QR[m]);
      UL[0] = QL[0]; UL[1] = QL[1] / UL[0]; UL[2] = QL[2] / UL[0]; UL[3] = QL[3] / UL[0];
      UL[4] = (QL[4] - (UL[1] * QL[1] + UL[2] * QL[2] + UL[3] * QL[3]) * T(0.5)) * (gm - T(1));
      UR[0] = QR[0]; UR[1] = QR[1] / UR[0]; UR[2] = QR[2] / UR[0]; UR[3] = QR[3] / UR[0];
      UR[4] = (QR[4] - (UR[1] * QR[1] + UR[2] * QR[2] + UR[3] * QR[3]) * T(0.5)) * (gm - T(1));
    } else {  // characteristic (sub_Residual.f90:1291-1347)
      T Uh[5];
      for (int m = 0; m < 5; m++) Uh[m] = T(0.5) * (U0[m][3] + U0[m][4]);
      T d1 = Uh[0], u1 = Uh[1] / d1, v1 = Uh[2] / d1, w1 = Uh[3] / d1;
      T p1 = (Uh[4] - (Uh[1] * u1 + Uh[2] * v1 + Uh[3] * w1) * T(0.5)) * (gm - T(1));
      T c1 = dsqrt(gm * p1 / d1);
      T V2 = (u1 * u1 + v1 * v1 + w1 * w1) * T(0.5);
      T tmp1 = (gm - T(1)) / c1, tmp3 = (gm - T(1)) / (c1 * c1), tmp5 = T(1) / (T(2) * c1), tmp0 = T(1) / tmp3;
      T Sm[5][5] = {{V2 - tmp0, -u1, -v1, -w1, T(1)},
                    {-v1, T(0), T(1), T(0), T(0)},
                    {-w1, T(0), T(0), T(1), T(0)},
                    {-u1 - V2 * tmp1, T(1) + tmp1 * u1, tmp1 * v1, tmp1 * w1, -tmp1},
                    {-u1 + V2 * tmp1, T(1) - tmp1 * u1, -tmp1 * v1, -tmp1 * w1, tmp1}};
      T S1[5][5] = {{-tmp3, T(0), T(0), -tmp5, tmp5},
                    {-tmp3 * u1, T(0), T(0), T(0.5) - u1 * tmp5, T(0.5) + u1 * tmp5},
                    {-tmp3 * v1, T(1), T(0), -v1 * tmp5, v1 * tmp5},
                    {-tmp3 * w1, T(0), T(1), -w1 * tmp5, w1 * tmp5},
                    {-tmp3 * V2, v1, w1, (c1 * u1 - V2 - tmp0) * tmp5, (c1 * u1 + V2 + tmp0) * tmp5}};
      T V0[5][8];
      for (int q = 0; q < 8; q++)
        for (int m = 0; m < 5; m++) {
          T acc = T(0);
          for (int jj = 0; jj < 5; jj++) acc = acc + Sm[m][jj] * U0[jj][q];
          V0[m][q] = acc;
        }
      T VL[5], VR[5], QL[5], QR[5];
      for (int m = 0; m < 5; m++) scheme_LR(V0[m], scheme, VL[m], VR[m]);
      for (int m = 0; m < 5; m++) {
        QL[m] = T(0); QR[m] = T(0);
        for (int jj = 0; jj < 5; jj++) { QL[m] = QL[m] + S1[m][jj] * VL[jj]; QR[m] = QR[m] + S1[m][jj] * VR[jj]; }
      }
      UL[0] = QL[0]; UL[1] = QL[1] / UL[0]; UL[2] = QL[2] / UL[0]; UL[3] = QL[3] / UL[0];
      UL[4] = (QL[4] - (UL[1] * QL[1] + UL[2] * QL[2] + UL[3] * QL[3]) * T(0.5)) * (gm - T(1));
      UR[0] = QR[0]; UR[1] = QR[1] / UR[0]; UR[2] = QR[2] / UR[0]; UR[3] = QR[3] / UR[0];
      UR[4] = (QR[4] - (UR[1] * QR[1] + UR[2] * QR[2] + UR[3] * QR[3]) * T(0.5)) * (gm - T(1));
    }
  }
  if (s.positivity == 1) {  // first-order fallback (sub_Residual.f90:283-299)
    const T lz = T(1.e-20);
    if (UL[0] <= lz || UL[4] <= lz) {
      long long cl = c0 + 3 * st;
      UL[0] = A.P[P_D * tb + cl]; UL[1] = A.P[P_U * tb + cl]; UL[2] = A.P[P_V * tb + cl]; UL[3] = A.P[P_W * tb + cl]; UL[4] = A.P[P_P * tb + cl];
    }
    if (UR[0] <= lz || UR[4] <= lz) {
      long long cr = c0 + 4 * st;
      UR[0] = A.P[P_D * tb + cr]; UR[1] = A.P[P_U * tb + cr]; UR[2] = A.P[P_V * tb + cr]; UR[3] = A.P[P_W * tb + cr]; UR[4] = A.P[P_P * tb + cr];
    }
  }
  T s1x = A.M[(M_NI1 + 3 * DIR) * tf + g], s1y = A.M[(M_NI2 + 3 * DIR) * tf + g], s1z = A.M[(M_NI3 + 3 * DIR) * tf + g];
  T s2x = A.M[(M_TI + 3 * DIR) * tf + g], s2y = A.M[(M_TI + 3 * DIR + 1) * tf + g], s2z = A.M[(M_TI + 3 * DIR + 2) * tf + g];
  T s3x = s1y * s2z - s1z * s2y, s3y = s1z * s2x - s1x * s2z, s3z = s1x * s2y - s1y * s2x;
  T QL[5], QR[5], F0[5];
  QL[0] = UL[0]; QL[1] = UL[1] * s1x + UL[2] * s1y + UL[3] * s1z; QL[2] = UL[1] * s2x + UL[2] * s2y + UL[3] * s2z;
  QL[3] = UL[1] * s3x + UL[2] * s3y + UL[3] * s3z; QL[4] = UL[4];
  QR[0] = UR[0]; QR[1] = UR[1] * s1x + UR[2] * s1y + UR[3] * s1z; QR[2] = UR[1] * s2x + UR[2] * s2y + UR[3] * s2z;
  QR[3] = UR[1] * s3x + UR[2] * s3y + UR[3] * s3z; QR[4] = UR[4];
  flux_1d(QL, QR, F0, T(s.gamma), IFLUX >= 0 ? IFLUX : s.flux);
  T S = A.M[(M_SI + DIR) * tf + g];
  Fo[0] = -F0[0] * S;
  Fo[1] = -(F0[1] * s1x + F0[2] * s2x + F0[3] * s3x) * S;
  Fo[2] = -(F0[1] * s1y + F0[2] * s2y + F0[3] * s3y) * S;
  Fo[3] = -(F0[1] * s1z + F0[2] * s2z + F0[3] * s3z) * S;
  Fo[4] = -F0[4] * S;
}

template <class T, int DIR, bool PRIM = false, int ISCH = -1, int IFLUX = -1>
__global__ void __launch_bounds__(256, InvFluxOccS<T, ISCH>::value) k_inv_flux(Arena<T> A) {
  const long long tf = A.tot_face;
  OCFD_GRID_STRIDE(g, tf) {
    int b = find_blk_h(A.pre_face, A.hint_face, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_face(B, g - B.oface, i, j, k);
    if (DIR == 0 && (j == B.ny || k == B.nz)) continue;
    if (DIR == 1 && (i == B.nx || k == B.nz)) continue;
    if (DIR == 2 && (i == B.nx || j == B.ny)) continue;
    // a physical k face with bc > 0 takes k_inv_kbc's central flux, which overwrites this one: skip
    // it (two of the three k planes of the batch's two-cell-thick airfoils)
    if (DIR == 2 && (k == 1 || k == B.nz) && (A.bck[B.obck + (i - 1) + (long long)(B.nx - 1) * (j - 1)] & (k == 1 ? 4 : 8))) continue;
    T F[5];
    inv_face<T, DIR, PRIM, ISCH, IFLUX>(A, B, A.sp[B.solve], b, i, j, k, g, F);
    T* Fo = A.Fi + (long long)DIR * 5 * tf + g;
#pragma unroll
    for (int m = 0; m < 5; m++) Fo[m * tf] = F[m];
  }
}

// physical k-faces: central flux of the averaged primitives (sub_Residual.f90:666-689), for the
// face (i, j, k) between cells k-1 and k
template <class T>
__device__ __forceinline__ void kbc_face(const Arena<T>& A, const BlkD& B, const SolveP& sp, int i, int j, int k, long long f, T* Fo) {
  const long long tb = A.tot_box, tf = A.tot_face;
  long long c0 = bix(B, i, j, k), c1 = bix(B, i, j, k - 1);
  T gm = T(sp.gamma);
  T d0 = (A.P[P_D * tb + c0] + A.P[P_D * tb + c1]) * T(0.5), uu0 = (A.P[P_U * tb + c0] + A.P[P_U * tb + c1]) * T(0.5);
  T v0 = (A.P[P_V * tb + c0] + A.P[P_V * tb + c1]) * T(0.5), w0 = (A.P[P_W * tb + c0] + A.P[P_W * tb + c1]) * T(0.5);
  T p0 = (A.P[P_P * tb + c0] + A.P[P_P * tb + c1]) * T(0.5);
  T E0 = p0 / (gm - T(1)) + d0 * (uu0 * uu0 + v0 * v0 + w0 * w0) * T(0.5);
  T n1 = A.M[M_NK1 * tf + f], n2 = A.M[M_NK2 * tf + f], n3 = A.M[M_NK3 * tf + f], Sk = A.M[M_SK * tf + f];
  T un = uu0 * n1 + v0 * n2 + w0 * n3;
  Fo[0] = -d0 * un * Sk;
  Fo[1] = -(d0 * un * uu0 + p0 * n1) * Sk;
  Fo[2] = -(d0 * un * v0 + p0 * n2) * Sk;
  Fo[3] = -(d0 * un * w0 + p0 * n3) * Sk;
  Fo[4] = -(E0 + p0) * un * Sk;
}

template <class T>
__global__ void k_inv_kbc(Arena<T> A) {
  const long long tf = A.tot_face;
  OCFD_GRID_STRIDE(g, A.tot_subcell) {
    int s = find_blk(A.pre_subcell, A.nsub, g);
    const SubD S = A.sub[s];
    if (!(S.bc > 0 && (S.face == 3 || S.face == 6))) continue;
    const BlkD& B = A.blk[S.blk];
    long long l = g - A.pre_subcell[s];
    const unsigned ni = (unsigned)(S.ie - S.ib), u = (unsigned)l;
    int i = S.ib + (int)(u % ni), j = S.jb + (int)(u / ni), k = S.kb;
    long long f = fix_(B, i, j, k);
    T F[5];
    kbc_face(A, B, A.sp[B.solve], i, j, k, f, F);
    T* Fo = A.Fi + 2LL * 5 * tf + f;
#pragma unroll
    for (int m = 0; m < 5; m++) Fo[m * tf] = F[m];
  }
}

// ============================================================================================
// viscous fluxes (flux_viscous_i/j/k, sub_Residual.f90:712-1247)
// ============================================================================================
// one face of direction DIR: its four viscous flux components (m = 1..4 of Res; the face's Fv
// plane entries).  Returns 0 with Fo[0..3] set; under OverLimit (no viscous flux, Surf = 0,
// sub_Residual.f90:734-750) 1 on a block-boundary face, whose Fo[0..2] are then 0, and 2 elsewhere
// (Fo untouched).  The flag is tested after the stencil loads (a branch on it first would hold
// every load of the face behind the flag's load).
template <class T, int DIR>
__device__ __forceinline__ int visc_face(const Arena<T>& A, const BlkD& B, const SolveP& s, int overlimit, int i, int j, int k,
                                         long long g, T* Fo) {
  const long long tb = A.tot_box, tf = A.tot_face;
  const T *Pu = A.P + P_U * tb, *Pv = A.P + P_V * tb, *Pw = A.P + P_W * tb, *PT = A.P + P_T * tb;
  auto avg = [&](const T* a, int i1, int j1, int k1, int i2, int j2, int k2) -> T { return T(0.5) * (a[bix(B, i1, j1, k1)] + a[bix(B, i2, j2, k2)]); };
  T ui, vi, wi, Ti, uj, vj, wj, Tj, uk, vk, wk, Tk;
  const int di = DIR == 0, dj = DIR == 1, dk = DIR == 2;
  const int im = i - di, jm = j - dj, km = k - dk;
  long long c0 = bix(B, i, j, k), c1 = bix(B, im, jm, km);
  if (DIR == 0) {
    ui = Pu[c0] - Pu[c1]; vi = Pv[c0] - Pv[c1]; wi = Pw[c0] - Pw[c1]; Ti = PT[c0] - PT[c1];
    bool zj = (i == 1 || i == B.nx) && (j == 1 || j == B.ny - 1), zk = (i == 1 || i == B.nx) && (k == 1 || k == B.nz - 1);
    T uj1 = T(0), vj1 = T(0), wj1 = T(0), Tj1 = T(0), uj2 = T(0), vj2 = T(0), wj2 = T(0), Tj2 = T(0);
    T uk1 = T(0), vk1 = T(0), wk1 = T(0), Tk1 = T(0), uk2 = T(0), vk2 = T(0), wk2 = T(0), Tk2 = T(0);
    if (!zj) {
      uj1 = avg(Pu, i, j - 1, k, i - 1, j - 1, k); vj1 = avg(Pv, i, j - 1, k, i - 1, j - 1, k); wj1 = avg(Pw, i, j - 1, k, i - 1, j - 1, k); Tj1 = avg(PT, i, j - 1, k, i - 1, j - 1, k);
      uj2 = avg(Pu, i, j + 1, k, i - 1, j + 1, k); vj2 = avg(Pv, i, j + 1, k, i - 1, j + 1, k); wj2 = avg(Pw, i, j + 1, k, i - 1, j + 1, k); Tj2 = avg(PT, i, j + 1, k, i - 1, j + 1, k);
    }
    if (!zk) {
      uk1 = avg(Pu, i, j, k - 1, i - 1, j, k - 1); vk1 = avg(Pv, i, j, k - 1, i - 1, j, k - 1); wk1 = avg(Pw, i, j, k - 1, i - 1, j, k - 1); Tk1 = avg(PT, i, j, k - 1, i - 1, j, k - 1);
      uk2 = avg(Pu, i, j, k + 1, i - 1, j, k + 1); vk2 = avg(Pv, i, j, k + 1, i - 1, j, k + 1); wk2 = avg(Pw, i, j, k + 1, i - 1, j, k + 1); Tk2 = avg(PT, i, j, k + 1, i - 1, j, k + 1);
    }
    uj = T(0.5) * (uj2 - uj1); vj = T(0.5) * (vj2 - vj1); wj = T(0.5) * (wj2 - wj1); Tj = T(0.5) * (Tj2 - Tj1);
    uk = T(0.5) * (uk2 - uk1); vk = T(0.5) * (vk2 - vk1); wk = T(0.5) * (wk2 - wk1); Tk = T(0.5) * (Tk2 - Tk1);
  } else if (DIR == 1) {
    uj = Pu[c0] - Pu[c1]; vj = Pv[c0] - Pv[c1]; wj = Pw[c0] - Pw[c1]; Tj = PT[c0] - PT[c1];
    bool zi = (j == 1 || j == B.ny) && (i == 1 || i == B.nx - 1), zk = (j == 1 || j == B.ny) && (k == 1 || k == B.nz - 1);
    T ui1 = T(0), vi1 = T(0), wi1 = T(0), Ti1 = T(0), ui2 = T(0), vi2 = T(0), wi2 = T(0), Ti2 = T(0);
    T uk1 = T(0), vk1 = T(0), wk1 = T(0), Tk1 = T(0), uk2 = T(0), vk2 = T(0), wk2 = T(0), Tk2 = T(0);
    if (!zi) {
      ui1 = avg(Pu, i - 1, j, k, i - 1, j - 1, k); vi1 = avg(Pv, i - 1, j, k, i - 1, j - 1, k); wi1 = avg(Pw, i - 1, j, k, i - 1, j - 1, k); Ti1 = avg(PT, i - 1, j, k, i - 1, j - 1, k);
      ui2 = avg(Pu, i + 1, j, k, i + 1, j - 1, k); vi2 = avg(Pv, i + 1, j, k, i + 1, j - 1, k); wi2 = avg(Pw, i + 1, j, k, i + 1, j - 1, k); Ti2 = avg(PT, i + 1, j, k, i + 1, j - 1, k);
    }
    if (!zk) {
      uk1 = avg(Pu, i, j, k - 1, i, j - 1, k - 1); vk1 = avg(Pv, i, j, k - 1, i, j - 1, k - 1); wk1 = avg(Pw, i, j, k - 1, i, j - 1, k - 1); Tk1 = avg(PT, i, j, k - 1, i, j - 1, k - 1);
      uk2 = avg(Pu, i, j, k + 1, i, j - 1, k + 1); vk2 = avg(Pv, i, j, k + 1, i, j - 1, k + 1); wk2 = avg(Pw, i, j, k + 1, i, j - 1, k + 1); Tk2 = avg(PT, i, j, k + 1, i, j - 1, k + 1);
    }
    ui = T(0.5) * (ui2 - ui1); vi = T(0.5) * (vi2 - vi1); wi = T(0.5) * (wi2 - wi1); Ti = T(0.5) * (Ti2 - Ti1);
    uk = T(0.5) * (uk2 - uk1); vk = T(0.5) * (vk2 - vk1); wk = T(0.5) * (wk2 - wk1); Tk = T(0.5) * (Tk2 - Tk1);
  } else {
    uk = Pu[c0] - Pu[c1]; vk = Pv[c0] - Pv[c1]; wk = Pw[c0] - Pw[c1]; Tk = PT[c0] - PT[c1];
    bool zi = (k == 1 || k == B.nz) && (i == 1 || i == B.nx - 1), zj = (k == 1 || k == B.nz) && (j == 1 || j == B.ny - 1);
    T ui1 = T(0), vi1 = T(0), wi1 = T(0), Ti1 = T(0), ui2 = T(0), vi2 = T(0), wi2 = T(0), Ti2 = T(0);
    T uj1 = T(0), vj1 = T(0), wj1 = T(0), Tj1 = T(0), uj2 = T(0), vj2 = T(0), wj2 = T(0), Tj2 = T(0);
    if (!zi) {
      ui1 = avg(Pu, i - 1, j, k, i - 1, j, k - 1); vi1 = avg(Pv, i - 1, j, k, i - 1, j, k - 1); wi1 = avg(Pw, i - 1, j, k, i - 1, j, k - 1); Ti1 = avg(PT, i - 1, j, k, i - 1, j, k - 1);
      ui2 = avg(Pu, i + 1, j, k, i + 1, j, k - 1); vi2 = avg(Pv, i + 1, j, k, i + 1, j, k - 1); wi2 = avg(Pw, i + 1, j, k, i + 1, j, k - 1); Ti2 = avg(PT, i + 1, j, k, i + 1, j, k - 1);
    }
    if (!zj) {
      uj1 = avg(Pu, i, j - 1, k, i, j - 1, k - 1); vj1 = avg(Pv, i, j - 1, k, i, j - 1, k - 1); wj1 = avg(Pw, i, j - 1, k, i, j - 1, k - 1); Tj1 = avg(PT, i, j - 1, k, i, j - 1, k - 1);
      uj2 = avg(Pu, i, j + 1, k, i, j + 1, k - 1); vj2 = avg(Pv, i, j + 1, k, i, j + 1, k - 1); wj2 = avg(Pw, i, j + 1, k, i, j + 1, k - 1); Tj2 = avg(PT, i, j + 1, k, i, j + 1, k - 1);
    }
    ui = T(0.5) * (ui2 - ui1); vi = T(0.5) * (vi2 - vi1); wi = T(0.5) * (wi2 - wi1); Ti = T(0.5) * (Ti2 - Ti1);
    uj = T(0.5) * (uj2 - uj1); vj = T(0.5) * (vj2 - vj1); wj = T(0.5) * (wj2 - wj1); Tj = T(0.5) * (Tj2 - Tj1);
  }
  if (overlimit == 1) {
    int idx = DIR == 0 ? i : (DIR == 1 ? j : k), nd = DIR == 0 ? B.nx : (DIR == 1 ? B.ny : B.nz);
    if (idx == 1 || idx == nd) { Fo[0] = T(0); Fo[1] = T(0); Fo[2] = T(0); return 1; }
    return 2;
  }
  const int J = DIR == 0 ? M_J1 : (DIR == 1 ? M_J2 : M_J3);
  T ix = A.M[(J + 0) * tf + g], iy = A.M[(J + 1) * tf + g], iz = A.M[(J + 2) * tf + g];
  T jx = A.M[(J + 3) * tf + g], jy = A.M[(J + 4) * tf + g], jz = A.M[(J + 5) * tf + g];
  T kx = A.M[(J + 6) * tf + g], ky = A.M[(J + 7) * tf + g], kz = A.M[(J + 8) * tf + g];
  T ux = ui * ix + uj * jx + uk * kx, vx = vi * ix + vj * jx + vk * kx, wx = wi * ix + wj * jx + wk * kx, Tx = Ti * ix + Tj * jx + Tk * kx;
  T uy = ui * iy + uj * jy + uk * ky, vy = vi * iy + vj * jy + vk * ky, wy = wi * iy + wj * jy + wk * ky, Ty = Ti * iy + Tj * jy + Tk * ky;
  T uz = ui * iz + uj * jz + uk * kz, vz = vi * iz + vj * jz + vk * kz, wz = wi * iz + wj * jz + wk * kz, Tz = Ti * iz + Tj * jz + Tk * kz;
  T mu0 = T(0.5) * (A.mu[c0] + A.mut[c0] + A.mu[c1] + A.mut[c1]);
  T PrL = T(s.prl), PrT = T(s.prt);
  T k0 = T(0.5) * T(s.cp) * (A.mu[c0] / PrL + A.mut[c0] / PrT + A.mu[c1] / PrL + A.mut[c1] / PrT);
  const T t1 = T(4.0 / 3.0), t2 = T(2.0 / 3.0);
  T s11 = mu0 * (t1 * ux - t2 * (vy + wz)), s12 = mu0 * (uy + vx), s13 = mu0 * (uz + wx);
  T s22 = mu0 * (t1 * vy - t2 * (ux + wz)), s23 = mu0 * (vz + wy), s33 = mu0 * (t1 * wz - t2 * (ux + vy));
  T u1 = (Pu[c0] + Pu[c1]) * T(0.5), v1 = (Pv[c0] + Pv[c1]) * T(0.5), w1 = (Pw[c0] + Pw[c1]) * T(0.5);
  T E1 = u1 * s11 + v1 * s12 + w1 * s13 + k0 * Tx;
  T E2 = u1 * s12 + v1 * s22 + w1 * s23 + k0 * Ty;
  T E3 = u1 * s13 + v1 * s23 + w1 * s33 + k0 * Tz;
  T s1x = A.M[(M_NI1 + 3 * DIR) * tf + g], s1y = A.M[(M_NI2 + 3 * DIR) * tf + g], s1z = A.M[(M_NI3 + 3 * DIR) * tf + g];
  T S = A.M[(M_SI + DIR) * tf + g];
  Fo[0] = (s11 * s1x + s12 * s1y + s13 * s1z) * S;
  Fo[1] = (s12 * s1x + s22 * s1y + s23 * s1z) * S;
  Fo[2] = (s13 * s1x + s23 * s1y + s33 * s1z) * S;
  Fo[3] = (E1 * s1x + E2 * s1y + E3 * s1z) * S;
  return 0;
}

template <class T, int DIR>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_visc_flux(Arena<T> A) {
  const long long tf = A.tot_face;
  OCFD_GRID_STRIDE(g, tf) {
    int b = find_blk_h(A.pre_face, A.hint_face, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_face(B, g - B.oface, i, j, k);
    if (DIR == 0 && (j == B.ny || k == B.nz)) continue;
    if (DIR == 1 && (i == B.nx || k == B.nz)) continue;
    if (DIR == 2 && (i == B.nx || j == B.ny)) continue;
    T F[4];
    const int r = visc_face<T, DIR>(A, B, A.sp[B.solve], A.flags[b], i, j, k, g, F);
    T* Fo = A.Fv + (long long)DIR * 4 * tf + g;
    if (r == 0) { Fo[0] = F[0]; Fo[tf] = F[1]; Fo[2 * tf] = F[2]; Fo[3 * tf] = F[3]; }
    else if (r == 1) { Fo[0] = F[0]; Fo[tf] = F[1]; Fo[2 * tf] = F[2]; }
  }
}

// ============================================================================================
// Res(1:5) assembly in the reference order (inviscid i "=", j "+=", k "+=", viscous i, j, k),
// spectral radii (comput_Lijk, sub_time_acceleraction.f90:7-56) and local dt (comput_dt, 61-112)
// ============================================================================================
// the cell part of the assembly: spectral radii (comput_Lijk, sub_time_acceleraction.f90:7-56) and
// local dt (comput_dt, 61-112) from the primitives, then the stores of Res(1:5) = Rm, Lc, Lv, dt;
// f / fi1 / fj1 / fk1 are the cell's faces in the face index space, g its cell index.  RES / LDT:
// store Res / compute and store Lc, Lv, dt (the two parts read disjoint inputs)
template <class T, bool RES = true, bool LDT = true>
__device__ __forceinline__ void cell_finish(const Arena<T>& A, const BlkD& B, const SolveP& s, int b, int i, int j, int k, long long g,
                                            long long f, long long fi1, long long fj1, long long fk1, const T* Rm) {
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  T L[6], dtv;
  if (LDT) {
    long long c = bix(B, i, j, k);
    T D0 = T(0);
    if (s.viscous == 1) {
      T gm = T(s.gamma), f43 = T((double)(4.0f / 3.0f));  // `4./3.` default-real literal
      D0 = fmax_(gm, f43) / A.P[P_D * tb + c] * (A.mu[c] / T(s.prl) + A.mut[c] / T(s.prt));
    }
    T vol = A.vol[g];
    T vol1 = T(1) / vol;
    T uu = A.P[P_U * tb + c], v = A.P[P_V * tb + c], w = A.P[P_W * tb + c], cc = A.P[P_C * tb + c];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      long long fo = d == 0 ? fi1 : (d == 1 ? fj1 : fk1);
      const T* n1 = A.M + (M_NI1 + 3 * d) * tf;
      const T* n2 = A.M + (M_NI2 + 3 * d) * tf;
      const T* n3 = A.M + (M_NI3 + 3 * d) * tf;
      const T* Sd = A.M + (M_SI + d) * tf;
      T un = T(0.5) * (uu * (n1[f] + n1[fo]) + v * (n2[f] + n2[fo]) + w * (n3[f] + n3[fo]));
      T S0 = (Sd[f] + Sd[fo]) * T(0.5);
      L[d] = (dabs(un) + cc) * S0;
      L[3 + d] = D0 * S0 * S0 * vol1;
    }
    if (s.local_dt == 1) {
      T dt_fac = A.flags[b] == 0 ? T(1) : T(0.1);
      dtv = dt_fac * T(s.cfl) * vol / (L[0] + L[1] + L[2] + T(1) * (L[3] + L[4] + L[5]));
      if (s.dtime_mesh == 1) dtv = dtv * A.dtm[g];
      if (dtv > T(s.dtmax)) dtv = T(s.dtmax);
      if (dtv < T(s.dtmin)) dtv = T(s.dtmin);
    } else {
      dtv = T(s.dt_global);
    }
  }
  if (RES) {
#pragma unroll
    for (int m = 0; m < 5; m++) A.Res[m * tc + g] = Rm[m];
  }
  if (LDT) {
#pragma unroll
    for (int d = 0; d < 3; d++) { A.Lc[d * tc + g] = L[d]; A.Lv[d * tc + g] = L[3 + d]; }
    A.dt[g] = dtv;
  }
}

// RES_ONLY: Lc, Lv and dt were computed by k_cell_dt (the two-stream residual)
template <class T, bool RES_ONLY = false>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_assemble(Arena<T> A) {
  const long long tf = A.tot_face, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    long long f = fix_(B, i, j, k), fi1 = fix_(B, i + 1, j, k), fj1 = fix_(B, i, j + 1, k), fk1 = fix_(B, i, j, k + 1);
    bool visc = s.viscous == 1 && A.flags[b] != 1;
    // all loads and arithmetic first, the stores (Res, Lc, Lv, dt) at the end: a store inside the
    // loop would keep every later load (the planes may alias for the compiler) behind it
    T Rm[5];
#pragma unroll
    for (int m = 0; m < 5; m++) {
      const T* F0 = A.Fi + (0 * 5 + m) * tf;
      const T* F1 = A.Fi + (1 * 5 + m) * tf;
      const T* F2 = A.Fi + (2 * 5 + m) * tf;
      T R = F0[fi1] - F0[f];
      R = R + F1[fj1] - F1[f];
      R = R + F2[fk1] - F2[f];
      if (visc && m >= 1) {
        const T* V0 = A.Fv + (0 * 4 + m - 1) * tf;
        const T* V1 = A.Fv + (1 * 4 + m - 1) * tf;
        const T* V2 = A.Fv + (2 * 4 + m - 1) * tf;
        R = R + V0[fi1] - V0[f];
        R = R + V1[fj1] - V1[f];
        R = R + V2[fk1] - V2[f];
      }
      Rm[m] = R;
    }
    cell_finish<T, true, !RES_ONLY>(A, B, s, b, i, j, k, g, f, fi1, fj1, fk1, Rm);
  }
}

// the spectral radii and dt of every cell (the assembly's cell part without Res)
template <class T>
__global__ void __launch_bounds__(256, OCFD_MEM_MINB) k_cell_dt(Arena<T> A) {
  OCFD_GRID_STRIDE(g, A.tot_cell) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    cell_finish<T, false, true>(A, B, A.sp[B.solve], b, i, j, k, g, fix_(B, i, j, k), fix_(B, i + 1, j, k), fix_(B, i, j + 1, k),
                                fix_(B, i, j, k + 1), nullptr);
  }
}

// ============================================================================================
// The Navier-Stokes residual of a tile of cells in one pass (one CTA per tile at a time): the
// inviscid face fluxes of direction i, then j, then k, are computed into shared memory and each
// cell adds its two faces' difference to its Res held in shared memory, then the viscous ones the
// same way, then the spectral radii, dt and the stores - the order of k_assemble, so the bits are
// those of k_inv_flux + k_inv_kbc + k_visc_flux + k_assemble, without the face-flux planes.  A
// face on a tile's border is computed by both tiles that share it.  The viscous fluxes of the
// block-boundary faces are still stored to Fv, where the forces read them.
// ============================================================================================
template <class T, int DIR, bool PRIM, int ISCH, int IFLUX>
__device__ __forceinline__ void tile_inv_dir(const Arena<T>& A, const BlkD& B, const SolveP& s, int b, int i0, int j0, int k0,
                                             int ni, int nj, int nk, T* Fs, T* Rs) {
  const int fa = ni + (DIR == 0), fb = nj + (DIR == 1), fc = nk + (DIR == 2);
  const int nf = fa * fb * fc, MF = A.tile_maxf, MC = A.tile_maxc;
  for (int q = threadIdx.x; q < nf; q += blockDim.x) {
    const int a = q % fa, r = q / fa, bb = r % fb, c = r / fb;
    const int i = i0 + a, j = j0 + bb, k = k0 + c;
    const long long g = fix_(B, i, j, k);
    T F[5];
    bool kbc = false;
    if (DIR == 2 && (k == 1 || k == B.nz)) kbc = (A.bck[B.obck + (i - 1) + (long long)(B.nx - 1) * (j - 1)] & (k == 1 ? 4 : 8)) != 0;
    if (kbc) kbc_face(A, B, s, i, j, k, g, F);
    else inv_face<T, DIR, PRIM, ISCH, IFLUX>(A, B, s, b, i, j, k, g, F);
#pragma unroll
    for (int m = 0; m < 5; m++) Fs[m * MF + q] = F[m];
  }
  __syncthreads();
  const int nc = ni * nj * nk, step = DIR == 0 ? 1 : (DIR == 1 ? fa : fa * fb);
  for (int q = threadIdx.x; q < nc; q += blockDim.x) {
    const int a = q % ni, r = q / ni, bb = r % nj, c = r / nj;
    const int lo = a + fa * (bb + fb * c);
#pragma unroll
    for (int m = 0; m < 5; m++) {
      const T* F = Fs + m * MF;
      Rs[m * MC + q] = DIR == 0 ? F[lo + step] - F[lo] : Rs[m * MC + q] + F[lo + step] - F[lo];
    }
  }
  __syncthreads();
}

template <class T, int DIR>
__device__ __forceinline__ void tile_visc_dir(const Arena<T>& A, const BlkD& B, const SolveP& s, int i0, int j0, int k0, int ni,
                                              int nj, int nk, T* Fs, T* Rs) {
  const long long tf = A.tot_face;
  const int fa = ni + (DIR == 0), fb = nj + (DIR == 1), fc = nk + (DIR == 2);
  const int nf = fa * fb * fc, MF = A.tile_maxf, MC = A.tile_maxc;
  const int nd = DIR == 0 ? B.nx : (DIR == 1 ? B.ny : B.nz);
  for (int q = threadIdx.x; q < nf; q += blockDim.x) {
    const int a = q % fa, r = q / fa, bb = r % fb, c = r / fb;
    const int i = i0 + a, j = j0 + bb, k = k0 + c;
    const long long g = fix_(B, i, j, k);
    T F[4];
    visc_face<T, DIR>(A, B, s, 0, i, j, k, g, F);
#pragma unroll
    for (int m = 0; m < 4; m++) Fs[m * MF + q] = F[m];
    const int idx = DIR == 0 ? i : (DIR == 1 ? j : k);
    if (idx == 1 || idx == nd) {
      T* Fo = A.Fv + (long long)DIR * 4 * tf + g;
      Fo[0] = F[0]; Fo[tf] = F[1]; Fo[2 * tf] = F[2]; Fo[3 * tf] = F[3];
    }
  }
  __syncthreads();
  const int nc = ni * nj * nk, step = DIR == 0 ? 1 : (DIR == 1 ? fa : fa * fb);
  for (int q = threadIdx.x; q < nc; q += blockDim.x) {
    const int a = q % ni, r = q / ni, bb = r % nj, c = r / nj;
    const int lo = a + fa * (bb + fb * c);
#pragma unroll
    for (int m = 1; m < 5; m++) {
      const T* F = Fs + (m - 1) * MF;
      Rs[m * MC + q] = Rs[m * MC + q] + F[lo + step] - F[lo];
    }
  }
  __syncthreads();
}

// OverLimit: no viscous flux; the block-boundary faces of Fv hold 0 in components 1..3
template <class T, int DIR>
__device__ __forceinline__ void tile_visc_zero(const Arena<T>& A, const BlkD& B, int i0, int j0, int k0, int ni, int nj, int nk) {
  const long long tf = A.tot_face;
  const int fa = ni + (DIR == 0), fb = nj + (DIR == 1), fc = nk + (DIR == 2);
  const int nd = DIR == 0 ? B.nx : (DIR == 1 ? B.ny : B.nz);
  for (int q = threadIdx.x; q < fa * fb * fc; q += blockDim.x) {
    const int a = q % fa, r = q / fa, bb = r % fb, c = r / fb;
    const int i = i0 + a, j = j0 + bb, k = k0 + c;
    const int idx = DIR == 0 ? i : (DIR == 1 ? j : k);
    if (idx == 1 || idx == nd) {
      T* Fo = A.Fv + (long long)DIR * 4 * tf + fix_(B, i, j, k);
      Fo[0] = T(0); Fo[tf] = T(0); Fo[2 * tf] = T(0);
    }
  }
}

// VISC: the viscous fluxes are computed in the tile too (else k_visc_flux wrote them to Fv, and the
// cells add them from there, in the same order).  INV: the inviscid fluxes are computed in the tile
// (else k_inv_flux / k_inv_kbc wrote them to Fi, and the cells start from their differences there)
template <class T, int ISCH, bool INV>
struct NsTileOcc { static constexpr int value = INV ? InvFluxOccS<T, ISCH>::value : OCFD_MEM_MINB; };
template <class T, bool PRIM, int ISCH, int IFLUX, bool VISC, bool INV = true>
__global__ void __launch_bounds__(256, NsTileOcc<T, ISCH, INV>::value) k_ns_tile(Arena<T> A) {
  extern __shared__ __align__(16) unsigned char ns_smem[];
  T* Fs = reinterpret_cast<T*>(ns_smem);
  T* Rs = Fs + 5 * A.tile_maxf;
  const int MC = A.tile_maxc;
  for (int t = blockIdx.x; t < A.ntile; t += gridDim.x) {
    const int4 tl = A.tiles[t];
    const int b = tl.x, i0 = tl.y, j0 = tl.z, k0 = tl.w;
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    const int ni = min(B.tdim[0], B.nx - i0), nj = min(B.tdim[1], B.ny - j0), nk = min(B.tdim[2], B.nz - k0);
    if (INV) {
      tile_inv_dir<T, 0, PRIM, ISCH, IFLUX>(A, B, s, b, i0, j0, k0, ni, nj, nk, Fs, Rs);
      tile_inv_dir<T, 1, PRIM, ISCH, IFLUX>(A, B, s, b, i0, j0, k0, ni, nj, nk, Fs, Rs);
      tile_inv_dir<T, 2, PRIM, ISCH, IFLUX>(A, B, s, b, i0, j0, k0, ni, nj, nk, Fs, Rs);
    } else {
      const long long tf = A.tot_face;
      for (int q = threadIdx.x; q < ni * nj * nk; q += blockDim.x) {
        const int i = i0 + q % ni, r = q / ni, j = j0 + r % nj, k = k0 + r / nj;
        const long long f = fix_(B, i, j, k), fi1 = fix_(B, i + 1, j, k), fj1 = fix_(B, i, j + 1, k), fk1 = fix_(B, i, j, k + 1);
        T Rm[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
          const T* F0 = A.Fi + (0 * 5 + m) * tf;
          const T* F1 = A.Fi + (1 * 5 + m) * tf;
          const T* F2 = A.Fi + (2 * 5 + m) * tf;
          T R = F0[fi1] - F0[f];
          R = R + F1[fj1] - F1[f];
          R = R + F2[fk1] - F2[f];
          Rm[m] = R;
        }
#pragma unroll
        for (int m = 0; m < 5; m++) Rs[m * MC + q] = Rm[m];
      }
      __syncthreads();
    }
    if (VISC && s.viscous == 1) {
      if (A.flags[b] != 1) {
        tile_visc_dir<T, 0>(A, B, s, i0, j0, k0, ni, nj, nk, Fs, Rs);
        tile_visc_dir<T, 1>(A, B, s, i0, j0, k0, ni, nj, nk, Fs, Rs);
        tile_visc_dir<T, 2>(A, B, s, i0, j0, k0, ni, nj, nk, Fs, Rs);
      } else {
        tile_visc_zero<T, 0>(A, B, i0, j0, k0, ni, nj, nk);
        tile_visc_zero<T, 1>(A, B, i0, j0, k0, ni, nj, nk);
        tile_visc_zero<T, 2>(A, B, i0, j0, k0, ni, nj, nk);
      }
    }
    const int nc = ni * nj * nk;
    for (int q = threadIdx.x; q < nc; q += blockDim.x) {
      const int i = i0 + q % ni, r = q / ni, j = j0 + r % nj, k = k0 + r / nj;
      const long long f = fix_(B, i, j, k), fi1 = fix_(B, i + 1, j, k), fj1 = fix_(B, i, j + 1, k), fk1 = fix_(B, i, j, k + 1);
      T Rm[5];
#pragma unroll
      for (int m = 0; m < 5; m++) Rm[m] = Rs[m * MC + q];
      if (!VISC && s.viscous == 1 && A.flags[b] != 1) {
        const long long tf = A.tot_face;
#pragma unroll
        for (int m = 1; m < 5; m++) {
          const T* V0 = A.Fv + (0 * 4 + m - 1) * tf;
          const T* V1 = A.Fv + (1 * 4 + m - 1) * tf;
          const T* V2 = A.Fv + (2 * 4 + m - 1) * tf;
          T R = Rm[m];
          R = R + V0[fi1] - V0[f];
          R = R + V1[fj1] - V1[f];
          R = R + V2[fk1] - V2[f];
          Rm[m] = R;
        }
      }
      cell_finish(A, B, s, b, i, j, k, cix(B, i, j, k), f, fi1, fj1, fk1, Rm);
    }
    __syncthreads();
  }
}

// ============================================================================================
// upwind implicit residual smoothing (Residual_smoothing, sub_time_acceleraction.f90:119-217, with
// tridiagonal 222-241): one thread per grid line of direction DIR, Res(1:5) of the line solved in
// one forward elimination and one back substitution.  The end cells of a line keep their values
// (Rs(1) = R(1), Rs(n) = R(n)), so lines of fewer than 3 cells are unchanged.  The elimination
// factor P(p) is common to the five variables; it is parked in DU plane 0 (free between the
// update's limiter and the next LU-SGS sweep), and Q_m(p) in Res(m) until the back substitution
// overwrites it with the smoothed value.
// ============================================================================================
template <class T, int DIR>
__global__ void __launch_bounds__(128) k_smooth(Arena<T> A) {
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  const long long nl = DIR == 0 ? A.tot_col : (DIR == 1 ? A.tot_lnj : A.tot_lnk);
  const long long* pre = DIR == 0 ? A.pre_col : (DIR == 1 ? A.pre_lnj : A.pre_lnk);
  OCFD_GRID_STRIDE(g, nl) {
    const int b = find_blk(pre, A.nblk, g);
    const BlkD& B = A.blk[b];
    const long long l = g - __ldg(pre + b);
    const int nxm = B.nx - 1, nym = B.ny - 1;
    int i = 1, j = 1, k = 1, n;
    long long sc, sf, sb;  // strides along the line in the cell, face and box index spaces
    if (DIR == 0) { j = (int)(l % nym) + 1; k = (int)(l / nym) + 1; n = nxm; sc = 1; sf = 1; sb = 1; }
    else if (DIR == 1) { i = (int)(l % nxm) + 1; k = (int)(l / nxm) + 1; n = nym; sc = nxm; sf = B.nx; sb = B.NX; }
    else { i = (int)(l % nxm) + 1; j = (int)(l / nxm) + 1; n = B.nz - 1; sc = (long long)nxm * nym; sf = (long long)B.nx * B.ny; sb = (long long)B.NX * B.NY; }
    if (n < 3) continue;
    const long long c1 = cix(B, i, j, k), f1 = fix_(B, i, j, k), b1 = bix(B, i, j, k);
    const T* Ld = A.Lc + DIR * tc;
    const T* La = A.Lc + (DIR == 0 ? 1 : 0) * tc;
    const T* Lb = A.Lc + (DIR == 2 ? 1 : 2) * tc;
    const T* n1 = A.M + (M_NI1 + 3 * DIR) * tf;
    const T* n2 = A.M + (M_NI2 + 3 * DIR) * tf;
    const T* n3 = A.M + (M_NI3 + 3 * DIR) * tf;
    double Pp = 0.0, Qp[5];
#pragma unroll
    for (int m = 0; m < 5; m++) Qp[m] = (double)A.Res[m * tc + c1];
    for (int q = 2; q <= n - 1; q++) {
      const long long c = c1 + (q - 1) * sc, f = f1 + (q - 1) * sf, bx = b1 + (q - 1) * sb;
      const double ld = (double)Ld[c];
      double ei = 1.0, r = ld / (double)La[c];
      if (r < ei) ei = r;
      r = ld / (double)Lb[c];
      if (r < ei) ei = r;
      const double uu = A.P[P_U * tb + bx], vv = A.P[P_V * tb + bx], ww = A.P[P_W * tb + bx], cc = A.P[P_C * tb + bx];
      const double Mn = 0.5 * (uu * ((double)n1[f] + (double)n1[f + sf]) + vv * ((double)n2[f] + (double)n2[f + sf]) +
                               ww * ((double)n3[f] + (double)n3[f + sf])) / cc;
      double as, bs, cs;
      if (Mn > 1.0) { as = -ei; bs = 1.0 + ei; cs = 0.0; }
      else if (Mn < -1.0) { as = 0.0; bs = 1.0 + ei; cs = -ei; }
      else { as = -ei; bs = 1.0 + 2.0 * ei; cs = -ei; }
      const double tmp = 1.0 / (as * Pp + bs);
      Pp = -cs * tmp;
      A.DU[c] = Pp;
#pragma unroll
      for (int m = 0; m < 5; m++) {
        Qp[m] = ((double)A.Res[m * tc + c] - as * Qp[m]) * tmp;
        A.Res[m * tc + c] = (T)Qp[m];
      }
    }
    double Rn[5];
    const long long cn = c1 + (n - 1) * sc;
#pragma unroll
    for (int m = 0; m < 5; m++) Rn[m] = (double)A.Res[m * tc + cn];
    for (int q = n - 1; q >= 2; q--) {
      const long long c = c1 + (q - 1) * sc;
      const double P = A.DU[c];
#pragma unroll
      for (int m = 0; m < 5; m++) {
        Rn[m] = P * Rn[m] + (double)A.Res[m * tc + c];
        A.Res[m * tc + c] = (T)Rn[m];
      }
    }
  }
}

// ============================================================================================
// LU-SGS (du_LU_SGS, sub_LU_SGS.f90:4-129): one launch per hyperplane i+j+k = plane, all blocks
// ============================================================================================
__device__ __forceinline__ void comput_DFn(int NV, double* DF, const double* U, const double* DU, double n1, double n2, double n3, double gamma) {
  double U2[7];
  for (int m = 0; m < NV; m++) U2[m] = U[m] + DU[m];
  double un1 = (U[1] * n1 + U[2] * n2 + U[3] * n3) / U[0];
  double p1 = (gamma - 1.0) * (U[4] - 0.5 * (sq(U[1]) + sq(U[2]) + sq(U[3])) / U[0]);
  double un2 = (U2[1] * n1 + U2[2] * n2 + U2[3] * n3) / U2[0];
  double pp2 = (gamma - 1.0) * (U2[4] - 0.5 * (sq(U2[1]) + sq(U2[2]) + sq(U2[3])) / U2[0]);
  DF[0] = U2[0] * un2 - U[0] * un1;
  DF[1] = (U2[1] * un2 + pp2 * n1) - (U[1] * un1 + p1 * n1);
  DF[2] = (U2[2] * un2 + pp2 * n2) - (U[2] * un1 + p1 * n2);
  DF[3] = (U2[3] * un2 + pp2 * n3) - (U[3] * un1 + p1 * n3);
  DF[4] = (U2[4] + pp2) * un2 - (U[4] + p1) * un1;
  if (NV >= 6) DF[5] = U2[5] * un2 - U[5] * un1;
  if (NV == 7) DF[6] = U2[6] * un2 - U[6] * un1;
}

template <class T, int NV, bool UPPER>
__global__ void k_lusgs(Arena<T> A, int plane) {
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, A.tot_col) {
    int b = find_blk(A.pre_col, A.nblk, g);
    const BlkD& B = A.blk[b];
    long long l = g - B.ocol;
    const unsigned nym = (unsigned)(B.ny - 1), u = (unsigned)l;
    int j = (int)(u % nym) + 1, k = (int)(u / nym) + 1;
    int i = plane - k - j;
    if (i < 1 || i > B.nx - 1) continue;
    const SolveP& s = A.sp[B.solve];
    const double w = s.w_lu, gamma = s.gamma;
    const bool visc = s.viscous == 1;
    long long c = cix(B, i, j, k);
    double Lci = A.Lc[c], Lcj = A.Lc[tc + c], Lck = A.Lc[2 * tc + c];
    double Lvi = A.Lv[c], Lvj = A.Lv[tc + c], Lvk = A.Lv[2 * tc + c];
    double alfa[NV];
    double a0 = (double)A.vold[c] / (double)A.dt[c] + w * (Lci + Lcj + Lck);
#pragma unroll
    for (int m = 0; m < NV; m++) alfa[m] = a0;
    if (visc) {
#pragma unroll
      for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + 2.0 * (Lvi + Lvj + Lvk);
      if (NV == 6) {
        if (!UPPER) alfa[5] = alfa[5] + (Lvi + Lvj + Lvk);
        else alfa[5] = alfa[5] + Lvi + Lvj + Lvk;
      }
    }
    if (s.time_method == -1) {  // dual time: + Sfac1 vol (sub_LU_SGS.f90:39, 92)
#pragma unroll
      for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + A.sfac[1] * (double)A.vold[c];
    }
    double acc[NV];
#pragma unroll
    for (int m = 0; m < NV; m++) acc[m] = 0.0;
    double du[3][NV];
    const int off = UPPER ? 1 : -1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      int ii = i + (d == 0 ? off : 0), jj = j + (d == 1 ? off : 0), kk = k + (d == 2 ? off : 0);
      bool has = UPPER ? (d == 0 ? i != B.nx - 1 : (d == 1 ? j != B.ny - 1 : k != B.nz - 1)) : (d == 0 ? i != 1 : (d == 1 ? j != 1 : k != 1));
      if (!has) {
#pragma unroll
        for (int m = 0; m < NV; m++) du[d][m] = 0.0;
        continue;
      }
      long long cn = cix(B, ii, jj, kk), bn = bix(B, ii, jj, kk);
      double Uv[NV], DUv[NV], DF[NV];
#pragma unroll
      for (int m = 0; m < NV; m++) {
        double u = A.U[m * tb + bn];
        Uv[m] = m >= 5 ? clamp0(u) : u;
        DUv[m] = A.DU[m * tc + cn];
      }
      long long fn = fix_(B, i, j, k);                                   // normal of the lower face
      long long fs = UPPER ? fix_(B, ii, jj, kk) : fn;                    // area: upper face in the upper sweep
      double n1 = A.M[(M_NI1 + 3 * d) * tf + fn], n2 = A.M[(M_NI2 + 3 * d) * tf + fn], n3 = A.M[(M_NI3 + 3 * d) * tf + fn];
      double S = A.M[(M_SI + d) * tf + fs];
      comput_DFn(NV, DF, Uv, DUv, n1, n2, n3, gamma);
      double Lcn = A.Lc[d * tc + cn], Lvn = A.Lv[d * tc + cn];
#pragma unroll
      for (int m = 0; m < NV; m++) {
        double v;
        if (!UPPER) v = 0.5 * (DF[m] * S + w * Lcn * DUv[m]);
        else v = -(0.5 * (DF[m] * S - w * Lcn * DUv[m]));
        if (visc) v = v + Lvn * DUv[m];
        du[d][m] = v;
      }
    }
#pragma unroll
    for (int m = 0; m < NV; m++) {
      if (!UPPER) A.DU[m * tc + c] = ((double)A.Res[m * tc + c] + du[0][m] + du[1][m] + du[2][m]) / alfa[m];
      else A.DU[m * tc + c] = A.DU[m * tc + c] + (du[0][m] + du[1][m] + du[2][m]) / alfa[m];
    }
    (void)acc;
  }
}

// ============================================================================================
// update U (LU-SGS: U = Un + DU; RK3 stage), then the limiter test (sub_limitflow.f90:24-150)
// ============================================================================================
__device__ __forceinline__ bool lim_bad(const SolveP& s, double d, double u, double v, double w, double p) {
  return d < s.ldmin || p < s.lpmin || d > s.ldmax || p > s.lpmax || fabs(u) > s.lumax || fabs(v) > s.lumax || fabs(w) > s.lumax;
}

template <class T, int NV, int MODE>  // MODE 0: LU-SGS; 1,2,3: RK3 stage KRK; 4: dual-time inner iteration; 5: explicit Euler
__global__ void k_update(Arena<T> A) {
  const long long tb = A.tot_box, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    long long c = bix(B, i, j, k);
    // every variable's new value first, then the stores: a store of U inside the loop would keep
    // the next variable's loads (U and DU may alias for the compiler) behind it
    double Un[NV];
#pragma unroll
    for (int m = 0; m < NV; m++) {
      double u;
      if (MODE == 0) {
        u = A.U[m * tb + c] + A.DU[m * tc + g];
      } else if (MODE == 4) {  // U = U + DU with U6/U7 as limit_vt left them (sub_time_advance.f90:138-147)
        double cur = A.U[m * tb + c];
        if (m >= 5) cur = clamp0(cur);
        u = cur + A.DU[m * tc + g];
      } else if (MODE == 5) {  // U = Un + dt Res/vol (sub_time_advance.f90:238-239)
        double du = (double)A.Res[m * tc + g] / (double)A.vol[g];
        u = A.Un[m * tb + c] + (double)A.dt[g] * du;
      } else {
        const double Ra = MODE == 1 ? 1.0 : (MODE == 2 ? 3.0 / 4.0 : 1.0 / 3.0);
        const double Rb = MODE == 1 ? 1.0 : (MODE == 2 ? 1.0 / 4.0 : 2.0 / 3.0);
        const double Rg = MODE == 1 ? 0.0 : (MODE == 2 ? 1.0 / 4.0 : 2.0 / 3.0);
        double du = (double)A.Res[m * tc + g] / (double)A.vol[g];
        double cur = A.U[m * tb + c];
        if (m >= 5) cur = clamp0(cur);
        u = Ra * A.Un[m * tb + c] + Rg * cur + (double)A.dt[g] * Rb * du;
      }
      Un[m] = u;
    }
#pragma unroll
    for (int m = 0; m < NV; m++) A.U[m * tb + c] = Un[m];
    if (s.limit_flow == 1) {
      double d1 = Un[0], u1 = Un[1] / d1, v1 = Un[2] / d1, w1 = Un[3] / d1;
      double p1 = (Un[4] - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1)) * (s.gamma - 1.0);
      A.DU[g] = d1; A.DU[tc + g] = u1; A.DU[2 * tc + g] = v1; A.DU[3 * tc + g] = w1; A.DU[4 * tc + g] = p1;
      if (lim_bad(s, d1, u1, v1, w1, p1)) atomicAdd(&A.flags[A.nblk + b], 1);
    }
  }
}

// dual time: physical-time derivative on the residual (sub_Residual.f90:94-104), U6/U7 clamped as
// limit_vt leaves them in the reference
template <class T, int NV>
__global__ void k_dual_res(Arena<T> A) {
  const long long tb = A.tot_box, tc = A.tot_cell;
  const double Sfac = A.sfac[0];
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    const long long c = bix(B, i, j, k);
    const double vol = A.vold[g];
#pragma unroll
    for (int m = 0; m < NV; m++) {
      double u = A.U[m * tb + c];
      if (m >= 5) u = clamp0(u);
      double r = (double)A.Res[m * tc + g] - (3.0 * u - 4.0 * A.Un[m * tb + c] + A.Un1[m * tb + c]) * vol * Sfac;
      A.Res[m * tc + g] = (T)r;
    }
  }
}
// dual time: end of a physical step, Un1 = Un, Un = U on the interior (sub_time_advance.f90:178-196)
template <class T, int NV>
__global__ void k_dual_shift(Arena<T> A) {
  const long long tb = A.tot_box, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    const long long c = bix(B, i, j, k);
#pragma unroll
    for (int m = 0; m < NV; m++) { A.Un1[m * tb + c] = A.Un[m * tb + c]; A.Un[m * tb + c] = A.U[m * tb + c]; }
  }
}
// dual time: Un = Un1 = U everywhere (Init_flow, sub_init.f90:278-296)
template <class T, int NV>
__global__ void k_dual_init(Arena<T> A) {
  const long long n = (long long)NV * A.tot_box;
  OCFD_GRID_STRIDE(g, n) { A.Un[g] = A.U[g]; A.Un1[g] = A.U[g]; }
}

// neighbour-average repair of bad cells (sub_limitflow.f90:84-150); DU planes 0..4 hold d,u,v,w,p
template <class T>
__global__ void k_limit_fix(Arena<T> A) {
  const long long tb = A.tot_box, tc = A.tot_cell;
  OCFD_GRID_STRIDE(g, tc) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    if (A.flags[A.nblk + b] == 0) continue;
    const BlkD& B = A.blk[b];
    const SolveP& s = A.sp[B.solve];
    const double *d1 = A.DU, *u1 = A.DU + tc, *v1 = A.DU + 2 * tc, *w1 = A.DU + 3 * tc, *p1 = A.DU + 4 * tc;
    if (!lim_bad(s, d1[g], u1[g], v1[g], w1[g], p1[g])) continue;
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    double d0 = 0, u0 = 0, v0 = 0, w0 = 0, p0 = 0;
    int kn = 0;
    for (int ka = -1; ka <= 1; ka++)
      for (int ja = -1; ja <= 1; ja++)
        for (int ia = -1; ia <= 1; ia++) {
          int k1 = k + ka, j1 = j + ja, i1 = i + ia;
          if (i1 > 0 && i1 < B.nx && j1 > 0 && j1 < B.ny && k1 > 0 && k1 < B.nz) {
            long long q = cix(B, i1, j1, k1);
            if (!lim_bad(s, d1[q], u1[q], v1[q], w1[q], p1[q])) { d0 += d1[q]; u0 += u1[q]; v0 += v1[q]; w0 += w1[q]; p0 += p1[q]; kn++; }
          }
        }
    if (kn == 0) {
      d0 = d1[g]; u0 = u1[g]; v0 = v1[g]; w0 = w1[g]; p0 = p1[g];
      if (d0 < s.ldmin) d0 = s.ldmin;
      if (d0 > s.ldmax) d0 = s.ldmax;
      if (p0 < s.lpmin) p0 = s.lpmin;
      if (p0 > s.lpmax) p0 = s.lpmax;
      if (fabs(u0) > s.lumax) u0 = copysign(s.lumax, u0);
      if (fabs(v0) > s.lumax) v0 = copysign(s.lumax, v0);
      if (fabs(w0) > s.lumax) w0 = copysign(s.lumax, w0);
    } else {
      double sn1 = 1.0 / (double)kn;
      d0 = d0 * sn1; u0 = u0 * sn1; v0 = v0 * sn1; w0 = w0 * sn1; p0 = p0 * sn1;
    }
    long long c = bix(B, i, j, k);
    A.U[c] = d0; A.U[tb + c] = d0 * u0; A.U[2 * tb + c] = d0 * v0; A.U[3 * tb + c] = d0 * w0;
    A.U[4 * tb + c] = p0 / (s.gamma - 1.0) + 0.5 * d0 * (u0 * u0 + v0 * v0 + w0 * w0);
    A.flags[b] = 1;  // sticky IF_OverLimit (sub_limitflow.f90:171)
  }
}

// limit_flow_SA (sub_limitflow.f90:182-231).  The reference visits the interior cells in (k, j, i)
// order and limits each in place: U6 < SAmin becomes SAmin; U6 > LSAmax becomes the average of the
// 3x3x3 neighbours whose value lies in [SAmin, LSAmax] at that moment (LSAmax if none).  So a
// neighbour earlier in the order holds its limited value and a later one its original value.
// Every limited value is at least SAmin, and an earlier cell's limited value is max(v, SAmin) of
// what it holds in the array before the clamp pass, whether it was above LSAmax (replaced by an
// average in [SAmin, LSAmax]) or not.  That makes the order matter only among the cells above
// LSAmax, which k_sa_limit_serial visits in order (reading earlier neighbours as max(v, SAmin) and
// later ones as they are); k_sa_limit_par then clamps every other cell to SAmin in parallel.
template <class T>
__global__ void k_sa_limit_check(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, A.tot_cell) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    if (A.sp[B.solve].limit_flow == 1 && A.U[5 * tb + bix(B, i, j, k)] > A.sp[B.solve].lsamax) A.flags[2 * A.nblk + b] = 1;
  }
}
template <class T>
__global__ void k_sa_limit_par(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, A.tot_cell) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    if (A.sp[B.solve].limit_flow != 1) continue;
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    long long c = 5 * tb + bix(B, i, j, k);
    if (A.U[c] < 1.e-8) A.U[c] = 1.e-8;
  }
}
// one CTA per block with a cell above LSAmax: the block is scanned in chunks of SAL_CHUNK cells in
// the reference's order (warp ballots find the chunk's cells above LSAmax), and thread 0 replaces
// those cells, in order, by the average of their neighbours
constexpr int SAL_THREADS = 512, SAL_PER = 8, SAL_CHUNK = SAL_THREADS * SAL_PER;
template <class T>
__global__ void __launch_bounds__(SAL_THREADS) k_sa_limit_serial(Arena<T> A) {
  __shared__ unsigned s_bad[SAL_CHUNK / 32];
  const int b = blockIdx.x;
  if (b >= A.nblk || A.flags[2 * A.nblk + b] == 0) return;   // the same for every thread of the CTA
  const BlkD& B = A.blk[b];
  const double SAmin = 1.e-8, LSAmax = A.sp[B.solve].lsamax;
  double* U6 = A.U + 5 * A.tot_box;
  const int nxm = B.nx - 1, nym = B.ny - 1, nzm = B.nz - 1;
  const long long ncl = (long long)nxm * nym * nzm;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto cell = [&](long long l, int& i, int& j, int& k) {
    const unsigned u = (unsigned)l, t = u / (unsigned)nxm;
    i = (int)(u - t * (unsigned)nxm) + 1; j = (int)(t % (unsigned)nym) + 1; k = (int)(t / (unsigned)nym) + 1;
  };
  for (long long base = 0; base < ncl; base += SAL_CHUNK) {
    bool any = false;
#pragma unroll
    for (int q = 0; q < SAL_PER; q++) {
      const long long l = base + q * SAL_THREADS + tid;   // word (q * SAL_THREADS + tid) / 32 = q * 16 + warp
      bool bad = false;
      if (l < ncl) {
        int i, j, k;
        cell(l, i, j, k);
        bad = U6[bix(B, i, j, k)] > LSAmax;
      }
      const unsigned m = __ballot_sync(0xffffffffu, bad);
      if (lane == 0) s_bad[q * (SAL_THREADS / 32) + warp] = m;
      any |= bad;
    }
    if (__syncthreads_or(any) && tid == 0) {
      for (int w = 0; w < SAL_CHUNK / 32; w++) {
        unsigned m = s_bad[w];
        while (m) {
          const int bit = __ffs(m) - 1;
          m &= m - 1;
          const long long l = base + w * 32 + bit;
          int i, j, k;
          cell(l, i, j, k);
          double s0 = 0.0;
          int kn = 0;
          for (int ka = -1; ka <= 1; ka++)
            for (int ja = -1; ja <= 1; ja++)
              for (int ia = -1; ia <= 1; ia++) {
                const int k1 = k + ka, j1 = j + ja, i1 = i + ia;
                if (i1 > 0 && i1 < B.nx && j1 > 0 && j1 < B.ny && k1 > 0 && k1 < B.nz) {
                  const long long l1 = (long long)(i1 - 1) + (long long)nxm * ((j1 - 1) + (long long)nym * (k1 - 1));
                  double q = U6[bix(B, i1, j1, k1)];
                  if (l1 < l && q < SAmin) q = SAmin;   // an earlier cell holds its limited value
                  if (q >= SAmin && q <= LSAmax) { s0 = s0 + q; kn++; }
                }
              }
          U6[bix(B, i, j, k)] = kn == 0 ? LSAmax : s0 / kn;
        }
      }
    }
    __syncthreads();   // this chunk's averages are written before the next chunk's scan reads them
  }
}

// force_vt_kw (sub_time_advance.f90:27-61)
template <class T, int NV>
__global__ void k_vtkw(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, A.tot_cell) {
    int b = find_blk_h(A.pre_cell, A.hint_cell, A.nblk, g);
    const BlkD& B = A.blk[b];
    int i, j, k;
    dec_cell(B, g - B.ocell, i, j, k);
    long long c = bix(B, i, j, k);
    if (A.U[5 * tb + c] < 0) A.U[5 * tb + c] = 1.e-10;
    if (NV == 7 && A.U[6 * tb + c] < 0) A.U[6 * tb + c] = 1.e-10;
  }
}

// RK3: Un = U over the box (Set_Un range -1..n+1 is a subset)
template <class T, int NV>
__global__ void k_copy_un(Arena<T> A) {
  const long long n = (long long)NV * A.tot_box;
  OCFD_GRID_STRIDE(g, n) A.Un[g] = A.U[g];
}

// ============================================================================================
// boundary conditions (Boundary_condition_onemesh, sub_boundary.f90:6-80): one CTA per block, its
// physical subfaces in file order (later subfaces may read ghost values earlier ones wrote)
// ============================================================================================
template <int NV>
__device__ void wall_bound_d(const SolveP& s, double* U, long long tb, long long c1, long long c2, double mu1, double dw) {  // 405-454
  double U1[NV], Ug[NV];
  for (int m = 0; m < NV; m++) U1[m] = U[m * tb + c1];
  if (s.twall > 0.0) {
    double gamma = s.gamma, Ma = s.ma;
    double d1 = U1[0], uu1 = U1[1] / d1, v1 = U1[2] / d1, w1 = U1[3] / d1;
    double p1 = (U1[4] - 0.5 * d1 * (uu1 * uu1 + v1 * v1 + w1 * w1)) * (gamma - 1.0);
    double T1 = gamma * Ma * Ma * p1 / d1;
    double p2 = p1, T2 = 2.0 * s.twall - T1;
    if (T2 < 0.5 * T1) T2 = 0.5 * T1;
    double uu2 = -uu1, v2 = -v1, w2 = -w1;
    double d2 = gamma * Ma * Ma * p2 / T2;
    Ug[0] = d2; Ug[1] = d2 * uu2; Ug[2] = d2 * v2; Ug[3] = d2 * w2;
    Ug[4] = p2 / (gamma - 1.0) + 0.5 * d2 * (uu2 * uu2 + v2 * v2 + w2 * w2);
  } else {
    Ug[0] = U1[0]; Ug[1] = -U1[1]; Ug[2] = -U1[2]; Ug[3] = -U1[3]; Ug[4] = U1[4];
  }
  if (NV == 6) Ug[5] = 0.0;
  if (NV == 7) {
    double wt = 60.0 * mu1 / (U1[0] * 0.075 * sq(dw) * s.re);
    Ug[5] = -U1[5];
    Ug[6] = (U1[0] + Ug[0]) * wt - U1[6];
  }
  for (int m = 0; m < NV; m++) U[m * tb + c2] = Ug[m];
}

// Physical boundary conditions.  The reference applies the subfaces of a block one after the
// other (ghost cells on edges are written by more than one subface, and far-field loops read
// ghost cells written by earlier subfaces), so the work is issued in rounds: round r applies the
// r-th subface of every block, all blocks and all cells of a subface in parallel, and the rounds
// run in order.
template <class T, int NV>
__device__ __forceinline__ void bc_cell(Arena<T>& A, const SubD& S, const BlkD& B, const SolveP& s, long long l) {
  const long long tb = A.tot_box, tf = A.tot_face;
  double* U = A.U;
  const int f = S.face;
  if ((S.bc == 2 && s.viscous == 1)) {  // boundary_wall (87-147)
    int i, j, k, gi, gj, gk;
    subcell_ijk(S, l, i, j, k);
    ghost_of(S, i, j, k, gi, gj, gk);
    long long c1 = bix(B, i, j, k);
    double dwv = NV == 7 ? (double)A.dwd[cix(B, i, j, k)] : 0.0;
    wall_bound_d<NV>(s, U, tb, c1, bix(B, gi, gj, gk), (double)A.mu[c1], dwv);
  } else if (S.bc == 4 || S.bc == 5 || S.bc == 6 || S.bc == 401) {  // far field / inflow / outflow / extrapolate (152-283, 458-504)
    const int Flag = S.bc == 5 ? 2 : (S.bc == 6 ? 1 : 0);
    const unsigned ni = (unsigned)(S.ie - S.ib + 1), nj = (unsigned)(S.je - S.jb + 1), u = (unsigned)l, t = u / ni;
    int i = S.ib + (int)(u - t * ni), j = S.jb + (int)(t % nj), k = S.kb + (int)(t / nj);
    int i1 = i, j1 = j, k1 = k, i2 = i, j2 = j, k2 = k;
    double n1, n2, n3, sg = (f <= 3) ? -1.0 : 1.0;
    if (f == 1) i2 = i - 1; else if (f == 2) j2 = j - 1; else if (f == 3) k2 = k - 1;
    else if (f == 4) i1 = i - 1; else if (f == 5) j1 = j - 1; else k1 = k - 1;
    int d = (f - 1) % 3;
    long long fi = fix_(B, i, j, k);
    n1 = A.Md[(M_NI1 + 3 * d) * tf + fi]; n2 = A.Md[(M_NI2 + 3 * d) * tf + fi]; n3 = A.Md[(M_NI3 + 3 * d) * tf + fi];
    if (sg < 0) { n1 = -n1; n2 = -n2; n3 = -n3; }
    long long c1 = bix(B, i1, j1, k1), c2 = bix(B, i2, j2, k2);
    if (S.bc == 401) {
      for (int m = 0; m < NV; m++) U[m * tb + c2] = U[m * tb + c1];
      return;
    }
    double gamma = s.gamma;
    double d1 = U[c1], u1 = U[tb + c1] / d1, v1 = U[2 * tb + c1] / d1, w1 = U[3 * tb + c1] / d1;
    double p1 = (U[4 * tb + c1] - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1)) * (gamma - 1.0);
    double c1s = sqrt(gamma * p1 / d1);
    double d2, u2, v2, w2, p2, Ma_n = 0.0;
    double d_inf = s.d_inf, u_inf = s.u_inf, v_inf = s.v_inf, w_inf = s.w_inf, p_inf = s.p_inf;
    if (Flag == 1) { d2 = d1; u2 = u1; v2 = v1; w2 = w1; p2 = p1; }
    else if (Flag == 2) { d2 = d_inf; u2 = u_inf; v2 = v_inf; w2 = w_inf; p2 = p_inf; }
    else {
      if (s.p_outlet <= -1.0) Ma_n = (u_inf * n1 + v_inf * n2 + w_inf * n3) * s.ma;
      else Ma_n = (u1 * n1 + v1 * n2 + w1 * n3) / c1s;
      if (Ma_n > 1.0) { d2 = d1; u2 = u1; v2 = v1; w2 = w1; p2 = p1; }
      else if (Ma_n > -1.e-6) {
        if (s.p_outlet > 0.0) {
          double pb = s.p_outlet, db = d1 + (pb - p1) / (c1s * c1s);
          double ub = u1 + (p1 - pb) / (d1 * c1s) * n1, vb = v1 + (p1 - pb) / (d1 * c1s) * n2, wb = w1 + (p1 - pb) / (d1 * c1s) * n3;
          p2 = 2.0 * pb - p1; d2 = 2.0 * db - d1; u2 = 2.0 * ub - u1; v2 = 2.0 * vb - v1; w2 = 2.0 * wb - w1;
        } else { d2 = d1; u2 = u1; v2 = v1; w2 = w1; p2 = p1; }
      } else if (Ma_n > -1.0) {
        double pb = 0.5 * (p1 + p_inf - d1 * c1s * ((u_inf - u1) * n1 + (v_inf - v1) * n2 + (w_inf - w1) * n3));
        double db = d_inf + (pb - p_inf) / (c1s * c1s);
        double ub = u_inf - (p_inf - pb) / (d1 * c1s) * n1, vb = v_inf - (p_inf - pb) / (d1 * c1s) * n2, wb = w_inf - (p_inf - pb) / (d1 * c1s) * n3;
        p2 = 2.0 * pb - p1; d2 = 2.0 * db - d1; u2 = 2.0 * ub - u1; v2 = 2.0 * vb - v1; w2 = 2.0 * wb - w1;
      } else { d2 = d_inf; u2 = u_inf; v2 = v_inf; w2 = w_inf; p2 = p_inf; }
    }
    U[c2] = d2; U[tb + c2] = d2 * u2; U[2 * tb + c2] = d2 * v2; U[3 * tb + c2] = d2 * w2;
    U[4 * tb + c2] = p2 / (gamma - 1.0) + 0.5 * d2 * (u2 * u2 + v2 * v2 + w2 * w2);
    if (Ma_n > 0.0 || Flag == 1) {
      if (NV >= 6) U[5 * tb + c2] = U[5 * tb + c1];
      if (NV == 7) U[6 * tb + c2] = U[6 * tb + c1];
    } else {
      if (NV == 6) U[5 * tb + c2] = 5.0;
      if (NV == 7) { U[5 * tb + c2] = d_inf * s.kt_inf; U[6 * tb + c2] = d_inf * s.wt_inf; }
    }
  } else {  // symmetry / slip wall (291-373)
    int d = (f - 1) % 3;
    int i, j, k, gi, gj, gk;
    subcell_ijk(S, l, i, j, k);
    ghost_of(S, i, j, k, gi, gj, gk);
    // the normal is taken at the boundary node plane (i=ib or ie, ...)
    int ni_ = i, nj_ = j, nk_ = k;
    if (f == 4) ni_ = S.ie; else if (f == 5) nj_ = S.je; else if (f == 6) nk_ = S.ke;
    long long fi = fix_(B, ni_, nj_, nk_);
    double n1 = A.Md[(M_NI1 + 3 * d) * tf + fi], n2 = A.Md[(M_NI2 + 3 * d) * tf + fi], n3 = A.Md[(M_NI3 + 3 * d) * tf + fi];
    long long c1 = bix(B, i, j, k), c2 = bix(B, gi, gj, gk);
    for (int m = 0; m < NV; m++) U[m * tb + c2] = U[m * tb + c1];
    double Vn = U[tb + c1] * n1 + U[2 * tb + c1] * n2 + U[3 * tb + c1] * n3;
    U[tb + c2] = U[tb + c2] - 2.0 * Vn * n1;
    U[2 * tb + c2] = U[2 * tb + c2] - 2.0 * Vn * n2;
    U[3 * tb + c2] = U[3 * tb + c2] - 2.0 * Vn * n3;
  }
}

// one round: entries e0..e1-1 of the boundary work list (subface, cells), ncell cells in total
template <class T, int NV>
__global__ void k_bc_round(Arena<T> A, int e0, int e1, long long ncell) {
  OCFD_GRID_STRIDE(g, ncell) {
    const long long gg = A.bc_pre[e0] + g;
    const int e = e0 + find_blk(A.bc_pre + e0, e1 - e0, gg);
    const SubD S = A.sub[A.bc_ent[e]];
    const BlkD& B = A.blk[S.blk];
    if (A.only_solve >= 0 && B.solve != A.only_solve) continue;
    bc_cell<T, NV>(A, S, B, A.sp[B.solve], gg - A.bc_pre[e]);
  }
}

// ============================================================================================
// block-interface halo (Umessage_send_mpi, sub_update_buffer_mpi.f90:42-141): LAP ghost layers
// of every inner subface are copied from the partner's interior with the (L1,L2,L3) permutation
// ============================================================================================
// cell l of subface S's copy, counted in the target's order: the source cell (i,j,k) in the
// subface's own block (its LAP layers next to the face) and the target cell in the partner block
// (its LAP ghost layers)
__device__ __forceinline__ void halo_idx(const SubD& S, long long l, int* src, int* dst) {
  int kb[3] = {S.ib, S.jb, S.kb}, ke[3] = {S.ie - 1, S.je - 1, S.ke - 1};
  int d = (S.face - 1) % 3;
  if (S.face > 3) kb[d] = kb[d] - LAP;
  ke[d] = kb[d] + LAP - 1;
  int kb1[3] = {S.ib1, S.jb1, S.kb1}, ke1[3] = {S.ie1 - 1, S.je1 - 1, S.ke1 - 1};
  int d1 = (S.face1 - 1) % 3;
  if (S.face1 <= 3) kb1[d1] = kb1[d1] - LAP;
  ke1[d1] = kb1[d1] + LAP - 1;
  const unsigned n0 = (unsigned)(ke1[0] - kb1[0] + 1), n1 = (unsigned)(ke1[1] - kb1[1] + 1);
  const unsigned u = (unsigned)l, t = u / n0;  // a copy's cell count is below 2^31
  int ka[3] = {(int)(u - t * n0), (int)(t % n1), (int)(t / n1)};
  int L[3] = {abs(S.L1), abs(S.L2), abs(S.L3)};
  int P[3] = {S.L1 >= 0 ? 1 : -1, S.L2 >= 0 ? 1 : -1, S.L3 >= 0 ? 1 : -1};
#pragma unroll
  for (int q = 0; q < 3; q++) {
    src[q] = (P[q] > 0 ? kb[q] : ke[q]) + ka[L[q] - 1] * P[q];
    dst[q] = kb1[q] + ka[q];
  }
}
template <class T>
__device__ __forceinline__ void halo_map(const Arena<T>& A, const SubD& S, long long l, long long& cs, long long& ct) {
  int src[3], dst[3];
  halo_idx(S, l, src, dst);
  cs = bix(A.blk[S.blk], src[0], src[1], src[2]);
  ct = bix(A.blk[S.nb1], dst[0], dst[1], dst[2]);
}

// every interface copy in one launch: valid when no copy reads or writes cells another copy
// writes (blocks at least LAP cells thick across their interfaces)
template <class T, int NV>
__global__ void k_halo(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, A.tot_halo) {
    int s = find_blk(A.pre_halo, A.nsub, g);
    if (A.only_solve >= 0 && A.blk[A.sub[s].nb1].solve != A.only_solve) continue;
    long long cs, ct;
    halo_map(A, A.sub[s], g - A.pre_halo[s], cs, ct);
    double v[NV];  // all loads before the stores (a store in between would hold the next load back)
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = A.U[m * tb + cs];
#pragma unroll
    for (int m = 0; m < NV; m++) A.U[m * tb + ct] = v[m];
  }
}

// one level of ordered interface copies: PHASE 0 gathers the level's sources into stage, PHASE 1
// scatters them, so a copy whose source reaches ghost cells reads them as the reference's
// subface-by-subface order leaves them (update_buffer_onemesh, sub_update_buffer_mpi.f90:55-140).
// ent[e0..e1) are the level's subfaces, pre[e] the first staged cell of entry e (from 0).
template <class T, int NV, int PHASE>
__global__ void k_halo_level(Arena<T> A, const int* ent, const long long* pre, int e0, int e1, long long cells, double* stage) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, cells) {
    int e = e0 + find_blk(pre + e0, e1 - e0, g);
    if (A.only_solve >= 0 && A.blk[A.sub[ent[e]].nb1].solve != A.only_solve) continue;
    long long cs, ct;
    halo_map(A, A.sub[ent[e]], g - pre[e], cs, ct);
    double v[NV];  // all loads before the stores
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = PHASE == 0 ? A.U[m * tb + cs] : stage[m * cells + g];
#pragma unroll
    for (int m = 0; m < NV; m++) {
      if (PHASE == 0) stage[m * cells + g] = v[m];
      else A.U[m * tb + ct] = v[m];
    }
  }
}

// copies between ranks of a block-sharded handle (Umessage_send_mpi / Umessage_recv_mpi,
// sub_update_buffer_mpi.f90:42-211): the pack gathers the source cells of the subfaces ent[0..n)
// (this rank's blocks, partner on another rank) into buf, cell-major with NV values per cell;
// the unpack scatters buf into the ghost cells of the subfaces sub[0..n) of other ranks' blocks
// whose partner (nb1, renumbered to this handle's block) is here.  Both sides count a copy's
// cells in the target's order, so the two buffers line up entry by entry.
template <class T, int NV>
__global__ void k_halo_pack(Arena<T> A, const int* ent, const long long* pre, int n, long long cells, double* buf) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, cells) {
    const int e = find_blk(pre, n, g);
    const SubD S = A.sub[ent[e]];
    int src[3], dst[3];
    halo_idx(S, g - pre[e], src, dst);
    const long long cs = bix(A.blk[S.blk], src[0], src[1], src[2]);
    double v[NV];  // all loads before the stores
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = A.U[m * tb + cs];
#pragma unroll
    for (int m = 0; m < NV; m++) buf[g * NV + m] = v[m];
  }
}
template <class T, int NV>
__global__ void k_halo_unpack(Arena<T> A, const SubD* sub, const long long* pre, int n, long long cells, const double* buf) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, cells) {
    const int e = find_blk(pre, n, g);
    const SubD S = sub[e];
    int src[3], dst[3];
    halo_idx(S, g - pre[e], src, dst);
    const long long ct = bix(A.blk[S.nb1], dst[0], dst[1], dst[2]);
    double v[NV];  // all loads before the stores
#pragma unroll
    for (int m = 0; m < NV; m++) v[m] = buf[g * NV + m];
#pragma unroll
    for (int m = 0; m < NV; m++) A.U[m * tb + ct] = v[m];
  }
}

// edge and vertex ghosts by averaging (get_U_conner, sub_update_buffer_mpi.f90:515-549)
template <class T, int NV>
__global__ void k_corner(Arena<T> A) {  // edges: grid (blocks, CTAs per block)
  const int b = blockIdx.x;
  if (b >= A.nblk) return;
  const BlkD& B = A.blk[b];
  if (A.only_solve >= 0 && B.solve != A.only_solve) return;
  const long long tb = A.tot_box;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  double* U = A.U;
  auto u = [&](int m, int i, int j, int k) -> double& { return U[m * tb + bix(B, i, j, k)]; };
  int nk = nz - 1, nj = ny - 1, ni = nx - 1;
  long long n = (long long)NV * 4 * (nk + nj + ni);
  for (long long l = (long long)blockIdx.y * blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.y * blockDim.x) {
    int m = (int)(l % NV);
    long long r = l / NV;
    int e = (int)(r % 4);
    long long t = r / 4;
    if (t < nk) {
      int k = (int)t + 1;
      if (e == 0) u(m, 0, 0, k) = (u(m, 1, 0, k) + u(m, 0, 1, k)) * 0.5;
      else if (e == 1) u(m, nx, 0, k) = (u(m, nx - 1, 0, k) + u(m, nx, 1, k)) * 0.5;
      else if (e == 2) u(m, 0, ny, k) = (u(m, 1, ny, k) + u(m, 0, ny - 1, k)) * 0.5;
      else u(m, nx, ny, k) = (u(m, nx - 1, ny, k) + u(m, nx, ny - 1, k)) * 0.5;
    } else if (t < nk + nj) {
      int j = (int)(t - nk) + 1;
      if (e == 0) u(m, 0, j, 0) = (u(m, 1, j, 0) + u(m, 0, j, 1)) * 0.5;
      else if (e == 1) u(m, nx, j, 0) = (u(m, nx - 1, j, 0) + u(m, nx, j, 1)) * 0.5;
      else if (e == 2) u(m, 0, j, nz) = (u(m, 1, j, nz) + u(m, 0, j, nz - 1)) * 0.5;
      else u(m, nx, j, nz) = (u(m, nx - 1, j, nz) + u(m, nx, j, nz - 1)) * 0.5;
    } else {
      int i = (int)(t - nk - nj) + 1;
      if (e == 0) u(m, i, 0, 0) = (u(m, i, 1, 0) + u(m, i, 0, 1)) * 0.5;
      else if (e == 1) u(m, i, ny, 0) = (u(m, i, ny - 1, 0) + u(m, i, ny, 1)) * 0.5;
      else if (e == 2) u(m, i, 0, nz) = (u(m, i, 1, nz) + u(m, i, 0, nz - 1)) * 0.5;
      else u(m, i, ny, nz) = (u(m, i, ny - 1, nz) + u(m, i, ny, nz - 1)) * 0.5;
    }
  }
}
// the 8 vertices of every block from the edge values (after k_corner)
template <class T, int NV>
__global__ void k_corner_vtx(Arena<T> A) {
  const long long tb = A.tot_box;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)A.nblk * NV * 8) return;
  const int b = (int)(g / (NV * 8));
  const BlkD& B = A.blk[b];
  if (A.only_solve >= 0 && B.solve != A.only_solve) return;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  double* U = A.U;
  auto u = [&](int m, int i, int j, int k) -> double& { return U[m * tb + bix(B, i, j, k)]; };
  {
    const int r = (int)(g % (NV * 8));
    int m = r % NV, v = r / NV;
    int ia = (v & 1) ? nx : 0, ja = (v & 2) ? ny : 0, kz = (v & 4) ? nz : 0;
    int ib = (v & 1) ? nx - 1 : 1, jb = (v & 2) ? ny - 1 : 1, kb = (v & 4) ? nz - 1 : 1;
    u(m, ia, ja, kz) = (2.0 * (u(m, ib, ja, kz) + u(m, ia, jb, kz) + u(m, ia, ja, kb)) - (u(m, ib, jb, kz) + u(m, ib, ja, kb) + u(m, ia, jb, kb))) / 3.0;
  }
}

// ============================================================================================
// residual norms (comput_max_Res_onemesh, sub_time_advance.f90:330-380): FP64, fixed chunks and
// a fixed reduction tree, so the result is deterministic
// ============================================================================================
template <class T, int NV>
__global__ void k_norms(Arena<T> A, double* part, unsigned long long* nan_at) {
  __shared__ double smax[NV][256], ssum[NV][256];
  const int4 ch = A.cchunk[blockIdx.x];
  const BlkD& B = A.blk[ch.x];
  const long long tc = A.tot_cell;
  double mx[NV], sm[NV];
#pragma unroll
  for (int m = 0; m < NV; m++) { mx[m] = 0.0; sm[m] = 0.0; }
  // the first NaN position of this thread's cells, published by one atomic after the loop (an
  // atomic inside it would order every later load behind the NaN test of the previous value)
  unsigned long long nan_first = ~0ULL;
#pragma unroll 4
  for (int l = threadIdx.x; l < ch.z; l += blockDim.x) {  // unrolled: loads of 4 cells in flight, sums in order
    long long g = B.ocell + ch.y + l;
#pragma unroll
    for (int m = 0; m < NV; m++) {
      double r = (double)__ldg(A.Res + m * tc + g);
      if (isnan(r)) nan_first = min(nan_first, (unsigned long long)(g * 8 + m));
      mx[m] = fmax(mx[m], fabs(r));
      sm[m] = sm[m] + r * r;
    }
  }
  if (nan_first != ~0ULL) atomicMin(nan_at, nan_first);
#pragma unroll
  for (int m = 0; m < NV; m++) { smax[m][threadIdx.x] = mx[m]; ssum[m][threadIdx.x] = sm[m]; }
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int m = 0; m < NV; m++) {
        smax[m][threadIdx.x] = fmax(smax[m][threadIdx.x], smax[m][threadIdx.x + w]);
        ssum[m][threadIdx.x] = ssum[m][threadIdx.x] + ssum[m][threadIdx.x + w];
      }
    __syncthreads();
  }
  if (threadIdx.x < NV) {
    part[(long long)blockIdx.x * 14 + threadIdx.x] = smax[threadIdx.x][0];
    part[(long long)blockIdx.x * 14 + 7 + threadIdx.x] = ssum[threadIdx.x][0];
  }
}
// per solve (one CTA each): every thread folds a fixed stride of the solve's chunks in order,
// then a fixed tree over the threads -- the same order whatever else the handle holds
template <class T>
__global__ void k_norms_combine(Arena<T> A, const double* part, double* out) {
  __shared__ double smx[7][128], ssm[7][128];
  const int sv = blockIdx.x, c0 = A.cspre[sv], c1 = A.cspre[sv + 1];
  double mx[7] = {0, 0, 0, 0, 0, 0, 0}, sm[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int c = c0 + (int)threadIdx.x; c < c1; c += blockDim.x)
#pragma unroll
    for (int m = 0; m < 7; m++) { mx[m] = fmax(mx[m], part[c * 14 + m]); sm[m] = sm[m] + part[c * 14 + 7 + m]; }
#pragma unroll
  for (int m = 0; m < 7; m++) { smx[m][threadIdx.x] = mx[m]; ssm[m][threadIdx.x] = sm[m]; }
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int m = 0; m < 7; m++) {
        smx[m][threadIdx.x] = fmax(smx[m][threadIdx.x], smx[m][threadIdx.x + w]);
        ssm[m][threadIdx.x] = ssm[m][threadIdx.x] + ssm[m][threadIdx.x + w];
      }
    __syncthreads();
  }
  if (threadIdx.x < 7) { out[sv * 14 + threadIdx.x] = smx[threadIdx.x][0]; out[sv * 14 + 7 + threadIdx.x] = ssm[threadIdx.x][0]; }
}

// ============================================================================================
// forces (comput_force, sub_Post.f90:4-265): per wall chunk partial sums of the 9 components
// ============================================================================================
template <class T>
__global__ void k_forces(Arena<T> A, double* part) {
  __shared__ double sh[9][256];
  const int4 ch = A.wchunk[blockIdx.x];
  const SubD S = A.sub[ch.x];
  const BlkD& B = A.blk[S.blk];
  const SolveP& s = A.sp[B.solve];
  const long long tb = A.tot_box, tf = A.tot_face;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double p_inf = s.p_inf, gamma = s.gamma;
  const int f = S.face, d = (f - 1) % 3;
  for (int l = threadIdx.x; l < ch.z; l += blockDim.x) {
    int i, j, k, gi, gj, gk;
    subcell_ijk(S, ch.y + l, i, j, k);
    ghost_of(S, i, j, k, gi, gj, gk);
    // the face index: the boundary node plane
    int fi_ = i, fj_ = j, fk_ = k;
    if (f == 4) fi_ = B.nx; else if (f == 5) fj_ = B.ny; else if (f == 6) fk_ = B.nz;
    long long fq = fix_(B, fi_, fj_, fk_);
    long long c1 = bix(B, i, j, k), c2 = bix(B, gi, gj, gk);
    auto pres = [&](long long c) {
      return (gamma - 1.0) * (A.U[4 * tb + c] - (sq(A.U[tb + c]) + sq(A.U[2 * tb + c]) + sq(A.U[3 * tb + c])) / A.U[c]);
    };
    double pw1 = pres(c1), pw2 = pres(c2);
    double Sa = (double)A.Md[(M_SI + d) * tf + fq];
    double Pw = f <= 3 ? -(0.5 * (pw1 + pw2) - p_inf) * Sa : (0.5 * (pw1 + pw2) - p_inf) * Sa;
    double n1 = A.Md[(M_NI1 + 3 * d) * tf + fq], n2 = A.Md[(M_NI2 + 3 * d) * tf + fq], n3 = A.Md[(M_NI3 + 3 * d) * tf + fq];
    // recorded viscous face flux (Surf1..6 = boundary entries of the viscous flux planes)
    double sf1 = 0.0, sf2 = 0.0, sf3 = 0.0;
    if (s.viscous == 1) {
      sf1 = (double)A.Fv[(d * 4 + 0) * tf + fq]; sf2 = (double)A.Fv[(d * 4 + 1) * tf + fq]; sf3 = (double)A.Fv[(d * 4 + 2) * tf + fq];
    }
    double xc = (A.xc[c1] + A.xc[c2]) * 0.5 - s.cen[0], yc = (A.yc[c1] + A.yc[c2]) * 0.5 - s.cen[1], zc = (A.zc[c1] + A.zc[c2]) * 0.5 - s.cen[2];
    acc[0] += Pw * n1; acc[1] += Pw * n2; acc[2] += Pw * n3;
    double fx0, fy0, fz0;
    if (f <= 3) { acc[3] += sf1; acc[4] += sf2; acc[5] += sf3; fx0 = Pw * n1 + sf1; fy0 = Pw * n2 + sf2; fz0 = Pw * n3 + sf3; }
    else { acc[3] -= sf1; acc[4] -= sf2; acc[5] -= sf3; fx0 = Pw * n1 - sf1; fy0 = Pw * n2 - sf2; fz0 = Pw * n3 - sf3; }
    // moments about the centroid
    acc[6] += (yc * fz0 - zc * fy0);
    acc[7] += (zc * fx0 - xc * fz0);
    acc[8] += (xc * fy0 - yc * fx0);
  }
  for (int q = 0; q < 9; q++) sh[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int q = 0; q < 9; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 9) part[(long long)blockIdx.x * 9 + threadIdx.x] = sh[threadIdx.x][0];
}

// freestream everywhere (init_flow_zero, sub_init.f90:324-357)
template <class T, int NV>
__global__ void k_init_flow(Arena<T> A) {
  const long long tb = A.tot_box;
  OCFD_GRID_STRIDE(g, tb) {
    int b = find_blk_h(A.pre_box, A.hint_box, A.nblk, g);
    if (A.only_solve >= 0 && A.blk[b].solve != A.only_solve) continue;
    const SolveP& s = A.sp[A.blk[b].solve];
    double d0 = 1.0, u0 = s.u_inf, v0 = s.v_inf, w0 = s.w_inf, p0 = 1.0 / (s.gamma * s.ma * s.ma);
    A.U[g] = d0; A.U[tb + g] = d0 * u0; A.U[2 * tb + g] = d0 * v0; A.U[3 * tb + g] = d0 * w0;
    A.U[4 * tb + g] = p0 / (s.gamma - 1.0) + 0.5 * d0 * (u0 * u0 + v0 * v0 + w0 * w0);
    if (NV == 6) A.U[5 * tb + g] = 5.0;
    if (NV == 7) { A.U[5 * tb + g] = 10.0 * s.kt_inf; A.U[6 * tb + g] = s.wt_inf; }
  }
}

}  // namespace ocfd
