// Setup kernels (run once per case, FP64, compiled with --fmad=false):
//   face areas / unit normals / unit tangents and volumes  (Comput_Goemetric_var, sub_geometry.f90:6-105)
//   cell centres on the 0..n box                            (sub_geometry.f90:93-104)
//   the four families of Jacobian metrics                   (sub_geometry.f90:110-341)
//   the mesh-quality time-step factor dtime_mesh            (check_mesh_quality_onemesh, 361-444)
//   wall distance, brute force over all wall nodes          (comput_wall_dist, sub_comput_dw.f90:43-101)
// The arithmetic follows the reference line by line so the metrics match a CPU FP64 evaluation
// bit for bit (IEEE division and square root are exact-rounded on the GPU as well).
#include <cuda_runtime.h>

#include "arena.h"
#include "setup.h"

namespace ocfd {

#define GS(g, n) for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < (n); g += (long long)gridDim.x * blockDim.x)

__device__ __forceinline__ int sfind(const long long* pre, int n, long long g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ double sq2(double x) { return x * x; }

struct GeoP {
  const BlkD* blk;
  int nblk;
  const long long *pre_face, *pre_cell, *pre_box, *pre_node;
  long long tot_face, tot_cell, tot_box, tot_node;
  const double *x, *y, *z;
  double* M;  // M_COUNT planes of tot_face
  double *Vi, *Vj, *Vk;
  double *vol, *dtm, *dw;
  double *xc, *yc, *zc;
};

__device__ __forceinline__ long long gn(const BlkD& B, int i, int j, int k) {
  return B.onode + (long long)i + (long long)B.NXn * ((long long)j + (long long)B.NYn * (long long)k);
}
__device__ __forceinline__ long long gf(const BlkD& B, int i, int j, int k) {
  return B.oface + (long long)(i - 1) + (long long)B.nx * ((long long)(j - 1) + (long long)B.ny * (long long)(k - 1));
}
__device__ __forceinline__ long long gb(const BlkD& B, int i, int j, int k) {
  return B.obox + (long long)(i + 3) + (long long)B.NX * ((long long)(j + 3) + (long long)B.NY * (long long)(k + 3));
}

__global__ void k_geom_face(GeoP G) {
  const long long tf = G.tot_face;
  GS(g, tf) {
    int b = sfind(G.pre_face, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.oface;
    int i = (int)(l % B.nx) + 1;
    long long t = l / B.nx;
    int j = (int)(t % B.ny) + 1, k = (int)(t / B.ny) + 1;
    const double *x = G.x, *y = G.y, *z = G.z;
    auto X = [&](int a, int c, int e) { return x[gn(B, a, c, e)]; };
    auto Y = [&](int a, int c, int e) { return y[gn(B, a, c, e)]; };
    auto Z = [&](int a, int c, int e) { return z[gn(B, a, c, e)]; };
    double t1x, t1y, t1z, t2x, t2y, t2z, s1x, s1y, s1z, ss, xa, ya, za, t10;
    // i faces
    t1x = X(i, j + 1, k) - X(i, j, k + 1); t1y = Y(i, j + 1, k) - Y(i, j, k + 1); t1z = Z(i, j + 1, k) - Z(i, j, k + 1);
    t2x = X(i, j + 1, k + 1) - X(i, j, k); t2y = Y(i, j + 1, k + 1) - Y(i, j, k); t2z = Z(i, j + 1, k + 1) - Z(i, j, k);
    s1x = t1y * t2z - t1z * t2y; s1y = t1z * t2x - t1x * t2z; s1z = t1x * t2y - t1y * t2x;
    ss = sqrt(s1x * s1x + s1y * s1y + s1z * s1z);
    G.M[M_SI * tf + g] = ss * 0.5;
    if (ss >= 1.e-20) { G.M[M_NI1 * tf + g] = s1x / ss; G.M[M_NI2 * tf + g] = s1y / ss; G.M[M_NI3 * tf + g] = s1z / ss; }
    else { G.M[M_NI1 * tf + g] = 1.0; G.M[M_NI2 * tf + g] = 0.0; G.M[M_NI3 * tf + g] = 0.0; }
    t10 = 1.0 / (sqrt(t1x * t1x + t1y * t1y + t1z * t1z));  // tangent of the flux frame (sub_Residual.f90:251-253)
    G.M[(M_TI + 0) * tf + g] = t1x * t10; G.M[(M_TI + 1) * tf + g] = t1y * t10; G.M[(M_TI + 2) * tf + g] = t1z * t10;
    xa = (X(i, j, k) + X(i, j + 1, k) + X(i, j, k + 1) + X(i, j + 1, k + 1)) * 0.25;
    ya = (Y(i, j, k) + Y(i, j + 1, k) + Y(i, j, k + 1) + Y(i, j + 1, k + 1)) * 0.25;
    za = (Z(i, j, k) + Z(i, j + 1, k) + Z(i, j, k + 1) + Z(i, j + 1, k + 1)) * 0.25;
    G.Vi[g] = (s1x * xa + s1y * ya + s1z * za) * 0.5;
    // j faces
    t1x = X(i + 1, j, k + 1) - X(i, j, k); t1y = Y(i + 1, j, k + 1) - Y(i, j, k); t1z = Z(i + 1, j, k + 1) - Z(i, j, k);
    t2x = X(i + 1, j, k) - X(i, j, k + 1); t2y = Y(i + 1, j, k) - Y(i, j, k + 1); t2z = Z(i + 1, j, k) - Z(i, j, k + 1);
    s1x = t1y * t2z - t1z * t2y; s1y = t1z * t2x - t1x * t2z; s1z = t1x * t2y - t1y * t2x;
    ss = sqrt(s1x * s1x + s1y * s1y + s1z * s1z);
    G.M[M_SJ * tf + g] = ss * 0.5;
    if (ss >= 1.e-20) { G.M[M_NJ1 * tf + g] = s1x / ss; G.M[M_NJ2 * tf + g] = s1y / ss; G.M[M_NJ3 * tf + g] = s1z / ss; }
    else { G.M[M_NJ1 * tf + g] = 1.0; G.M[M_NJ2 * tf + g] = 0.0; G.M[M_NJ3 * tf + g] = 0.0; }
    t10 = 1.0 / (sqrt(t1x * t1x + t1y * t1y + t1z * t1z));  // sub_Residual.f90:416-418
    G.M[(M_TJ + 0) * tf + g] = t1x * t10; G.M[(M_TJ + 1) * tf + g] = t1y * t10; G.M[(M_TJ + 2) * tf + g] = t1z * t10;
    xa = (X(i, j, k) + X(i + 1, j, k) + X(i, j, k + 1) + X(i + 1, j, k + 1)) * 0.25;
    ya = (Y(i, j, k) + Y(i + 1, j, k) + Y(i, j, k + 1) + Y(i + 1, j, k + 1)) * 0.25;
    za = (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j, k + 1) + Z(i + 1, j, k + 1)) * 0.25;
    G.Vj[g] = (s1x * xa + s1y * ya + s1z * za) * 0.5;
    // k faces
    t1x = X(i + 1, j + 1, k) - X(i, j, k); t1y = Y(i + 1, j + 1, k) - Y(i, j, k); t1z = Z(i + 1, j + 1, k) - Z(i, j, k);
    t2x = X(i, j + 1, k) - X(i + 1, j, k); t2y = Y(i, j + 1, k) - Y(i + 1, j, k); t2z = Z(i, j + 1, k) - Z(i + 1, j, k);
    s1x = t1y * t2z - t1z * t2y; s1y = t1z * t2x - t1x * t2z; s1z = t1x * t2y - t1y * t2x;
    ss = sqrt(s1x * s1x + s1y * s1y + s1z * s1z);
    G.M[M_SK * tf + g] = ss * 0.5;
    if (ss >= 1.e-20) { G.M[M_NK1 * tf + g] = s1x / ss; G.M[M_NK2 * tf + g] = s1y / ss; G.M[M_NK3 * tf + g] = s1z / ss; }
    else { G.M[M_NK1 * tf + g] = 1.0; G.M[M_NK2 * tf + g] = 0.0; G.M[M_NK3 * tf + g] = 0.0; }
    t10 = 1.0 / (sqrt(t1x * t1x + t1y * t1y + t1z * t1z));  // sub_Residual.f90:576-578
    G.M[(M_TK + 0) * tf + g] = t1x * t10; G.M[(M_TK + 1) * tf + g] = t1y * t10; G.M[(M_TK + 2) * tf + g] = t1z * t10;
    xa = (X(i, j, k) + X(i + 1, j, k) + X(i, j + 1, k) + X(i + 1, j + 1, k)) * 0.25;
    ya = (Y(i, j, k) + Y(i + 1, j, k) + Y(i, j + 1, k) + Y(i + 1, j + 1, k)) * 0.25;
    za = (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)) * 0.25;
    G.Vk[g] = (s1x * xa + s1y * ya + s1z * za) * 0.5;
  }
}

__global__ void k_geom_vol(GeoP G) {
  GS(g, G.tot_cell) {
    int b = sfind(G.pre_cell, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.ocell;
    int i = (int)(l % (B.nx - 1)) + 1;
    long long t = l / (B.nx - 1);
    int j = (int)(t % (B.ny - 1)) + 1, k = (int)(t / (B.ny - 1)) + 1;
    G.vol[g] = (G.Vi[gf(B, i + 1, j, k)] - G.Vi[gf(B, i, j, k)] + G.Vj[gf(B, i, j + 1, k)] - G.Vj[gf(B, i, j, k)] + G.Vk[gf(B, i, j, k + 1)] -
                G.Vk[gf(B, i, j, k)]) / 3.0;
  }
}

__global__ void k_geom_xc(GeoP G) {
  GS(g, G.tot_box) {
    int b = sfind(G.pre_box, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.obox;
    int i = (int)(l % B.NX) - 3;
    long long t = l / B.NX;
    int j = (int)(t % B.NY) - 3, k = (int)(t / B.NY) - 3;
    if (i < 0 || i > B.nx || j < 0 || j > B.ny || k < 0 || k > B.nz) { G.xc[g] = 0.0; G.yc[g] = 0.0; G.zc[g] = 0.0; continue; }
    const double* c3[3] = {G.x, G.y, G.z};
    double* o3[3] = {G.xc, G.yc, G.zc};
    for (int q = 0; q < 3; q++) {
      const double* x = c3[q];
      o3[q][g] = (x[gn(B, i, j, k)] + x[gn(B, i, j + 1, k)] + x[gn(B, i, j, k + 1)] + x[gn(B, i, j + 1, k + 1)] + x[gn(B, i + 1, j, k)] +
                  x[gn(B, i + 1, j + 1, k)] + x[gn(B, i + 1, j, k + 1)] + x[gn(B, i + 1, j + 1, k + 1)]) * 0.125;
    }
  }
}

__device__ __forceinline__ void jac9(double xi, double yi, double zi, double xj, double yj, double zj, double xk, double yk, double zk, double* M,
                                     long long tf, long long g, int base) {
  double Jac1 = xi * yj * zk + yi * zj * xk + zi * xj * yk - xi * zj * yk - yi * xj * zk - zi * yj * xk;
  if (fabs(Jac1) < 1.e-20) Jac1 = 1.e-20;
  double Jac = 1.0 / Jac1;
  M[(base + 0) * tf + g] = Jac * (yj * zk - zj * yk);
  M[(base + 1) * tf + g] = Jac * (zj * xk - xj * zk);
  M[(base + 2) * tf + g] = Jac * (xj * yk - yj * xk);
  M[(base + 3) * tf + g] = Jac * (yk * zi - zk * yi);
  M[(base + 4) * tf + g] = Jac * (zk * xi - xk * zi);
  M[(base + 5) * tf + g] = Jac * (xk * yi - yk * xi);
  M[(base + 6) * tf + g] = Jac * (yi * zj - zi * yj);
  M[(base + 7) * tf + g] = Jac * (zi * xj - xi * zj);
  M[(base + 8) * tf + g] = Jac * (xi * yj - yi * xj);
}

// FAM 1: (I-1/2,J,K), 2: (I,J-1/2,K), 3: (I,J,K-1/2), 0: cell centres
template <int FAM>
__global__ void k_geom_jac(GeoP G) {
  const long long tf = G.tot_face;
  GS(g, tf) {
    int b = sfind(G.pre_face, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.oface;
    int i = (int)(l % B.nx) + 1;
    long long t = l / B.nx;
    int j = (int)(t % B.ny) + 1, k = (int)(t / B.ny) + 1;
    int nx = B.nx, ny = B.ny, nz = B.nz;
    if (FAM == 1 && (j > ny - 1 || k > nz - 1)) continue;
    if (FAM == 2 && (i > nx - 1 || k > nz - 1)) continue;
    if (FAM == 3 && (i > nx - 1 || j > ny - 1)) continue;
    if (FAM == 0 && (i > nx - 1 || j > ny - 1 || k > nz - 1)) continue;
    auto xc = [&](int a, int c, int e) { return G.xc[gb(B, a, c, e)]; };
    auto yc = [&](int a, int c, int e) { return G.yc[gb(B, a, c, e)]; };
    auto zc = [&](int a, int c, int e) { return G.zc[gb(B, a, c, e)]; };
    double xi, yi, zi, xj, yj, zj, xk, yk, zk;
    if (FAM == 1) {
      xi = xc(i, j, k) - xc(i - 1, j, k); yi = yc(i, j, k) - yc(i - 1, j, k); zi = zc(i, j, k) - zc(i - 1, j, k);
      double xj1, yj1, zj1, xj2, yj2, zj2, xk1, yk1, zk1, xk2, yk2, zk2;
      if ((i == 1 || i == nx) && (j == 1 || j == ny - 1)) {
        xj1 = xc(i, j - 1, k); yj1 = yc(i, j - 1, k); zj1 = zc(i, j - 1, k); xj2 = xc(i, j + 1, k); yj2 = yc(i, j + 1, k); zj2 = zc(i, j + 1, k);
      } else {
        xj1 = 0.5 * (xc(i, j - 1, k) + xc(i - 1, j - 1, k)); yj1 = 0.5 * (yc(i, j - 1, k) + yc(i - 1, j - 1, k)); zj1 = 0.5 * (zc(i, j - 1, k) + zc(i - 1, j - 1, k));
        xj2 = 0.5 * (xc(i, j + 1, k) + xc(i - 1, j + 1, k)); yj2 = 0.5 * (yc(i, j + 1, k) + yc(i - 1, j + 1, k)); zj2 = 0.5 * (zc(i, j + 1, k) + zc(i - 1, j + 1, k));
      }
      if ((i == 1 || i == nx) && (k == 1 || k == nz - 1)) {
        xk1 = xc(i, j, k - 1); yk1 = yc(i, j, k - 1); zk1 = zc(i, j, k - 1); xk2 = xc(i, j, k + 1); yk2 = yc(i, j, k + 1); zk2 = zc(i, j, k + 1);
      } else {
        xk1 = 0.5 * (xc(i, j, k - 1) + xc(i - 1, j, k - 1)); yk1 = 0.5 * (yc(i, j, k - 1) + yc(i - 1, j, k - 1)); zk1 = 0.5 * (zc(i, j, k - 1) + zc(i - 1, j, k - 1));
        xk2 = 0.5 * (xc(i, j, k + 1) + xc(i - 1, j, k + 1)); yk2 = 0.5 * (yc(i, j, k + 1) + yc(i - 1, j, k + 1)); zk2 = 0.5 * (zc(i, j, k + 1) + zc(i - 1, j, k + 1));
      }
      xj = 0.5 * (xj2 - xj1); yj = 0.5 * (yj2 - yj1); zj = 0.5 * (zj2 - zj1);
      xk = 0.5 * (xk2 - xk1); yk = 0.5 * (yk2 - yk1); zk = 0.5 * (zk2 - zk1);
      jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, G.M, tf, g, M_J1);
    } else if (FAM == 2) {
      xj = xc(i, j, k) - xc(i, j - 1, k); yj = yc(i, j, k) - yc(i, j - 1, k); zj = zc(i, j, k) - zc(i, j - 1, k);
      double xi1, yi1, zi1, xi2, yi2, zi2, xk1, yk1, zk1, xk2, yk2, zk2;
      if ((j == 1 || j == ny) && (i == 1 || i == nx - 1)) {
        xi1 = xc(i - 1, j, k); yi1 = yc(i - 1, j, k); zi1 = zc(i - 1, j, k); xi2 = xc(i + 1, j, k); yi2 = yc(i + 1, j, k); zi2 = zc(i + 1, j, k);
      } else {
        xi1 = 0.5 * (xc(i - 1, j, k) + xc(i - 1, j - 1, k)); yi1 = 0.5 * (yc(i - 1, j, k) + yc(i - 1, j - 1, k)); zi1 = 0.5 * (zc(i - 1, j, k) + zc(i - 1, j - 1, k));
        xi2 = 0.5 * (xc(i + 1, j, k) + xc(i + 1, j - 1, k)); yi2 = 0.5 * (yc(i + 1, j, k) + yc(i + 1, j - 1, k)); zi2 = 0.5 * (zc(i + 1, j, k) + zc(i + 1, j - 1, k));
      }
      if ((j == 1 || j == ny) && (k == 1 || k == nz - 1)) {
        xk1 = xc(i, j, k - 1); yk1 = yc(i, j, k - 1); zk1 = zc(i, j, k - 1); xk2 = xc(i, j, k + 1); yk2 = yc(i, j, k + 1); zk2 = zc(i, j, k + 1);
      } else {
        xk1 = 0.5 * (xc(i, j, k - 1) + xc(i, j - 1, k - 1)); yk1 = 0.5 * (yc(i, j, k - 1) + yc(i, j - 1, k - 1)); zk1 = 0.5 * (zc(i, j, k - 1) + zc(i, j - 1, k - 1));
        xk2 = 0.5 * (xc(i, j, k + 1) + xc(i, j - 1, k + 1)); yk2 = 0.5 * (yc(i, j, k + 1) + yc(i, j - 1, k + 1)); zk2 = 0.5 * (zc(i, j, k + 1) + zc(i, j - 1, k + 1));
      }
      xi = 0.5 * (xi2 - xi1); yi = 0.5 * (yi2 - yi1); zi = 0.5 * (zi2 - zi1);
      xk = 0.5 * (xk2 - xk1); yk = 0.5 * (yk2 - yk1); zk = 0.5 * (zk2 - zk1);
      jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, G.M, tf, g, M_J2);
    } else if (FAM == 3) {
      xk = xc(i, j, k) - xc(i, j, k - 1); yk = yc(i, j, k) - yc(i, j, k - 1); zk = zc(i, j, k) - zc(i, j, k - 1);
      double xi1, yi1, zi1, xi2, yi2, zi2, xj1, yj1, zj1, xj2, yj2, zj2;
      if ((k == 1 || k == nz) && (i == 1 || i == nx - 1)) {
        xi1 = xc(i - 1, j, k); yi1 = yc(i - 1, j, k); zi1 = zc(i - 1, j, k); xi2 = xc(i + 1, j, k); yi2 = yc(i + 1, j, k); zi2 = zc(i + 1, j, k);
      } else {
        xi1 = 0.5 * (xc(i - 1, j, k) + xc(i - 1, j, k - 1)); yi1 = 0.5 * (yc(i - 1, j, k) + yc(i - 1, j, k - 1)); zi1 = 0.5 * (zc(i - 1, j, k) + zc(i - 1, j, k - 1));
        xi2 = 0.5 * (xc(i + 1, j, k) + xc(i + 1, j, k - 1)); yi2 = 0.5 * (yc(i + 1, j, k) + yc(i + 1, j, k - 1)); zi2 = 0.5 * (zc(i + 1, j, k) + zc(i + 1, j, k - 1));
      }
      if ((k == 1 || k == nz) && (j == 1 || j == ny - 1)) {
        xj1 = xc(i, j - 1, k); yj1 = yc(i, j - 1, k); zj1 = zc(i, j - 1, k); xj2 = xc(i, j + 1, k); yj2 = yc(i, j + 1, k); zj2 = zc(i, j + 1, k);
      } else {
        xj1 = 0.5 * (xc(i, j - 1, k) + xc(i, j - 1, k - 1)); yj1 = 0.5 * (yc(i, j - 1, k) + yc(i, j - 1, k - 1)); zj1 = 0.5 * (zc(i, j - 1, k) + zc(i, j - 1, k - 1));
        xj2 = 0.5 * (xc(i, j + 1, k) + xc(i, j + 1, k - 1)); yj2 = 0.5 * (yc(i, j + 1, k) + yc(i, j + 1, k - 1)); zj2 = 0.5 * (zc(i, j + 1, k) + zc(i, j + 1, k - 1));
      }
      xi = 0.5 * (xi2 - xi1); yi = 0.5 * (yi2 - yi1); zi = 0.5 * (zi2 - zi1);
      xj = 0.5 * (xj2 - xj1); yj = 0.5 * (yj2 - yj1); zj = 0.5 * (zj2 - zj1);
      jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, G.M, tf, g, M_J3);
    } else {
      xi = xc(i + 1, j, k) - xc(i - 1, j, k); yi = yc(i + 1, j, k) - yc(i - 1, j, k); zi = zc(i + 1, j, k) - zc(i - 1, j, k);
      xj = xc(i, j + 1, k) - xc(i, j - 1, k); yj = yc(i, j + 1, k) - yc(i, j - 1, k); zj = zc(i, j + 1, k) - zc(i, j - 1, k);
      xk = xc(i, j, k + 1) - xc(i, j, k - 1); yk = yc(i, j, k + 1) - yc(i, j, k - 1); zk = zc(i, j, k + 1) - zc(i, j, k - 1);
      jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, G.M, tf, g, M_J0);
    }
  }
}

__global__ void k_mesh_quality(GeoP G) {
  GS(g, G.tot_cell) {
    int b = sfind(G.pre_cell, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.ocell;
    int i = (int)(l % (B.nx - 1)) + 1;
    long long t = l / (B.nx - 1);
    int j = (int)(t % (B.ny - 1)) + 1, k = (int)(t / (B.ny - 1)) + 1;
    auto xc = [&](int a, int c, int e) { return G.xc[gb(B, a, c, e)]; };
    auto yc = [&](int a, int c, int e) { return G.yc[gb(B, a, c, e)]; };
    auto zc = [&](int a, int c, int e) { return G.zc[gb(B, a, c, e)]; };
    double fl1 = sqrt(sq2(xc(i, j, k) - xc(i - 1, j, k)) + sq2(yc(i, j, k) - yc(i - 1, j, k)) + sq2(zc(i, j, k) - zc(i - 1, j, k))) /
                 sqrt(sq2(xc(i, j, k) - xc(i + 1, j, k)) + sq2(yc(i, j, k) - yc(i + 1, j, k)) + sq2(zc(i, j, k) - zc(i + 1, j, k)));
    double fl2 = sqrt(sq2(xc(i, j, k) - xc(i, j - 1, k)) + sq2(yc(i, j, k) - yc(i, j - 1, k)) + sq2(zc(i, j, k) - zc(i, j - 1, k))) /
                 sqrt(sq2(xc(i, j, k) - xc(i, j + 1, k)) + sq2(yc(i, j, k) - yc(i, j + 1, k)) + sq2(zc(i, j, k) - zc(i, j + 1, k)));
    double fl3 = sqrt(sq2(xc(i, j, k) - xc(i, j, k - 1)) + sq2(yc(i, j, k) - yc(i, j, k - 1)) + sq2(zc(i, j, k) - zc(i, j, k - 1))) /
                 sqrt(sq2(xc(i, j, k) - xc(i, j, k + 1)) + sq2(yc(i, j, k) - yc(i, j, k + 1)) + sq2(zc(i, j, k) - zc(i, j, k + 1)));
    if (fl1 < 1.0) fl1 = 1.0 / fl1;
    if (fl2 < 1.0) fl2 = 1.0 / fl2;
    if (fl3 < 1.0) fl3 = 1.0 / fl3;
    double fl = (fl1 < fl2) ? fl2 : fl1;  // max(max(fl1,fl2),fl3) with std::max semantics
    fl = (fl < fl3) ? fl3 : fl;
    double x1, x2, y1, y2, z1, z2, ft1, ft2, ft3;
    x1 = xc(i, j, k) - xc(i - 1, j, k); x2 = xc(i + 1, j, k) - xc(i, j, k);
    y1 = yc(i, j, k) - yc(i - 1, j, k); y2 = yc(i + 1, j, k) - yc(i, j, k);
    z1 = zc(i, j, k) - zc(i - 1, j, k); z2 = zc(i + 1, j, k) - zc(i, j, k);
    ft1 = (x1 * x2 + y1 * y2 + z1 * z2) / sqrt((x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2));
    x1 = xc(i, j, k) - xc(i, j - 1, k); x2 = xc(i, j + 1, k) - xc(i, j, k);
    y1 = yc(i, j, k) - yc(i, j - 1, k); y2 = yc(i, j + 1, k) - yc(i, j, k);
    z1 = zc(i, j, k) - zc(i, j - 1, k); z2 = zc(i, j + 1, k) - zc(i, j, k);
    ft2 = (x1 * x2 + y1 * y2 + z1 * z2) / sqrt((x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2));
    x1 = xc(i, j, k) - xc(i, j, k - 1); x2 = xc(i, j, k + 1) - xc(i, j, k);
    y1 = yc(i, j, k) - yc(i, j, k - 1); y2 = yc(i, j, k + 1) - yc(i, j, k);
    z1 = zc(i, j, k) - zc(i, j, k - 1); z2 = zc(i, j, k + 1) - zc(i, j, k);
    ft3 = (x1 * x2 + y1 * y2 + z1 * z2) / sqrt((x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2));
    double fmn = (ft2 < ft1) ? ft2 : ft1;  // min(min(ft1,ft2),ft3) with std::min semantics
    fmn = (ft3 < fmn) ? ft3 : fmn;
    double ft = (1.0 * fmn < 1.0) ? 1.0 * fmn : 1.0;
    ft = acos(ft);
    double Af = 0.9 * exp(-4.0 * sq2(fl - 1.0)) + 0.1;
    double Aa = 0.9 * exp(-sq2(4.0 / 3.1415926535 * ft)) + 0.1;
    G.dtm[g] = (Aa < Af) ? Aa : Af;
  }
}

// wall distance (comput_wall_dist, sub_comput_dw.f90:43-101): for every node the minimum of
// sqrt(dx^2+dy^2+dz^2) over the wall nodes of its own solve, initial value 1e8.  The search is
// pruned by the chunks' bounding boxes: a first pass bounds the minimum from above by the
// farthest-corner distance of every box, the second evaluates only boxes whose nearest-point
// distance can reach that bound.  The minimum is taken over squared distances and rooted once:
// sqrt is monotone and correctly rounded, so this equals the minimum of the rooted values.
__global__ void k_wall_dist_nodes(GeoP G, const double* Xw, const WallChunk* ch, const int* wcpre, double* dis) {
  GS(g, G.tot_face) {
    int b = sfind(G.pre_face, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.oface;
    int i = (int)(l % B.nx) + 1;
    long long t = l / B.nx;
    int j = (int)(t % B.ny) + 1, k = (int)(t / B.ny) + 1;
    long long q = gn(B, i, j, k);
    const double px = G.x[q], py = G.y[q], pz = G.z[q];
    const int c0 = wcpre[B.solve], c1 = wcpre[B.solve + 1];
    double ub = 1.0e300;
    for (int c = c0; c < c1; c++) {
      const WallChunk& C = ch[c];
      double fx = fmax(fabs(px - C.lo[0]), fabs(px - C.hi[0]));
      double fy = fmax(fabs(py - C.lo[1]), fabs(py - C.hi[1]));
      double fz = fmax(fabs(pz - C.lo[2]), fabs(pz - C.hi[2]));
      ub = fmin(ub, fx * fx + fy * fy + fz * fz);
    }
    ub = ub * (1.0 + 1.0e-12);
    double best = 1.0e300;
    for (int c = c0; c < c1; c++) {
      const WallChunk& C = ch[c];
      double ex = fmax(fmax(C.lo[0] - px, px - C.hi[0]), 0.0);
      double ey = fmax(fmax(C.lo[1] - py, py - C.hi[1]), 0.0);
      double ez = fmax(fmax(C.lo[2] - pz, pz - C.hi[2]), 0.0);
      double lb = (ex * ex + ey * ey + ez * ez) * (1.0 - 1.0e-12);
      if (lb > ub || lb > best) continue;
      for (long long w = C.w0; w < C.w1; w++) {
        double d2 = sq2(px - Xw[3 * w]) + sq2(py - Xw[3 * w + 1]) + sq2(pz - Xw[3 * w + 2]);
        if (d2 < best) best = d2;
      }
    }
    double dmin = 1.e8;
    if (best < 1.0e300) {
      double d1 = sqrt(best);
      if (d1 < dmin) dmin = d1;
    }
    dis[g] = dmin;
  }
}
__global__ void k_wall_dist_cells(GeoP G, const double* dis) {
  GS(g, G.tot_cell) {
    int b = sfind(G.pre_cell, G.nblk, g);
    const BlkD& B = G.blk[b];
    long long l = g - B.ocell;
    int i = (int)(l % (B.nx - 1)) + 1;
    long long t = l / (B.nx - 1);
    int j = (int)(t % (B.ny - 1)) + 1, k = (int)(t / (B.ny - 1)) + 1;
    G.dw[g] = (dis[gf(B, i, j, k)] + dis[gf(B, i, j + 1, k)] + dis[gf(B, i, j, k + 1)] + dis[gf(B, i, j + 1, k + 1)] + dis[gf(B, i + 1, j, k)] +
               dis[gf(B, i + 1, j + 1, k)] + dis[gf(B, i + 1, j, k + 1)] + dis[gf(B, i + 1, j + 1, k + 1)]) * 0.125;
  }
}

template <class F>
__global__ void k_convert(const double* src, F* dst, long long n) {
  GS(g, n) dst[g] = (F)src[g];
}

static int grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t run_geometry(const GeoArgs& a, cudaStream_t st) {
  GeoP G;
  G.blk = a.blk; G.nblk = a.nblk;
  G.pre_face = a.pre_face; G.pre_cell = a.pre_cell; G.pre_box = a.pre_box; G.pre_node = nullptr;
  G.tot_face = a.tot_face; G.tot_cell = a.tot_cell; G.tot_box = a.tot_box; G.tot_node = a.tot_node;
  G.x = a.x; G.y = a.y; G.z = a.z;
  G.M = a.M; G.Vi = a.scratch; G.Vj = a.scratch + a.tot_face; G.Vk = a.scratch + 2 * a.tot_face;
  G.vol = a.vol; G.dtm = a.dtm; G.dw = a.dw; G.xc = a.xc; G.yc = a.yc; G.zc = a.zc;
  k_geom_face<<<grid_for(a.tot_face), 256, 0, st>>>(G);
  k_geom_vol<<<grid_for(a.tot_cell), 256, 0, st>>>(G);
  k_geom_xc<<<grid_for(a.tot_box), 256, 0, st>>>(G);
  k_geom_jac<1><<<grid_for(a.tot_face), 256, 0, st>>>(G);
  k_geom_jac<2><<<grid_for(a.tot_face), 256, 0, st>>>(G);
  k_geom_jac<3><<<grid_for(a.tot_face), 256, 0, st>>>(G);
  k_geom_jac<0><<<grid_for(a.tot_face), 256, 0, st>>>(G);
  k_mesh_quality<<<grid_for(a.tot_cell), 256, 0, st>>>(G);
  if (a.Xw) {  // set whenever distances are computed here, also without wall nodes (all 1e8 then)
    k_wall_dist_nodes<<<grid_for(a.tot_face), 128, 0, st>>>(G, a.Xw, a.wch, a.wcpre, a.scratch);
    k_wall_dist_cells<<<grid_for(a.tot_cell), 256, 0, st>>>(G, a.scratch);
  }
  return cudaGetLastError();
}

cudaError_t convert_to_float(const double* src, float* dst, long long n, cudaStream_t st) {
  k_convert<float><<<grid_for(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

}  // namespace ocfd
