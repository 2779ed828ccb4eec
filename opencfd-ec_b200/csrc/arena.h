// Device data layout shared by the host orchestration (capi.cu) and the kernels.
//
// All blocks of all solves of a handle live in one set of arrays ("arena"), one cudaMalloc per
// array, structure-of-arrays and variable-major: variable m of a box array is the plane
// A + m*tot_box.  Each block owns a contiguous range of every index space:
//   box  : cells 1-LAP..n+LAP-1 in each direction (nx+7)(ny+7)(nz+7), i fastest
//   face : face / node-indexed metrics 1..nx x 1..ny x 1..nz
//   node : node coordinates with one ghost layer 0..nx+1 x 0..ny+1 x 0..nz+1
//   cell : interior cells 1..nx-1 x 1..ny-1 x 1..nz-1 (Res, DU, dt, Lc, Lv, vol, ...)
#pragma once
#include <cstdint>
#include <vector_types.h>

namespace ocfd {

struct BlkD {
  int nx, ny, nz;     // nodes
  int NX, NY, NZ;     // box extents nx+7, ny+7, nz+7
  int NXn, NYn, NZn;  // node box extents nx+2 ...
  int solve;          // owning solve
  long long obox, oface, onode, ocell;  // offsets into each index space
  long long obci, obcj, obck;           // offsets of the physical-boundary flag arrays
  long long ocol;                        // offset in the (j,k) column space used by LU-SGS
  int sub0, nsub;                        // subface table range
  // cells whose primitives a residual reads: 1-glo[d] .. n-1+ghi[d] in direction d (glo/ghi = 4,
  // all LAP ghost layers, on a face with an interface cell; else the reach of the boundary scheme,
  // at least 1), RX x RY x RZ cells from offset oreg of that index space; and the 0..n layer
  // ((nx+1)(ny+1)(nz+1) cells) from offset or1
  int glo[3], ghi[3];
  int RX, RY, RZ;
  long long oreg, or1;
  int tdim[3];  // cells per residual tile in i, j, k (the last tile of a direction may be shorter)
};

// One subface of the .inc table (sub_IO.f90:700-705), 0-based block numbers.
struct SubD {
  int blk;
  int ib, ie, jb, je, kb, ke, bc, face, f_no;
  int ib1, ie1, jb1, je1, kb1, ke1, nb1, face1, f_no1, L1, L2, L3;
};

// Per-solve constants (set_const_para values + derived), read by every kernel through
// sp[blk.solve].
struct SolveP {
  int nvar, scheme, bound_scheme, flux, recon, turb, viscous, local_dt, dtime_mesh, limit_flow, positivity, time_method;
  double gamma, ma, re, cv, cp, prl, prt, tsb, twall, kt_inf, wt_inf;
  double a_alfa, a_beta, cfl, dt_global, dtmin, dtmax, w_lu, mut_max, p_outlet;
  double ldmin, ldmax, lpmin, lpmax, lumax, lsamax;
  double p00, d_inf, u_inf, v_inf, w_inf, p_inf;
  double cen[3];
};

// metric planes in the face arrays
enum : int {
  M_SI = 0, M_SJ = 1, M_SK = 2,
  M_NI1 = 3, M_NI2, M_NI3, M_NJ1, M_NJ2, M_NJ3, M_NK1, M_NK2, M_NK3,
  M_J1 = 12,  // ix1,iy1,iz1,jx1,jy1,jz1,kx1,ky1,kz1 : 12..20
  M_J2 = 21,  // ..2 family : 21..29
  M_J3 = 30,  // ..3 family : 30..38
  M_J0 = 39,  // cell-centre family : 39..47
  M_TI = 48,  // unit tangent s2 of the i faces (x,y,z) : 48..50 (node diagonal, sub_Residual.f90:251-253)
  M_TJ = 51,  // j faces : 51..53 (sub_Residual.f90:416-418)
  M_TK = 54,  // k faces : 54..56 (sub_Residual.f90:576-578)
  M_COUNT = 57
};
// primitive planes in the box arrays
enum : int { P_D = 0, P_U, P_V, P_W, P_P, P_T, P_C, P_COUNT };

constexpr int HINT_SHIFT = 10;  // 1024 elements per block-hint chunk

template <class T>
struct Arena {
  // layout
  const BlkD* blk;
  int nblk;
  const long long* pre_box;   // nblk+1 prefix sums of box sizes
  // block of element q << HINT_SHIFT of the box, cell and face index spaces (a lookup start for
  // the block of any element: at most a few block starts lie inside one chunk)
  const int *hint_box, *hint_cell, *hint_face;
  const long long* pre_cell;  // nblk+1
  const long long* pre_face;  // nblk+1
  // nblk+1: the primitive region and the 0..n layer (BlkD::oreg / or1) with their block hints; the
  // region's total is read from pre_reg[nblk] on the device, since a reset_solve that changes a
  // solve's boundary scheme changes it without touching a captured step
  const long long *pre_reg, *pre_r1;
  const int *hint_reg, *hint_r1;
  const long long* pre_col;   // nblk+1, (ny-1)(nz-1) columns per block
  const long long* pre_lnj;   // nblk+1, (nx-1)(nz-1) j-lines per block
  const long long* pre_lnk;   // nblk+1, (nx-1)(ny-1) k-lines per block
  const SubD* sub;
  int nsub;
  const long long* pre_subcell;  // nsub+1 prefix sums of face cells per subface (transverse ranges b..e-1)
  const long long* pre_halo;     // nsub+1 prefix sums of halo target cells per inner subface (LAP deep)
  const int4* cchunk;            // norm chunks (blk, first local cell, count, -), in block order
  int ncchunk;
  const int* cspre;              // nsolve+1: chunks of solve q are [cspre[q], cspre[q+1])
  const int* bc_ent;             // boundary work list: subface of each entry, grouped in rounds
  const long long* bc_pre;       // prefix sums of the entries' cells (per round, from 0)
  const int4* wchunk;            // force chunks (subface, first local face cell, count, -)
  int nwchunk;
  const SolveP* sp;
  int nsolve;
  long long tot_box, tot_cell, tot_face, tot_node, tot_col, tot_subcell, tot_halo, tot_lnj, tot_lnk;
  long long tot_r1;
  const int4* tiles;  // residual tiles (block, first cell i, j, k), block by block, i fastest
  int ntile, tile_maxf, tile_maxc;  // largest face count of one direction / cell count of a tile
  int tile_maxb;                     // largest (tile + one layer) box, (ti+2)(tj+2)(tk+2) cells
  // geometry
  const double *x, *y, *z;   // node
  const double* Md;          // 48 FP64 metric planes (face)
  const T* M;                // metric planes in the flux precision (== Md for FP64)
  const double *vold, *dwd;  // cell
  const T *vol, *dtm, *dw;   // cell, flux precision
  const double *xc, *yc, *zc;  // box
  const unsigned char *bci, *bcj, *bck;  // physical-face flags: bit0 lo face, bit1 hi face
  // state
  double* U;   // NV box planes
  double* Un;  // NV box planes (RK3: stage start; dual time: time level n)
  double* Un1;  // NV box planes (dual time: time level n-1)
  const double* sfac;  // dual time: Sfac, Sfac1 of the current residual evaluation
  T* P;        // P_COUNT box planes
  T* mu;       // box
  T* mut;      // box
  T* Kt;       // box (SST)
  T* Wt;       // box (SST)
  T* f1;       // face (SST)
  T* Res;      // NV cell planes
  double* DU;  // NV cell planes (also FP64 limiter scratch after the update)
  T* dt;       // cell
  T* Lc;       // 3 cell planes
  T* Lv;       // 3 cell planes
  T* Fi;       // inviscid face fluxes: plane dir*5+m
  T* Fv;       // viscous face fluxes: plane dir*4+(m-1), m = 1..4 for Res(2..5); boundary entries are Surf1..6
  T* Ft;       // turbulence face fluxes: plane dir*2+q
  int* flags;  // 4 planes of nblk ints: IF_OverLimit, limited-cell count, SA above LSAmax, BC error
  // -1: kernels cover every solve; q >= 0: the initialisation, BC, halo and corner kernels touch
  // only solve q's blocks (a solve of a batch re-initialised while the others keep their state)
  int only_solve;
};

}  // namespace ocfd
