// LU-SGS sweeps (du_LU_SGS, sub_LU_SGS.f90:4-129) as one persistent pipelined-wavefront kernel
// per sweep instead of one launch per hyperplane.
//
// The lower sweep needs DU(i-1,j,k), DU(i,j-1,k), DU(i,j,k-1) before DU(i,j,k); any order that
// respects these dependencies gives bitwise the same DU as the reference's i+j+k = plane order,
// because every cell evaluates the same expression from the same operands.
//
// Each block is cut into tiles of TJ x TK (j,k) columns.  A CTA of TJ*TK threads owns one tile
// and marches along i with a skew: at local step t, thread (lj,lk) updates i = t - lj - lk.
// Everything a cell's neighbours need from it (U, DU, the spectral radii of the shared face) is
// handed over through shared memory or registers, so every cell's data is read from HBM once per
// sweep, and the data of the next step is prefetched into registers while the current step's
// dependent chain runs.  Across tile boundaries the neighbour tile publishes the number of steps
// it has completed (st.release.gpu after a CTA barrier); the consumer waits (ld.acquire.gpu,
// bounded spin) until the producer is far enough ahead and then reads the values through L2.
//
// Deadlock freedom: CTAs take tiles from a global counter in topological order (J+K ascending
// for the lower sweep, descending for the upper), so every producer of a tile was handed out
// earlier to a CTA that is already running and that itself depends only on earlier tiles.  Every
// wait is bounded; a timeout sets an error flag and the CTA finishes its tile without waiting
// (the host reports OCFD_ERR_TIMEOUT).
#pragma once
#include <type_traits>

#include "solver.cuh"

namespace ocfd {

struct LuTile {
  int blk, j0, k0, pad;  // first column (1-based j, k) of the tile
};

struct LuArgs {
  const LuTile* tiles;  // lower-sweep order: J+K ascending, the longer tiles first within a level
  const LuTile* rtiles; // upper-sweep order: J+K descending, the longer tiles first within a level
  const LuTile* utiles; // the upper sweep's order when both sweeps share one launch (k_lusgs_wave4_ul)
  int ntiles;
  int* counter;         // [0] lower, [1] upper tile counters
  int* progress;        // per tile: steps completed in the current sweep
  int* progress_up;     // k_lusgs_wave4_ul: the upper sweep's progress
  int* blkdone;         // k_lusgs_wave4_ul: per block, lower tiles finished
  int* tile_of;         // per block: first tile index, tiles per row (nJ), tiles per column (nK)
  int* err;             // timeout flag
  int TJ, TK;
  long long spin_limit;
};

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// wait until *p >= need; returns false on timeout
__device__ __forceinline__ bool wait_ge(const int* p, int need, long long limit, int& seen) {
  long long it = 0;
  int v;
  while ((v = ld_acquire(p)) < need) {
    if (++it > limit) { seen = v; return false; }
    if (it > 32) __nanosleep(32);
  }
  seen = v;
  return true;
}

// data of one cell that the sweep reads from HBM
template <int NV>
struct LuCell {
  double U[NV];    // conserved state (U6/U7 clamped as limit_vt leaves them)
  double R[NV];    // lower sweep: Res; upper sweep: DU* of the lower sweep
  double Lc[3], Lv[3];
  double a0;       // vol/dt + w (Lci+Lcj+Lck)
  double n[3][3];  // unit normals of the faces shared with the three upstream neighbours
  double S[3];     // their areas
};

template <class T, int NV, bool UPPER>
__device__ __forceinline__ void lu_load(const Arena<T>& A, const BlkD& B, int i, int j, int k, double w, LuCell<NV>& c) {
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  const long long ci = cix(B, i, j, k), bi = bix(B, i, j, k);
#pragma unroll
  for (int m = 0; m < NV; m++) {
    double u = A.U[m * tb + bi];
    c.U[m] = m >= 5 ? clamp0(u) : u;
    c.R[m] = UPPER ? A.DU[m * tc + ci] : (double)A.Res[m * tc + ci];
  }
#pragma unroll
  for (int d = 0; d < 3; d++) { c.Lc[d] = A.Lc[d * tc + ci]; c.Lv[d] = A.Lv[d * tc + ci]; }
  c.a0 = (double)A.vold[ci] / (double)A.dt[ci] + w * (c.Lc[0] + c.Lc[1] + c.Lc[2]);
  const long long f = fix_(B, i, j, k);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    // normal of the cell's lower face in direction d; the area of the lower face (lower sweep)
    // or of the upper face (upper sweep, the reference pairs n(i) with S(i+1), sub_LU_SGS.f90:96-97)
    c.n[d][0] = A.M[(M_NI1 + 3 * d) * tf + f];
    c.n[d][1] = A.M[(M_NI2 + 3 * d) * tf + f];
    c.n[d][2] = A.M[(M_NI3 + 3 * d) * tf + f];
    long long fs = f;
    if (UPPER) fs = fix_(B, i + (d == 0), j + (d == 1), k + (d == 2));
    c.S[d] = A.M[(M_SI + d) * tf + fs];
  }
}

// what a cell hands to its downstream neighbours in j and k
template <int NV>
struct LuOut {
  double U[NV], DU[NV];
  double Lcj, Lck, Lvj, Lvk;
};

template <class T, int NV, bool UPPER>
__global__ void __launch_bounds__(64) k_lusgs_wave(Arena<T> A, LuArgs L) {
  __shared__ int s_tile;
  __shared__ LuOut<NV> s_out[2][64];
  const long long tb = A.tot_box, tc = A.tot_cell;
  const int TJ = L.TJ, TK = L.TK;
  const int lt = threadIdx.x, lj = lt % TJ, lk = lt / TJ;
  for (;;) {
    if (lt == 0) s_tile = atomicAdd(&L.counter[UPPER ? 1 : 0], 1);
    __syncthreads();
    const int q = s_tile;
    if (q >= L.ntiles) break;
    const LuTile tl = UPPER ? L.rtiles[q] : L.tiles[q];
    const BlkD& B = A.blk[tl.blk];
    const SolveP& s = A.sp[B.solve];
    const int nxm = B.nx - 1, nym = B.ny - 1, nzm = B.nz - 1;
    const int j = UPPER ? (tl.j0 + TJ - 1 - lj) : (tl.j0 + lj);
    const int k = UPPER ? (tl.k0 + TK - 1 - lk) : (tl.k0 + lk);
    const bool active = j >= 1 && j <= nym && k >= 1 && k <= nzm;
    const int* tb3 = L.tile_of + 3 * tl.blk;
    const int first = tb3[0], nJ = tb3[1], nK = tb3[2];
    const int J = (tl.j0 - 1) / TJ, K = (tl.k0 - 1) / TK;
    int pj = -1, pk = -1;
    if (!UPPER) {
      if (J > 0) pj = first + (J - 1) + nJ * K;
      if (K > 0) pk = first + J + nJ * (K - 1);
    } else {
      if (J < nJ - 1) pj = first + (J + 1) + nJ * K;
      if (K < nK - 1) pk = first + J + nJ * (K + 1);
    }
    const int my = first + J + nJ * K;
    const int nsteps = nxm + TJ + TK - 2;
    const double w = s.w_lu, gamma = s.gamma;
    const bool visc = s.viscous == 1;
    const int off = UPPER ? 1 : -1;
    // neighbour columns outside the tile (read through L2 from the producer tile)
    const bool jx = (lj == 0) && (UPPER ? j != nym : j != 1);
    const bool kx = (lk == 0) && (UPPER ? k != nzm : k != 1);
    // the cell of step t is i(t); prefetch the first one
    auto i_of = [&](int t) { int il = t - lj - lk; return UPPER ? (nxm - il) : (il + 1); };
    auto on_at = [&](int t) { int il = t - lj - lk; return active && il >= 0 && il < nxm; };
    LuCell<NV> cur, nxt;
    if (on_at(0)) lu_load<T, NV, UPPER>(A, B, i_of(0), j, k, w, cur);
    double prevU[NV], prevDU[NV], prevLci = 0.0, prevLvi = 0.0;  // the i-upstream cell (this thread's last one)
#pragma unroll
    for (int m = 0; m < NV; m++) { prevU[m] = 0.0; prevDU[m] = 0.0; }
    int seen_j = 0, seen_k = 0;
    for (int t = 0; t < nsteps; t++) {
      const bool on = on_at(t);
      const int i = i_of(t);
      // prefetch the next step's cell while this step's chain runs
      if (on_at(t + 1)) lu_load<T, NV, UPPER>(A, B, i_of(t + 1), j, k, w, nxt);
      if (lt == 0) {
        bool ok = true;
        if (pj >= 0 && seen_j < min(t + TJ, nsteps)) ok &= wait_ge(L.progress + pj, min(t + TJ, nsteps), L.spin_limit, seen_j);
        if (pk >= 0 && seen_k < min(t + TK, nsteps)) ok &= wait_ge(L.progress + pk, min(t + TK, nsteps), L.spin_limit, seen_k);
        if (!ok) atomicExch(L.err, 1);
      }
      __syncthreads();
      LuOut<NV> out;
      if (on) {
        double alfa[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) alfa[m] = cur.a0;
        if (visc) {
          double lv = cur.Lv[0] + cur.Lv[1] + cur.Lv[2];
#pragma unroll
          for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + 2.0 * lv;
          if (NV == 6) {
            if (!UPPER) alfa[5] = alfa[5] + lv;
            else alfa[5] = alfa[5] + cur.Lv[0] + cur.Lv[1] + cur.Lv[2];
          }
        }
        double acc[3][NV];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const bool has = UPPER ? (d == 0 ? i != nxm : (d == 1 ? j != nym : k != nzm)) : (d == 0 ? i != 1 : (d == 1 ? j != 1 : k != 1));
          if (!has) {
#pragma unroll
            for (int m = 0; m < NV; m++) acc[d][m] = 0.0;
            continue;
          }
          double Un[NV], DUn[NV], Lcn, Lvn;
          if (d == 0) {
#pragma unroll
            for (int m = 0; m < NV; m++) { Un[m] = prevU[m]; DUn[m] = prevDU[m]; }
            Lcn = prevLci; Lvn = prevLvi;
          } else if ((d == 1 && !jx) || (d == 2 && !kx)) {
            const LuOut<NV>& o = s_out[(t + 1) & 1][d == 1 ? lt - 1 : lt - TJ];
#pragma unroll
            for (int m = 0; m < NV; m++) { Un[m] = o.U[m]; DUn[m] = o.DU[m]; }
            Lcn = d == 1 ? o.Lcj : o.Lck;
            Lvn = d == 1 ? o.Lvj : o.Lvk;
          } else {
            const int jj = j + (d == 1 ? off : 0), kk = k + (d == 2 ? off : 0);
            const long long cn = cix(B, i, jj, kk), bn = bix(B, i, jj, kk);
#pragma unroll
            for (int m = 0; m < NV; m++) {
              double u = A.U[m * tb + bn];
              Un[m] = m >= 5 ? clamp0(u) : u;
              DUn[m] = __ldcg(A.DU + m * tc + cn);
            }
            Lcn = A.Lc[d * tc + cn];
            Lvn = A.Lv[d * tc + cn];
          }
          double DF[NV];
          comput_DFn(NV, DF, Un, DUn, cur.n[d][0], cur.n[d][1], cur.n[d][2], gamma);
#pragma unroll
          for (int m = 0; m < NV; m++) {
            double v;
            if (!UPPER) v = 0.5 * (DF[m] * cur.S[d] + w * Lcn * DUn[m]);
            else v = -(0.5 * (DF[m] * cur.S[d] - w * Lcn * DUn[m]));
            if (visc) v = v + Lvn * DUn[m];
            acc[d][m] = v;
          }
        }
        const long long c = cix(B, i, j, k);
#pragma unroll
        for (int m = 0; m < NV; m++) {
          double r;
          if (!UPPER) r = (cur.R[m] + acc[0][m] + acc[1][m] + acc[2][m]) / alfa[m];
          else r = cur.R[m] + (acc[0][m] + acc[1][m] + acc[2][m]) / alfa[m];
          A.DU[m * tc + c] = r;
          out.DU[m] = r;
          out.U[m] = cur.U[m];
          prevU[m] = cur.U[m];
          prevDU[m] = r;
        }
        out.Lcj = cur.Lc[1]; out.Lck = cur.Lc[2]; out.Lvj = cur.Lv[1]; out.Lvk = cur.Lv[2];
        prevLci = cur.Lc[0];
        prevLvi = cur.Lv[0];
        s_out[t & 1][lt] = out;
      }
      __syncthreads();
      if (lt == 0) st_release(L.progress + my, t + 1);
      cur = nxt;
    }
    __syncthreads();
  }
}


// ============================================================================================
// Version 3: the work of one column split over four thread groups of TC threads each.
//
//   group d = 0, 1, 2 ("direction threads"): the flux-difference term of the upstream neighbour
//                   in direction d (i, j, k): DF = F(U+DU)n - F(U)n, times S, plus the spectral
//                   radius terms; the old-state half F(U)n is computed a step ahead, so only the
//                   DU-dependent half sits on the dependency chain;
//   group 3       ("owner"): sums Res + the three terms in the reference's order, divides by
//                   the diagonal, writes DU and publishes (DU, p(U+DU)) for the downstream cells.
//
// Per step: barrier B1, direction threads compute their terms into shared memory while owners
// load the next cell; barrier B2, owners finish the cell while direction threads prepare the
// next step (old-state terms from prefetched data) and one thread polls the upstream tiles'
// progress.  Every cell still evaluates the reference expression with the same operands in the
// same order, so the bits equal the hyperplane order.
// ============================================================================================
template <int NV>
struct LuDir {      // direction-thread data of one step (old state only)
  double n1, n2, n3, S;
  double Unb[NV];   // neighbour state, U6/U7 clamped as limit_vt leaves them (cross-tile only)
  double wLc, Lv;   // Lc and Lv of the neighbour in this direction (cross-tile only)
};


__device__ __forceinline__ double ldro(const double* p) { return __ldg(p); }
// CTA-wide barrier on a named barrier (warp-uniform callers; the owner and direction warps
// reach it from different loops, each warp executing the same instruction in all its lanes)
template <int NT>
__device__ __forceinline__ void cta_bar() { asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); }
__device__ __forceinline__ double ldro(const float* p) { return (double)__ldg(p); }

// cp.async (sm_80+) of one 4- or 8-byte value into shared memory, and the group controls: each
// thread waits only for its own copies and reads only the slots it filled itself
__device__ __forceinline__ void cpa(void* dst, const void* src, int bytes) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(dst);
  if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(src) : "memory");
}
template <class X>
__device__ __forceinline__ void cpa(X* dst, const X* src) { cpa((void*)dst, (const void*)src, (int)sizeof(X)); }
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Per-column input data of the sweep, staged through a ring of LU_RING steps in dynamic shared
// memory: step t's loads are issued two steps before the step uses them, so their HBM latency
// overlaps two steps of the dependency chain instead of half a step.
constexpr int LU_RING = 3;
template <class T, int NV, bool UPPER, int TC>
struct LuRing {
  using RT = typename std::conditional<UPPER, double, T>::type;  // R: Res (lower) or DU* (upper)
  double oU[LU_RING][NV][TC];      // owner: the cell's state
  double ovol[LU_RING][TC];
  double dU[LU_RING][3][NV][TC];   // direction threads: the cross-tile neighbour's state
  RT oR[LU_RING][NV][TC];
  T odt[LU_RING][TC];
  T oLc[LU_RING][3][TC], oLv[LU_RING][3][TC];
  T dn[LU_RING][3][4][TC];         // n1, n2, n3 of the face and S (the lower or the upper face)
  T dL[LU_RING][3][2][TC];         // Lc, Lv of the cross-tile neighbour
};

#ifndef OCFD_LU_MINB
#define OCFD_LU_MINB (64 / TC)
#endif
template <class T, int NV, bool UPPER, int TC>
__global__ void __launch_bounds__(4 * TC + 32, OCFD_LU_MINB) k_lusgs_wave3(Arena<T> A, LuArgs L) {
  extern __shared__ __align__(16) unsigned char s_dyn[];
  LuRing<T, NV, UPPER, TC>& R = *reinterpret_cast<LuRing<T, NV, UPPER, TC>*>(s_dyn);
  __shared__ int s_tile;
  __shared__ double s_acc[3][NV][TC];      // direction terms of the current step
  __shared__ double s_pub[NV][TC];         // DU of each column's last cell
  __shared__ double s_diag[2][TC];         // the diagonal of the current step (all variables; the SA variable's)
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  const int TJ = L.TJ, TK = L.TK;
  // thread groups: 0..2 direction threads, 3 owner (TC threads each), 4 the poller warp (lane 0
  // publishes this tile's progress and waits for the upstream tiles')
  constexpr int NT = 4 * TC + 32;
  const int tid = threadIdx.x, grp = tid < 4 * TC ? tid / TC : 4, c = tid % TC;
  const int lj = c % TJ, lk = c / TJ;
  const bool owner = grp == 3;
  const int d = grp;  // direction of a direction thread
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(&L.counter[UPPER ? 1 : 0], 1);
    __syncthreads();
    const int q = s_tile;
    if (q >= L.ntiles) break;
    const LuTile tl = UPPER ? L.rtiles[q] : L.tiles[q];
    const BlkD& B = A.blk[tl.blk];
    const SolveP& s = A.sp[B.solve];
    const int nxm = B.nx - 1, nym = B.ny - 1, nzm = B.nz - 1;
    const int j = UPPER ? (tl.j0 + TJ - 1 - lj) : (tl.j0 + lj);
    const int k = UPPER ? (tl.k0 + TK - 1 - lk) : (tl.k0 + lk);
    const bool active = j >= 1 && j <= nym && k >= 1 && k <= nzm;
    const int* tb3 = L.tile_of + 3 * tl.blk;
    const int first = tb3[0], nJ = tb3[1], nK = tb3[2];
    const int J = (tl.j0 - 1) / TJ, K = (tl.k0 - 1) / TK;
    int pj = -1, pk = -1;
    if (!UPPER) {
      if (J > 0) pj = first + (J - 1) + nJ * K;
      if (K > 0) pk = first + J + nJ * (K - 1);
    } else {
      if (J < nJ - 1) pj = first + (J + 1) + nJ * K;
      if (K < nK - 1) pk = first + J + nJ * (K + 1);
    }
    const int my = first + J + nJ * K;
    const int nsteps = nxm + TJ + TK - 2;
    const double w = s.w_lu, gamma = s.gamma;
    const bool visc = s.viscous == 1;
    const bool dual = s.time_method == -1;
    const double sfac1 = dual ? A.sfac[1] : 0.0;
    const int off = UPPER ? 1 : -1;
    auto i_of = [&](int t) { int il = t - lj - lk; return UPPER ? (nxm - il) : (il + 1); };
    auto on_at = [&](int t) { int il = t - lj - lk; return active && il >= 0 && il < nxm; };
    // does the cell of step t have an upstream neighbour in direction d inside the block?
    auto has_at = [&](int t) {
      const int i = i_of(t);
      return UPPER ? (d == 0 ? i != nxm : (d == 1 ? j != nym : k != nzm)) : (d == 0 ? i != 1 : (d == 1 ? j != 1 : k != 1));
    };
    // a neighbour column in another tile: its DU comes through L2 after the progress wait
    const bool xt = !owner && ((d == 1 && lj == 0) || (d == 2 && lk == 0));
    const int pubcol = d == 0 ? c : (d == 1 ? c - 1 : c - TJ);
    // the column's index bases (cell, box and face spaces; add i) and this thread's upstream
    // neighbour offset in direction d, so a step's indices are additions
    const long long cb = B.ocell - 1 + (long long)nxm * ((j - 1) + (long long)nym * (k - 1));
    const long long bb = B.obox + 3 + (long long)B.NX * ((j + 3) + (long long)B.NY * (k + 3));
    const long long fb = B.oface - 1 + (long long)B.nx * ((j - 1) + (long long)B.ny * (k - 1));
    const long long dcn = d == 0 ? off : (d == 1 ? (long long)off * nxm : (long long)off * nxm * nym);
    const long long dbn = d == 0 ? off : (d == 1 ? (long long)off * B.NX : (long long)off * B.NX * B.NY);
    const long long dfs = !UPPER ? 0 : (d == 0 ? 1 : (d == 1 ? (long long)B.nx : (long long)B.nx * B.ny));

    // step t's face data of direction d (and, across a tile edge, the neighbour's old state) into
    // ring slot t % LU_RING; one commit group per step, empty when the step has nothing to load
    auto issue_dir = [&](int t) {
      if (on_at(t) && has_at(t)) {
        const int sl = t % LU_RING, i = i_of(t);
        const long long f = fb + i;
        cpa(&R.dn[sl][d][0][c], A.M + (M_NI1 + 3 * d) * tf + f);
        cpa(&R.dn[sl][d][1][c], A.M + (M_NI2 + 3 * d) * tf + f);
        cpa(&R.dn[sl][d][2][c], A.M + (M_NI3 + 3 * d) * tf + f);
        // the lower face's area (lower sweep) or the upper face's (upper sweep, sub_LU_SGS.f90:96-97)
        cpa(&R.dn[sl][d][3][c], A.M + (M_SI + d) * tf + f + dfs);
        if (xt) {  // in-tile neighbours publish their old state in shared memory
          const long long bn = bb + i + dbn, cn = cb + i + dcn;
#pragma unroll
          for (int m = 0; m < NV; m++) cpa(&R.dU[sl][d][m][c], A.U + m * tb + bn);
          cpa(&R.dL[sl][d][0][c], A.Lc + d * tc + cn);
          cpa(&R.dL[sl][d][1][c], A.Lv + d * tc + cn);
        }
      }
      cpa_commit();
    };
    auto take_dir = [&](int t, LuDir<NV>& x) {
      const int sl = t % LU_RING;
      x.n1 = (double)R.dn[sl][d][0][c]; x.n2 = (double)R.dn[sl][d][1][c]; x.n3 = (double)R.dn[sl][d][2][c];
      x.S = (double)R.dn[sl][d][3][c];
      if (!xt) return;
#pragma unroll
      for (int m = 0; m < NV; m++) {
        const double u = R.dU[sl][d][m][c];
        x.Unb[m] = m >= 5 ? clamp0(u) : u;
      }
      x.wLc = (double)R.dL[sl][d][0][c];
      x.Lv = (double)R.dL[sl][d][1][c];
    };
    using RT = typename LuRing<T, NV, UPPER, TC>::RT;
    auto issue_own = [&](int t) {
      if (on_at(t)) {
        const int sl = t % LU_RING, i = i_of(t);
        const long long bi = bb + i, ci = cb + i;
#pragma unroll
        for (int m = 0; m < NV; m++) {
          cpa(&R.oU[sl][m][c], A.U + m * tb + bi);
          // upper sweep: R is DU* of the lower sweep, read before this column overwrites it
          if (UPPER) cpa(&R.oR[sl][m][c], (const RT*)(A.DU + m * tc + ci));
          else cpa(&R.oR[sl][m][c], (const RT*)(A.Res + m * tc + ci));
        }
        cpa(&R.ovol[sl][c], A.vold + ci);
        cpa(&R.odt[sl][c], A.dt + ci);
#pragma unroll
        for (int q2 = 0; q2 < 3; q2++) { cpa(&R.oLc[sl][q2][c], A.Lc + q2 * tc + ci); cpa(&R.oLv[sl][q2][c], A.Lv + q2 * tc + ci); }
      }
      cpa_commit();
    };

    // direction thread state for the current step: old-state half of the flux difference.  The
    // flux difference DF = F(U+DU)n - F(U)n is evaluated in the flux precision DFT (FP32 in the
    // mixed form, as the reconstruction and the fluxes; FP64 otherwise); its products with S and
    // the spectral-radius terms, the sum and the division by the diagonal stay FP64.
    using DFT = T;
    DFT un1 = 0, F1[NV], n1 = 0, n2 = 0, n3 = 0, Unb[NV];
    double S = 0.0, wLc = 0.0, Lvn = 0.0;
    bool has = false;
    // comput_DFn's U terms (sub_LU_SGS.f90:135-157) of step t; an in-tile neighbour's old state is
    // read from its owner's ring slot of step t-1 (complete since the owner's wait in step t-1,
    // ordered before this read by barrier B2 of step t-1)
    auto prep_dir = [&](int t, const LuDir<NV>& x) {
      has = on_at(t) && has_at(t);
      if (!has) return;
      n1 = (DFT)x.n1; n2 = (DFT)x.n2; n3 = (DFT)x.n3; S = x.S;
      if (xt) {
        Lvn = x.Lv;
        wLc = w * x.wLc;
#pragma unroll
        for (int m = 0; m < NV; m++) Unb[m] = (DFT)x.Unb[m];
      } else {
        const int pb = (t + LU_RING - 1) % LU_RING;
        Lvn = (double)R.oLv[pb][d][pubcol];
        wLc = w * (double)R.oLc[pb][d][pubcol];
#pragma unroll
        for (int m = 0; m < NV; m++) {
          const double u = R.oU[pb][m][pubcol];
          Unb[m] = (DFT)(m >= 5 ? clamp0(u) : u);
        }
      }
      const DFT g1 = (DFT)(gamma - 1.0), half = (DFT)0.5;
      un1 = (Unb[1] * n1 + Unb[2] * n2 + Unb[3] * n3) / Unb[0];
      const DFT p1 = g1 * (Unb[4] - half * (sq(Unb[1]) + sq(Unb[2]) + sq(Unb[3])) / Unb[0]);
      F1[0] = Unb[0] * un1;
      F1[1] = Unb[1] * un1 + p1 * n1;
      F1[2] = Unb[2] * un1 + p1 * n2;
      F1[3] = Unb[3] * un1 + p1 * n3;
      F1[4] = (Unb[4] + p1) * un1;
#pragma unroll
      for (int m = 5; m < NV; m++) F1[m] = Unb[m] * un1;
    };
    // the diagonal of step t's cell from the owner's ring slot (sub_LU_SGS.f90:50-62, 90-92): the
    // value of every variable, and the SA variable's (its extra Lv term)
    auto diag_own = [&](int t) {
      const int sl = t % LU_RING;
      const double vol = R.ovol[sl][c], dt = (double)R.odt[sl][c];
      const double a0 = vol / dt + w * ((double)R.oLc[sl][0][c] + (double)R.oLc[sl][1][c] + (double)R.oLc[sl][2][c]);
      double al = a0, als = a0;
      if (visc) {
        const double lv0 = R.oLv[sl][0][c], lv1 = R.oLv[sl][1][c], lv2 = R.oLv[sl][2][c];
        const double lv = lv0 + lv1 + lv2;
        al = al + 2.0 * lv;
        als = als + 2.0 * lv;
        if (NV == 6) {  // lower: + (Lv sum); upper: + Lv1 + Lv2 + Lv3 term by term (sub_LU_SGS.f90:60-62, 90-92)
          if (!UPPER) als = als + lv;
          else als = als + lv0 + lv1 + lv2;
        }
      }
      if (dual) {  // dual time: + Sfac1 vol (sub_LU_SGS.f90:39, 92)
        al = al + sfac1 * vol;
        als = als + sfac1 * vol;
      }
      // the mixed form multiplies by the diagonal's FP64 reciprocal (taken here, off the chain);
      // the FP64 form divides as the reference does
      s_diag[0][c] = sizeof(T) == 4 ? 1.0 / al : al;
      s_diag[1][c] = sizeof(T) == 4 ? 1.0 / (NV == 6 ? als : al) : (NV == 6 ? als : al);
    };

    int seen_j = 0, seen_k = 0;
    auto poll = [&](int t) {  // upstream tiles far enough for step t
      bool ok = true;
      if (pj >= 0 && seen_j < min(t + TJ, nsteps)) ok &= wait_ge(L.progress + pj, min(t + TJ, nsteps), L.spin_limit, seen_j);
      if (pk >= 0 && seen_k < min(t + TK, nsteps)) ok &= wait_ge(L.progress + pk, min(t + TK, nsteps), L.spin_limit, seen_k);
      if (!ok) atomicExch(L.err, 1);
    };

    // The owner warps and the direction warps run separate loops (so each keeps only its own
    // registers live); both take the same two CTA barriers per step.
    //   phase A (after B1): direction threads evaluate their flux-difference term (the dependency
    //     chain); the owner prepares the cell's diagonal and R (off the chain) and prefetches.
    //   phase B (after B2): the final divisions are shared: direction thread d computes DU of
    //     variable d, the owner the variables 3..NV-1; direction threads then prepare the next
    //     step's old-state terms, and thread 0 completes the poll of the upstream tiles.
    auto diag_of = [&](int m) { return (NV == 6 && m == 5) ? s_diag[1][c] : s_diag[0][c]; };
    auto finish_val = [&](int m, int t) {  // sub_LU_SGS.f90:63-72 (lower), 108-117 (upper)
      const double rm = (double)R.oR[t % LU_RING][m][c];
      double r;
      if (sizeof(T) == 4) {
        if (!UPPER) r = (rm + s_acc[0][m][c] + s_acc[1][m][c] + s_acc[2][m][c]) * diag_of(m);
        else r = rm + (s_acc[0][m][c] + s_acc[1][m][c] + s_acc[2][m][c]) * diag_of(m);
      } else {
        if (!UPPER) r = (rm + s_acc[0][m][c] + s_acc[1][m][c] + s_acc[2][m][c]) / diag_of(m);
        else r = rm + (s_acc[0][m][c] + s_acc[1][m][c] + s_acc[2][m][c]) / diag_of(m);
      }
      return r;
    };
    auto finish = [&](int m, int t, long long ci) {
      const double r = finish_val(m, t);
      A.DU[m * tc + ci] = r;
      s_pub[m][c] = r;
    };
    if (grp == 4) {
      // poller warp: its flag traffic (release of this tile's progress after B1, acquire of the
      // upstream tiles' progress) never sits on the compute warps' paths
      // waits one step ahead of the compute warps (the upstream tiles run at least one step
      // further ahead than the dependency needs), so the cross-tile DU of step t+1 can be loaded
      // during step t
      if (tid == 4 * TC) { poll(0); if (1 < nsteps) poll(1); }
      cta_bar<NT>();  // B0
      for (int t = 0; t < nsteps; t++) {
        cta_bar<NT>();  // B1
        if (tid == 4 * TC && t > 0) st_release(L.progress + my, t);
        cta_bar<NT>();  // B2
        if (tid == 4 * TC && t + 2 < nsteps) poll(t + 2);
      }
    } else if (owner) {
      issue_own(0);
      issue_own(1);
      cta_bar<NT>();  // B0
      for (int t = 0; t < nsteps; t++) {
        cta_bar<NT>();  // B1
        cpa_wait<1>();  // step t's group (only step t+1's may be outstanding)
        if (on_at(t)) diag_own(t);
        issue_own(t + 2);  // into the slot step t-1 used
        cta_bar<NT>();  // B2: the three direction terms of step t are in shared memory
        if (on_at(t)) {
          const long long ci = cb + i_of(t);
          double r[NV];  // every value before the stores, so the divisions overlap
#pragma unroll
          for (int m = 3; m < NV; m++) r[m] = finish_val(m, t);
#pragma unroll
          for (int m = 3; m < NV; m++) { A.DU[m * tc + ci] = r[m]; s_pub[m][c] = r[m]; }
        }
      }
    } else {
      {
        issue_dir(0);
        cpa_wait<0>();
        LuDir<NV> dn;
        take_dir(0, dn);
        prep_dir(0, dn);
        issue_dir(1);
      }
      double xdu[NV];  // cross-tile neighbour's DU of the current step, loaded one step early
      auto load_xdu = [&](int t) {
        const long long cn = cb + i_of(t) + dcn;
#pragma unroll
        for (int m = 0; m < NV; m++) xdu[m] = __ldcg(A.DU + m * tc + cn);
      };
      cta_bar<NT>();  // B0: the poller's first waits are done
      if (xt && has) load_xdu(0);
      for (int t = 0; t < nsteps; t++) {
        cta_bar<NT>();  // B1: step t-1 finished (DU in s_pub and in HBM), upstream tiles ready
        issue_dir(t + 2);  // into the slot step t-1 used
        if (has) {
          double DUn[NV];
          if (!xt) {
#pragma unroll
            for (int m = 0; m < NV; m++) DUn[m] = s_pub[m][pubcol];
          } else {
#pragma unroll
            for (int m = 0; m < NV; m++) DUn[m] = xdu[m];
          }
          DFT U2[NV];
#pragma unroll
          for (int m = 0; m < NV; m++) U2[m] = (DFT)((double)Unb[m] + DUn[m]);
          const DFT g1 = (DFT)(gamma - 1.0), half = (DFT)0.5;
          const DFT un2 = (U2[1] * n1 + U2[2] * n2 + U2[3] * n3) / U2[0];
          const DFT pp2 = g1 * (U2[4] - half * (sq(U2[1]) + sq(U2[2]) + sq(U2[3])) / U2[0]);
          DFT DF[NV];
          DF[0] = U2[0] * un2 - F1[0];
          DF[1] = (U2[1] * un2 + pp2 * n1) - F1[1];
          DF[2] = (U2[2] * un2 + pp2 * n2) - F1[2];
          DF[3] = (U2[3] * un2 + pp2 * n3) - F1[3];
          DF[4] = (U2[4] + pp2) * un2 - F1[4];
#pragma unroll
          for (int m = 5; m < NV; m++) DF[m] = U2[m] * un2 - F1[m];
#pragma unroll
          for (int m = 0; m < NV; m++) {
            double v;
            if (sizeof(T) == 4) {   // the mixed form: off-diagonal products in FP32, the sum stays FP64
              const float du = (float)DUn[m];
              float x;
              if (!UPPER) x = 0.5f * ((float)DF[m] * (float)S + (float)wLc * du);
              else x = -(0.5f * ((float)DF[m] * (float)S - (float)wLc * du));
              if (visc) x = x + (float)Lvn * du;
              v = (double)x;
            } else {
              if (!UPPER) v = 0.5 * ((double)DF[m] * S + wLc * DUn[m]);
              else v = -(0.5 * ((double)DF[m] * S - wLc * DUn[m]));
              if (visc) v = v + Lvn * DUn[m];
            }
            s_acc[d][m][c] = v;
          }
        } else if (on_at(t)) {
#pragma unroll
          for (int m = 0; m < NV; m++) s_acc[d][m][c] = 0.0;
        }
        cta_bar<NT>();  // B2
        if (on_at(t)) finish(d, t, cb + i_of(t));
        cpa_wait<1>();  // step t+1's group (only step t+2's may be outstanding)
        {
          LuDir<NV> dn;
          take_dir(t + 1, dn);
          prep_dir(t + 1, dn);
        }
        if (xt && has) load_xdu(t + 1);  // ready since the poller's wait of step t-1
      }
    }
    cpa_wait<0>();  // no copy of this tile is still landing when the next tile reuses the ring
    __syncthreads();
    if (tid == 0) st_release(L.progress + my, nsteps);
  }
}

template <class T, int NV, bool UPPER, int TC>
inline size_t lu_wave3_smem() { return sizeof(LuRing<T, NV, UPPER, TC>); }
// the ring lives in dynamic shared memory (above the 48 KB static limit for TC = 64)
template <class T, int NV, bool UPPER, int TC>
inline void lu_wave3_prepare() {
  cudaFuncSetAttribute(k_lusgs_wave3<T, NV, UPPER, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lu_wave3_smem<T, NV, UPPER, TC>());
}

// ============================================================================================
// Version 4: the version-3 wavefront (same tiles, per-cell arithmetic and finish order, so the
// same bits) with its inputs staged by 32-byte sector instead of by element, and its two helper
// tasks (waiting for the upstream tiles, releasing this tile's progress) on two warps that take
// only barrier B1, so neither an acquire poll nor a release fence sits inside a step's phase.
//
// Every input of a column is a plane read along i, one element per step, so each plane is a
// stream: its aligned 32-byte sectors land in two 32-byte slots per column, four 16-byte chunks
// (chunk q = (address >> 4) & 3, so consecutive sectors alternate between the slots), copied by
// two 16-byte cp.async when the march enters a new sector, LU4_D steps before the step that
// first reads it.  A stream then costs one copy pair per 4 (FP64) or 8 (FP32) steps instead of
// one scattered element copy per step: the sweep's global requests fall 2x (FP64) to 4x (FP32),
// each a whole sector.  Measured on config 2: 8 % faster than version 3 at 64-column tiles; the
// sweep stays bound by the latency of a step (dependent FP64 divisions, barriers, and the address
// arithmetic of the streams), not by the load/store path.
//
// Slot lifetime: when step s issues (after barrier B1 of step s) every read of steps < s is done
// (B1 orders it), and the sectors still to be read cover the elements of steps s .. s+LU4_D,
// LU4_D+1 <= 5 consecutive elements: at most two sectors of 8-byte elements.  So an issue never
// lands in a slot that a pending read or an in-flight copy uses.
//
// The arena pads every allocation by 32 bytes, so the sector of an array's last element is in
// bounds.  Bytes of a sector outside the column's own elements are copied and never read.
// ============================================================================================
constexpr int LU4_D = 2;

static_assert(LU4_D >= 1 && LU4_D <= 4, "two sector slots hold LU4_D + 1 <= 5 consecutive FP64 elements");

// named barrier ID over NT threads (warp-uniform callers)
template <int ID, int NT>
__device__ __forceinline__ void cta_bar_id() { asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(NT) : "memory"); }

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(src) : "memory");
}
// the aligned sector holding p into the column's slots (col: the column's chunk 0, CS: chunk stride)
__device__ __forceinline__ void sec_copy(unsigned char* col, int CS, const void* p) {
  const size_t a = (size_t)p & ~(size_t)31;
  unsigned char* dst = col + (int)((a >> 4) & 3) * CS;
  cpa16(dst, (const void*)a);
  cpa16(dst + CS, (const void*)(a + 16));
}
// stage p's sector when the march enters it at this step (lower sweep: addresses rise, a sector
// starts at offset 0; upper sweep: they fall, a sector starts at its last element) or when the
// stream's run starts here (fresh)
template <bool UPPER, class X>
__device__ __forceinline__ void sec_stage(unsigned char* col, int CS, const X* p, bool fresh) {
  const unsigned lo = (unsigned)(size_t)p & 31u;
  if (fresh || lo == (UPPER ? 32u - (unsigned)sizeof(X) : 0u)) sec_copy(col, CS, p);
}
template <class X>
__device__ __forceinline__ X sec_get(const unsigned char* col, int CS, const X* p) {
  const size_t a = (size_t)p;
  return *reinterpret_cast<const X*>(col + (int)((a >> 4) & 3) * CS + (int)(a & 15));
}

// dynamic shared memory of version 4 (byte offsets); every stream holds four chunks
template <int NV, int TC>
struct Lu4Smem {
  static constexpr int CS = TC * 16;          // chunk stride of the column-indexed streams
  static constexpr int XN = TC / 2 + 2;       // tile-edge columns: TJ + TK <= TC / 2 + 2 as TK >= 2
  static constexpr int XS = XN * 16;          // chunk stride of the edge streams
  static constexpr int NOWN = 2 * NV + 8;     // owner: U[NV], R[NV], vol, dt, Lc[3], Lv[3]
  static constexpr int NXT = NV + 2;          // edge: the cross-tile neighbour's U[NV], Lc, Lv
  static constexpr int OWN = 0;
  static constexpr int DIR = OWN + NOWN * 4 * CS;  // per direction: n1, n2, n3, S
  static constexpr int XT = DIR + 3 * 4 * 4 * CS;
  static constexpr int BYTES = XT + NXT * 4 * XS;
  // owner stream numbers
  static constexpr int SU = 0, SR = NV, SVOL = 2 * NV, SDT = 2 * NV + 1, SLC = 2 * NV + 2, SLV = 2 * NV + 5;
};

// one tile of a version-4 sweep (lower or upper) for k_lusgs_wave4_ul, its progress published in
// progress[]; the shared arrays are declared here, the dynamic ring is the kernel's
template <class T, int NV, bool UPPER, int TC>
__device__ __forceinline__ void lu4_tile(const Arena<T>& A, const LuArgs& L, const LuTile tl, int* progress) {
  using SM = Lu4Smem<NV, TC>;
  constexpr int CS = SM::CS, XS = SM::XS;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  __shared__ double s_acc[3][NV][TC];      // direction terms of the current step
  __shared__ double s_pub[NV][TC];         // DU of each column's last cell
  __shared__ double s_diag[2][TC];         // the diagonal of the current step (all variables; the SA variable's)
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  const int TJ = L.TJ, TK = L.TK;
  constexpr int NT = 4 * TC + 64, NC = 4 * TC;
  const int tid = threadIdx.x, grp = tid < 4 * TC ? tid / TC : (tid < 4 * TC + 32 ? 4 : 5), c = tid % TC;
  const int lj = c % TJ, lk = c / TJ;
  const bool owner = grp == 3;
  const int d = grp;  // direction of a direction thread
  auto obuf = [&](int s, int cc) { return s_dyn + SM::OWN + s * 4 * CS + cc * 16; };
  unsigned char* const dbuf = s_dyn + SM::DIR + (d < 3 ? d : 0) * 16 * CS + c * 16;  // stream s at + 4 s CS
  unsigned char* const xbuf = s_dyn + SM::XT + (d == 1 ? lk : TK + lj) * 16;        // stream s at + 4 s XS
  using RT = typename std::conditional<UPPER, double, T>::type;  // R: Res (lower) or DU* (upper)
#include "lusgs4_tile.inc"
}

template <class T, int NV, bool UPPER, int TC>
__global__ void __launch_bounds__(4 * TC + 64, OCFD_LU_MINB) k_lusgs_wave4(Arena<T> A, LuArgs L) {
  using SM = Lu4Smem<NV, TC>;
  constexpr int CS = SM::CS, XS = SM::XS;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  __shared__ int s_tile;
  __shared__ double s_acc[3][NV][TC];      // direction terms of the current step
  __shared__ double s_pub[NV][TC];         // DU of each column's last cell
  __shared__ double s_diag[2][TC];         // the diagonal of the current step (all variables; the SA variable's)
  const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
  const int TJ = L.TJ, TK = L.TK;
  // thread groups: 0..2 direction threads, 3 owner (TC threads each), 4 the poller warp (waits
  // for the upstream tiles' progress), 5 the publisher warp (releases this tile's progress).  The
  // two helper warps take barriers B0 and B1 only; B2 is a separate named barrier of the 4 TC
  // compute threads, so neither a release fence nor an acquire poll sits inside a step's phase.
  constexpr int NT = 4 * TC + 64, NC = 4 * TC;
  const int tid = threadIdx.x, grp = tid < 4 * TC ? tid / TC : (tid < 4 * TC + 32 ? 4 : 5), c = tid % TC;
  const int lj = c % TJ, lk = c / TJ;
  const bool owner = grp == 3;
  const int d = grp;  // direction of a direction thread
  if (TJ * TK != TC || TJ + TK > SM::XN) {  // tile shape outside the edge-stream table: refuse
    if (tid == 0) atomicExch(L.err, 1);
    return;
  }
  auto obuf = [&](int s, int cc) { return s_dyn + SM::OWN + s * 4 * CS + cc * 16; };
  unsigned char* const dbuf = s_dyn + SM::DIR + (d < 3 ? d : 0) * 16 * CS + c * 16;  // stream s at + 4 s CS
  unsigned char* const xbuf = s_dyn + SM::XT + (d == 1 ? lk : TK + lj) * 16;        // stream s at + 4 s XS
  using RT = typename std::conditional<UPPER, double, T>::type;  // R: Res (lower) or DU* (upper)
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(&L.counter[UPPER ? 1 : 0], 1);
    __syncthreads();
    const int q = s_tile;
    if (q >= L.ntiles) break;
    const LuTile tl = UPPER ? L.rtiles[q] : L.tiles[q];
    int* const progress = L.progress;
#include "lusgs4_tile.inc"
  }
}

__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Both sweeps of version 4 in one launch.  LU-SGS is block-local, so a block's upper sweep can
// start as soon as its own lower sweep is done, while the deeper blocks still run their lower
// sweeps.  Tiles come from one counter: every lower tile first (J+K order), then the upper tiles in
// L.utiles, ordered by the step at which each could start (its block's lower sweep done, then its
// upper upstream tiles), so every tile a CTA waits on was handed out before its own.  A finished
// lower tile adds one to its block's count in L.blkdone (release); an upper tile waits (bounded)
// until the count reaches the block's tiles.  The upper sweep publishes into L.progress_up.
template <class T, int NV, int TC>
__global__ void __launch_bounds__(4 * TC + 64, OCFD_LU_MINB) k_lusgs_wave4_ul(Arena<T> A, LuArgs L) {
  using SM = Lu4Smem<NV, TC>;
  __shared__ int s_tile;
  const int tid = threadIdx.x;
  if (L.TJ * L.TK != TC || L.TJ + L.TK > SM::XN) {
    if (tid == 0) atomicExch(L.err, 1);
    return;
  }
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(&L.counter[0], 1);
    __syncthreads();
    const int q = s_tile;
    if (q >= 2 * L.ntiles) break;
    if (q < L.ntiles) {
      const LuTile tl = L.tiles[q];
      lu4_tile<T, NV, false, TC>(A, L, tl, L.progress);
      if (tid == 0) red_release_add(L.blkdone + tl.blk, 1);  // after this tile's release of its progress
    } else {
      const LuTile tl = L.utiles[q - L.ntiles];
      if (tid == 0) {
        const int* tb3 = L.tile_of + 3 * tl.blk;
        int seen = 0;
        if (!wait_ge(L.blkdone + tl.blk, tb3[1] * tb3[2], L.spin_limit, seen)) atomicExch(L.err, 1);
      }
      __syncthreads();
      lu4_tile<T, NV, true, TC>(A, L, tl, L.progress_up);
    }
  }
}

template <class T, int NV, bool UPPER, int TC>
inline size_t lu_wave4_smem() { return (size_t)Lu4Smem<NV, TC>::BYTES; }
template <class T, int NV, bool UPPER, int TC>
inline void lu_wave4_prepare() {
  cudaFuncSetAttribute(k_lusgs_wave4<T, NV, UPPER, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lu_wave4_smem<T, NV, UPPER, TC>());
}
template <class T, int NV, int TC>
inline void lu_wave4_ul_prepare() {
  cudaFuncSetAttribute(k_lusgs_wave4_ul<T, NV, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lu_wave4_smem<T, NV, false, TC>());
}

}  // namespace ocfd
