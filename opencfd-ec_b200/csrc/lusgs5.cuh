// LU-SGS sweeps, version 5: inputs packed in sweep order, one bulk copy per step.
//
// The sweeps (du_LU_SGS, sub_LU_SGS.f90:4-129) march every tile of TJ x TK (j,k) columns along i
// with a skew (column (lj,lk) is at i = t - lj - lk + 1 at step t of the lower sweep), so each
// step reads one scattered cell per column from every input plane.  Here a pack kernel, run once
// per residual before the lower sweep, writes those cells in the order the sweep consumes them:
// one record per (tile, step) holding, for the tile's columns and a one-column ring around them,
// every input of that step.  The sweep then fetches a whole step with one cp.async.bulk per
// record into a ring of shared-memory stages, completed on an mbarrier; it has no per-column
// address arithmetic or staging bookkeeping left.  Geometry (volumes, face normals and areas) is
// packed once, when the handle is created.
//
// Both sweeps read the same records: the cells of the upper sweep's step t are those of the lower
// sweep's step nsteps-1-t, and a column's upstream neighbours of the upper sweep (i+1, j+1, k+1)
// sit in the next record and in the ring's far side.  The lower sweep writes DU* per record
// (coalesced); the upper sweep bulk-copies it as its right-hand side, overwrites it with the final
// DU (what its downstream tiles read) and writes the final DU to the cell-ordered DU planes for
// the update.
//
// Thread roles: one thread per column (TC threads) evaluates the reference expression of its
// cell, in the same order and precision as versions 2-4 (the bits equal the hyperplane order);
// one helper warp issues the bulk copies, releases this tile's progress and waits for the
// upstream tiles (bounded).  One CTA barrier per step: it orders the neighbours' DU of the
// previous step (shared memory), frees the ring stage of step t-2 for the next copy, and carries
// the helper's acquire of the upstream tiles' progress to the threads that then load the
// cross-tile DU (through L2, one step ahead).
#pragma once
#include <stdint.h>

#include "lusgs.cuh"

namespace ocfd {

// record layout (bytes; every section 16-byte aligned) and per-tile record offsets
struct LuStream {
  const LuTile* tmy;       // tiles in block order (index = first + J + nJ*K)
  const long long* rec0;   // first record of each tile (block order); a tile has nrec + 2 records
  unsigned char* dyn;      // per-step records: U (ring), R = Res, dt, Lc (ring), Lv (ring)
  unsigned char* geo;      // static records: vol, n (lower faces), S (lower faces), S (upper faces)
  double* dus;             // DU records: DU* after the lower sweep, DU after the upper
  int dyn_bytes, geo_bytes, dus_bytes;
  int E;                   // columns of the ring-extended tile, (TJ+2)(TK+2)
  int nstage;              // ring stages in shared memory (as many as fit, 4 to 8)
  int o_U, o_R, o_dt, o_Lc, o_Lv;     // in a dyn record
  int o_vol, o_n, o_Slo, o_Sup;        // in a geo record
};


__host__ __device__ inline int lu5_align16(int b) { return (b + 15) & ~15; }

// section offsets for precision T, NV variables, TC columns, E ring columns
template <class T, int NV>
inline void lu5_layout(LuStream& S, int TC, int E) {
  int o = 0;
  S.o_U = o; o = lu5_align16(o + 8 * NV * E);
  S.o_R = o; o = lu5_align16(o + (int)sizeof(T) * NV * TC);
  S.o_dt = o; o = lu5_align16(o + (int)sizeof(T) * TC);
  S.o_Lc = o; o = lu5_align16(o + (int)sizeof(T) * 3 * E);
  S.o_Lv = o; o = lu5_align16(o + (int)sizeof(T) * 3 * E);
  S.dyn_bytes = o;
  o = 0;
  S.o_vol = o; o = lu5_align16(o + 8 * TC);
  S.o_n = o; o = lu5_align16(o + (int)sizeof(T) * 9 * TC);
  S.o_Slo = o; o = lu5_align16(o + (int)sizeof(T) * 3 * TC);
  S.o_Sup = o; o = lu5_align16(o + (int)sizeof(T) * 3 * TC);
  S.geo_bytes = o;
  S.dus_bytes = lu5_align16(8 * NV * TC);
  S.E = E;
  // ring depth: as many stages as fit next to the kernel's static arrays in half of the SM's
  // 228 KB (two CTAs per SM: every tile of a 2 M-cell case resident at once), 4 at the least
  const int stat = (2 + 3) * NV * TC * 8 + 2 * TC * 8 + 16 + 1024;
  const int stg = S.dyn_bytes + S.geo_bytes + S.dus_bytes + 16;
  S.nstage = (233472 / 2 - 1024 - stat) / stg;
  if (S.nstage > 8) S.nstage = 8;
  if (S.nstage < 4) S.nstage = 4;
}

// the cell of ring column (lj, lk) of a tile in stored record s (record r = s - 1 of the lower
// sweep): i = r - lj - lk + 1; false when it lies outside the block
__device__ __forceinline__ bool lu5_cell(const BlkD& B, const LuTile& tl, int s, int lj, int lk, int& i, int& j, int& k) {
  i = s - 1 - lj - lk + 1;
  j = tl.j0 + lj;
  k = tl.k0 + lk;
  return i >= 1 && i <= B.nx - 1 && j >= 1 && j <= B.ny - 1 && k >= 1 && k <= B.nz - 1;
}

// per-step inputs of every tile in sweep order; grid.y = tile (block order)
template <class T, int NV>
__global__ void k_lu_pack_dyn(Arena<T> A, LuStream S, int TJ, int TK) {
  const int q = blockIdx.y;
  const LuTile tl = S.tmy[q];
  const BlkD& B = A.blk[tl.blk];
  const int nrec = B.nx - 1 + TJ + TK - 2;
  const int E = S.E, TC = TJ * TK, W = TJ + 2;
  const long long tb = A.tot_box, tc = A.tot_cell;
  const long long n = (long long)(nrec + 2) * E;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(g / E), e = (int)(g - (long long)s * E);
    const int lj = e % W - 1, lk = e / W - 1;
    unsigned char* rec = S.dyn + (S.rec0[q] + s) * (long long)S.dyn_bytes;
    double* U = (double*)(rec + S.o_U);
    T* Lc = (T*)(rec + S.o_Lc);
    T* Lv = (T*)(rec + S.o_Lv);
    int i, j, k;
    const bool ok = lu5_cell(B, tl, s, lj, lk, i, j, k);
    const bool core = lj >= 0 && lj < TJ && lk >= 0 && lk < TK;
    double u[NV];
    T lc[3], lv[3], r[NV], dt = T(0);
    if (ok) {
      const long long bi = bix(B, i, j, k), ci = cix(B, i, j, k);
#pragma unroll
      for (int m = 0; m < NV; m++) {
        const double x = A.U[m * tb + bi];
        u[m] = m >= 5 ? clamp0(x) : x;   // as limit_vt leaves U6 / U7 (sub_time_advance.f90:410-443)
      }
#pragma unroll
      for (int d = 0; d < 3; d++) { lc[d] = A.Lc[d * tc + ci]; lv[d] = A.Lv[d * tc + ci]; }
      if (core) {
#pragma unroll
        for (int m = 0; m < NV; m++) r[m] = A.Res[m * tc + ci];
        dt = A.dt[ci];
      }
    } else {
#pragma unroll
      for (int m = 0; m < NV; m++) { u[m] = 0.0; r[m] = T(0); }
#pragma unroll
      for (int d = 0; d < 3; d++) { lc[d] = T(0); lv[d] = T(0); }
    }
#pragma unroll
    for (int m = 0; m < NV; m++) U[m * E + e] = u[m];
#pragma unroll
    for (int d = 0; d < 3; d++) { Lc[d * E + e] = lc[d]; Lv[d * E + e] = lv[d]; }
    if (core) {
      const int c = lj + TJ * lk;
      T* R = (T*)(rec + S.o_R);
#pragma unroll
      for (int m = 0; m < NV; m++) R[m * TC + c] = r[m];
      ((T*)(rec + S.o_dt))[c] = dt;
    }
  }
}

// static geometry records (once per handle); grid.y = tile (block order)
template <class T>
__global__ void k_lu_pack_geo(Arena<T> A, LuStream S, int TJ, int TK) {
  const int q = blockIdx.y;
  const LuTile tl = S.tmy[q];
  const BlkD& B = A.blk[tl.blk];
  const int nrec = B.nx - 1 + TJ + TK - 2;
  const int TC = TJ * TK;
  const long long tf = A.tot_face;
  const long long n = (long long)(nrec + 2) * TC;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(g / TC), c = (int)(g - (long long)s * TC);
    const int lj = c % TJ, lk = c / TJ;
    unsigned char* rec = S.geo + (S.rec0[q] + s) * (long long)S.geo_bytes;
    int i, j, k;
    const bool ok = lu5_cell(B, tl, s, lj, lk, i, j, k);
    double vol = 0.0;
    T nn[9], slo[3], sup[3];
#pragma unroll
    for (int x = 0; x < 9; x++) nn[x] = T(0);
#pragma unroll
    for (int d = 0; d < 3; d++) { slo[d] = T(0); sup[d] = T(0); }
    if (ok) {
      vol = A.vold[cix(B, i, j, k)];
      const long long f = fix_(B, i, j, k);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        nn[3 * d + 0] = A.M[(M_NI1 + 3 * d) * tf + f];
        nn[3 * d + 1] = A.M[(M_NI2 + 3 * d) * tf + f];
        nn[3 * d + 2] = A.M[(M_NI3 + 3 * d) * tf + f];
        slo[d] = A.M[(M_SI + d) * tf + f];
        // the upper sweep pairs the lower face's normal with the upper face's area
        // (sub_LU_SGS.f90:96-97, 105-106, 114-115)
        sup[d] = A.M[(M_SI + d) * tf + fix_(B, i + (d == 0), j + (d == 1), k + (d == 2))];
      }
    }
    ((double*)(rec + S.o_vol))[c] = vol;
    T* N = (T*)(rec + S.o_n);
#pragma unroll
    for (int x = 0; x < 9; x++) N[x * TC + c] = nn[x];
#pragma unroll
    for (int d = 0; d < 3; d++) { ((T*)(rec + S.o_Slo))[d * TC + c] = slo[d]; ((T*)(rec + S.o_Sup))[d * TC + c] = sup[d]; }
  }
}

// ---- mbarrier + bulk copy (sm_90+ PTX; no multicast) --------------------------------------
__device__ __forceinline__ unsigned lu5_s(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void lu5_mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(lu5_s(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void lu5_mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void lu5_mbar_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(lu5_s(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void lu5_bulk(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(lu5_s(dst)), "l"(src), "r"(bytes), "r"(lu5_s(bar)) : "memory");
}
__device__ __forceinline__ bool lu5_mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(lu5_s(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// bounded wait for the phase of the given parity; false on timeout
__device__ __forceinline__ bool lu5_mbar_wait(uint64_t* bar, unsigned parity, long long limit) {
  long long it = 0;
  while (!lu5_mbar_test(bar, parity)) {
    if (++it > limit) return false;
  }
  return true;
}

// barrier 1 of the compute groups alone (warp-uniform callers; barrier 0 is __syncthreads)
template <int NT>
__device__ __forceinline__ void lu5_bar_compute() { asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); }

template <class T, int NV, bool UPPER>
__host__ __device__ inline int lu5_stage_bytes(const LuStream& S) { return S.dyn_bytes + S.geo_bytes + (UPPER ? S.dus_bytes : 0); }

template <class T, int NV, int TC>
inline size_t lu5_smem(const LuStream& S, bool upper) {
  return (size_t)S.nstage * (S.dyn_bytes + S.geo_bytes + (upper ? S.dus_bytes : 0)) + 16 * S.nstage;
}
// shared memory of the kernel outside the ring (DU exchange, direction terms, diagonal, tile id)
template <int NV, int TC>
constexpr size_t lu5_static_smem() { return (2 + 3) * NV * TC * 8 + 2 * TC * 8 + 16; }

// Thread groups of a CTA (TC threads each, one per column): 0, 1, 2 the direction threads (the
// flux-difference term of the upstream neighbour in i, j, k; its old-state half is prepared a
// step ahead, so only the DU-dependent half sits on the dependency chain), 3 the owner (the
// diagonal, and the final sum and division of the variables 3..NV-1; direction thread d finishes
// variable d), then one helper warp.  Two CTA barriers per step: B1 (the previous step's DU is in
// shared memory; a ring stage is free), B2 (the three terms and the diagonal are in shared memory).
template <class T, int NV, bool UPPER, int TC>
__global__ void __launch_bounds__(4 * TC + 32, 2) k_lusgs_wave5(Arena<T> A, LuArgs L, LuStream S) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ double s_du[2][NV][TC];     // DU of each column's cell of the last two steps
  __shared__ double s_acc[3][NV][TC];    // the direction terms of the current step
  __shared__ double s_diag[2][TC];       // the diagonal: every variable's, the SA variable's
  __shared__ int s_tile;
  const int NS = S.nstage;
  const int stage_bytes = lu5_stage_bytes<T, NV, UPPER>(S);
  uint64_t* bars = (uint64_t*)(s_dyn + (size_t)NS * stage_bytes);
  auto stage = [&](long long seq) { return s_dyn + (size_t)(seq % NS) * stage_bytes; };
  auto wait_rec = [&](long long seq) { return lu5_mbar_wait(bars + seq % NS, (unsigned)((seq / NS) & 1), L.spin_limit); };
  const int tid = threadIdx.x;
  const int grp = tid < 4 * TC ? tid / TC : 4;
  const int TJ = L.TJ, TK = L.TK, E = S.E, W = TJ + 2;
  const int c = tid % TC, lj = c % TJ, lk = c / TJ;
  const int ec = (lj + 1) + W * (lk + 1);   // this column in the ring-extended tile
  const int HT = 4 * TC;                     // the helper thread
  constexpr bool MIXED = sizeof(T) == 4;     // the mixed form (FP32 fluxes, FP64 state / diagonal)
  const long long tc = A.tot_cell;
  if (tid == HT) {
    for (int q = 0; q < NS; q++) lu5_mbar_init(bars + q, 1);
    lu5_mbar_fence_init();
  }
  __syncthreads();
  long long seq0 = 0;   // records this CTA has loaded before the current tile
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(&L.counter[UPPER ? 1 : 0], 1);
    __syncthreads();
    const int qq = s_tile;
    if (qq >= L.ntiles) break;
    const LuTile tl = UPPER ? L.rtiles[qq] : L.tiles[qq];
    const BlkD& B = A.blk[tl.blk];
    const SolveP& sp = A.sp[B.solve];
    const int nxm = B.nx - 1, nym = B.ny - 1, nzm = B.nz - 1;
    const int* tb3 = L.tile_of + 3 * tl.blk;
    const int first = tb3[0], nJ = tb3[1], nK = tb3[2];
    const int J = (tl.j0 - 1) / TJ, K = (tl.k0 - 1) / TK;
    const int my = first + J + nJ * K;
    int pj = -1, pk = -1;   // upstream tiles (block order)
    if (!UPPER) {
      if (J > 0) pj = my - 1;
      if (K > 0) pk = my - nJ;
    } else {
      if (J < nJ - 1) pj = my + 1;
      if (K < nK - 1) pk = my + nJ;
    }
    const int nsteps = nxm + TJ + TK - 2;
    const int nrecs = nsteps + 2;
    const long long r0 = S.rec0[my];
    // the x-th record loaded is stored record x (lower) or nrecs-1-x (upper); step t's own
    // record is load t+1, its neighbours' record load t (the previous step's own one)
    auto rec_of_load = [&](int x) { return UPPER ? (nrecs - 1 - x) : x; };
    const double w = sp.w_lu, gamma = sp.gamma;
    const bool visc = sp.viscous == 1;
    const bool dual = sp.time_method == -1;
    const double sfac1 = dual ? A.sfac[1] : 0.0;
    const int j = tl.j0 + lj, k = tl.k0 + lk;
    const bool active = j <= nym && k <= nzm;
    auto own_s = [&](int t) { return UPPER ? (nsteps - t) : (t + 1); };
    auto cell_i = [&](int t) { return own_s(t) - lj - lk; };
    auto on_at = [&](int t) { const int i = cell_i(t); return active && t < nsteps && i >= 1 && i <= nxm; };
    auto has = [&](int d, int i) {
      return UPPER ? (d == 0 ? i != nxm : (d == 1 ? j != nym : k != nzm)) : (d == 0 ? i != 1 : (d == 1 ? j != 1 : k != 1));
    };
    // the final value of variable m at step t (sub_LU_SGS.f90:65-67 lower, 120-122 upper).  The
    // FP64 form divides by the diagonal as the reference does; the mixed form multiplies by its
    // FP64 reciprocal, taken by the owner off the dependency chain
    auto finish = [&](int m, int t) {
      const unsigned char* so = stage(seq0 + t + 1);
      const double dg = (NV == 6 && m == 5) ? s_diag[1][c] : s_diag[0][c];
      double r;
      if (!UPPER) {
        const double x = (double)((const T*)(so + S.o_R))[m * TC + c] + s_acc[0][m][c] + s_acc[1][m][c] + s_acc[2][m][c];
        r = MIXED ? x * dg : x / dg;
      } else {
        const double x = s_acc[0][m][c] + s_acc[1][m][c] + s_acc[2][m][c];
        r = ((const double*)(so + S.dyn_bytes + S.geo_bytes))[m * TC + c] + (MIXED ? x * dg : x / dg);
      }
      return r;
    };
    auto store = [&](int m, int t, double r) {
      s_du[t & 1][m][c] = r;
      S.dus[(r0 + own_s(t)) * (S.dus_bytes / 8) + m * TC + c] = r;
      if (UPPER) A.DU[m * tc + cix(B, cell_i(t), j, k)] = r;
    };

    if (grp == 4) {
      // ---- helper: bulk copies, progress release, upstream waits ----------------------
      auto issue = [&](int x) {
        if (x < 0 || x >= nrecs) return;
        const long long seq = seq0 + x;
        unsigned char* st = stage(seq);
        uint64_t* bar = bars + seq % NS;
        const long long rs = r0 + rec_of_load(x);
        lu5_mbar_expect(bar, (unsigned)stage_bytes);
        lu5_bulk(st, S.dyn + rs * S.dyn_bytes, S.dyn_bytes, bar);
        lu5_bulk(st + S.dyn_bytes, S.geo + rs * S.geo_bytes, S.geo_bytes, bar);
        if (UPPER) lu5_bulk(st + S.dyn_bytes + S.geo_bytes, (const unsigned char*)S.dus + rs * S.dus_bytes, S.dus_bytes, bar);
      };
      int seen_j = 0, seen_k = 0;
      auto poll = [&](int t) {   // the upstream tiles have done the steps whose DU step t reads
        if (t >= nsteps) return;
        bool ok = true;
        if (pj >= 0 && seen_j < min(t + TJ, nsteps)) ok &= wait_ge(L.progress + pj, min(t + TJ, nsteps), L.spin_limit, seen_j);
        if (pk >= 0 && seen_k < min(t + TK, nsteps)) ok &= wait_ge(L.progress + pk, min(t + TK, nsteps), L.spin_limit, seen_k);
        if (!ok) atomicExch(L.err, 1);
      };
      if (tid == HT) {
        for (int x = 0; x < NS - 1; x++) issue(x);
        poll(0);
        poll(1);
      }
      __syncthreads();   // B0
      for (int t = 0; t < nsteps; t++) {
        __syncthreads();   // B1 (the compute groups' B2 is a named barrier without the helper, so
                           // the release fence and the upstream wait below overlap their step)
        if (tid == HT) {
          if (t > 0) st_release(L.progress + my, t);
          issue(t + NS - 1);   // into the stage of load t-1, last read before B1
          poll(t + 2);
        }
      }
    } else if (grp == 3) {
      // ---- owner: diagonal (sub_LU_SGS.f90:29-39, 82-92), finish of variables 3..NV-1 ----
      __syncthreads();   // B0
      for (int t = 0; t < nsteps; t++) {
        __syncthreads();   // B1
        const bool on = on_at(t);
        if (on) {
          if (!wait_rec(seq0 + t + 1)) atomicExch(L.err, 1);
          const unsigned char* so = stage(seq0 + t + 1);
          const T* Lco = (const T*)(so + S.o_Lc);
          const T* Lvo = (const T*)(so + S.o_Lv);
          const double vol = ((const double*)(so + S.dyn_bytes + S.o_vol))[c];
          const double dt = (double)((const T*)(so + S.o_dt))[c];
          const double a0 = vol / dt + w * ((double)Lco[ec] + (double)Lco[E + ec] + (double)Lco[2 * E + ec]);
          double al = a0, als = a0;
          if (visc) {
            const double lv0 = Lvo[ec], lv1 = Lvo[E + ec], lv2 = Lvo[2 * E + ec];
            const double lv = lv0 + lv1 + lv2;
            al = al + 2.0 * lv;
            als = als + 2.0 * lv;
            if (NV == 6) {
              if (!UPPER) als = als + lv;
              else als = als + lv0 + lv1 + lv2;
            }
          }
          if (dual) {
            al = al + sfac1 * vol;
            als = als + sfac1 * vol;
          }
          s_diag[0][c] = MIXED ? 1.0 / al : al;
          s_diag[1][c] = MIXED ? 1.0 / als : als;
        }
        lu5_bar_compute<4 * TC>();   // B2
        if (on) {
          double r[NV];
#pragma unroll
          for (int m = 3; m < NV; m++) r[m] = finish(m, t);
#pragma unroll
          for (int m = 3; m < NV; m++) store(m, t, r[m]);
        }
      }
    } else {
      // ---- direction thread d --------------------------------------------------------
      const int d = grp;
      const int dnb = UPPER ? 1 : -1;
      const int en = d == 0 ? ec : (d == 1 ? ec + dnb : ec + dnb * W);       // the neighbour's ring column
      const int cn = d == 0 ? c : (d == 1 ? c + dnb : c + dnb * TJ);          // ... and its column (in-tile)
      // a neighbour in another tile: its DU comes through L2 after the helper's wait.  Lower j-1 of
      // column (0, lk) is column (TJ-1, lk) of tile J-1, TJ-1 records later (the skew); upper j+1
      // of column (TJ-1, lk) is column (0, lk) of tile J+1, TJ-1 records earlier; likewise in k
      const bool xt = d == 1 ? (UPPER ? (lj == TJ - 1 && pj >= 0) : (lj == 0 && pj >= 0))
                             : (d == 2 ? (UPPER ? (lk == TK - 1 && pk >= 0) : (lk == 0 && pk >= 0)) : false);
      const long long pr0 = !xt ? 0 : S.rec0[d == 1 ? pj : pk];
      const int colp = d == 1 ? (UPPER ? TJ * lk : (TJ - 1 + TJ * lk)) : (UPPER ? lj : (lj + TJ * (TK - 1)));
      const int dsp = d == 1 ? (UPPER ? -(TJ - 1) : (TJ - 1)) : (UPPER ? -(TK - 1) : (TK - 1));
      auto load_x = [&](int t, double* xd) {
        const double* src = S.dus + (pr0 + own_s(t) + dsp) * (S.dus_bytes / 8) + colp;
#pragma unroll
        for (int m = 0; m < NV; m++) xd[m] = __ldcg(src + m * TC);
      };
      // old-state half of step t's term: comput_DFn's F(U)n (sub_LU_SGS.f90:135-157), in the flux
      // precision; the neighbour's U, Lc, Lv are in the previous step's record, the face's normal
      // and area in this step's
      using DFT = T;
      DFT Ub[NV], F1[NV], n1 = 0, n2 = 0, n3 = 0;
      double Sd = 0.0, wLc = 0.0, Lvd = 0.0;
      bool hd = false;
      auto prep = [&](int t) {
        hd = on_at(t) && has(d, cell_i(t));
        if (!hd) return;
        const unsigned char* so = stage(seq0 + t + 1);
        const unsigned char* sn = stage(seq0 + t);
        const T* Nn = (const T*)(so + S.dyn_bytes + S.o_n);
        const T* Sa = (const T*)(so + S.dyn_bytes + (UPPER ? S.o_Sup : S.o_Slo));
        n1 = (DFT)Nn[(3 * d) * TC + c];
        n2 = (DFT)Nn[(3 * d + 1) * TC + c];
        n3 = (DFT)Nn[(3 * d + 2) * TC + c];
        Sd = (double)Sa[d * TC + c];
        wLc = w * (double)((const T*)(sn + S.o_Lc))[d * E + en];
        Lvd = (double)((const T*)(sn + S.o_Lv))[d * E + en];
        const double* Un = (const double*)(sn + S.o_U);
#pragma unroll
        for (int m = 0; m < NV; m++) Ub[m] = (DFT)Un[m * E + en];
        const DFT g1 = (DFT)(gamma - 1.0), half = (DFT)0.5;
        const DFT un1 = (Ub[1] * n1 + Ub[2] * n2 + Ub[3] * n3) / Ub[0];
        const DFT p1 = g1 * (Ub[4] - half * (sq(Ub[1]) + sq(Ub[2]) + sq(Ub[3])) / Ub[0]);
        F1[0] = Ub[0] * un1;
        F1[1] = Ub[1] * un1 + p1 * n1;
        F1[2] = Ub[2] * un1 + p1 * n2;
        F1[3] = Ub[3] * un1 + p1 * n3;
        F1[4] = (Ub[4] + p1) * un1;
#pragma unroll
        for (int m = 5; m < NV; m++) F1[m] = Ub[m] * un1;
      };
      bool ok = wait_rec(seq0);
      ok &= wait_rec(seq0 + 1);
      if (!ok) atomicExch(L.err, 1);
      prep(0);
      double xdu[NV];
#pragma unroll
      for (int m = 0; m < NV; m++) xdu[m] = 0.0;
      __syncthreads();   // B0: the helper's first waits are done
      if (xt && hd) load_x(0, xdu);
      for (int t = 0; t < nsteps; t++) {
        __syncthreads();   // B1: step t-1's DU is in s_du
        double nxdu[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) nxdu[m] = 0.0;
        if (xt && on_at(t + 1) && has(d, cell_i(t + 1))) load_x(t + 1, nxdu);   // ready since the wait before B1
        if (hd) {
          double DUn[NV];
#pragma unroll
          for (int m = 0; m < NV; m++) DUn[m] = xt ? xdu[m] : s_du[(t + 1) & 1][m][cn];
          DFT U2[NV];
#pragma unroll
          for (int m = 0; m < NV; m++) U2[m] = (DFT)((double)Ub[m] + DUn[m]);
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
            if (MIXED) {   // the off-diagonal products in FP32 (the accumulation stays FP64)
              const float du = (float)DUn[m];
              float x;
              if (!UPPER) x = 0.5f * ((float)DF[m] * (float)Sd + (float)wLc * du);
              else x = -(0.5f * ((float)DF[m] * (float)Sd - (float)wLc * du));
              if (visc) x = x + (float)Lvd * du;
              v = (double)x;
            } else {
              if (!UPPER) v = 0.5 * ((double)DF[m] * Sd + wLc * DUn[m]);
              else v = -(0.5 * ((double)DF[m] * Sd - wLc * DUn[m]));
              if (visc) v = v + Lvd * DUn[m];
            }
            s_acc[d][m][c] = v;
          }
        } else if (on_at(t)) {
#pragma unroll
          for (int m = 0; m < NV; m++) s_acc[d][m][c] = 0.0;
        }
        lu5_bar_compute<4 * TC>();   // B2: the terms and the diagonal of step t are in shared memory
        if (on_at(t)) store(d, t, finish(d, t));
        if (t + 1 < nsteps) {
          if (on_at(t + 1) && !wait_rec(seq0 + t + 2)) atomicExch(L.err, 1);
          prep(t + 1);
        }
#pragma unroll
        for (int m = 0; m < NV; m++) xdu[m] = nxdu[m];
      }
    }
    __syncthreads();   // the tile's last step is done everywhere
    if (tid == HT) st_release(L.progress + my, nsteps);
    seq0 += nrecs;
  }
}

template <class T, int NV, bool UPPER, int TC>
inline void lu_wave5_prepare(const LuStream& S) {
  cudaFuncSetAttribute(k_lusgs_wave5<T, NV, UPPER, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lu5_smem<T, NV, TC>(S, UPPER));
}

}  // namespace ocfd
