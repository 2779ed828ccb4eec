// C-ABI of libocfd_b200.so (include/ocfd_ec_gpu.h): host orchestration of the device hot path.
//
// A handle holds all blocks of one case resident on the current device: one arena (arena.h),
// the block / subface tables, the setup geometry and the captured CUDA graph of one
// NS_Time_advance step.  All compute happens in the kernels of solver.cuh / setup.cu; the host
// code below only builds tables, fills the node-coordinate ghost layer (a copy / linear
// extrapolation, sub_update_buffer_mpi.f90:230-512) and moves data.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ocfd_ec_gpu.h"
#include "arena.h"
#include "lusgs.cuh"
#include "lusgs5.cuh"
#include "runner.h"
#include "setup.h"

using namespace ocfd;

namespace {

struct DevMem {
  std::vector<void*> ptrs;
  size_t bytes = 0;
  template <class T>
  T* alloc(size_t n, cudaError_t& err) {
    if (err != cudaSuccess) return nullptr;
    if (n == 0) n = 1;
    void* p = nullptr;
    // 32 bytes of padding: the LU-SGS sweep stages whole aligned 32-byte sectors, and the sector
    // of an array's last element may reach up to 28 bytes past its end
    err = cudaMalloc(&p, n * sizeof(T) + 32);
    if (err != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n * sizeof(T) + 32);
    ptrs.push_back(p);
    bytes += n * sizeof(T);
    return (T*)p;
  }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

constexpr int LAPH = 4;

}  // namespace

// One rank's share of a block-sharded case (ocfd_create_part)
struct PartCtx {
  int rank = 0;
  std::vector<int> loc2glob;             // local block -> global block
  long long ncell_global = 0;            // interior cells of the whole case (RMS denominator)
  std::vector<std::vector<double>> X;    // per local block: node coordinates with the ghost layer
  std::vector<double> Xw;                // wall nodes of the whole case
  std::vector<int> send_ent;             // local subface of each outgoing copy (grouped by peer)
  std::vector<long long> send_pre;       // their cell prefix sums (closing entry included)
  std::vector<SubD> recv_sub;            // incoming copies: the remote subface, nb1 = local block
  std::vector<long long> recv_pre;
  std::vector<int> peers;                // ranks exchanged with, ascending
  std::vector<long long> send_off, recv_off;  // per peer, in doubles (npeer + 1 each)
  ocfd_comm comm{};
  bool xchg = true;                      // false while the tile-width autotuner runs
  int comm_err = 0;
  int* d_send_ent = nullptr;
  long long* d_send_pre = nullptr;
  SubD* d_recv_sub = nullptr;
  long long* d_recv_pre = nullptr;
  double* d_send = nullptr;
  double* d_recv = nullptr;
};

struct ocfd_handle {
  ocfd_params P;                   // parameters of solve 0
  std::vector<ocfd_params> Ps;     // per solve
  std::vector<int> sblk0;          // first block of each solve (nsolve + 1 entries)
  std::vector<long long> ncell_s;  // interior cells per solve
  int nvar = 5, prec = 0, nblk = 0, nsolve = 1;
  std::vector<BlkD> blk;
  std::vector<SubD> sub;
  std::vector<long long> pre_box, pre_cell, pre_face, pre_col, pre_subcell, pre_halo, pre_lnj, pre_lnk, pre_reg, pre_r1;
  long long tot_reg = 0, tot_r1 = 0;
  std::vector<unsigned char> phys;  // per block and face (d*2+side): every face cell physical
  int4* d_tiles = nullptr;
  int ntile = 0, tile_maxf = 0, tile_maxc = 0, tile_maxb = 0;
  long long *d_pre_reg = nullptr, *d_pre_r1 = nullptr;
  int *d_hint_reg = nullptr, *d_hint_r1 = nullptr;
  std::vector<int4> cchunk, wchunk;
  std::vector<SolveP> sps;
  long long tot_box = 0, tot_cell = 0, tot_face = 0, tot_node = 0, tot_col = 0, tot_subcell = 0, tot_halo = 0;
  long long ncell = 0;
  int max_plane = 3;
  DevMem mem;
  // device pointers
  BlkD* d_blk = nullptr;
  SubD* d_sub = nullptr;
  SolveP* d_sp = nullptr;
  long long *d_pre_box = nullptr, *d_pre_cell = nullptr, *d_pre_face = nullptr, *d_pre_col = nullptr, *d_pre_subcell = nullptr, *d_pre_halo = nullptr;
  int *d_hint_box = nullptr, *d_hint_cell = nullptr, *d_hint_face = nullptr;
  long long *d_pre_lnj = nullptr, *d_pre_lnk = nullptr;  // j-line and k-line prefix sums (residual smoothing)
  int4 *d_cchunk = nullptr, *d_wchunk = nullptr;
  int* d_cspre = nullptr;
  std::vector<int> cspre;
  std::vector<int> bc_ent, bc_rounds;   // boundary work list (entries grouped by round)
  std::vector<long long> bc_pre;
  int* d_bc_ent = nullptr;
  long long* d_bc_pre = nullptr;
  std::vector<int> halo_ent, halo_levels;  // ordered interface copies (entries grouped by level)
  std::vector<long long> halo_pre;
  int* d_halo_ent = nullptr;
  long long* d_halo_pre = nullptr;
  double* d_halo_stage = nullptr;
  double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr, *d_Md = nullptr, *d_vold = nullptr, *d_dtmd = nullptr, *d_dwd = nullptr;
  double *d_xc = nullptr, *d_yc = nullptr, *d_zc = nullptr;
  float *d_Mf = nullptr, *d_volf = nullptr, *d_dtmf = nullptr, *d_dwf = nullptr;
  unsigned char *d_bci = nullptr, *d_bcj = nullptr, *d_bck = nullptr;
  double *d_U = nullptr, *d_Un = nullptr, *d_Un1 = nullptr, *d_DU = nullptr, *d_sfac = nullptr;
  int dual_started = 0;   // Comput_Residual_one_mesh's saved first-call flag (sub_Residual.f90:25-33)
  double sfac_h[2] = {0.0, 0.0};
  void *d_P = nullptr, *d_mu = nullptr, *d_mut = nullptr, *d_Kt = nullptr, *d_Wt = nullptr, *d_f1 = nullptr;
  void *d_Res = nullptr, *d_dt = nullptr, *d_Lc = nullptr, *d_Lv = nullptr, *d_Fi = nullptr, *d_Fv = nullptr, *d_Ft = nullptr;
  int* d_flags = nullptr;
  double *d_norm_part = nullptr, *d_norm_out = nullptr, *d_force_part = nullptr, *d_stage = nullptr;
  unsigned long long* d_nan = nullptr;
  double* h_pin = nullptr;  // pinned read-back area of the monitors: norms, NaN location, wait flag, force partials
  long long max_box_b = 0;
  Arena<double> A64;
  Arena<float> A32;
  LuArgs lu{};
  LuArgs lu_var[2]{};          // LU-SGS tile tables for TC = 32, 64
  int lu_tc = 32;              // the tile width in use
  LuStream lus{};              // version-5 sweep records (built for the 64-column tile table)
  int lus_v = -1;              // tile table the records were built for (-1: none)
  bool lus_geo = false;        // static geometry records packed
  RunInfo info{};
  int nsm = 148;
  int* d_lu_err = nullptr;
  std::unique_ptr<Runner> run;
  cudaStream_t st = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  std::unique_ptr<PartCtx> part;   // set for block-sharded handles
  int kstep = 0;
  double tt = 0.0;
  std::string err;
};

static int fail(ocfd_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}
static int cuda_fail(ocfd_handle* h, cudaError_t e, const char* where) {
  return fail(h, e == cudaErrorMemoryAllocation ? OCFD_ERR_OOM : OCFD_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
// error paths that allocate nothing (ocfd_residual_static): the message is formatted on the
// stack and copied into the handle's error string, whose capacity (512 bytes) every handle
// reserves at creation, so the copy never reallocates
static int fail_c(ocfd_handle* h, int code, const char* msg) {
  if (h) h->err.assign(msg, std::min<size_t>(std::strlen(msg), 511));
  return code;
}
static int cuda_fail_c(ocfd_handle* h, cudaError_t e, const char* where) {
  char buf[256];
  std::snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
  return fail_c(h, e == cudaErrorMemoryAllocation ? OCFD_ERR_OOM : OCFD_ERR_CUDA, buf);
}

extern "C" const char* ocfd_version(void) { return "ocfd-b200 abi 1 sm_100a (FP64 + mixed FP32/FP64)"; }

extern "C" int ocfd_default_params(ocfd_params* p) {  // set_default_parameter, sub_read_parameter.f90:30-106
  if (!p) return OCFD_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->ma = 1.0; p->re = 1000.0; p->gamma = 1.4; p->aoa = 0.0; p->aos = 0.0; p->p_outlet = -1.0;
  p->iflag_turbulence_model = 0; p->if_viscous = 1; p->iflag_local_dt = 1; p->dt_global = 0.01; p->cfl = 1.0;
  p->dtmax = 10.0; p->dtmin = 1.e-9; p->time_method = 0; p->w_lu = 1.0; p->if_dtime_mesh = 1;
  p->iflag_scheme = 5; p->iflag_flux = 5; p->iflag_reconstruction = 0; p->t_inf = 288.15; p->twall = -1.0;
  p->kt_inf = 1.e-5; p->wt_inf = 0.01; p->mut_max = -1.0; p->bound_scheme = 4; p->ref_s = 1.0; p->ref_l = 1.0;
  p->cood_y_up = 1; p->iflag_limit_flow = 1; p->prl = 0.7; p->prt = 0.9;
  p->ldmin = 1.e-6; p->ldmax = 1000.0; p->lpmin = 1.e-6; p->lpmax = 1000.0; p->lumax = 1000.0; p->lsamax = 1000.0;
  p->if_scheme_positivity = 1; p->precision = OCFD_PREC_FP64;
  p->step_inner_limit = 20; p->res_inner_limit = 1.e-10;  // sub_read_parameter.f90:69-70
  return OCFD_OK;
}

extern "C" int ocfd_finalize_params(ocfd_params* p) {  // set_const_para, sub_read_parameter.f90:371-429
  if (!p) return OCFD_ERR_ARG;
  const double PI = 3.1415926535897932;
  p->twall = p->twall / p->t_inf;
  p->lpmin = p->lpmin / (p->gamma * p->ma * p->ma);
  p->lpmax = p->lpmax / (p->gamma * p->ma * p->ma);
  if (p->bound_scheme == -1) p->bound_scheme = p->iflag_scheme;
  if (p->if_viscous == 0) p->iflag_turbulence_model = 0;
  if (p->iflag_turbulence_model == 2 || p->iflag_turbulence_model == 21) p->nvar = 6;
  else if (p->iflag_turbulence_model == 3) p->nvar = 7;
  else p->nvar = 5;
  p->aoa = p->aoa * PI / 180.0;
  p->aos = p->aos * PI / 180.0;
  if (p->cood_y_up == 1) { p->a_alfa = p->aoa; p->a_beta = p->aos; }
  else { p->a_alfa = p->aos; p->a_beta = p->aoa; }
  p->cv = 1.0 / (p->gamma * (p->gamma - 1.0) * p->ma * p->ma);
  p->cp = p->cv * p->gamma;
  return OCFD_OK;
}

static void fill_solve(const ocfd_params& p, int nvar, SolveP& s) {
  s.nvar = nvar; s.scheme = p.iflag_scheme; s.bound_scheme = p.bound_scheme; s.flux = p.iflag_flux; s.recon = p.iflag_reconstruction;
  s.turb = p.if_viscous ? p.iflag_turbulence_model : 0; s.viscous = p.if_viscous; s.local_dt = p.iflag_local_dt; s.dtime_mesh = p.if_dtime_mesh;
  s.limit_flow = p.iflag_limit_flow; s.positivity = p.if_scheme_positivity; s.time_method = p.time_method;
  s.gamma = p.gamma; s.ma = p.ma; s.re = p.re; s.cv = p.cv; s.cp = p.cp; s.prl = p.prl; s.prt = p.prt; s.tsb = 110.4 / p.t_inf;
  s.twall = p.twall; s.kt_inf = p.kt_inf; s.wt_inf = p.wt_inf; s.a_alfa = p.a_alfa; s.a_beta = p.a_beta; s.cfl = p.cfl;
  s.dt_global = p.dt_global; s.dtmin = p.dtmin; s.dtmax = p.dtmax; s.w_lu = p.w_lu; s.mut_max = p.mut_max; s.p_outlet = p.p_outlet;
  s.ldmin = p.ldmin; s.ldmax = p.ldmax; s.lpmin = p.lpmin; s.lpmax = p.lpmax; s.lumax = p.lumax; s.lsamax = p.lsamax;
  s.p00 = 1.0 / (p.gamma * p.ma * p.ma);
  s.d_inf = 1.0;
  s.u_inf = std::cos(p.a_alfa) * std::cos(p.a_beta);
  s.v_inf = std::sin(p.a_alfa) * std::cos(p.a_beta);
  s.w_inf = std::sin(p.a_beta);
  s.p_inf = 1.0 / (p.gamma * p.ma * p.ma);
  s.cen[0] = p.centroid[0]; s.cen[1] = p.centroid[1]; s.cen[2] = p.centroid[2];
}

// node coordinates with one ghost layer: interface copy (Coordinate_send_mpi, 250-352), linear
// extrapolation on physical faces and edge / vertex averaging (coordinate_boundary_and_corner,
// get_xyz_conner, 413-512)
static void coordinate_ghosts(const std::vector<BlkD>& blk, const std::vector<SubD>& sub, std::vector<std::vector<double>>& X) {
  auto at = [&](int b, int c, int i, int j, int k) -> double& {
    const BlkD& B = blk[b];
    return X[b][(size_t)c * B.NXn * B.NYn * B.NZn + (size_t)i + (size_t)B.NXn * ((size_t)j + (size_t)B.NYn * k)];
  };
  for (const SubD& S : sub) {
    if (S.bc >= 0) continue;
    int kb[3] = {S.ib, S.jb, S.kb}, ke[3] = {S.ie, S.je, S.ke};
    int d = (S.face - 1) % 3;
    if (S.face <= 3) kb[d] += 1; else kb[d] -= 1;
    ke[d] = kb[d];
    int kb1[3] = {S.ib1, S.jb1, S.kb1}, ke1[3] = {S.ie1, S.je1, S.ke1};
    int d1 = (S.face1 - 1) % 3;
    if (S.face1 <= 3) kb1[d1] -= 1; else kb1[d1] += 1;
    ke1[d1] = kb1[d1];
    int L[3] = {std::abs(S.L1), std::abs(S.L2), std::abs(S.L3)};
    int Pq[3] = {S.L1 >= 0 ? 1 : -1, S.L2 >= 0 ? 1 : -1, S.L3 >= 0 ? 1 : -1};
    int ks[3];
    for (int q = 0; q < 3; q++) ks[q] = Pq[q] > 0 ? kb[q] : ke[q];
    for (int kk = kb1[2]; kk <= ke1[2]; kk++)
      for (int jj = kb1[1]; jj <= ke1[1]; jj++)
        for (int ii = kb1[0]; ii <= ke1[0]; ii++) {
          int ka[3] = {ii - kb1[0], jj - kb1[1], kk - kb1[2]};
          int i1 = ks[0] + ka[L[0] - 1] * Pq[0], j1 = ks[1] + ka[L[1] - 1] * Pq[1], k1 = ks[2] + ka[L[2] - 1] * Pq[2];
          for (int c = 0; c < 3; c++) at(S.nb1, c, ii, jj, kk) = at(S.blk, c, i1, j1, k1);
        }
  }
  for (const SubD& S : sub) {
    if (S.bc < 0) continue;
    int b = S.blk, i1 = S.ib, i2 = S.ie, j1 = S.jb, j2 = S.je, k1 = S.kb, k2 = S.ke;
    for (int c = 0; c < 3; c++) {
      if (S.face == 1) { for (int k = k1; k <= k2; k++) for (int j = j1; j <= j2; j++) at(b, c, i1 - 1, j, k) = 2.0 * at(b, c, i1, j, k) - at(b, c, i1 + 1, j, k); }
      else if (S.face == 2) { for (int k = k1; k <= k2; k++) for (int i = i1; i <= i2; i++) at(b, c, i, j1 - 1, k) = 2.0 * at(b, c, i, j1, k) - at(b, c, i, j1 + 1, k); }
      else if (S.face == 3) { for (int j = j1; j <= j2; j++) for (int i = i1; i <= i2; i++) at(b, c, i, j, k1 - 1) = 2.0 * at(b, c, i, j, k1) - at(b, c, i, j, k1 + 1); }
      else if (S.face == 4) { for (int k = k1; k <= k2; k++) for (int j = j1; j <= j2; j++) at(b, c, i2 + 1, j, k) = 2.0 * at(b, c, i2, j, k) - at(b, c, i2 - 1, j, k); }
      else if (S.face == 5) { for (int k = k1; k <= k2; k++) for (int i = i1; i <= i2; i++) at(b, c, i, j2 + 1, k) = 2.0 * at(b, c, i, j2, k) - at(b, c, i, j2 - 1, k); }
      else { for (int j = j1; j <= j2; j++) for (int i = i1; i <= i2; i++) at(b, c, i, j, k2 + 1) = 2.0 * at(b, c, i, j, k2) - at(b, c, i, j, k2 - 1); }
    }
  }
  for (size_t b = 0; b < blk.size(); b++) {
    if (X[b].empty()) continue;  // a block of another rank whose nodes no ghost layer here reaches
    int nx = blk[b].nx, ny = blk[b].ny, nz = blk[b].nz;
    for (int c = 0; c < 3; c++) {
      auto x = [&](int i, int j, int k) -> double& { return at((int)b, c, i, j, k); };
      for (int k = 1; k <= nz; k++) {
        x(0, 0, k) = (x(1, 0, k) + x(0, 1, k)) * 0.5;
        x(nx + 1, 0, k) = (x(nx, 0, k) + x(nx + 1, 1, k)) * 0.5;
        x(0, ny + 1, k) = (x(1, ny + 1, k) + x(0, ny, k)) * 0.5;
        x(nx + 1, ny + 1, k) = (x(nx, ny + 1, k) + x(nx + 1, ny, k)) * 0.5;
      }
      for (int j = 1; j <= ny; j++) {
        x(0, j, 0) = (x(1, j, 0) + x(0, j, 1)) * 0.5;
        x(nx + 1, j, 0) = (x(nx, j, 0) + x(nx + 1, j, 1)) * 0.5;
        x(0, j, nz + 1) = (x(1, j, nz + 1) + x(0, j, nz)) * 0.5;
        x(nx + 1, j, nz + 1) = (x(nx, j, nz + 1) + x(nx + 1, j, nz)) * 0.5;
      }
      for (int i = 1; i <= nx; i++) {
        x(i, 0, 0) = (x(i, 1, 0) + x(i, 0, 1)) * 0.5;
        x(i, ny + 1, 0) = (x(i, ny, 0) + x(i, ny + 1, 1)) * 0.5;
        x(i, 0, nz + 1) = (x(i, 1, nz + 1) + x(i, 0, nz)) * 0.5;
        x(i, ny + 1, nz + 1) = (x(i, ny, nz + 1) + x(i, ny + 1, nz)) * 0.5;
      }
      for (int v = 0; v < 8; v++) {
        int ia = (v & 1) ? nx + 1 : 0, ib = (v & 1) ? nx : 1;
        int ja = (v & 2) ? ny + 1 : 0, jb = (v & 2) ? ny : 1;
        int ka = (v & 4) ? nz + 1 : 0, kb = (v & 4) ? nz : 1;
        x(ia, ja, ka) = (2.0 * (x(ib, ja, ka) + x(ia, jb, ka) + x(ia, ja, kb)) - (x(ib, jb, ka) + x(ib, ja, kb) + x(ia, jb, kb))) / 3.0;
      }
    }
  }
}

static long long subcell_count(const SubD& S) {
  if (S.face == 1 || S.face == 4) return (long long)(S.je - S.jb) * (S.ke - S.kb);
  if (S.face == 2 || S.face == 5) return (long long)(S.ie - S.ib) * (S.ke - S.kb);
  return (long long)(S.ie - S.ib) * (S.je - S.jb);
}

template <class T>
static void fill_arena(ocfd_handle* h, Arena<T>& A, const T* M, const T* vol, const T* dtm, const T* dw) {
  A.blk = h->d_blk; A.nblk = h->nblk;
  A.pre_box = h->d_pre_box; A.pre_cell = h->d_pre_cell; A.pre_face = h->d_pre_face; A.pre_col = h->d_pre_col;
  A.hint_box = h->d_hint_box; A.hint_cell = h->d_hint_cell; A.hint_face = h->d_hint_face;
  A.pre_reg = h->d_pre_reg; A.pre_r1 = h->d_pre_r1; A.hint_reg = h->d_hint_reg; A.hint_r1 = h->d_hint_r1;
  A.tot_r1 = h->tot_r1;
  A.tiles = h->d_tiles; A.ntile = h->ntile; A.tile_maxf = h->tile_maxf; A.tile_maxc = h->tile_maxc; A.tile_maxb = h->tile_maxb;
  A.pre_lnj = h->d_pre_lnj; A.pre_lnk = h->d_pre_lnk; A.tot_lnj = h->pre_lnj[h->nblk]; A.tot_lnk = h->pre_lnk[h->nblk];
  A.sub = h->d_sub; A.nsub = (int)h->sub.size();
  A.pre_subcell = h->d_pre_subcell; A.pre_halo = h->d_pre_halo;
  A.cchunk = h->d_cchunk; A.ncchunk = (int)h->cchunk.size(); A.cspre = h->d_cspre;
  A.bc_ent = h->d_bc_ent; A.bc_pre = h->d_bc_pre;
  A.wchunk = h->d_wchunk; A.nwchunk = (int)h->wchunk.size();
  A.sp = h->d_sp; A.nsolve = h->nsolve;
  A.tot_box = h->tot_box; A.tot_cell = h->tot_cell; A.tot_face = h->tot_face; A.tot_node = h->tot_node; A.tot_col = h->tot_col;
  A.tot_subcell = h->tot_subcell; A.tot_halo = h->tot_halo;
  A.x = h->d_x; A.y = h->d_y; A.z = h->d_z; A.Md = h->d_Md; A.M = M;
  A.vold = h->d_vold; A.dwd = h->d_dwd; A.vol = vol; A.dtm = dtm; A.dw = dw;
  A.xc = h->d_xc; A.yc = h->d_yc; A.zc = h->d_zc;
  A.bci = h->d_bci; A.bcj = h->d_bcj; A.bck = h->d_bck;
  A.U = h->d_U; A.Un = h->d_Un; A.Un1 = h->d_Un1; A.sfac = h->d_sfac; A.P = (T*)h->d_P; A.mu = (T*)h->d_mu; A.mut = (T*)h->d_mut; A.Kt = (T*)h->d_Kt; A.Wt = (T*)h->d_Wt;
  A.f1 = (T*)h->d_f1; A.Res = (T*)h->d_Res; A.DU = h->d_DU; A.dt = (T*)h->d_dt; A.Lc = (T*)h->d_Lc; A.Lv = (T*)h->d_Lv;
  A.Fi = (T*)h->d_Fi; A.Fv = (T*)h->d_Fv; A.Ft = (T*)h->d_Ft; A.flags = h->d_flags;
  A.only_solve = -1;
}

template <class T>
static cudaError_t up(T* d, const std::vector<T>& v) {
  if (v.empty()) return cudaSuccess;
  return cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// mu = 1/Re everywhere (allocate_mem_Blocks, sub_init.f90:507), Re of each block's solve
static void reset_mu(ocfd_handle* h) {
  size_t n = (size_t)h->tot_box;
  std::vector<double> v(n);
  for (int b = 0; b < h->nblk; b++)
    std::fill(v.begin() + h->pre_box[b], v.begin() + h->pre_box[b + 1], 1.0 / h->Ps[h->blk[b].solve].re);
  if (h->prec == OCFD_PREC_MIXED) {
    std::vector<float> vf(v.begin(), v.end());
    cudaMemcpy(h->d_mu, vf.data(), n * 4, cudaMemcpyHostToDevice);
  } else {
    cudaMemcpy(h->d_mu, v.data(), n * 8, cudaMemcpyHostToDevice);
  }
}

// every work array back to its state right after allocation (zeros; mu = 1/Re), so that steps
// run before the caller's first step leave no trace (edge ghosts of mu and mu_t are never
// recomputed and carry history, sub_turbulence_SA.f90:37-45)
static void reset_work(ocfd_handle* h) {
  const long long tb = h->tot_box, tf = h->tot_face, tc = h->tot_cell;
  const size_t ts = h->prec == OCFD_PREC_MIXED ? sizeof(float) : sizeof(double);
  const int NV = h->nvar;
  cudaDeviceSynchronize();
  cudaMemset(h->d_P, 0, ts * P_COUNT * tb);
  cudaMemset(h->d_mut, 0, ts * tb);
  if (h->d_Kt) { cudaMemset(h->d_Kt, 0, ts * tb); cudaMemset(h->d_Wt, 0, ts * tb); cudaMemset(h->d_f1, 0, ts * tf); }
  cudaMemset(h->d_Res, 0, ts * NV * tc);
  cudaMemset(h->d_dt, 0, ts * tc);
  cudaMemset(h->d_Lc, 0, ts * 3 * tc);
  cudaMemset(h->d_Lv, 0, ts * 3 * tc);
  cudaMemset(h->d_DU, 0, sizeof(double) * std::max(NV, 5) * tc);
  if (h->d_Fv) cudaMemset(h->d_Fv, 0, ts * 12 * tf);
  if (h->d_Ft) cudaMemset(h->d_Ft, 0, ts * 6 * tf);
  if (h->d_Un) cudaMemset(h->d_Un, 0, sizeof(double) * NV * tb);
  if (h->d_Un1) cudaMemset(h->d_Un1, 0, sizeof(double) * NV * tb);
  cudaMemset(h->d_flags, 0, sizeof(int) * 4 * h->nblk);
  cudaMemset(h->d_lu_err, 0, sizeof(int));
  reset_mu(h);
}

// version-5 record layout for the handle's precision and NVAR
static void lu5_layout_for(int prec, int NV, LuStream& S, int TC, int E) {
  if (prec == OCFD_PREC_MIXED) {
    if (NV == 5) lu5_layout<float, 5>(S, TC, E);
    else if (NV == 6) lu5_layout<float, 6>(S, TC, E);
    else lu5_layout<float, 7>(S, TC, E);
  } else {
    if (NV == 5) lu5_layout<double, 5>(S, TC, E);
    else if (NV == 6) lu5_layout<double, 6>(S, TC, E);
    else lu5_layout<double, 7>(S, TC, E);
  }
}

// (re)builds the runner for LU-SGS tile table v (0: TC = 32, 1: TC = 64) and wavefront kernel
// version ver (2, 3 or 4); drops a captured graph
static void select_lu(ocfd_handle* h, int v, int ver) {
  if (ver == 5 && h->lus_v != v) ver = 4;   // records exist for one tile table only
  h->lu = h->lu_var[v];
  h->lu_tc = v == 0 ? 32 : 64;
  h->info.lu_fused = ver == 6 ? 1 : 0;      // 6: version 4 with both sweeps in one launch
  if (ver == 6) ver = 4;
  h->info.lu_version = ver;
  h->info.lu = &h->lu;
  h->info.lu_tc = h->lu_tc;
  h->info.lu_grid = std::max(1, std::min(h->lu.ntiles, h->nsm * 8));
  h->info.lus = ver == 5 ? &h->lus : nullptr;
  if (ver == 5) {
    // resident CTAs per SM from the shared memory a CTA takes (ring + exchange arrays + margin)
    const int TC = h->lu_tc;
    for (int up = 0; up < 2; up++) {
      const long long ring = (long long)h->lus.nstage * (h->lus.dyn_bytes + h->lus.geo_bytes + (up ? h->lus.dus_bytes : 0)) + 16 * h->lus.nstage;
      const long long per = ring + 40LL * h->nvar * TC + 16LL * TC + 2048;
      const int occ = (int)std::max(1LL, std::min(233472LL / (per + 1024), std::min(2LL, 2048LL / (4 * TC + 32))));
      h->info.lu5_grid[up] = std::max(1, std::min(h->lu.ntiles, h->nsm * occ));
    }
  }
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  if (h->prec == OCFD_PREC_MIXED) h->run.reset(make_runner_mixed(h->A32, h->info));
  else h->run.reset(make_runner_fp64(h->A64, h->info));
  if (ver == 5 && h->run && !h->lus_geo) {
    h->run->lu5_pack_geo(h->st);
    h->lus_geo = true;
  }
}

// LU-SGS autotuner: each candidate (tile table v, kernel version ver) sweeps the freshly
// initialised case (two warm-up and three timed steps, CUDA events around the two sweeps); the
// fastest is kept.  The state is re-initialised afterwards by the caller, and the choice does not
// change any result (every tiling and version gives the hyperplane-order bits).
static void autotune_lu(ocfd_handle* h, const std::vector<std::pair<int, int>>& cand) {
  cudaEvent_t ev[6];
  for (int q = 0; q < 6; q++) cudaEventCreate(&ev[q]);
  float best = 1e30f;
  std::pair<int, int> bestv = cand[0];
  for (const auto& vv : cand) {
    const int v = vv.first;
    select_lu(h, v, vv.second);
    h->run->init_flow(h->st);
    for (int s = 0; s < 2; s++) h->run->step(h->st);
    float tot = 0.0f;
    for (int s = 0; s < 3; s++) {
      h->run->step(h->st, ev);
      cudaEventSynchronize(ev[5]);
      float a = 0.0f, b2 = 0.0f;
      cudaEventElapsedTime(&a, ev[1], ev[2]);
      cudaEventElapsedTime(&b2, ev[2], ev[3]);
      tot += a + b2;
    }
    if (cudaGetLastError() == cudaSuccess && tot < best) { best = tot; bestv = vv; }
  }
  for (int q = 0; q < 6; q++) cudaEventDestroy(ev[q]);
  reset_work(h);
  select_lu(h, bestv.first, bestv.second);
}

extern "C" int ocfd_lu_tile_width(const ocfd_handle* h) { return h ? h->lu_tc : 0; }
extern "C" int ocfd_lu_kernel_version(const ocfd_handle* h) { return h ? h->info.lu_version : 0; }
extern "C" int ocfd_lu_one_launch(const ocfd_handle* h) {
  return h && !h->info.lu_planes && h->info.lu_version == 4 && h->info.lu_fused ? 1 : 0;
}

// all solves of a handle share the model switches that select kernels; Mach, angles, Re, CFL,
// schemes, fluxes and limits may differ per solve
static int check_params(const ocfd_params* ps, int nsolve) {
  const ocfd_params& p0 = ps[0];
  for (int q = 0; q < nsolve; q++) {
    const ocfd_params& p = ps[q];
    int tm = p.if_viscous ? p.iflag_turbulence_model : 0;
    if (tm != 0 && tm != 2 && tm != 3) return OCFD_ERR_UNSUPPORTED;
    if (p.time_method != 0 && p.time_method != 1 && p.time_method != 3 && p.time_method != -1) return OCFD_ERR_UNSUPPORTED;
    if (p.if_residual_smoothing != 0 && p.if_residual_smoothing != 1) return OCFD_ERR_ARG;
    if (p.time_method == -1 && p.step_inner_limit < 1) return OCFD_ERR_ARG;
    if (p.iflag_flux < 1 || p.iflag_flux > 6) return OCFD_ERR_ARG;
    int tm0 = p0.if_viscous ? p0.iflag_turbulence_model : 0;
    if (tm != tm0 || p.if_viscous != p0.if_viscous || p.time_method != p0.time_method || p.precision != p0.precision ||
        p.if_residual_smoothing != p0.if_residual_smoothing)
      return OCFD_ERR_ARG;
  }
  return OCFD_OK;
}

// the exchange hook of a sharded handle's runner: hands the packed buffers to the caller's
// exchange callback; returns 1 when the receive buffer holds this update's copies
static int part_exchange(void* ctx, cudaStream_t st) {
  ocfd_handle* h = (ocfd_handle*)ctx;
  PartCtx& P = *h->part;
  if (!P.xchg) return 0;
  int rc = P.comm.exchange(P.comm.user, (void*)st, (int)P.peers.size(), P.peers.data(), P.d_send, P.send_off.data(), P.d_recv,
                           P.recv_off.data());
  if (rc && !P.comm_err) P.comm_err = rc;
  return rc ? 0 : 1;
}

// the cells whose primitives a residual reads (BlkD::glo/ghi, the pre_reg prefix): all LAPH ghost
// layers across a block face with an interface cell; across a wholly physical face only as deep
// as that face's stencils reach.  The face at the boundary uses CD2 (cells 0 and 1), the next
// LAPH-2 faces the boundary scheme, which reaches 1 cell below its face's left cell for the 2nd /
// 3rd-order schemes (and UD1), 2 for WENO5 / UD5 and 3 for WENO7; the interior scheme starts
// LAPH faces in and reaches layer 0 at most.  Depends on each solve's boundary scheme, so a
// reset_solve recomputes it.
static void region_tables(ocfd_handle* h) {
  const int nblk = h->nblk;
  h->pre_reg.assign(nblk + 1, 0);
  for (int b = 0; b < nblk; b++) {
    BlkD& B = h->blk[b];
    const int bs = h->Ps[B.solve].bound_scheme;
    const int reach = bs == OCFD_SCHEME_WENO7 ? 3 : ((bs == OCFD_SCHEME_WENO5 || bs == OCFD_SCHEME_UD5) ? 2 : 1);
    for (int d = 0; d < 3; d++) {
      B.glo[d] = h->phys[b * 6 + d * 2] ? reach : LAPH;
      B.ghi[d] = h->phys[b * 6 + d * 2 + 1] ? reach : LAPH;
    }
    B.RX = B.nx - 1 + B.glo[0] + B.ghi[0];
    B.RY = B.ny - 1 + B.glo[1] + B.ghi[1];
    B.RZ = B.nz - 1 + B.glo[2] + B.ghi[2];
    B.oreg = h->pre_reg[b];
    h->pre_reg[b + 1] = h->pre_reg[b] + (long long)B.RX * B.RY * B.RZ;
  }
  h->tot_reg = h->pre_reg[nblk];
}

// residual tiles: about 512 cells, 16 along i, 4 along k (fewer on thinner blocks, whose tiles
// grow in j instead), in block order with i fastest so that neighbouring tiles run together
static std::vector<int4> tile_table(ocfd_handle* h) {
  std::vector<int4> t;
  h->tile_maxf = 1;
  h->tile_maxc = 1;
  h->tile_maxb = 1;
  int TI = 16, TK = 4, NC = 512;  // OCFD_RES_TILE="i,k,cells" overrides (tile-shape measurements)
  if (const char* e = std::getenv("OCFD_RES_TILE")) {
    int a = 0, c = 0, n = 0;
    if (std::sscanf(e, "%d,%d,%d", &a, &c, &n) == 3 && a > 0 && c > 0 && n >= a * c && n <= 1024) { TI = a; TK = c; NC = n; }
  }
  for (int b = 0; b < h->nblk; b++) {
    BlkD& B = h->blk[b];
    const int ti = std::min(TI, B.nx - 1), tk = std::min(TK, B.nz - 1);
    const int tj = std::min(B.ny - 1, std::max(1, NC / (ti * tk)));
    B.tdim[0] = ti; B.tdim[1] = tj; B.tdim[2] = tk;
    h->tile_maxc = std::max(h->tile_maxc, ti * tj * tk);
    h->tile_maxb = std::max(h->tile_maxb, (ti + 2) * (tj + 2) * (tk + 2));
    h->tile_maxf = std::max({h->tile_maxf, (ti + 1) * tj * tk, ti * (tj + 1) * tk, ti * tj * (tk + 1)});
    for (int k = 1; k < B.nz; k += tk)
      for (int j = 1; j < B.ny; j += tj)
        for (int i = 1; i < B.nx; i += ti) t.push_back(make_int4(b, i, j, k));
  }
  return t;
}

static std::vector<int> hint_table(const std::vector<long long>& pre, int nblk) {
  std::vector<int> hv((size_t)(pre[nblk] >> HINT_SHIFT) + 1);
  int b = 0;
  for (size_t q = 0; q < hv.size(); q++) {
    const long long g = (long long)q << HINT_SHIFT;
    while (b + 1 < nblk && pre[b + 1] <= g) b++;
    hv[q] = b;
  }
  return hv;
}

static int create_impl(const ocfd_params* ps, int nsolve, const int* nblk_s, const int* nijk, const double* const* xyz, const int* nsub,
                       const int* inc, const double* const* dw, ocfd_handle** out, std::unique_ptr<PartCtx> part = nullptr) {
  if (!ps || nsolve <= 0 || !nblk_s || !nijk || !xyz || !nsub || !inc || !out) return OCFD_ERR_ARG;
  int nblk = 0;
  for (int q = 0; q < nsolve; q++) {
    if (nblk_s[q] <= 0) return OCFD_ERR_ARG;
    nblk += nblk_s[q];
  }
  if (int rc = check_params(ps, nsolve)) return rc;
  std::unique_ptr<ocfd_handle> hp(new ocfd_handle());
  ocfd_handle* h = hp.get();
  h->err.reserve(512);
  h->part = std::move(part);
  const ocfd_params* p = ps;
  h->P = ps[0];
  h->Ps.assign(ps, ps + nsolve);
  h->nsolve = nsolve;
  h->sblk0.assign(nsolve + 1, 0);
  for (int q = 0; q < nsolve; q++) h->sblk0[q + 1] = h->sblk0[q] + nblk_s[q];
  int tm = p->if_viscous ? p->iflag_turbulence_model : 0;
  h->nvar = (tm == 2) ? 6 : (tm == 3 ? 7 : 5);
  h->prec = p->precision;
  h->nblk = nblk;
  h->sps.resize(nsolve);
  for (int q = 0; q < nsolve; q++) fill_solve(ps[q], h->nvar, h->sps[q]);
  // ---- tables
  h->blk.resize(nblk);
  h->pre_box.assign(nblk + 1, 0); h->pre_cell.assign(nblk + 1, 0); h->pre_face.assign(nblk + 1, 0); h->pre_col.assign(nblk + 1, 0);
  h->pre_lnj.assign(nblk + 1, 0); h->pre_lnk.assign(nblk + 1, 0);
  long long onode = 0, obci = 0, obcj = 0, obck = 0;
  const int* q = inc;
  for (int b = 0; b < nblk; b++) {
    BlkD& B = h->blk[b];
    B.nx = nijk[3 * b]; B.ny = nijk[3 * b + 1]; B.nz = nijk[3 * b + 2];
    if (B.nx < 2 || B.ny < 2 || B.nz < 2) return OCFD_ERR_ARG;
    B.NX = B.nx + 7; B.NY = B.ny + 7; B.NZ = B.nz + 7;
    B.NXn = B.nx + 2; B.NYn = B.ny + 2; B.NZn = B.nz + 2;
    B.solve = (int)(std::upper_bound(h->sblk0.begin(), h->sblk0.end(), b) - h->sblk0.begin()) - 1;
    B.obox = h->pre_box[b]; B.oface = h->pre_face[b]; B.ocell = h->pre_cell[b]; B.ocol = h->pre_col[b]; B.onode = onode;
    B.obci = obci; B.obcj = obcj; B.obck = obck;
    long long box = (long long)B.NX * B.NY * B.NZ;
    if (box >= (1LL << 31)) return OCFD_ERR_ARG;  // the kernels decode block-local indices in 32 bits
    h->max_box_b = std::max(h->max_box_b, box);
    h->pre_box[b + 1] = h->pre_box[b] + box;
    h->pre_face[b + 1] = h->pre_face[b] + (long long)B.nx * B.ny * B.nz;
    h->pre_cell[b + 1] = h->pre_cell[b] + (long long)(B.nx - 1) * (B.ny - 1) * (B.nz - 1);
    h->pre_col[b + 1] = h->pre_col[b] + (long long)(B.ny - 1) * (B.nz - 1);
    h->pre_lnj[b + 1] = h->pre_lnj[b] + (long long)(B.nx - 1) * (B.nz - 1);
    h->pre_lnk[b + 1] = h->pre_lnk[b] + (long long)(B.nx - 1) * (B.ny - 1);
    onode += (long long)B.NXn * B.NYn * B.NZn;
    obci += (long long)(B.ny - 1) * (B.nz - 1);
    obcj += (long long)(B.nx - 1) * (B.nz - 1);
    obck += (long long)(B.nx - 1) * (B.ny - 1);
    h->max_plane = std::max(h->max_plane, B.nx + B.ny + B.nz - 3);
    B.sub0 = (int)h->sub.size(); B.nsub = nsub[b];
    for (int s = 0; s < nsub[b]; s++, q += 21) {
      SubD S;
      S.blk = b;
      S.ib = q[0]; S.ie = q[1]; S.jb = q[2]; S.je = q[3]; S.kb = q[4]; S.ke = q[5]; S.bc = q[6]; S.face = q[7]; S.f_no = q[8];
      S.ib1 = q[9]; S.ie1 = q[10]; S.jb1 = q[11]; S.je1 = q[12]; S.kb1 = q[13]; S.ke1 = q[14]; S.nb1 = q[15] - 1; S.face1 = q[16];
      S.f_no1 = q[17]; S.L1 = q[18]; S.L2 = q[19]; S.L3 = q[20];
      if (S.face < 1 || S.face > 6) return fail(nullptr, OCFD_ERR_ARG, "bad face");
      // partner block numbers are 1-based within the solve
      const int sb0 = h->sblk0[B.solve], sbn = h->sblk0[B.solve + 1] - sb0;
      // nb1 = -1 (partner on another rank) only in a sharded handle
      if (S.bc < 0 && !(h->part && S.nb1 == -1) && (S.nb1 < 0 || S.nb1 >= sbn)) return OCFD_ERR_ARG;
      if (S.bc < 0 && S.nb1 >= 0) S.nb1 += sb0;
      if (S.bc > 0 && !(S.bc == 2 || S.bc == 3 || S.bc == 4 || S.bc == 5 || S.bc == 6 || S.bc == 401)) return OCFD_ERR_UNSUPPORTED;
      h->sub.push_back(S);
    }
  }
  h->tot_box = h->pre_box[nblk]; h->tot_face = h->pre_face[nblk]; h->tot_cell = h->pre_cell[nblk]; h->tot_col = h->pre_col[nblk];
  h->tot_node = onode;
  h->ncell = h->tot_cell;
  h->ncell_s.assign(nsolve, 0);
  for (int b = 0; b < nblk; b++) h->ncell_s[h->blk[b].solve] += h->pre_cell[b + 1] - h->pre_cell[b];
  if (h->part) h->ncell_s[0] = h->part->ncell_global;
  int ns = (int)h->sub.size();
  h->pre_subcell.assign(ns + 1, 0); h->pre_halo.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++) {
    const SubD& S = h->sub[s];
    h->pre_subcell[s + 1] = h->pre_subcell[s] + subcell_count(S);
    long long nh = 0;
    if (S.bc < 0 && S.nb1 >= 0) {
      int kb1[3] = {S.ib1, S.jb1, S.kb1}, ke1[3] = {S.ie1 - 1, S.je1 - 1, S.ke1 - 1};
      int d1 = (S.face1 - 1) % 3;
      if (S.face1 <= 3) kb1[d1] -= LAPH;
      ke1[d1] = kb1[d1] + LAPH - 1;
      nh = (long long)(ke1[0] - kb1[0] + 1) * (ke1[1] - kb1[1] + 1) * (ke1[2] - kb1[2] + 1);
    }
    h->pre_halo[s + 1] = h->pre_halo[s] + nh;
  }
  h->tot_subcell = h->pre_subcell[ns]; h->tot_halo = h->pre_halo[ns];
  h->cspre.assign(nsolve + 1, 0);
  for (int b = 0; b < nblk; b++) {
    long long n = h->pre_cell[b + 1] - h->pre_cell[b];
    for (long long s0 = 0; s0 < n; s0 += 8192) h->cchunk.push_back(make_int4(b, (int)s0, (int)std::min<long long>(8192, n - s0), 0));
    h->cspre[h->blk[b].solve + 1] = (int)h->cchunk.size();
  }
  for (int s = 0; s < ns; s++) {
    if (h->sub[s].bc != 2) continue;
    long long n = subcell_count(h->sub[s]);
    // 512 wall faces per chunk: enough CTAs for a wing's few thousand wall faces
    for (long long s0 = 0; s0 < n; s0 += 512) h->wchunk.push_back(make_int4(s, (int)s0, (int)std::min<long long>(512, n - s0), 0));
  }
  // boundary rounds: round r holds the r-th subface of every block (physical subfaces only); the
  // cells of an entry are the subface's face cells (walls, symmetry) or its inclusive node range
  // (far field, inflow, outflow, extrapolation), as the boundary kernels iterate them
  {
    int maxsub = 0;
    for (const BlkD& B : h->blk) maxsub = std::max(maxsub, B.nsub);
    for (int r = 0; r < maxsub; r++) {
      int e0 = (int)h->bc_ent.size();
      long long cells = 0;
      for (int b = 0; b < nblk; b++) {
        const BlkD& B = h->blk[b];
        if (r >= B.nsub) continue;
        const SubD& S = h->sub[B.sub0 + r];
        if (S.bc <= 0) continue;
        long long n;
        if (S.bc == 4 || S.bc == 5 || S.bc == 6 || S.bc == 401)
          n = (long long)(S.ie - S.ib + 1) * (S.je - S.jb + 1) * (S.ke - S.kb + 1);
        else
          n = subcell_count(S);
        if (n <= 0) continue;
        h->bc_pre.push_back(cells);
        h->bc_ent.push_back(B.sub0 + r);
        cells += n;
      }
      h->bc_pre.push_back(cells);  // closing entry of the round
      h->bc_ent.push_back(-1);
      h->bc_rounds.push_back(e0); h->bc_rounds.push_back((int)h->bc_ent.size() - 1); h->bc_rounds.push_back((int)cells);
    }
  }
  // interface copies.  update_buffer_onemesh copies subface after subface in block order, each
  // through its own buffer (sub_update_buffer_mpi.f90:55-140).  When no copy touches cells that
  // another copy writes (every block at least LAP cells thick across its interfaces) the order is
  // immaterial and one launch does them all.  Otherwise copy t is placed one level after every
  // earlier copy whose target it reads or writes, and no earlier than any earlier copy that reads
  // its target; each level gathers all its sources before it scatters.
  long long max_level_cells = 0;
  {
    struct Rng { int b, lo[3], hi[3]; };
    auto ranges = [](const SubD& S, Rng& R, Rng& W) {
      int kb[3] = {S.ib, S.jb, S.kb}, ke[3] = {S.ie - 1, S.je - 1, S.ke - 1};
      int d = (S.face - 1) % 3;
      if (S.face > 3) kb[d] -= LAPH;
      ke[d] = kb[d] + LAPH - 1;
      int kb1[3] = {S.ib1, S.jb1, S.kb1}, ke1[3] = {S.ie1 - 1, S.je1 - 1, S.ke1 - 1};
      int d1 = (S.face1 - 1) % 3;
      if (S.face1 <= 3) kb1[d1] -= LAPH;
      ke1[d1] = kb1[d1] + LAPH - 1;
      R.b = S.blk; W.b = S.nb1;
      for (int a = 0; a < 3; a++) { R.lo[a] = kb[a]; R.hi[a] = ke[a]; W.lo[a] = kb1[a]; W.hi[a] = ke1[a]; }
    };
    auto meet = [](const Rng& a, const Rng& b) {
      if (a.b != b.b) return false;
      for (int q = 0; q < 3; q++)
        if (a.hi[q] < b.lo[q] || b.hi[q] < a.lo[q]) return false;
      return true;
    };
    std::vector<int> inner;
    std::vector<Rng> R, W;
    for (int s = 0; s < ns; s++) {
      if (h->sub[s].bc >= 0 || h->pre_halo[s + 1] == h->pre_halo[s]) continue;
      Rng r, w;
      ranges(h->sub[s], r, w);
      inner.push_back(s); R.push_back(r); W.push_back(w);
    }
    const int ni = (int)inner.size();
    std::vector<int> lvl(ni, 0);
    bool ordered = false;
    for (int t = 0; t < ni; t++) {
      if (meet(R[t], W[t])) ordered = true;
      for (int q = 0; q < t; q++) {
        if (meet(W[q], R[t]) || meet(W[q], W[t])) { lvl[t] = std::max(lvl[t], lvl[q] + 1); ordered = true; }
        if (meet(R[q], W[t])) { lvl[t] = std::max(lvl[t], lvl[q]); ordered = true; }
      }
    }
    if (ordered) {
      const int nl = ni ? *std::max_element(lvl.begin(), lvl.end()) + 1 : 0;
      for (int v = 0; v < nl; v++) {
        const int e0 = (int)h->halo_ent.size();
        long long cells = 0;
        for (int t = 0; t < ni; t++) {
          if (lvl[t] != v) continue;
          h->halo_pre.push_back(cells);
          h->halo_ent.push_back(inner[t]);
          cells += h->pre_halo[inner[t] + 1] - h->pre_halo[inner[t]];
        }
        h->halo_pre.push_back(cells);
        h->halo_ent.push_back(-1);
        h->halo_levels.push_back(e0); h->halo_levels.push_back((int)h->halo_ent.size() - 1); h->halo_levels.push_back((int)cells);
        max_level_cells = std::max(max_level_cells, cells);
      }
    }
  }
  // physical-face flags (set_BcK, sub_init.f90:545-577)
  std::vector<unsigned char> bci(obci, 0), bcj(obcj, 0), bck(obck, 0);
  for (const SubD& S : h->sub) {
    if (S.bc < 0) continue;
    const BlkD& B = h->blk[S.blk];
    unsigned char bit = S.face <= 3 ? 1 : 2;
    if (S.face == 1 || S.face == 4) for (int k = S.kb; k <= S.ke - 1; k++) for (int j = S.jb; j <= S.je - 1; j++) bci[B.obci + (j - 1) + (long long)(B.ny - 1) * (k - 1)] |= bit;
    if (S.face == 2 || S.face == 5) for (int k = S.kb; k <= S.ke - 1; k++) for (int i = S.ib; i <= S.ie - 1; i++) bcj[B.obcj + (i - 1) + (long long)(B.nx - 1) * (k - 1)] |= bit;
    // k faces also mark bc > 0 (bits 4 / 8): their inviscid flux is the central one of k_inv_kbc
    const unsigned char kbit = bit | (S.bc > 0 ? (unsigned char)(bit << 2) : 0);
    if (S.face == 3 || S.face == 6) for (int j = S.jb; j <= S.je - 1; j++) for (int i = S.ib; i <= S.ie - 1; i++) bck[B.obck + (i - 1) + (long long)(B.nx - 1) * (j - 1)] |= kbit;
  }
  // block faces whose every face cell carries a physical condition (the region tables below)
  h->phys.assign((size_t)nblk * 6, 0);
  for (int b = 0; b < nblk; b++) {
    const BlkD& B = h->blk[b];
    const int n[3] = {B.nx - 1, B.ny - 1, B.nz - 1};
    for (int d = 0; d < 3; d++) {
      const int na = d == 0 ? n[1] : n[0], nb = d == 2 ? n[1] : n[2];
      const unsigned char* f = d == 0 ? &bci[B.obci] : (d == 1 ? &bcj[B.obcj] : &bck[B.obck]);
      for (int side = 0; side < 2; side++) {
        bool all = true;
        for (long long l = 0; l < (long long)na * nb && all; l++) all = (f[l] & (side == 0 ? 1 : 2)) != 0;
        h->phys[b * 6 + d * 2 + side] = all;
      }
    }
  }
  region_tables(h);
  const std::vector<int4> tiles = tile_table(h);
  h->ntile = (int)tiles.size();
  h->tot_r1 = 0;
  h->pre_r1.assign(nblk + 1, 0);
  for (int b = 0; b < nblk; b++) {
    BlkD& B = h->blk[b];
    B.or1 = h->pre_r1[b];
    h->pre_r1[b + 1] = h->pre_r1[b] + (long long)(B.nx + 1) * (B.ny + 1) * (B.nz + 1);
  }
  h->tot_r1 = h->pre_r1[nblk];
  // node coordinates + ghost layer
  std::vector<std::vector<double>> X(nblk);
  for (int b = 0; b < nblk; b++) {
    const BlkD& B = h->blk[b];
    size_t nn = (size_t)B.NXn * B.NYn * B.NZn;
    X[b].assign(3 * nn, 0.0);
    size_t np = (size_t)B.nx * B.ny * B.nz;
    for (int c = 0; c < 3; c++)
      for (int k = 1; k <= B.nz; k++)
        for (int j = 1; j <= B.ny; j++)
          for (int i = 1; i <= B.nx; i++)
            X[b][c * nn + i + (size_t)B.NXn * (j + (size_t)B.NYn * k)] = xyz[b][c * np + (i - 1) + (size_t)B.nx * ((j - 1) + (size_t)B.ny * (k - 1))];
  }
  if (h->part) X = h->part->X;  // ghost layer from the whole case, across rank boundaries too
  else coordinate_ghosts(h->blk, h->sub, X);
  std::vector<double> hx(onode), hy(onode), hz(onode);
  for (int b = 0; b < nblk; b++) {
    const BlkD& B = h->blk[b];
    size_t nn = (size_t)B.NXn * B.NYn * B.NZn;
    std::memcpy(&hx[B.onode], &X[b][0], nn * 8);
    std::memcpy(&hy[B.onode], &X[b][nn], nn * 8);
    std::memcpy(&hz[B.onode], &X[b][2 * nn], nn * 8);
  }
  std::vector<double> Xw;
  std::vector<long long> wpre(nsolve + 1, 0);  // wall nodes of solve q: [wpre[q], wpre[q+1])
  int turb = h->sps[0].turb;
  bool need_dw = turb != 0 && !(dw && dw[0]);
  if (need_dw && h->part) {  // the wall nodes of every rank's blocks
    Xw = h->part->Xw;
    wpre[1] = (long long)(Xw.size() / 3);
  } else if (need_dw) {
    for (int sq_ = 0; sq_ < nsolve; sq_++) {
     for (const SubD& S : h->sub) {
      if (S.bc != 2 || h->blk[S.blk].solve != sq_) continue;
      const BlkD& B = h->blk[S.blk];
      for (int k = S.kb; k <= S.ke; k++)
        for (int j = S.jb; j <= S.je; j++)
          for (int i = S.ib; i <= S.ie; i++) {
            size_t o = (size_t)i + (size_t)B.NXn * ((size_t)j + (size_t)B.NYn * k);
            size_t nn = (size_t)B.NXn * B.NYn * B.NZn;
            Xw.push_back(X[S.blk][o]); Xw.push_back(X[S.blk][nn + o]); Xw.push_back(X[S.blk][2 * nn + o]);
          }
     }
     wpre[sq_ + 1] = (long long)(Xw.size() / 3);
    }
  }
  X.clear();
  // ---- device memory
  cudaError_t e = cudaSuccess;
  DevMem& M = h->mem;
  const long long tb = h->tot_box, tf = h->tot_face, tc = h->tot_cell;
  const int NV = h->nvar;
  const size_t ts = h->prec == OCFD_PREC_MIXED ? sizeof(float) : sizeof(double);
  h->d_blk = M.alloc<BlkD>(nblk, e);
  h->d_sub = M.alloc<SubD>(std::max(1, ns), e);
  h->d_sp = M.alloc<SolveP>(nsolve, e);
  // block hints of the box, cell and face index spaces (find_blk_h)
  auto hints = [&](const std::vector<long long>& pre) { return hint_table(pre, nblk); };
  const std::vector<int> hint_box = hints(h->pre_box), hint_cell = hints(h->pre_cell), hint_face = hints(h->pre_face);
  const std::vector<int> hint_reg = hints(h->pre_reg), hint_r1 = hints(h->pre_r1);
  h->d_hint_reg = M.alloc<int>(hint_box.size(), e);  // the largest a reset_solve can make it
  h->d_tiles = M.alloc<int4>(tiles.size(), e);
  h->d_hint_r1 = M.alloc<int>(hint_r1.size(), e);
  h->d_pre_reg = M.alloc<long long>(nblk + 1, e);
  h->d_pre_r1 = M.alloc<long long>(nblk + 1, e);
  h->d_hint_box = M.alloc<int>(hint_box.size(), e);
  h->d_hint_cell = M.alloc<int>(hint_cell.size(), e);
  h->d_hint_face = M.alloc<int>(hint_face.size(), e);
  h->d_pre_box = M.alloc<long long>(nblk + 1, e); h->d_pre_cell = M.alloc<long long>(nblk + 1, e);
  h->d_pre_face = M.alloc<long long>(nblk + 1, e); h->d_pre_col = M.alloc<long long>(nblk + 1, e);
  h->d_pre_lnj = M.alloc<long long>(nblk + 1, e); h->d_pre_lnk = M.alloc<long long>(nblk + 1, e);
  h->d_pre_subcell = M.alloc<long long>(ns + 1, e); h->d_pre_halo = M.alloc<long long>(ns + 1, e);
  h->d_cspre = M.alloc<int>(nsolve + 1, e);
  h->d_bc_ent = M.alloc<int>(std::max<size_t>(1, h->bc_ent.size()), e);
  h->d_bc_pre = M.alloc<long long>(std::max<size_t>(1, h->bc_pre.size()), e);
  if (!h->halo_levels.empty()) {
    h->d_halo_ent = M.alloc<int>(h->halo_ent.size(), e);
    h->d_halo_pre = M.alloc<long long>(h->halo_pre.size(), e);
    h->d_halo_stage = M.alloc<double>((size_t)NV * max_level_cells, e);
  }
  h->d_cchunk = M.alloc<int4>(h->cchunk.size(), e); h->d_wchunk = M.alloc<int4>(std::max<size_t>(1, h->wchunk.size()), e);
  h->d_x = M.alloc<double>(onode, e); h->d_y = M.alloc<double>(onode, e); h->d_z = M.alloc<double>(onode, e);
  h->d_Md = M.alloc<double>((size_t)M_COUNT * tf, e);
  h->d_vold = M.alloc<double>(tc, e); h->d_dtmd = M.alloc<double>(tc, e); h->d_dwd = M.alloc<double>(tc, e);
  h->d_xc = M.alloc<double>(tb, e); h->d_yc = M.alloc<double>(tb, e); h->d_zc = M.alloc<double>(tb, e);
  h->d_bci = M.alloc<unsigned char>(obci, e); h->d_bcj = M.alloc<unsigned char>(obcj, e); h->d_bck = M.alloc<unsigned char>(obck, e);
  h->d_U = M.alloc<double>((size_t)NV * tb, e);
  if (p->time_method != 0) h->d_Un = M.alloc<double>((size_t)NV * tb, e);
  if (p->time_method == -1) h->d_Un1 = M.alloc<double>((size_t)NV * tb, e);
  h->d_sfac = M.alloc<double>(2, e);
  h->d_DU = M.alloc<double>((size_t)std::max(NV, 5) * tc, e);
  h->d_P = M.alloc<char>(ts * P_COUNT * tb, e);
  h->d_mu = M.alloc<char>(ts * tb, e);
  h->d_mut = M.alloc<char>(ts * tb, e);
  if (turb == 3) { h->d_Kt = M.alloc<char>(ts * tb, e); h->d_Wt = M.alloc<char>(ts * tb, e); h->d_f1 = M.alloc<char>(ts * tf, e); }
  h->d_Res = M.alloc<char>(ts * NV * tc, e);
  h->d_dt = M.alloc<char>(ts * tc, e);
  h->d_Lc = M.alloc<char>(ts * 3 * tc, e);
  h->d_Lv = M.alloc<char>(ts * 3 * tc, e);
  h->d_Fi = M.alloc<char>(std::max(ts * 15 * tf, sizeof(double) * 3 * tf), e);
  if (p->if_viscous) h->d_Fv = M.alloc<char>(ts * 12 * tf, e);
  if (turb != 0) h->d_Ft = M.alloc<char>(ts * 6 * tf, e);
  h->d_flags = M.alloc<int>(4 * nblk, e);
  h->d_norm_part = M.alloc<double>(14 * h->cchunk.size(), e);
  h->d_norm_out = M.alloc<double>(14 * h->nsolve, e);
  h->d_force_part = M.alloc<double>(9 * std::max<size_t>(1, h->wchunk.size()), e);
  h->d_nan = M.alloc<unsigned long long>(1, e);
  h->d_stage = M.alloc<double>((size_t)NV * h->max_box_b, e);
  if (h->prec == OCFD_PREC_MIXED) {
    h->d_Mf = M.alloc<float>((size_t)M_COUNT * tf, e);
    h->d_volf = M.alloc<float>(tc, e); h->d_dtmf = M.alloc<float>(tc, e); h->d_dwf = M.alloc<float>(tc, e);
  }
  double* d_Xw = nullptr;
  long long* d_wpre = nullptr;
  WallChunk* d_wch = nullptr;
  int* d_wcpre = nullptr;
  std::vector<WallChunk> wch;
  std::vector<int> wcpre(nsolve + 1, 0);
  if (need_dw) {
    for (int q = 0; q < nsolve; q++) {
      for (long long w0 = wpre[q]; w0 < wpre[q + 1]; w0 += 64) {
        WallChunk C;
        C.w0 = w0; C.w1 = std::min(w0 + 64, wpre[q + 1]);
        for (int a = 0; a < 3; a++) { C.lo[a] = 1e300; C.hi[a] = -1e300; }
        for (long long w = C.w0; w < C.w1; w++)
          for (int a = 0; a < 3; a++) { C.lo[a] = std::min(C.lo[a], Xw[3 * w + a]); C.hi[a] = std::max(C.hi[a], Xw[3 * w + a]); }
        wch.push_back(C);
      }
      wcpre[q + 1] = (int)wch.size();
    }
  }
  if (need_dw) {  // a handle without wall nodes still runs the search: every distance is then 1e8
    d_Xw = M.alloc<double>(std::max<size_t>(3, Xw.size()), e); d_wpre = M.alloc<long long>(nsolve + 1, e);
    d_wch = M.alloc<WallChunk>(std::max<size_t>(1, wch.size()), e); d_wcpre = M.alloc<int>(nsolve + 1, e);
  }
  if (e != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "allocation"); }
  // ---- uploads
  if ((e = up(h->d_blk, h->blk)) || (e = up(h->d_sub, h->sub)) || (e = up(h->d_sp, h->sps)) ||
      (e = up(h->d_hint_box, hint_box)) || (e = up(h->d_hint_cell, hint_cell)) || (e = up(h->d_hint_face, hint_face)) ||
      (e = up(h->d_pre_box, h->pre_box)) || (e = up(h->d_pre_cell, h->pre_cell)) || (e = up(h->d_pre_face, h->pre_face)) ||
      (e = up(h->d_pre_reg, h->pre_reg)) || (e = up(h->d_pre_r1, h->pre_r1)) || (e = up(h->d_hint_reg, hint_reg)) ||
      (e = up(h->d_hint_r1, hint_r1)) || (e = up(h->d_tiles, tiles)) ||
      (e = up(h->d_pre_col, h->pre_col)) || (e = up(h->d_pre_subcell, h->pre_subcell)) || (e = up(h->d_pre_halo, h->pre_halo)) ||
      (e = up(h->d_pre_lnj, h->pre_lnj)) || (e = up(h->d_pre_lnk, h->pre_lnk)) ||
      (e = up(h->d_cchunk, h->cchunk)) || (e = up(h->d_cspre, h->cspre)) || (e = up(h->d_bc_ent, h->bc_ent)) || (e = up(h->d_bc_pre, h->bc_pre)) || (e = up(h->d_wchunk, h->wchunk)) || (e = up(h->d_x, hx)) || (e = up(h->d_y, hy)) ||
      (e = up(h->d_z, hz)) || (e = up(h->d_bci, bci)) || (e = up(h->d_bcj, bcj)) || (e = up(h->d_bck, bck))) {
    M.release();
    return cuda_fail(nullptr, e, "upload");
  }
  if (!h->halo_levels.empty()) { up(h->d_halo_ent, h->halo_ent); up(h->d_halo_pre, h->halo_pre); }
  if (d_Xw) {
    if (!Xw.empty()) cudaMemcpy(d_Xw, Xw.data(), Xw.size() * 8, cudaMemcpyHostToDevice);
    up(d_wpre, wpre); up(d_wcpre, wcpre);
    if (!wch.empty()) up(d_wch, wch);
  }
  if (dw && dw[0] && turb != 0) {
    std::vector<double> hdw(tc);
    for (int b = 0; b < nblk; b++) std::memcpy(&hdw[h->pre_cell[b]], dw[b], (h->pre_cell[b + 1] - h->pre_cell[b]) * 8);
    cudaMemcpy(h->d_dwd, hdw.data(), tc * 8, cudaMemcpyHostToDevice);
  }
  reset_mu(h);
  if ((e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)) != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "stream"); }
  // ---- geometry on the device
  GeoArgs G;
  G.blk = h->d_blk; G.nblk = nblk; G.pre_face = h->d_pre_face; G.pre_cell = h->d_pre_cell; G.pre_box = h->d_pre_box;
  G.tot_face = tf; G.tot_cell = tc; G.tot_box = tb; G.tot_node = onode;
  G.x = h->d_x; G.y = h->d_y; G.z = h->d_z; G.M = h->d_Md; G.scratch = (double*)h->d_Fi;
  G.vol = h->d_vold; G.dtm = h->d_dtmd; G.dw = h->d_dwd; G.xc = h->d_xc; G.yc = h->d_yc; G.zc = h->d_zc;
  G.Xw = d_Xw; G.nwall = need_dw ? (long long)(Xw.size() / 3) : 0; G.wpre = d_wpre; G.wch = d_wch; G.wcpre = d_wcpre;
  if ((e = run_geometry(G, h->st)) != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "geometry"); }
  if (h->prec == OCFD_PREC_MIXED) {
    convert_to_float(h->d_Md, h->d_Mf, (long long)M_COUNT * tf, h->st);
    convert_to_float(h->d_vold, h->d_volf, tc, h->st);
    convert_to_float(h->d_dtmd, h->d_dtmf, tc, h->st);
    convert_to_float(h->d_dwd, h->d_dwf, tc, h->st);
  }
  if ((e = cudaStreamSynchronize(h->st)) != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "geometry sync"); }
  // ---- LU-SGS wavefront tiles: TJ x TK = TC columns per CTA, ordered by J+K.  Tables are built
  //      for both tile widths (TC = 32 and 64); the faster one on this case is picked at the end
  //      of creation (OCFD_LU_TC=32|64 fixes it; the one-thread-per-column form uses TC = 64)
  const int lu_v2 = std::getenv("OCFD_LU_V2") ? 1 : 0;
  int lu_force = 0;
  if (const char* e2 = std::getenv("OCFD_LU_TC")) lu_force = std::atoi(e2) == 64 ? 64 : 32;
  if (lu_v2) lu_force = 64;
  h->d_lu_err = M.alloc<int>(1, e);
  int* d_counter = M.alloc<int>(2, e);
  for (int v = 0; v < 2; v++) {
    const int tcv = v == 0 ? 32 : 64;
    int min_nzm = 1 << 30;
    for (const BlkD& B : h->blk) min_nzm = std::min(min_nzm, B.nz - 1);
    int TK = min_nzm <= 2 ? 2 : (min_nzm <= 4 ? 4 : 8);
    if (tcv == 32 && TK == 8) TK = 4;
    int TJ = tcv / TK;
    std::vector<int> tile_of(3 * nblk);
    std::vector<std::pair<int, LuTile>> order;
    std::vector<LuTile> tiles;
    int first = 0;
    for (int b = 0; b < nblk; b++) {
      const BlkD& B = h->blk[b];
      int nJ = (B.ny - 1 + TJ - 1) / TJ, nK = (B.nz - 1 + TK - 1) / TK;
      tile_of[3 * b] = first; tile_of[3 * b + 1] = nJ; tile_of[3 * b + 2] = nK;
      for (int K = 0; K < nK; K++)
        for (int J = 0; J < nJ; J++) order.push_back({J + K, LuTile{b, 1 + J * TJ, 1 + K * TK, 0}});
      first += nJ * nK;
    }
    // within a level (tiles that do not wait on one another) the longer tiles first, so that the
    // blocks with the longest i-lines start their march early
    auto longer = [&](const LuTile& a, const LuTile& c) { return h->blk[a.blk].nx > h->blk[c.blk].nx; };
    std::stable_sort(order.begin(), order.end(), [&](const std::pair<int, LuTile>& a, const std::pair<int, LuTile>& b) {
      return a.first != b.first ? a.first < b.first : longer(a.second, b.second);
    });
    for (auto& o : order) tiles.push_back(o.second);
    std::vector<std::pair<int, LuTile>> rorder(order.begin(), order.end());
    std::stable_sort(rorder.begin(), rorder.end(), [&](const std::pair<int, LuTile>& a, const std::pair<int, LuTile>& b) {
      // the upper sweep: a tile waits on the next level's tiles of its block (J+1, K+1)
      const int la = -(a.first + 0), lb = -(b.first + 0);
      return la != lb ? la < lb : longer(a.second, b.second);
    });
    std::vector<LuTile> rtiles;
    for (auto& o : rorder) rtiles.push_back(o.second);
    // the upper sweep's order when both sweeps share one launch: by the step at which a tile could
    // start (its block's lower sweep done, then the skew of its upstream tiles); an upstream tile
    // (J+1 or K+1) always sorts strictly earlier, so every wait is on a tile handed out before
    std::vector<std::pair<long long, LuTile>> uorder;
    for (const LuTile& t : tiles) {
      const BlkD& B = h->blk[t.blk];
      const int nJ = tile_of[3 * t.blk + 1], nK = tile_of[3 * t.blk + 2];
      const int J = (t.j0 - 1) / TJ, K = (t.k0 - 1) / TK;
      const long long lower_done = (long long)(nJ - 1) * TJ + (long long)(nK - 1) * TK + (B.nx - 1 + TJ + TK - 2);
      uorder.push_back({lower_done + (long long)(nJ - 1 - J) * TJ + (long long)(nK - 1 - K) * TK, t});
    }
    std::stable_sort(uorder.begin(), uorder.end(), [](const std::pair<long long, LuTile>& a, const std::pair<long long, LuTile>& b) { return a.first < b.first; });
    std::vector<LuTile> utiles;
    for (auto& o : uorder) utiles.push_back(o.second);
    LuTile* d_tiles = M.alloc<LuTile>(tiles.size(), e);
    LuTile* d_utiles = M.alloc<LuTile>(utiles.size(), e);
    LuTile* d_rtiles = M.alloc<LuTile>(rtiles.size(), e);
    int* d_tile_of = M.alloc<int>(tile_of.size(), e);
    int* d_progress = M.alloc<int>(first, e);
    int* d_progress_up = M.alloc<int>(first, e);
    int* d_blkdone = M.alloc<int>(nblk, e);
    if (e != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "lu tables"); }
    cudaMemcpy(d_tiles, tiles.data(), tiles.size() * sizeof(LuTile), cudaMemcpyHostToDevice);
    cudaMemcpy(d_utiles, utiles.data(), utiles.size() * sizeof(LuTile), cudaMemcpyHostToDevice);
    cudaMemcpy(d_rtiles, rtiles.data(), rtiles.size() * sizeof(LuTile), cudaMemcpyHostToDevice);
    cudaMemcpy(d_tile_of, tile_of.data(), tile_of.size() * sizeof(int), cudaMemcpyHostToDevice);
    LuArgs& L = h->lu_var[v];
    L.tiles = d_tiles; L.rtiles = d_rtiles; L.utiles = d_utiles; L.ntiles = first; L.counter = d_counter; L.progress = d_progress;
    L.progress_up = d_progress_up; L.blkdone = d_blkdone;
    L.tile_of = d_tile_of; L.err = h->d_lu_err; L.TJ = TJ; L.TK = TK;
    L.spin_limit = 4000000;  // x ~64 ns: a few hundred ms before a stuck wait gives up
    if (const char* sl = std::getenv("OCFD_LU_SPIN_LIMIT")) L.spin_limit = std::max(0LL, std::atoll(sl));
    // version-5 records for the 64-column table: tiles in block order and their first records
    if (v == 1 && !h->part && std::getenv("OCFD_LU_V5")) {
      std::vector<LuTile> tmy(first);
      std::vector<long long> rec0(first + 1, 0);
      for (int b = 0; b < nblk; b++) {
        const BlkD& B = h->blk[b];
        const int nJ = tile_of[3 * b + 1], nK = tile_of[3 * b + 2];
        for (int K = 0; K < nK; K++)
          for (int J = 0; J < nJ; J++) {
            const int q = tile_of[3 * b] + J + nJ * K;
            tmy[q] = LuTile{b, 1 + J * TJ, 1 + K * TK, 0};
            rec0[q + 1] = (B.nx - 1 + TJ + TK - 2) + 2;
          }
      }
      for (int q = 0; q < first; q++) rec0[q + 1] += rec0[q];
      LuStream& S = h->lus;
      lu5_layout_for(h->prec, NV, S, TJ * TK, (TJ + 2) * (TK + 2));
      const long long nrec = rec0[first];
      LuTile* d_tmy = M.alloc<LuTile>(tmy.size(), e);
      long long* d_rec0 = M.alloc<long long>(rec0.size(), e);
      S.dyn = M.alloc<unsigned char>((size_t)nrec * S.dyn_bytes, e);
      S.geo = M.alloc<unsigned char>((size_t)nrec * S.geo_bytes, e);
      S.dus = (double*)M.alloc<unsigned char>((size_t)nrec * S.dus_bytes, e);
      if (e != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "lu records"); }
      cudaMemcpy(d_tmy, tmy.data(), tmy.size() * sizeof(LuTile), cudaMemcpyHostToDevice);
      cudaMemcpy(d_rec0, rec0.data(), rec0.size() * sizeof(long long), cudaMemcpyHostToDevice);
      S.tmy = d_tmy;
      S.rec0 = d_rec0;
      h->lus_v = 1;
    }
  }
  // ---- runner
  h->info.nvar = NV; h->info.time_method = p->time_method; h->info.viscous = p->if_viscous; h->info.turb = turb;
  h->info.smoothing = p->if_residual_smoothing;
  h->info.max_plane = h->max_plane;
  h->info.ncchunk = (int)h->cchunk.size(); h->info.nwchunk = (int)h->wchunk.size();
  h->info.lu_planes = std::getenv("OCFD_LUSGS_PLANES") ? 1 : 0;
  h->info.bc_rounds = h->bc_rounds.data(); h->info.nround = (int)(h->bc_rounds.size() / 3);
  h->info.halo_levels = h->halo_levels.data(); h->info.nhlevel = (int)(h->halo_levels.size() / 3);
  h->info.halo_ent = h->d_halo_ent; h->info.halo_pre = h->d_halo_pre; h->info.halo_stage = h->d_halo_stage;
  if (h->part) {
    PartCtx& Pc = *h->part;
    const long long ns_cells = Pc.send_pre.back(), nr_cells = Pc.recv_pre.back();
    Pc.d_send_ent = M.alloc<int>(std::max<size_t>(1, Pc.send_ent.size()), e);
    Pc.d_send_pre = M.alloc<long long>(Pc.send_pre.size(), e);
    Pc.d_recv_sub = M.alloc<SubD>(std::max<size_t>(1, Pc.recv_sub.size()), e);
    Pc.d_recv_pre = M.alloc<long long>(Pc.recv_pre.size(), e);
    Pc.d_send = M.alloc<double>((size_t)NV * std::max(1LL, ns_cells), e);
    Pc.d_recv = M.alloc<double>((size_t)NV * std::max(1LL, nr_cells), e);
    if (e != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "exchange buffers"); }
    if (!Pc.send_ent.empty()) up(Pc.d_send_ent, Pc.send_ent);
    up(Pc.d_send_pre, Pc.send_pre);
    if (!Pc.recv_sub.empty()) up(Pc.d_recv_sub, Pc.recv_sub);
    up(Pc.d_recv_pre, Pc.recv_pre);
    for (long long& o : Pc.send_off) o *= NV;
    for (long long& o : Pc.recv_off) o *= NV;
    h->info.exchange = part_exchange; h->info.exchange_ctx = h;
    h->info.xs_ent = Pc.d_send_ent; h->info.xs_pre = Pc.d_send_pre; h->info.nxs = (int)Pc.send_ent.size(); h->info.xs_cells = ns_cells;
    h->info.xr_sub = Pc.d_recv_sub; h->info.xr_pre = Pc.d_recv_pre; h->info.nxr = (int)Pc.recv_sub.size(); h->info.xr_cells = nr_cells;
    h->info.xsend = Pc.d_send; h->info.xrecv = Pc.d_recv;
  }
  h->info.recon_prim = 1;
  for (int q = 0; q < nsolve; q++) if (ps[q].iflag_reconstruction != 0) h->info.recon_prim = 0;
  h->info.int_scheme = ps[0].iflag_scheme;
  h->info.int_flux = ps[0].iflag_flux;
  for (int q = 1; q < nsolve; q++) {
    if (ps[q].iflag_scheme != h->info.int_scheme) h->info.int_scheme = -1;
    if (ps[q].iflag_flux != h->info.int_flux) h->info.int_flux = -1;
  }
  {
    const char* fz = std::getenv("OCFD_RES_FUSED");  // the tile forms of the residual (opt-in: slower on config 2)
    h->info.res_fused = fz ? std::max(0, std::min(3, std::atoi(fz))) : 0;

    // the SA residual as one tile kernel (config 2 FP64 residual 1.85 -> 1.82 ms); OCFD_SA_SPLIT
    // restores the face-flux kernels + k_sa_res
    h->info.sa_fused = std::getenv("OCFD_SA_SPLIT") ? 0 : 1;
    // the viscosity / turbulence chain on a second, high-priority stream beside the inviscid fluxes
    // (config 2 FP64 step 3.32 -> 3.25 ms, mixed 2.50 -> 2.44, 64-airfoil batch 3.55 -> 3.45).
    // OCFD_RES_STREAMS=0: the whole residual on the handle's stream; 1: the inviscid fluxes on the
    // second stream, at the default priority
    const char* rs = std::getenv("OCFD_RES_STREAMS");
    h->info.res_streams = rs ? std::max(0, std::min(2, std::atoi(rs))) : 2;
  }
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  if (h->prec == OCFD_PREC_MIXED) fill_arena<float>(h, h->A32, h->d_Mf, h->d_volf, h->d_dtmf, h->d_dwf);
  else fill_arena<double>(h, h->A64, h->d_Md, h->d_vold, h->d_dtmd, h->d_dwd);
  // LU-SGS kernel candidates: OCFD_LU_TC fixes the tile width, OCFD_LU_V3 / OCFD_LU_V4 the
  // wavefront version (OCFD_LU_V2 both); the autotuner picks among the rest.  OCFD_LU_ONE_LAUNCH
  // replaces version 4 by its one-launch form (candidate 6: k_lusgs_wave4_ul)
  const int lu_ver_force = lu_v2 ? 2 : (std::getenv("OCFD_LU_V3") ? 3 : (std::getenv("OCFD_LU_V4") ? 4 : (std::getenv("OCFD_LU_V5") ? 5 : 0)));
  const bool lu_one = std::getenv("OCFD_LU_ONE_LAUNCH") != nullptr;
  std::vector<std::pair<int, int>> lu_cand;
  for (int v = 0; v < 2; v++) {
    if (lu_force && (lu_force == 64) != (v == 1)) continue;
    for (int ver : {5, 4, 3}) {
      if (lu_ver_force && ver != lu_ver_force) continue;
      if (ver == 5 && (h->lus_v != v || lu_ver_force != 5)) continue;
      lu_cand.push_back({v, ver == 4 && lu_one ? 6 : ver});
    }
  }
  if (lu_cand.empty()) lu_cand.push_back({1, 4});
  if (lu_ver_force == 2) lu_cand.assign(1, {1, 2});
  select_lu(h, lu_cand[0].first, lu_cand[0].second);
  if (!h->run) { M.release(); return OCFD_ERR_UNSUPPORTED; }
  if (lu_cand.size() > 1 && !h->info.lu_planes && !std::getenv("OCFD_NO_AUTOTUNE")) {
    if (h->part) h->part->xchg = false;  // the timed steps are discarded: no exchange with other ranks
    autotune_lu(h, lu_cand);
    if (h->part) h->part->xchg = true;
  }
  h->run->init_flow(h->st);
  if (p->time_method == -1) h->run->dual_init(h->st);
  if ((e = cudaStreamSynchronize(h->st)) != cudaSuccess) { M.release(); return cuda_fail(nullptr, e, "init"); }
  int bcerr = 0;
  {
    std::vector<int> fl(4 * nblk);
    cudaMemcpy(fl.data(), h->d_flags, fl.size() * 4, cudaMemcpyDeviceToHost);
    for (int b = 0; b < nblk; b++) bcerr |= fl[3 * nblk + b];
  }
  if (bcerr) { M.release(); return OCFD_ERR_UNSUPPORTED; }
  if (h->part && h->part->comm_err) { M.release(); return OCFD_ERR_COMM; }
  *out = hp.release();
  return OCFD_OK;
}

extern "C" int ocfd_create(const ocfd_params* p, int nblk, const int* nijk, const double* const* xyz, const int* nsub, const int* inc,
                           const double* const* dw, ocfd_handle** out) {
  if (!p || nblk <= 0) return OCFD_ERR_ARG;
  return create_impl(p, 1, &nblk, nijk, xyz, nsub, inc, dw, out);
}

extern "C" int ocfd_create_batch(const ocfd_params* ps, int nsolve, const int* nblk, const int* nijk, const double* const* xyz,
                                 const int* nsub, const int* inc, const double* const* dw, ocfd_handle** out) {
  return create_impl(ps, nsolve, nblk, nijk, xyz, nsub, inc, dw, out);
}

// ---- block-sharded handles ------------------------------------------------------------------
// The whole case is described on every rank (as every MPI rank of the reference knows the whole
// block list and .inc table); the node ghost layer and the wall nodes are taken from the whole
// case here, then the rank's blocks go through create_impl with interfaces to other ranks marked
// (partner -1) and the exchange lists attached.
// whole-case block and subface tables of a sharded case (0-based partner blocks)
static int parse_whole(int nblk, const int* nijk, const int* nsub, const int* inc, const int* owner, std::vector<BlkD>& fb,
                       std::vector<SubD>& fs, std::vector<int>& fsub0) {
  fb.assign(nblk, BlkD{});
  fs.clear();
  fsub0.assign(nblk + 1, 0);
  const int* q = inc;
  for (int b = 0; b < nblk; b++) {
    BlkD& B = fb[b];
    B.nx = nijk[3 * b]; B.ny = nijk[3 * b + 1]; B.nz = nijk[3 * b + 2];
    if (B.nx < 2 || B.ny < 2 || B.nz < 2 || owner[b] < 0 || nsub[b] < 0) return OCFD_ERR_ARG;
    B.NX = B.nx + 7; B.NY = B.ny + 7; B.NZ = B.nz + 7;
    B.NXn = B.nx + 2; B.NYn = B.ny + 2; B.NZn = B.nz + 2;
    fsub0[b] = (int)fs.size();
    for (int r = 0; r < nsub[b]; r++, q += 21) {
      SubD S{};
      S.blk = b;
      S.ib = q[0]; S.ie = q[1]; S.jb = q[2]; S.je = q[3]; S.kb = q[4]; S.ke = q[5]; S.bc = q[6]; S.face = q[7]; S.f_no = q[8];
      S.ib1 = q[9]; S.ie1 = q[10]; S.jb1 = q[11]; S.je1 = q[12]; S.kb1 = q[13]; S.ke1 = q[14]; S.nb1 = q[15] - 1; S.face1 = q[16];
      S.f_no1 = q[17]; S.L1 = q[18]; S.L2 = q[19]; S.L3 = q[20];
      if (S.face < 1 || S.face > 6 || (S.bc < 0 && (S.nb1 < 0 || S.nb1 >= nblk || S.face1 < 1 || S.face1 > 6))) return OCFD_ERR_ARG;
      fs.push_back(S);
    }
  }
  fsub0[nblk] = (int)fs.size();
  // interfaces between ranks: both blocks at least LAP cells thick across them, so that no copy
  // between ranks reads a ghost cell another copy writes
  auto thick = [&](int b, int face) {
    const BlkD& B = fb[b];
    int n = (face - 1) % 3 == 0 ? B.nx : ((face - 1) % 3 == 1 ? B.ny : B.nz);
    return n - 1 >= LAPH;
  };
  for (const SubD& S : fs)
    if (S.bc < 0 && owner[S.blk] != owner[S.nb1] && (!thick(S.blk, S.face) || !thick(S.nb1, S.face1))) return OCFD_ERR_UNSUPPORTED;
  return OCFD_OK;
}

// the exchange lists of one rank, per peer in ascending rank order; within a peer both sides list
// the copies in the whole case's subface order (block by block, subface by subface), so the
// sender's and the receiver's entries line up; sizes in cells (the target's LAP ghost layers)
static void make_plan(const std::vector<SubD>& fs, const std::vector<int>& fsub0, const int* owner, int nblk, int rank,
                      const std::vector<int>& glob2loc, const std::vector<int>& lsub0, PartCtx& Pc) {
  auto target_cells = [](const SubD& S) {
    int kb1[3] = {S.ib1, S.jb1, S.kb1}, ke1[3] = {S.ie1 - 1, S.je1 - 1, S.ke1 - 1};
    int d1 = (S.face1 - 1) % 3;
    if (S.face1 <= 3) kb1[d1] -= LAPH;
    ke1[d1] = kb1[d1] + LAPH - 1;
    return (long long)(ke1[0] - kb1[0] + 1) * (ke1[1] - kb1[1] + 1) * (ke1[2] - kb1[2] + 1);
  };
  int nrank = 0;
  for (int b = 0; b < nblk; b++) nrank = std::max(nrank, owner[b] + 1);
  Pc.send_pre.assign(1, 0); Pc.recv_pre.assign(1, 0); Pc.send_off.assign(1, 0); Pc.recv_off.assign(1, 0);
  Pc.send_ent.clear(); Pc.recv_sub.clear(); Pc.peers.clear();
  for (int peer = 0; peer < nrank; peer++) {
    if (peer == rank) continue;
    bool any = false;
    for (int t = 0; t < (int)fs.size(); t++) {
      const SubD& S = fs[t];
      if (S.bc < 0 && owner[S.blk] == rank && owner[S.nb1] == peer) {  // outgoing: local source, target on the peer
        Pc.send_ent.push_back(lsub0[glob2loc[S.blk]] + (t - fsub0[S.blk]));
        Pc.send_pre.push_back(Pc.send_pre.back() + target_cells(S));
        any = true;
      }
    }
    for (int t = 0; t < (int)fs.size(); t++) {
      const SubD& S = fs[t];
      if (S.bc < 0 && owner[S.blk] == peer && owner[S.nb1] == rank) {  // incoming: source on the peer, local target
        SubD R = S;
        R.blk = -1;
        R.nb1 = glob2loc[S.nb1];
        Pc.recv_sub.push_back(R);
        Pc.recv_pre.push_back(Pc.recv_pre.back() + target_cells(S));
        any = true;
      }
    }
    if (!any) continue;
    Pc.peers.push_back(peer);
    Pc.send_off.push_back(Pc.send_pre.back());
    Pc.recv_off.push_back(Pc.recv_pre.back());
  }
}

static void local_numbering(int nblk, const int* owner, int rank, const int* nsub, std::vector<int>& loc2glob, std::vector<int>& glob2loc,
                            std::vector<int>& lsub0) {
  loc2glob.clear();
  glob2loc.assign(nblk, -1);
  for (int b = 0; b < nblk; b++)
    if (owner[b] == rank) { glob2loc[b] = (int)loc2glob.size(); loc2glob.push_back(b); }
  lsub0.assign(loc2glob.size() + 1, 0);
  for (size_t l = 0; l < loc2glob.size(); l++) lsub0[l + 1] = lsub0[l] + nsub[loc2glob[l]];
}

extern "C" int ocfd_part_plan(int nblk, const int* nijk, const int* nsub, const int* inc, const int* owner, int rank, int* peers,
                              long long* send_off, long long* recv_off) {
  if (nblk <= 0 || !nijk || !nsub || !inc || !owner || rank < 0) return OCFD_ERR_ARG;
  std::vector<BlkD> fb;
  std::vector<SubD> fs;
  std::vector<int> fsub0, glob2loc, lsub0;
  if (int rc = parse_whole(nblk, nijk, nsub, inc, owner, fb, fs, fsub0)) return rc;
  PartCtx Pc;
  local_numbering(nblk, owner, rank, nsub, Pc.loc2glob, glob2loc, lsub0);
  make_plan(fs, fsub0, owner, nblk, rank, glob2loc, lsub0, Pc);
  const int np = (int)Pc.peers.size();
  for (int q = 0; q < np; q++)
    if (peers) peers[q] = Pc.peers[q];
  for (int q = 0; q <= np; q++) {
    if (send_off) send_off[q] = Pc.send_off[q];
    if (recv_off) recv_off[q] = Pc.recv_off[q];
  }
  return np;
}

// ---- block-sharded handles ------------------------------------------------------------------
// The whole case is described on every rank (as every MPI rank of the reference knows the whole
// block list and .inc table); the node ghost layer and the wall nodes are taken from the whole
// case here, then the rank's blocks go through create_impl with interfaces to other ranks marked
// (partner -1) and the exchange lists attached.
extern "C" int ocfd_create_part(const ocfd_params* p, int nblk, const int* nijk, const double* const* xyz, const int* nsub,
                                const int* inc, const double* const* dw, const int* owner, int rank, const ocfd_comm* comm,
                                ocfd_handle** out) {
  if (!p || nblk <= 0 || !nijk || !xyz || !nsub || !inc || !owner || !comm || !comm->exchange || !comm->allreduce || !out || rank < 0)
    return OCFD_ERR_ARG;
  std::unique_ptr<PartCtx> Pc(new PartCtx());
  Pc->rank = rank;
  Pc->comm = *comm;
  std::vector<BlkD> fb;
  std::vector<SubD> fs;
  std::vector<int> fsub0, glob2loc, lsub0;
  if (int rc = parse_whole(nblk, nijk, nsub, inc, owner, fb, fs, fsub0)) return rc;
  local_numbering(nblk, owner, rank, nsub, Pc->loc2glob, glob2loc, lsub0);
  if (Pc->loc2glob.empty()) return OCFD_ERR_ARG;
  for (const BlkD& B : fb) Pc->ncell_global += (long long)(B.nx - 1) * (B.ny - 1) * (B.nz - 1);
  // node coordinates with the ghost layer, from the whole case: this rank's blocks and the blocks
  // whose nodes their ghost layer copies
  std::vector<std::vector<double>> X(nblk);
  for (int b = 0; b < nblk; b++) {
    const BlkD& B = fb[b];
    if (owner[b] != rank) {
      bool touches = false;
      for (int t = fsub0[b]; t < fsub0[b + 1]; t++) touches |= fs[t].bc < 0 && owner[fs[t].nb1] == rank;
      if (!touches) continue;
    }
    size_t nn = (size_t)B.NXn * B.NYn * B.NZn, np = (size_t)B.nx * B.ny * B.nz;
    X[b].assign(3 * nn, 0.0);
    for (int c = 0; c < 3; c++)
      for (int k = 1; k <= B.nz; k++)
        for (int j = 1; j <= B.ny; j++)
          for (int i = 1; i <= B.nx; i++)
            X[b][c * nn + i + (size_t)B.NXn * (j + (size_t)B.NYn * k)] = xyz[b][c * np + (i - 1) + (size_t)B.nx * ((j - 1) + (size_t)B.ny * (k - 1))];
  }
  {
    std::vector<SubD> used;  // copies into this rank's blocks and the physical faces of its blocks, in order
    for (const SubD& S : fs)
      if ((S.bc < 0 && owner[S.nb1] == rank) || (S.bc >= 0 && owner[S.blk] == rank)) used.push_back(S);
    coordinate_ghosts(fb, used, X);
  }
  for (int b : Pc->loc2glob) Pc->X.push_back(std::move(X[b]));
  // wall nodes of the whole case (comput_dw searches the walls of every block)
  for (const SubD& S : fs) {
    if (S.bc != OCFD_BC_WALL) continue;
    const BlkD& B = fb[S.blk];
    size_t np = (size_t)B.nx * B.ny * B.nz;
    for (int k = S.kb; k <= S.ke; k++)
      for (int j = S.jb; j <= S.je; j++)
        for (int i = S.ib; i <= S.ie; i++) {
          size_t o = (size_t)(i - 1) + (size_t)B.nx * ((size_t)(j - 1) + (size_t)B.ny * (k - 1));
          for (int c = 0; c < 3; c++) Pc->Xw.push_back(xyz[S.blk][c * np + o]);
        }
  }
  make_plan(fs, fsub0, owner, nblk, rank, glob2loc, lsub0, *Pc);
  // the local case: this rank's blocks, interfaces to other ranks with partner 0 (-1 after the
  // 1-based conversion)
  const int nl = (int)Pc->loc2glob.size();
  std::vector<int> lnijk, lnsub, linc;
  std::vector<const double*> lxyz, ldw;
  for (int l = 0; l < nl; l++) {
    const int b = Pc->loc2glob[l];
    lnijk.insert(lnijk.end(), nijk + 3 * b, nijk + 3 * b + 3);
    lxyz.push_back(xyz[b]);
    if (dw && dw[0]) ldw.push_back(dw[b]);
    lnsub.push_back(nsub[b]);
    for (int t = fsub0[b]; t < fsub0[b + 1]; t++) {
      const int* r = inc + 21 * (size_t)t;
      const size_t o = linc.size();
      linc.insert(linc.end(), r, r + 21);
      if (fs[t].bc < 0) linc[o + 15] = owner[fs[t].nb1] == rank ? glob2loc[fs[t].nb1] + 1 : 0;
    }
  }
  return create_impl(p, 1, &nl, lnijk.data(), lxyz.data(), lnsub.data(), linc.data(), ldw.empty() ? nullptr : ldw.data(), out,
                     std::move(Pc));
}

extern "C" int ocfd_part_blocks(const ocfd_handle* h, int* global_ids) {
  if (!h) return 0;
  for (int b = 0; b < h->nblk; b++)
    if (global_ids) global_ids[b] = h->part ? h->part->loc2glob[b] : b;
  return h->nblk;
}

extern "C" int ocfd_nsolve(const ocfd_handle* h) { return h ? h->nsolve : 0; }

extern "C" long long ocfd_footprint(const ocfd_params* p, int nblk, const int* nijk) {
  if (!p || nblk <= 0 || !nijk) return -1;
  long long tb = 0, tf = 0, tc = 0, tn = 0, maxbox = 0;
  for (int b = 0; b < nblk; b++) {
    long long nx = nijk[3 * b], ny = nijk[3 * b + 1], nz = nijk[3 * b + 2];
    if (nx < 2 || ny < 2 || nz < 2) return -1;
    long long box = (nx + 7) * (ny + 7) * (nz + 7);
    tb += box; tf += nx * ny * nz; tc += (nx - 1) * (ny - 1) * (nz - 1); tn += (nx + 2) * (ny + 2) * (nz + 2);
    maxbox = std::max(maxbox, box);
  }
  const int tm = p->if_viscous ? p->iflag_turbulence_model : 0;
  const long long NV = tm == 2 ? 6 : (tm == 3 ? 7 : 5);
  const long long ts = p->precision == OCFD_PREC_MIXED ? 4 : 8;
  long long bytes = 0;
  bytes += 3 * tn * 8 + M_COUNT * tf * 8 + 3 * tc * 8 + 3 * tb * 8;              // geometry (FP64)
  bytes += NV * tb * 8 * (p->time_method == 0 ? 1 : (p->time_method == -1 ? 3 : 2)) + std::max(NV, 5LL) * tc * 8;  // U, Un, Un1, DU
  bytes += ts * (P_COUNT + 2) * tb + ts * (NV + 7) * tc;                          // P, mu, mut, Res, dt, Lc, Lv
  bytes += std::max(ts * 15 * tf, 24 * tf) + (p->if_viscous ? ts * 12 * tf : 0) + (tm ? ts * 6 * tf : 0);
  if (tm == 3) bytes += ts * (2 * tb + tf);
  if (p->precision == OCFD_PREC_MIXED) bytes += 4 * (M_COUNT * tf + 3 * tc);
  bytes += NV * maxbox * 8;                                                       // state staging
  if (std::getenv("OCFD_LU_V5")) {                                                // LU-SGS version-5 records
    int min_nzm = 1 << 30;
    for (int b = 0; b < nblk; b++) min_nzm = std::min(min_nzm, nijk[3 * b + 2] - 1);
    const int TK = min_nzm <= 2 ? 2 : (min_nzm <= 4 ? 4 : 8), TJ = 64 / TK;
    LuStream S{};
    lu5_layout_for(p->precision, (int)NV, S, 64, (TJ + 2) * (TK + 2));
    long long nrec = 0;
    for (int b = 0; b < nblk; b++) {
      const long long nJ = (nijk[3 * b + 1] - 1 + TJ - 1) / TJ, nK = (nijk[3 * b + 2] - 1 + TK - 1) / TK;
      nrec += nJ * nK * (nijk[3 * b] - 1 + TJ + TK);
    }
    bytes += nrec * (S.dyn_bytes + S.geo_bytes + S.dus_bytes);
  }
  return bytes + bytes / 20 + (16LL << 20);                                       // tables, chunks, margin
}

extern "C" int ocfd_synchronize(ocfd_handle* h) {
  if (!h) return OCFD_ERR_ARG;
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "synchronize");
  return OCFD_OK;
}

extern "C" int ocfd_destroy(ocfd_handle* h) {
  if (!h) return OCFD_OK;
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->h_pin) cudaFreeHost(h->h_pin);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->run.reset();
  h->mem.release();
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return OCFD_OK;
}

extern "C" const char* ocfd_last_error(const ocfd_handle* h) { return h ? h->err.c_str() : "null handle"; }

extern "C" long long ocfd_state_size(const ocfd_handle* h, int b) {
  if (!h || b < 0 || b >= h->nblk) return -1;
  const BlkD& B = h->blk[b];
  return (long long)h->nvar * B.NX * B.NY * B.NZ;
}

extern "C" int ocfd_set_state(ocfd_handle* h, int b, const double* U) {
  if (!h || !U || b < 0 || b >= h->nblk) return OCFD_ERR_ARG;
  const BlkD& B = h->blk[b];
  long long box = (long long)B.NX * B.NY * B.NZ;
  cudaError_t e = cudaMemcpyAsync(h->d_stage, U, (size_t)h->nvar * box * 8, cudaMemcpyHostToDevice, h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "set_state");
  h->run->scatter_state(h->st, b, h->d_stage, box);
  if (h->P.time_method == -1) h->run->dual_init(h->st);  // a restart sets both earlier time levels
  if ((e = cudaStreamSynchronize(h->st)) != cudaSuccess) return cuda_fail(h, e, "set_state");
  return OCFD_OK;
}

extern "C" int ocfd_get_state(ocfd_handle* h, int b, double* U) {
  if (!h || !U || b < 0 || b >= h->nblk) return OCFD_ERR_ARG;
  const BlkD& B = h->blk[b];
  long long box = (long long)B.NX * B.NY * B.NZ;
  h->run->gather_state(h->st, b, h->d_stage, box);
  cudaError_t e = cudaMemcpyAsync(U, h->d_stage, (size_t)h->nvar * box * 8, cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "get_state");
  return OCFD_OK;
}

// a slot of a batch given a new case on the same mesh: the solve's constants, its arrays that carry
// history from step to step (mu and mu_t with their never-recomputed edge ghosts, the SST k, omega
// and f1 planes, the limiter flags) back to their state after allocation, then freestream, BC,
// halo and corners on its blocks; the other solves and the captured step graph are untouched
extern "C" int ocfd_reset_solve(ocfd_handle* h, int q, const ocfd_params* p) {
  if (!h || !p || q < 0 || q >= h->nsolve) return OCFD_ERR_ARG;
  if (h->part) return fail(h, OCFD_ERR_UNSUPPORTED, "reset_solve: not for sharded handles");
  if (p->time_method == -1) return fail(h, OCFD_ERR_UNSUPPORTED, "reset_solve: dual time keeps per-handle history (use a new handle)");
  std::vector<ocfd_params> ps = h->Ps;
  ps[q] = *p;
  if (int rc = check_params(ps.data(), h->nsolve)) return fail(h, rc, "reset_solve: parameters incompatible with the handle's other solves");
  // the step's kernels were picked for the handle's reconstruction and, for WENO5 / MUSCL3 with
  // Roe in every solve, compiled with the Roe flux (RunInfo::recon_prim / int_scheme / int_flux)
  if (h->info.recon_prim && p->iflag_reconstruction != 0)
    return fail(h, OCFD_ERR_UNSUPPORTED, "reset_solve: the handle reconstructs primitive variables only");
  const bool roe_fixed = h->info.recon_prim && h->info.int_flux == OCFD_FLUX_ROE &&
                         (h->info.int_scheme == OCFD_SCHEME_WENO5 || h->info.int_scheme == OCFD_SCHEME_MUSCL3);
  if (roe_fixed && p->iflag_flux != OCFD_FLUX_ROE)
    return fail(h, OCFD_ERR_UNSUPPORTED, "reset_solve: the handle's step is built for the Roe flux");
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "reset_solve");
  h->Ps[q] = *p;
  fill_solve(*p, h->nvar, h->sps[q]);
  const int b0 = h->sblk0[q], b1 = h->sblk0[q + 1];
  const long long x0 = h->pre_box[b0], x1 = h->pre_box[b1], f0 = h->pre_face[b0], f1 = h->pre_face[b1];
  const size_t ts = h->prec == OCFD_PREC_MIXED ? sizeof(float) : sizeof(double);
  std::vector<char> mu((size_t)(x1 - x0) * ts);
  for (long long l = 0; l < x1 - x0; l++) {
    if (ts == 4) ((float*)mu.data())[l] = (float)(1.0 / p->re);
    else ((double*)mu.data())[l] = 1.0 / p->re;
  }
  region_tables(h);  // the boundary scheme sets how many ghost layers the primitives cover
  const std::vector<int> hint_reg = hint_table(h->pre_reg, h->nblk);
  if (!e) e = cudaMemcpy(h->d_blk, h->blk.data(), sizeof(BlkD) * h->nblk, cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(h->d_pre_reg, h->pre_reg.data(), sizeof(long long) * (h->nblk + 1), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(h->d_hint_reg, hint_reg.data(), sizeof(int) * hint_reg.size(), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(h->d_sp + q, &h->sps[q], sizeof(SolveP), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy((char*)h->d_mu + x0 * ts, mu.data(), mu.size(), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemset((char*)h->d_mut + x0 * ts, 0, (x1 - x0) * ts);
  if (!e && h->d_Kt) e = cudaMemset((char*)h->d_Kt + x0 * ts, 0, (x1 - x0) * ts);
  if (!e && h->d_Wt) e = cudaMemset((char*)h->d_Wt + x0 * ts, 0, (x1 - x0) * ts);
  if (!e && h->d_f1) e = cudaMemset((char*)h->d_f1 + f0 * ts, 0, (f1 - f0) * ts);
  for (int pl = 0; pl < 4 && !e; pl++) e = cudaMemset(h->d_flags + pl * h->nblk + b0, 0, sizeof(int) * (b1 - b0));
  if (e != cudaSuccess) return cuda_fail(h, e, "reset_solve");
  h->run->reset_solve(h->st, q);
  e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "reset_solve");
  return OCFD_OK;
}

extern "C" int ocfd_init_flow(ocfd_handle* h) {
  if (!h) return OCFD_ERR_ARG;
  h->run->init_flow(h->st);
  if (h->P.time_method == -1) h->run->dual_init(h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "init_flow");
  if (h->part && h->part->comm_err) return fail(h, OCFD_ERR_COMM, "halo exchange callback failed");
  h->kstep = 0;
  h->tt = 0.0;
  return OCFD_OK;
}

static int ensure_graph(ocfd_handle* h) {
  if (h->gexec) return OCFD_OK;
  if (std::getenv("OCFD_NO_GRAPH") || h->part) return OCFD_OK;  // a sharded step calls back to the host
  cudaError_t e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(h, e, "capture begin");
  h->run->step(h->st);
  e = cudaStreamEndCapture(h->st, &h->graph);
  if (e != cudaSuccess) return cuda_fail(h, e, "capture end");
  e = cudaGraphInstantiate(&h->gexec, h->graph, 0);
  if (e != cudaSuccess) return cuda_fail(h, e, "graph instantiate");
  return OCFD_OK;
}

// Sfac, Sfac1 of the next residual evaluation of a dual-time handle (the first one of the handle's
// life uses the first-order values, sub_Residual.f90:25-33), copied to the device on its stream
static void dual_factors(ocfd_handle* h) {
  const double dt = h->P.dt_global;
  if (h->dual_started == 0) { h->dual_started = 1; h->sfac_h[0] = 1.0 / (3.0 * dt); h->sfac_h[1] = 1.0 / dt; }
  else { h->sfac_h[0] = 1.0 / (2.0 * dt); h->sfac_h[1] = 3.0 / (2.0 * dt); }
  cudaMemcpyAsync(h->d_sfac, h->sfac_h, 2 * sizeof(double), cudaMemcpyHostToDevice, h->st);
}

static int residual_impl(ocfd_handle* h, double* rmax, double* rrms, int nout);

// NS_Time_Dual_LU_SGS (sub_time_advance.f90:126-202): inner iterations until the largest residual
// RMS of every solve is at most Res_Inner_Limit or Step_Inner_Limit is reached, then the time
// levels shift; the graph holds one inner iteration
static int advance_dual(ocfd_handle* h, int nsteps) {
  std::vector<double> rmax(7 * (size_t)h->nsolve), rrms(7 * (size_t)h->nsolve);
  for (int s = 0; s < nsteps; s++) {
    for (int kt = 1; kt <= h->P.step_inner_limit; kt++) {
      dual_factors(h);
      if (h->gexec) {
        cudaError_t e = cudaGraphLaunch(h->gexec, h->st);
        if (e != cudaSuccess) return cuda_fail(h, e, "graph launch");
      } else {
        h->run->step(h->st);
      }
      int rc = residual_impl(h, rmax.data(), rrms.data(), h->nsolve);
      if (rc) return rc;
      double mx = 0.0;
      for (int q = 0; q < h->nsolve; q++) {
        double m0 = rrms[7 * q];
        for (int m = 0; m < h->nvar; m++) m0 = std::max(m0, rrms[7 * q + m]);
        mx = std::max(mx, m0);
      }
      if (mx <= h->P.res_inner_limit) break;
    }
    h->run->dual_end(h->st);
    h->tt = h->tt + h->P.dt_global;
    h->kstep = h->kstep + 1;
  }
  return OCFD_OK;
}

extern "C" int ocfd_advance(ocfd_handle* h, int nsteps, int* kstep, double* tt) {
  if (!h || nsteps < 0) return OCFD_ERR_ARG;
  int rc = ensure_graph(h);
  if (rc) return rc;
  if (h->P.time_method == -1) {
    rc = advance_dual(h, nsteps);
    if (rc) return rc;
    nsteps = 0;
  }
  for (int s = 0; s < nsteps; s++) {
    if (h->gexec) {
      cudaError_t e = cudaGraphLaunch(h->gexec, h->st);
      if (e != cudaSuccess) return cuda_fail(h, e, "graph launch");
    } else {
      h->run->step(h->st);
    }
    h->tt = h->tt + h->P.dt_global;
    h->kstep = h->kstep + 1;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(h, e, "advance");
  if (h->part && h->part->comm_err) return fail(h, OCFD_ERR_COMM, "halo exchange callback failed");
  if (kstep) *kstep = h->kstep;
  if (tt) *tt = h->tt;
  return OCFD_OK;
}

extern "C" int ocfd_compute_residual(ocfd_handle* h, int with_lusgs) {
  if (!h) return OCFD_ERR_ARG;
  if (h->P.time_method == -1) dual_factors(h);
  h->run->residual(h->st, with_lusgs != 0);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "compute_residual");
  return OCFD_OK;
}

// pinned host area the monitors are read back into (one asynchronous copy each, one wait per call);
// allocated at the first read-back
static double* pin_area(ocfd_handle* h) {
  if (!h->h_pin) {
    const size_t n = 14 * (size_t)h->nsolve + 2 + 9 * std::max<size_t>(1, h->wchunk.size());
    if (cudaMallocHost((void**)&h->h_pin, n * sizeof(double)) != cudaSuccess) h->h_pin = nullptr;
  }
  return h->h_pin;
}

// norms of every solve (nout = 1: solve 0 only); NaN -> OCFD_ERR_NAN with the first location
static int residual_impl(ocfd_handle* h, double* rmax, double* rrms, int nout) {
  double* pin = pin_area(h);
  if (!pin) return fail(h, OCFD_ERR_OOM, "pinned read-back area");
  const size_t no = 14 * (size_t)h->nsolve;
  cudaMemsetAsync(h->d_nan, 0xFF, 8, h->st);  // "no NaN seen": all ones
  h->run->norms(h->st, h->d_norm_part, h->d_norm_out, h->d_nan);
  cudaMemcpyAsync(pin, h->d_norm_out, no * 8, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(pin + no, h->d_nan, 8, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(pin + no + 1, h->d_lu_err, 4, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "residual");
  std::vector<double> out(pin, pin + no);
  unsigned long long nan_at = 0;
  std::memcpy(&nan_at, pin + no, 8);
  int lu_err = 0;
  std::memcpy(&lu_err, pin + no + 1, 4);
  bool other_nan = false, other_lu = false;
  if (h->part) {  // MPI_ALLREDUCE of the maxima and the sums of squares (sub_time_advance.f90:373-374)
    double mx[9], sm[7];
    for (int m = 0; m < 7; m++) { mx[m] = out[m]; sm[m] = out[7 + m]; }
    mx[7] = nan_at != ~0ULL ? 1.0 : 0.0;
    mx[8] = lu_err ? 1.0 : 0.0;
    const ocfd_comm& C = h->part->comm;
    if (C.allreduce(C.user, mx, 9, 1) || C.allreduce(C.user, sm, 7, 0)) return fail(h, OCFD_ERR_COMM, "norm all-reduce callback failed");
    for (int m = 0; m < 7; m++) { out[m] = mx[m]; out[7 + m] = sm[m]; }
    other_nan = mx[7] != 0.0 && nan_at == ~0ULL;
    other_lu = mx[8] != 0.0 && !lu_err;
  }
  for (int q = 0; q < nout; q++)
    for (int m = 0; m < 7; m++) {
      rmax[7 * q + m] = m < h->nvar ? out[14 * q + m] : 0.0;
      rrms[7 * q + m] = m < h->nvar ? std::sqrt(out[14 * q + 7 + m] / (double)h->ncell_s[q]) : 0.0;
    }
  if (lu_err) {
    cudaMemset(h->d_lu_err, 0, 4);
    return fail(h, OCFD_ERR_TIMEOUT, "LU-SGS wavefront: a bounded wait between tiles timed out");
  }
  if (other_lu) return fail(h, OCFD_ERR_TIMEOUT, "LU-SGS wavefront: a bounded wait timed out on another rank");
  if (other_nan) return fail(h, OCFD_ERR_NAN, "NaN in residual on another rank");
  if (nan_at != ~0ULL) {
    long long g = (long long)(nan_at / 8);
    int m = (int)(nan_at % 8);
    int b = (int)(std::upper_bound(h->pre_cell.begin(), h->pre_cell.end(), g) - h->pre_cell.begin()) - 1;
    const BlkD& B = h->blk[b];
    long long l = g - h->pre_cell[b];
    int i = (int)(l % (B.nx - 1)) + 1, j = (int)((l / (B.nx - 1)) % (B.ny - 1)) + 1, k = (int)(l / ((long long)(B.nx - 1) * (B.ny - 1))) + 1;
    char buf[200];
    if (h->part)
      std::snprintf(buf, sizeof buf, "NaN in residual: block %d i,j,k,m = %d %d %d %d", h->part->loc2glob[b] + 1, i, j, k, m + 1);
    else if (h->nsolve > 1)
      std::snprintf(buf, sizeof buf, "NaN in residual: solve %d block %d i,j,k,m = %d %d %d %d", B.solve, b - h->sblk0[B.solve] + 1, i, j, k, m + 1);
    else
      std::snprintf(buf, sizeof buf, "NaN in residual: block %d i,j,k,m = %d %d %d %d", b + 1, i, j, k, m + 1);
    return fail(h, OCFD_ERR_NAN, buf);
  }
  return OCFD_OK;
}

extern "C" int ocfd_residual(ocfd_handle* h, double* rmax, double* rrms) {
  if (!h || !rmax || !rrms) return OCFD_ERR_ARG;
  return residual_impl(h, rmax, rrms, 1);
}

extern "C" int ocfd_residual_all(ocfd_handle* h, double* rmax, double* rrms) {
  if (!h || !rmax || !rrms) return OCFD_ERR_ARG;
  return residual_impl(h, rmax, rrms, h->nsolve);
}

// ---- residual norms without any allocation --------------------------------------------------
// ocfd_residual_static uses one statically sized device area per device, shared by every handle
// of the process: per-chunk partial max / sum of squares, per-solve totals, and the NaN location.
// Each call overwrites all partials and totals it reads; only the NaN location must start at its
// sentinel (all ones), which the call resets on the handle's stream before the norm kernels.
// each block's interior cells are cut into norm chunks of at most 8192 cells, so 4096 chunks hold
// 33,554,432 cells only when the blocks are large; a handle of many small blocks reaches 4096
// chunks with fewer cells
constexpr int kStaticNormChunks = 4096;
constexpr int kStaticNormSolves = 256;
static __device__ __align__(256) double g_static_norm[(kStaticNormChunks + kStaticNormSolves) * 14];
static __device__ __align__(256) unsigned long long g_static_nan;

__global__ void k_static_nan_reset(unsigned long long* nan_at) { *nan_at = ~0ULL; }

namespace {
struct StaticNormArea {
  double* part = nullptr;
  double* out = nullptr;
  unsigned long long* nan = nullptr;
};
constexpr int kMaxDevices = 64;
StaticNormArea g_static_area[kMaxDevices];
std::mutex g_static_mu;
}  // namespace

// device addresses of the static area on the current device (looked up once per device)
static int static_norm_area(ocfd_handle* h, StaticNormArea& a) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail_c(h, e, "residual_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail_c(h, OCFD_ERR_ARG, "residual_static: device ordinal beyond 63");
  std::lock_guard<std::mutex> lk(g_static_mu);
  StaticNormArea& c = g_static_area[dev];
  if (!c.part) {
    void* p = nullptr;
    void* n = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_static_norm)) != cudaSuccess) return cuda_fail_c(h, e, "residual_static: cudaGetSymbolAddress");
    if ((e = cudaGetSymbolAddress(&n, g_static_nan)) != cudaSuccess) return cuda_fail_c(h, e, "residual_static: cudaGetSymbolAddress");
    c.part = (double*)p;
    c.out = (double*)p + (size_t)kStaticNormChunks * 14;
    c.nan = (unsigned long long*)n;
  }
  a = c;
  return OCFD_OK;
}

extern "C" int ocfd_residual_static(ocfd_handle* h, double* rmax, double* rrms) {
  if (!h || !rmax || !rrms) return OCFD_ERR_ARG;
  if (h->part) return fail_c(h, OCFD_ERR_UNSUPPORTED, "residual_static: not for sharded handles (the norms are all-reduced); use ocfd_residual");
  if ((long long)h->cchunk.size() > kStaticNormChunks) {
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "residual_static: the handle has %lld norm chunks (each block's interior cells in chunks of at most 8192), "
                  "more than 4096; use ocfd_residual", (long long)h->cchunk.size());
    return fail_c(h, OCFD_ERR_ARG, buf);
  }
  if (h->nsolve > kStaticNormSolves) return fail_c(h, OCFD_ERR_ARG, "residual_static: the handle has more than 256 solves; use ocfd_residual");
  StaticNormArea a;
  if (int rc = static_norm_area(h, a)) return rc;
  k_static_nan_reset<<<1, 1, 0, h->st>>>(a.nan);
  h->run->norms(h->st, a.part, a.out, a.nan);
  double out[14];
  unsigned long long nan_at = 0;
  int lu_err = 0;
  cudaMemcpyAsync(out, a.out, sizeof(out), cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(&nan_at, a.nan, 8, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(&lu_err, h->d_lu_err, 4, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail_c(h, e, "residual_static");
  for (int m = 0; m < 7; m++) {
    rmax[m] = m < h->nvar ? out[m] : 0.0;
    rrms[m] = m < h->nvar ? std::sqrt(out[7 + m] / (double)h->ncell_s[0]) : 0.0;
  }
  if (lu_err) {
    cudaMemsetAsync(h->d_lu_err, 0, 4, h->st);
    cudaStreamSynchronize(h->st);
    return fail_c(h, OCFD_ERR_TIMEOUT, "LU-SGS wavefront: a bounded wait between tiles timed out");
  }
  if (nan_at != ~0ULL) return fail_c(h, OCFD_ERR_NAN, "NaN in residual (location: ocfd_residual)");
  return OCFD_OK;
}

// forces of every solve: partial sums per wall chunk, then per block in subface order, then over
// the solve's blocks (sub_Post.f90:31-202)
static int forces_impl(ocfd_handle* h, double* ft, double* cl, double* cd, double* cs, int nout) {
  size_t nw = h->wchunk.size();
  double* pin = pin_area(h);
  if (!pin) return fail(h, OCFD_ERR_OOM, "pinned read-back area");
  double* pf = pin + 14 * (size_t)h->nsolve + 2;
  std::vector<double> part(9 * std::max<size_t>(nw, 1), 0.0);
  if (nw) {
    h->run->forces(h->st, h->d_force_part);
    cudaMemcpyAsync(pf, h->d_force_part, nw * 9 * 8, cudaMemcpyDeviceToHost, h->st);
  }
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "forces");
  if (nw) std::copy(pf, pf + 9 * nw, part.begin());
  std::vector<double> blk(9 * h->nblk, 0.0);
  for (size_t c = 0; c < nw; c++) {
    int b = h->sub[h->wchunk[c].x].blk;
    for (int q = 0; q < 9; q++) blk[9 * b + q] = blk[9 * b + q] + part[9 * c + q];
  }
  for (int sv = 0; sv < nout; sv++) {
    double Ft[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = h->sblk0[sv]; b < h->sblk0[sv + 1]; b++)
      for (int q = 0; q < 9; q++) Ft[q] = Ft[q] + blk[9 * b + q];
    if (h->part && h->part->comm.allreduce(h->part->comm.user, Ft, 9, 0))  // MPI_ALLREDUCE, sub_Post.f90:202
      return fail(h, OCFD_ERR_COMM, "force all-reduce callback failed");
    const ocfd_params& P = h->Ps[sv];
    double* f = ft + 9 * sv;
    for (int q = 0; q < 6; q++) f[q] = 2.0 * Ft[q] / P.ref_s;
    for (int q = 6; q < 9; q++) f[q] = 2.0 * Ft[q] / (P.ref_s * P.ref_l);
    double Fx = f[0] + f[3], Fy = f[1] + f[4], Fz = f[2] + f[5];
    double L, D, S;
    if (P.cood_y_up == 1) { L = Fy * std::cos(P.aoa) - Fx * std::sin(P.aoa); D = Fx * std::cos(P.aoa) + Fy * std::sin(P.aoa); S = Fz; }
    else { L = Fz * std::cos(P.aoa) - Fx * std::sin(P.aoa); D = Fx * std::cos(P.aoa) + Fz * std::sin(P.aoa); S = Fy; }
    if (cl) cl[sv] = L;
    if (cd) cd[sv] = D;
    if (cs) cs[sv] = S;
  }
  return OCFD_OK;
}

extern "C" int ocfd_forces(ocfd_handle* h, double* ft, double* cl, double* cd, double* cs) {
  if (!h || !ft) return OCFD_ERR_ARG;
  return forces_impl(h, ft, cl, cd, cs, 1);
}

extern "C" int ocfd_forces_all(ocfd_handle* h, double* ft, double* cl, double* cd, double* cs) {
  if (!h || !ft) return OCFD_ERR_ARG;
  return forces_impl(h, ft, cl, cd, cs, h->nsolve);
}

extern "C" void* ocfd_stream(ocfd_handle* h) { return h ? (void*)h->st : nullptr; }

// kernel nodes of the captured step graph (memset nodes excluded); without a graph, the count
// the runner derives from its launch sequence
extern "C" int ocfd_launches_per_step(ocfd_handle* h) {
  if (!h) return 0;
  if (ensure_graph(h) == OCFD_OK && h->graph) {
    size_t n = 0;
    if (cudaGraphGetNodes(h->graph, nullptr, &n) == cudaSuccess && n > 0) {
      std::vector<cudaGraphNode_t> nodes(n);
      if (cudaGraphGetNodes(h->graph, nodes.data(), &n) == cudaSuccess) {
        int k = 0;
        for (size_t q = 0; q < n; q++) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
        }
        return k;
      }
    }
  }
  return h->run->launches_per_step();
}

extern "C" int ocfd_profile(ocfd_handle* h, int nsteps, double* phase_ms) {
  if (!h || !phase_ms || nsteps < 1) return OCFD_ERR_ARG;
  cudaEvent_t ev[6];
  for (int q = 0; q < 6; q++) cudaEventCreate(&ev[q]);
  for (int q = 0; q < 8; q++) phase_ms[q] = 0.0;
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < nsteps && e == cudaSuccess; s++) {
    h->run->step(h->st, ev);
    e = cudaStreamSynchronize(h->st);
    float ms[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < 5 && e == cudaSuccess; q++) e = cudaEventElapsedTime(&ms[q], ev[q], ev[q + 1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[5], ev[0], ev[5]);
    for (int q = 0; q < 6; q++) phase_ms[q] += ms[q];
    h->tt = h->tt + h->P.dt_global;
    h->kstep = h->kstep + 1;
  }
  for (int q = 0; q < 6; q++) cudaEventDestroy(ev[q]);
  if (e != cudaSuccess) return cuda_fail(h, e, "profile");
  return OCFD_OK;
}

extern "C" int ocfd_limiter_status(ocfd_handle* h, int b, int* n, int* ov) {
  if (!h || b < 0 || b >= h->nblk) return OCFD_ERR_ARG;
  int a = 0, c = 0;
  cudaMemcpyAsync(&a, h->d_flags + h->nblk + b, 4, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(&c, h->d_flags + b, 4, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return cuda_fail(h, e, "limiter_status");
  if (n) *n = a;
  if (ov) *ov = c;
  return OCFD_OK;
}

// ---- debug / parity array access --------------------------------------------------------
namespace {
struct ArrDesc {
  int space;  // 0 box, 1 face, 2 cell, 3 node
  int nv;
  const void* base;
  bool is_double;
  long long plane;  // plane stride
  int lo[3], hi[3];
};
}  // namespace

static bool describe(const ocfd_handle* h, int b, const std::string& s, ArrDesc& d) {
  const BlkD& B = h->blk[b];
  bool dbl = h->prec != OCFD_PREC_MIXED;
  auto set_box = [&](int l, int hoff) { d.space = 0; for (int q = 0; q < 3; q++) d.lo[q] = l; d.hi[0] = B.nx + hoff; d.hi[1] = B.ny + hoff; d.hi[2] = B.nz + hoff; d.plane = h->tot_box; };
  auto set_face = [&]() { d.space = 1; for (int q = 0; q < 3; q++) d.lo[q] = 1; d.hi[0] = B.nx; d.hi[1] = B.ny; d.hi[2] = B.nz; d.plane = h->tot_face; };
  auto set_cell = [&]() { d.space = 2; for (int q = 0; q < 3; q++) d.lo[q] = 1; d.hi[0] = B.nx - 1; d.hi[1] = B.ny - 1; d.hi[2] = B.nz - 1; d.plane = h->tot_cell; };
  d.nv = 1;
  static const char* mnames[] = {"Si", "Sj", "Sk", "ni1", "ni2", "ni3", "nj1", "nj2", "nj3", "nk1", "nk2", "nk3",
                                 "ix1", "iy1", "iz1", "jx1", "jy1", "jz1", "kx1", "ky1", "kz1", "ix2", "iy2", "iz2", "jx2", "jy2", "jz2", "kx2", "ky2", "kz2",
                                 "ix3", "iy3", "iz3", "jx3", "jy3", "jz3", "kx3", "ky3", "kz3", "ix0", "iy0", "iz0", "jx0", "jy0", "jz0", "kx0", "ky0", "kz0"};
  for (int q = 0; q < 48; q++)
    if (s == mnames[q]) { set_face(); d.base = h->d_Md + (size_t)q * h->tot_face; d.is_double = true; return true; }
  if (s == "U") { set_box(-3, 3); d.nv = h->nvar; d.base = h->d_U; d.is_double = true; return true; }
  if (s == "mu") { set_box(-1, 1); d.base = h->d_mu; d.is_double = dbl; return true; }
  if (s == "mu_t") { set_box(-1, 1); d.base = h->d_mut; d.is_double = dbl; return true; }
  if (s == "xc") { set_box(-3, 3); d.base = h->d_xc; d.is_double = true; return true; }
  if (s == "yc") { set_box(-3, 3); d.base = h->d_yc; d.is_double = true; return true; }
  if (s == "zc") { set_box(-3, 3); d.base = h->d_zc; d.is_double = true; return true; }
  if (s == "vol") { set_cell(); d.base = h->d_vold; d.is_double = true; return true; }
  if (s == "dw") { set_cell(); d.base = h->d_dwd; d.is_double = true; return true; }
  if (s == "dtime_mesh") { set_cell(); d.base = h->d_dtmd; d.is_double = true; return true; }
  if (s == "dt") { set_cell(); d.base = h->d_dt; d.is_double = dbl; return true; }
  if (s == "Res") { set_cell(); d.nv = h->nvar; d.base = h->d_Res; d.is_double = dbl; return true; }
  if (s == "DU") { set_cell(); d.nv = h->nvar; d.base = h->d_DU; d.is_double = true; return true; }
  return false;
}

extern "C" int ocfd_array_shape(const ocfd_handle* h, int b, const char* name, int* lo, int* hi, int* nv) {
  if (!h || !name || b < 0 || b >= h->nblk) return OCFD_ERR_ARG;
  ArrDesc d;
  if (!describe(h, b, name, d)) return OCFD_ERR_ARG;
  for (int q = 0; q < 3; q++) { lo[q] = d.lo[q]; hi[q] = d.hi[q]; }
  *nv = d.nv;
  return OCFD_OK;
}

// copies the array in the requested Fortran bounds; variable-major planes are interleaved back
// to the Fortran (m fastest) order
extern "C" int ocfd_get_array(ocfd_handle* h, int b, const char* name, double* out) {
  if (!h || !name || !out || b < 0 || b >= h->nblk) return OCFD_ERR_ARG;
  ArrDesc d;
  if (!describe(h, b, name, d)) return OCFD_ERR_ARG;
  const BlkD& B = h->blk[b];
  long long off, n0, n1, n2;
  int base_lo;
  if (d.space == 0) { off = B.obox; n0 = B.NX; n1 = B.NY; n2 = B.NZ; base_lo = -3; }
  else if (d.space == 1) { off = B.oface; n0 = B.nx; n1 = B.ny; n2 = B.nz; base_lo = 1; }
  else { off = B.ocell; n0 = B.nx - 1; n1 = B.ny - 1; n2 = B.nz - 1; base_lo = 1; }
  long long cnt = n0 * n1 * n2;
  size_t es = d.is_double ? 8 : 4;
  std::vector<char> tmp(cnt * es * d.nv);
  for (int m = 0; m < d.nv; m++) {
    cudaError_t e = cudaMemcpy(&tmp[m * cnt * es], (const char*)d.base + (size_t)(m * d.plane + off) * es, cnt * es, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(h, e, "get_array");
  }
  long long w0 = d.hi[0] - d.lo[0] + 1, w1 = d.hi[1] - d.lo[1] + 1;
  for (int k = d.lo[2]; k <= d.hi[2]; k++)
    for (int j = d.lo[1]; j <= d.hi[1]; j++)
      for (int i = d.lo[0]; i <= d.hi[0]; i++) {
        long long src = (i - base_lo) + n0 * ((j - base_lo) + n1 * (long long)(k - base_lo));
        long long dst = (i - d.lo[0]) + w0 * ((j - d.lo[1]) + w1 * (long long)(k - d.lo[2]));
        for (int m = 0; m < d.nv; m++) {
          double v = d.is_double ? ((double*)tmp.data())[m * cnt + src] : (double)((float*)tmp.data())[m * cnt + src];
          out[dst * d.nv + m] = v;
        }
      }
  return OCFD_OK;
}
