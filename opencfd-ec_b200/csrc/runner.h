// Step runner interface: one implementation per (flux precision, NVAR), created by
// make_runner_fp64 / make_runner_mixed (solver_fp64.cu, solver_mixed.cu).
#pragma once
#include <cuda_runtime.h>

#include "arena.h"

namespace ocfd {

struct LuArgs;
struct LuStream;

struct RunInfo {
  int nvar, time_method, viscous, turb;
  int smoothing;          // 1: upwind implicit residual smoothing after the assembly
  int max_plane;          // max over blocks of nx+ny+nz-3 (last LU-SGS hyperplane)
  int ncchunk, nwchunk;   // reduction chunk counts
  int lu_planes;          // 1: one launch per hyperplane (reference order); 0: pipelined wavefront
  const LuArgs* lu;       // wavefront tables (host copy of the kernel argument)
  int lu_grid;            // CTAs of the wavefront kernel
  int lu_version;         // 2: one thread per column; 3: four thread groups per column, staged by element; 4: staged by sector;
                          // 5: inputs packed in sweep order, one bulk copy per step (lus)
  const LuStream* lus;    // version 5: record layout and buffers (host copy of the kernel argument)
  int lu5_grid[2];        // version 5: CTAs of the lower / upper sweep (resident CTAs, at most the tiles)
  int lu_tc;              // columns per tile (32 or 64)
  int lu_fused;           // version 4: both sweeps in one launch (k_lusgs_wave4_ul)
  int recon_prim;         // 1: every solve reconstructs primitive variables
  int int_scheme;         // the interior scheme (Iflag_Scheme) if every solve uses the same one, else -1
  int int_flux;           // the flux (Iflag_Flux) if every solve uses the same one, else -1
  int sa_fused;           // 1: the SA fluxes and Res(6) in one tile kernel (k_sa_tile)
  int res_streams;        // 0: one stream; 1: the inviscid fluxes on a second stream beside the viscosity /
                          // turbulence chain; 2: the chain on a second, high-priority stream instead
  int res_fused;          // 0: the NS residual as face-flux kernels + k_assemble; 1: k_ns_tile (all fluxes in the
                          // tile); 2: k_visc_flux, then k_ns_tile with the inviscid fluxes in the tile; 3:
                          // k_inv_flux, then k_ns_tile with the viscous fluxes in the tile
  const int* bc_rounds;   // per boundary round: first entry, end entry, cells
  int nround;
  // ordered interface-copy levels (empty: all copies independent, one launch); per level the
  // first entry, end entry and cells; entries index halo_ent / halo_pre on the device
  const int* halo_levels;
  int nhlevel;
  const int* halo_ent;
  const long long* halo_pre;
  double* halo_stage;     // NV x (largest level) doubles
  // block-sharded handles: copies to other ranks are packed into xsend (entries xs_ent, cell
  // prefix xs_pre), exchange(ctx, stream) hands the buffers over (returns 1 when xrecv holds
  // fresh data to unpack), copies from other ranks are unpacked from xrecv (entries xr_sub)
  int (*exchange)(void* ctx, cudaStream_t st);
  void* exchange_ctx;
  const int* xs_ent;
  const long long* xs_pre;
  int nxs;
  long long xs_cells;
  const SubD* xr_sub;
  const long long* xr_pre;
  int nxr;
  long long xr_cells;
  double* xsend;
  double* xrecv;
};

class Runner {
 public:
  virtual ~Runner() {}
  // one NS_Time_advance (sub_time_advance.f90:6-23) on stream st; when ev is non-null, events
  // ev[0..5] are recorded at the phase boundaries (see ocfd_profile)
  virtual void step(cudaStream_t st, cudaEvent_t* ev = nullptr) = 0;
  // kernel launches of one step
  virtual int launches_per_step() const = 0;
  // residual only (Comput_Residual_one_mesh without LU-SGS), for parity checks
  virtual void residual(cudaStream_t st, bool lusgs) = 0;
  // freestream + BC + halo + corners (init_flow_zero, sub_init.f90:302-410)
  virtual void init_flow(cudaStream_t st) = 0;
  // dual time: Un = Un1 = U (after an initialisation or a restart) / end of a physical step
  // (Un1 = Un, Un = U, then the vt/k/w clamps of NS_Time_advance)
  virtual void dual_init(cudaStream_t st) = 0;
  virtual void dual_end(cudaStream_t st) = 0;
  // BC + halo + corners only
  virtual void bc_halo(cudaStream_t st) = 0;
  // freestream + BC + halo + corners of solve q's blocks only (a batch slot re-initialised)
  virtual void reset_solve(cudaStream_t st, int q) = 0;
  // residual norms: 14 doubles per solve into out (max[7], sum of squares[7])
  virtual void norms(cudaStream_t st, double* part, double* out, unsigned long long* nan_at) = 0;
  // force partial sums: 9 doubles per wall chunk
  virtual void forces(cudaStream_t st, double* part) = 0;
  // version-5 LU-SGS: the static geometry records (once, after the geometry is computed)
  virtual void lu5_pack_geo(cudaStream_t st) = 0;
  // AoS Fortran U(NV, box) of one block <-> device planes
  virtual void scatter_state(cudaStream_t st, int blk, const double* aos, long long box_b) = 0;
  virtual void gather_state(cudaStream_t st, int blk, double* aos, long long box_b) = 0;
};

Runner* make_runner_fp64(const Arena<double>& A, const RunInfo& I);
Runner* make_runner_mixed(const Arena<float>& A, const RunInfo& I);

}  // namespace ocfd
