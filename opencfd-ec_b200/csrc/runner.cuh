// Kernel sequencing of one time step, templated on the flux precision T and NVAR.
#pragma once
#include "lusgs.cuh"
#include "lusgs5.cuh"
#include "runner.h"
#include "solver.cuh"

namespace ocfd {

static inline int grid_of(long long n, int threads = 256) {
  long long g = (n + threads - 1) / threads;
  if (g > 148LL * 16) g = 148LL * 16;
  return g < 1 ? 1 : (int)g;
}

template <class T, int NV>
__global__ void k_scatter_state(Arena<T> A, int b, const double* aos, long long box_b) {
  const BlkD& B = A.blk[b];
  OCFD_GRID_STRIDE(l, box_b) {
#pragma unroll
    for (int m = 0; m < NV; m++) A.U[m * A.tot_box + B.obox + l] = aos[l * NV + m];
  }
}
template <class T, int NV>
__global__ void k_gather_state(Arena<T> A, int b, double* aos, long long box_b) {
  const BlkD& B = A.blk[b];
  OCFD_GRID_STRIDE(l, box_b) {
#pragma unroll
    for (int m = 0; m < NV; m++) aos[l * NV + m] = A.U[m * A.tot_box + B.obox + l];
  }
}

template <class T, int NV>
class RunnerT : public Runner {
 public:
  ~RunnerT() override {
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    if (ev_mu_) cudaEventDestroy(ev_mu_);
    if (st2_) cudaStreamDestroy(st2_);
  }
  RunnerT(const Arena<T>& A, const RunInfo& I) : A_(A), I_(I) {
    if (I.res_streams && I.viscous && !I.res_fused) {
      if (I.res_streams == 2) {  // the chain on a high-priority stream, the inviscid fluxes on the handle's
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        cudaStreamCreateWithPriority(&st2_, cudaStreamNonBlocking, hi);
      } else {
        cudaStreamCreateWithFlags(&st2_, cudaStreamNonBlocking);
      }
      cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming);
      cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming);
      cudaEventCreateWithFlags(&ev_mu_, cudaEventDisableTiming);
    }
    if (I.lu) L_ = *I.lu;
    lu_wave3_prepare<T, NV, false, 32>();
    lu_wave3_prepare<T, NV, true, 32>();
    lu_wave3_prepare<T, NV, false, 64>();
    lu_wave3_prepare<T, NV, true, 64>();
    lu_wave4_prepare<T, NV, false, 32>();
    lu_wave4_prepare<T, NV, true, 32>();
    lu_wave4_prepare<T, NV, false, 64>();
    lu_wave4_prepare<T, NV, true, 64>();
    lu_wave4_ul_prepare<T, NV, 32>();
    lu_wave4_ul_prepare<T, NV, 64>();
    if (I.sa_fused && NV == 6) {
      const size_t sm = sa_smem();
      if (sm > 48 * 1024) cudaFuncSetAttribute(k_sa_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      int occ = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sa_tile<T>, 256, sm);
      sa_grid_ = std::max(1, std::min(A_.ntile, 148 * std::max(1, occ)));
    }
    if (I.res_fused == 3) {
      const size_t sm = sizeof(T) * 5 * ((size_t)A_.tile_maxf + A_.tile_maxc);
      auto kern = k_ns_tile<T, true, -1, -1, true, false>;
      if (sm > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      int occ = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, sm);
      ns_grid_[4] = std::max(1, std::min(A_.ntile, 148 * std::max(1, occ)));
    } else if (I.res_fused) {
      ns_prepare<true, S_WENO5, F_ROE>();
      ns_prepare<true, S_MUSCL3, F_ROE>();
      ns_prepare<true, -1, -1>();
      ns_prepare<false, -1, -1>();
    }
    if (I.lus) {
      S_ = *I.lus;
      if (L_.TJ * L_.TK == 64) { lu_wave5_prepare<T, NV, false, 64>(S_); lu_wave5_prepare<T, NV, true, 64>(S_); }
      else { lu_wave5_prepare<T, NV, false, 32>(S_); lu_wave5_prepare<T, NV, true, 32>(S_); }
    }
  }

  void residual(cudaStream_t st, bool lusgs) override {
    const Arena<T>& A = A_;
    const long long tb = A.tot_box, tf = A.tot_face, tc = A.tot_cell;
    k_prim<T><<<grid_of(tb), 256, 0, st>>>(A);  // sized for the box: the region is read on the device
    // specialised instantiations for the WENO5 / MUSCL3 + Roe pairs (residual phase -3 % on
    // config 2 FP64, -8 % on config 1; MUSCL3 + AUSMPW was measured slower and is left general)
    const bool weno5_roe = I_.recon_prim && I_.int_scheme == S_WENO5 && I_.int_flux == F_ROE;
    const bool muscl3_roe = I_.recon_prim && I_.int_scheme == S_MUSCL3 && I_.int_flux == F_ROE;
    // the inviscid fluxes read only the primitives and the metrics: on two streams they run beside
    // the viscosity / turbulence chain and the viscous fluxes (FP64 arithmetic beside memory
    // latency), joined before the assembly; the chain, the longer path, gets the higher priority
    const bool fork = st2_ != nullptr;
    auto inviscid = [&](cudaStream_t s) {
      if (weno5_roe) inv_flux<true, S_WENO5, F_ROE>(s);
      else if (muscl3_roe) inv_flux<true, S_MUSCL3, F_ROE>(s);
      else if (I_.recon_prim) inv_flux<true, -1, -1>(s);
      else inv_flux<false, -1, -1>(s);
      k_inv_kbc<T><<<grid_of(A.tot_subcell), 256, 0, s>>>(A);
    };
    // cs: the viscosity / turbulence chain and the viscous fluxes; is: the inviscid fluxes
    cudaStream_t cs = st, is = st;
    if (fork) {
      cudaEventRecord(ev_fork_, st);
      cudaStreamWaitEvent(st2_, ev_fork_, 0);
      if (I_.res_streams == 2) cs = st2_;
      else is = st2_;
    }
    if (fork) inviscid(is);
    if (I_.viscous) {
      k_mu<T><<<grid_of(tc), 256, 0, cs>>>(A);
      if (I_.turb == 2 && NV == 6) {
        k_sa_pre<T><<<grid_of(A.tot_r1), 256, 0, cs>>>(A);
        if (I_.sa_fused) {
          k_sa_tile<T><<<sa_grid_, 256, sa_smem(), cs>>>(A);
        } else {
          k_sa_flux<T, 0><<<grid_of(tf), 256, 0, cs>>>(A);
          k_sa_flux<T, 1><<<grid_of(tf), 256, 0, cs>>>(A);
          k_sa_flux<T, 2><<<grid_of(tf), 256, 0, cs>>>(A);
          k_sa_res<T><<<grid_of(tc), 256, 0, cs>>>(A);
        }
        k_mu_finish<T, 1><<<grid_of(A.tot_r1), 256, 0, cs>>>(A);
      } else if (I_.turb == 3 && NV == 7) {
        k_sst_pre<T><<<grid_of(A.tot_r1), 256, 0, cs>>>(A);
        k_sst_src<T><<<grid_of(tc), 256, 0, cs>>>(A);
        k_sst_mut_ghost<T, 0><<<grid_of(tb), 256, 0, cs>>>(A);
        k_sst_mut_ghost<T, 1><<<grid_of(tb), 256, 0, cs>>>(A);
        k_sst_mut_ghost<T, 2><<<grid_of(tb), 256, 0, cs>>>(A);
        k_amut<T><<<grid_of(A.tot_subcell), 256, 0, cs>>>(A);
        k_sst_flux<T, 0><<<grid_of(tf), 256, 0, cs>>>(A);
        k_sst_flux<T, 1><<<grid_of(tf), 256, 0, cs>>>(A);
        k_sst_flux<T, 2><<<grid_of(tf), 256, 0, cs>>>(A);
        k_sst_res<T><<<grid_of(tc), 256, 0, cs>>>(A);
        k_mu_finish<T, 1><<<grid_of(A.tot_r1), 256, 0, cs>>>(A);
      } else {
        cudaMemsetAsync(A.mut, 0, sizeof(T) * tb, cs);
      }
      k_amut<T><<<grid_of(A.tot_subcell), 256, 0, cs>>>(A);
    }
    // forked, FP64: the spectral radii and dt (they need mu and mu_t) follow the inviscid fluxes on
    // their stream, beside the viscous fluxes, and the assembly stores Res only (config 2 step
    // -36 us).  The mixed form keeps them in the assembly: written just before the LU-SGS sweeps,
    // its FP32 Lc, Lv and dt are still in L2 when the sweeps read them (-19 us; batch -47 us)
    const bool ldt_apart = fork && sizeof(T) == 8;
    if (ldt_apart) {
      cudaEventRecord(ev_mu_, cs);
      cudaStreamWaitEvent(is, ev_mu_, 0);
      k_cell_dt<T><<<grid_of(tc), 256, 0, is>>>(A);
    }
    if (I_.res_fused == 3) {
      inviscid(st);
      k_ns_tile<T, true, -1, -1, true, false><<<ns_grid_[4], 256, sizeof(T) * 5 * ((size_t)A.tile_maxf + A.tile_maxc), st>>>(A);
    } else if (I_.res_fused) {
      if (I_.res_fused == 2 && I_.viscous) {
        k_visc_flux<T, 0><<<grid_of(tf), 256, 0, st>>>(A);
        k_visc_flux<T, 1><<<grid_of(tf), 256, 0, st>>>(A);
        k_visc_flux<T, 2><<<grid_of(tf), 256, 0, st>>>(A);
      }
      if (weno5_roe) ns_tile<true, S_WENO5, F_ROE>(st);
      else if (muscl3_roe) ns_tile<true, S_MUSCL3, F_ROE>(st);
      else if (I_.recon_prim) ns_tile<true, -1, -1>(st);
      else ns_tile<false, -1, -1>(st);
    } else {
      if (!fork) inviscid(st);
      if (I_.viscous) {
        // forked: the k-direction viscous fluxes follow the inviscid ones (and k_cell_dt) on their
        // stream once mu and mu_t are final, which evens the two streams (same-box A/B: config 2
        // FP64 step -6 us, mixed -16 us, batch -24 us; moving a second direction measured slower)
        if (fork && !ldt_apart) {
          cudaEventRecord(ev_mu_, cs);
          cudaStreamWaitEvent(is, ev_mu_, 0);
        }
        k_visc_flux<T, 0><<<grid_of(tf), 256, 0, cs>>>(A);
        k_visc_flux<T, 1><<<grid_of(tf), 256, 0, cs>>>(A);
        k_visc_flux<T, 2><<<grid_of(tf), 256, 0, fork ? is : cs>>>(A);
      }
      if (fork) {  // join the second stream back into the handle's
        cudaStream_t other = cs == st ? is : cs;
        cudaEventRecord(ev_join_, other);
        cudaStreamWaitEvent(st, ev_join_, 0);
        if (ldt_apart) k_assemble<T, true><<<grid_of(tc), 256, 0, st>>>(A);
        else k_assemble<T><<<grid_of(tc), 256, 0, st>>>(A);
      } else {
        k_assemble<T><<<grid_of(tc), 256, 0, st>>>(A);
      }
    }
    if (I_.time_method == -1) k_dual_res<T, NV><<<grid_of(tc), 256, 0, st>>>(A);
    if (I_.smoothing) {  // after the spectral radii, before dt (sub_Residual.f90:110-113); dt does not read Res
      k_smooth<T, 0><<<grid_of(A.tot_col, 128), 128, 0, st>>>(A);
      k_smooth<T, 1><<<grid_of(A.tot_lnj, 128), 128, 0, st>>>(A);
      k_smooth<T, 2><<<grid_of(A.tot_lnk, 128), 128, 0, st>>>(A);
    }
    if (lusgs) {
      lusgs_sweep(st, false);
      lusgs_sweep(st, true);
    }
  }

  size_t sa_smem() const { return sizeof(T) * (2 * (size_t)A_.tile_maxf + 2 * (size_t)A_.tile_maxc + (size_t)A_.tile_maxb); }
  template <bool PRIM, int ISCH, int IFLUX>
  size_t ns_smem() const { return sizeof(T) * 5 * ((size_t)A_.tile_maxf + A_.tile_maxc); }
  template <bool PRIM, int ISCH, int IFLUX>
  void ns_prepare() {
    const size_t sm = ns_smem<PRIM, ISCH, IFLUX>();
    auto kern = I_.res_fused == 1 ? k_ns_tile<T, PRIM, ISCH, IFLUX, true> : k_ns_tile<T, PRIM, ISCH, IFLUX, false>;
    if (sm > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, sm);
    ns_grid_[ns_slot<PRIM, ISCH, IFLUX>()] = std::max(1, std::min(A_.ntile, 148 * std::max(1, occ)));
  }
  template <bool PRIM, int ISCH, int IFLUX>
  static constexpr int ns_slot() { return !PRIM ? 3 : (ISCH == S_WENO5 ? 0 : (ISCH == S_MUSCL3 ? 1 : 2)); }
  template <bool PRIM, int ISCH, int IFLUX>
  void ns_tile(cudaStream_t st) {
    const int g = ns_grid_[ns_slot<PRIM, ISCH, IFLUX>()];
    if (I_.res_fused == 1) k_ns_tile<T, PRIM, ISCH, IFLUX, true><<<g, 256, ns_smem<PRIM, ISCH, IFLUX>(), st>>>(A_);
    else k_ns_tile<T, PRIM, ISCH, IFLUX, false><<<g, 256, ns_smem<PRIM, ISCH, IFLUX>(), st>>>(A_);
  }

  template <bool PRIM, int ISCH, int IFLUX>
  void inv_flux(cudaStream_t st) {
    const long long tf = A_.tot_face;
    k_inv_flux<T, 0, PRIM, ISCH, IFLUX><<<grid_of(tf), 256, 0, st>>>(A_);
    k_inv_flux<T, 1, PRIM, ISCH, IFLUX><<<grid_of(tf), 256, 0, st>>>(A_);
    k_inv_flux<T, 2, PRIM, ISCH, IFLUX><<<grid_of(tf), 256, 0, st>>>(A_);
  }

  void lusgs_sweep(cudaStream_t st, bool upper) {
    const Arena<T>& A = A_;
    if (I_.lu_planes) {
      int gc = grid_of(A.tot_col, 128);
      if (!upper) for (int p = 3; p <= I_.max_plane; p++) k_lusgs<T, NV, false><<<gc, 128, 0, st>>>(A, p);
      else for (int p = I_.max_plane; p >= 3; p--) k_lusgs<T, NV, true><<<gc, 128, 0, st>>>(A, p);
    } else {
      if (upper && I_.lu_version == 4 && I_.lu_fused) return;  // ran with the lower sweep's launch
      if (!upper) cudaMemsetAsync(L_.counter, 0, 2 * sizeof(int), st);
      cudaMemsetAsync(L_.progress, 0, sizeof(int) * L_.ntiles, st);
      if (I_.lu_version == 5) {
        const int TC = L_.TJ * L_.TK;
        const int g = I_.lu5_grid[upper ? 1 : 0];
        if (!upper) k_lu_pack_dyn<T, NV><<<dim3(8, L_.ntiles), 256, 0, st>>>(A, S_, L_.TJ, L_.TK);
        if (TC == 64) {
          if (!upper) k_lusgs_wave5<T, NV, false, 64><<<g, 4 * 64 + 32, lu5_smem<T, NV, 64>(S_, false), st>>>(A, L_, S_);
          else k_lusgs_wave5<T, NV, true, 64><<<g, 4 * 64 + 32, lu5_smem<T, NV, 64>(S_, true), st>>>(A, L_, S_);
        } else {
          if (!upper) k_lusgs_wave5<T, NV, false, 32><<<g, 4 * 32 + 32, lu5_smem<T, NV, 32>(S_, false), st>>>(A, L_, S_);
          else k_lusgs_wave5<T, NV, true, 32><<<g, 4 * 32 + 32, lu5_smem<T, NV, 32>(S_, true), st>>>(A, L_, S_);
        }
      } else if (I_.lu_version == 2) {
        if (!upper) k_lusgs_wave<T, NV, false><<<I_.lu_grid, 64, 0, st>>>(A, L_);
        else k_lusgs_wave<T, NV, true><<<I_.lu_grid, 64, 0, st>>>(A, L_);
      } else if (I_.lu_version == 4 && I_.lu_fused) {  // both sweeps in one launch, issued with the lower one
        cudaMemsetAsync(L_.progress_up, 0, sizeof(int) * L_.ntiles, st);
        cudaMemsetAsync(L_.blkdone, 0, sizeof(int) * A.nblk, st);
        if (I_.lu_tc == 64) k_lusgs_wave4_ul<T, NV, 64><<<I_.lu_grid, 4 * 64 + 64, lu_wave4_smem<T, NV, false, 64>(), st>>>(A, L_);
        else k_lusgs_wave4_ul<T, NV, 32><<<I_.lu_grid, 4 * 32 + 64, lu_wave4_smem<T, NV, false, 32>(), st>>>(A, L_);
      } else if (I_.lu_version == 4 && I_.lu_tc == 64) {
        if (!upper) k_lusgs_wave4<T, NV, false, 64><<<I_.lu_grid, 4 * 64 + 64, lu_wave4_smem<T, NV, false, 64>(), st>>>(A, L_);
        else k_lusgs_wave4<T, NV, true, 64><<<I_.lu_grid, 4 * 64 + 64, lu_wave4_smem<T, NV, true, 64>(), st>>>(A, L_);
      } else if (I_.lu_version == 4) {
        if (!upper) k_lusgs_wave4<T, NV, false, 32><<<I_.lu_grid, 4 * 32 + 64, lu_wave4_smem<T, NV, false, 32>(), st>>>(A, L_);
        else k_lusgs_wave4<T, NV, true, 32><<<I_.lu_grid, 4 * 32 + 64, lu_wave4_smem<T, NV, true, 32>(), st>>>(A, L_);
      } else if (I_.lu_tc == 64) {
        if (!upper) k_lusgs_wave3<T, NV, false, 64><<<I_.lu_grid, 4 * 64 + 32, lu_wave3_smem<T, NV, false, 64>(), st>>>(A, L_);
        else k_lusgs_wave3<T, NV, true, 64><<<I_.lu_grid, 4 * 64 + 32, lu_wave3_smem<T, NV, true, 64>(), st>>>(A, L_);
      } else {
        if (!upper) k_lusgs_wave3<T, NV, false, 32><<<I_.lu_grid, 4 * 32 + 32, lu_wave3_smem<T, NV, false, 32>(), st>>>(A, L_);
        else k_lusgs_wave3<T, NV, true, 32><<<I_.lu_grid, 4 * 32 + 32, lu_wave3_smem<T, NV, true, 32>(), st>>>(A, L_);
      }
    }
  }

  void bc_halo(cudaStream_t st) override { bc_halo_with(st, A_); }

  // freestream + BC + halo + corners of solve q's blocks only (the other solves keep their state)
  void reset_solve(cudaStream_t st, int q) override {
    Arena<T> A = A_;
    A.only_solve = q;
    k_init_flow<T, NV><<<grid_of(A.tot_box), 256, 0, st>>>(A);
    bc_halo_with(st, A);
  }

  void bc_halo_with(cudaStream_t st, const Arena<T>& A) {
    for (int r = 0; r < I_.nround; r++) {
      const int* R = I_.bc_rounds + 3 * r;
      if (R[2] > 0) k_bc_round<T, NV><<<grid_of(R[2]), 256, 0, st>>>(A, R[0], R[1], (long long)R[2]);
    }
    if (A.tot_halo > 0 && I_.nhlevel == 0) k_halo<T, NV><<<grid_of(A.tot_halo), 256, 0, st>>>(A);
    for (int v = 0; v < I_.nhlevel; v++) {
      const int* H = I_.halo_levels + 3 * v;
      k_halo_level<T, NV, 0><<<grid_of(H[2]), 256, 0, st>>>(A, I_.halo_ent, I_.halo_pre, H[0], H[1], (long long)H[2], I_.halo_stage);
      k_halo_level<T, NV, 1><<<grid_of(H[2]), 256, 0, st>>>(A, I_.halo_ent, I_.halo_pre, H[0], H[1], (long long)H[2], I_.halo_stage);
    }
    if (I_.exchange) {
      if (I_.xs_cells > 0) k_halo_pack<T, NV><<<grid_of(I_.xs_cells), 256, 0, st>>>(A, I_.xs_ent, I_.xs_pre, I_.nxs, I_.xs_cells, I_.xsend);
      const int fresh = I_.exchange(I_.exchange_ctx, st);
      if (fresh && I_.xr_cells > 0) k_halo_unpack<T, NV><<<grid_of(I_.xr_cells), 256, 0, st>>>(A, I_.xr_sub, I_.xr_pre, I_.nxr, I_.xr_cells, I_.xrecv);
    }
    k_corner<T, NV><<<dim3(A.nblk, 8), 256, 0, st>>>(A);
    k_corner_vtx<T, NV><<<grid_of((long long)A.nblk * NV * 8, 128), 128, 0, st>>>(A);
  }

  void limit(cudaStream_t st) {
    const Arena<T>& A = A_;
    k_limit_fix<T><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
    if (NV == 6) {  // order: the cells above LSAmax first, then the clamp of all others
      k_sa_limit_check<T><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
      k_sa_limit_serial<T><<<A.nblk, SAL_THREADS, 0, st>>>(A);
      k_sa_limit_par<T><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
    }
  }

  void step(cudaStream_t st, cudaEvent_t* ev = nullptr) override {
    const Arena<T>& A = A_;
    auto rec = [&](int q) { if (ev) cudaEventRecord(ev[q], st); };
    rec(0);
    if (I_.time_method == -1) {  // one inner iteration of NS_Time_Dual_LU_SGS (sub_time_advance.f90:136-166)
      residual_phases(st, ev);
      cudaMemsetAsync(A.flags + A.nblk, 0, sizeof(int) * 2 * A.nblk, st);
      k_update<T, NV, 4><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
      limit(st);
      rec(4);
      bc_halo(st);
      rec(5);
      return;
    }
    if (I_.time_method == 0) {
      residual_phases(st, ev);
      cudaMemsetAsync(A.flags + A.nblk, 0, sizeof(int) * 2 * A.nblk, st);
      k_update<T, NV, 0><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
      limit(st);
      rec(4);
      bc_halo(st);
    } else if (I_.time_method == 1) {  // NS_Time_advance_1Euler (sub_time_advance.f90:217-260)
      k_copy_un<T, NV><<<grid_of((long long)NV * A.tot_box), 256, 0, st>>>(A);
      residual(st, false);
      cudaMemsetAsync(A.flags + A.nblk, 0, sizeof(int) * 2 * A.nblk, st);
      k_update<T, NV, 5><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
      limit(st);
      bc_halo(st);
      rec(1); rec(2); rec(3); rec(4);
    } else {
      k_copy_un<T, NV><<<grid_of((long long)NV * A.tot_box), 256, 0, st>>>(A);
      for (int krk = 1; krk <= 3; krk++) {
        residual(st, false);
        cudaMemsetAsync(A.flags + A.nblk, 0, sizeof(int) * 2 * A.nblk, st);
        if (krk == 1) k_update<T, NV, 1><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
        else if (krk == 2) k_update<T, NV, 2><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
        else k_update<T, NV, 3><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
        limit(st);
        bc_halo(st);
      }
      rec(1); rec(2); rec(3); rec(4);
    }
    if (NV >= 6) k_vtkw<T, NV><<<grid_of(A.tot_cell), 256, 0, st>>>(A);
    rec(5);
  }

  // residual + LU-SGS with phase events (LU-SGS path)
  void residual_phases(cudaStream_t st, cudaEvent_t* ev) {
    residual(st, false);
    if (ev) cudaEventRecord(ev[1], st);
    lusgs_sweep(st, false);
    if (ev) cudaEventRecord(ev[2], st);
    lusgs_sweep(st, true);
    if (ev) cudaEventRecord(ev[3], st);
  }
  int launches_per_step() const override {
    // primitives, then the Navier-Stokes part: inviscid fluxes (3) + k-face central fluxes,
    // viscous fluxes (3), assembly, or the tile forms in their place
    const int vis = I_.viscous ? 3 : 0;
    int res = 1 + (I_.smoothing ? 3 : 0);
    if (I_.res_fused == 1) res += 1;
    else if (I_.res_fused == 2) res += vis + 1;
    else if (I_.res_fused == 3) res += 4 + 1;
    else res += 4 + vis + 1 + (st2_ && sizeof(T) == 8 ? 1 : 0);  // forked FP64: k_cell_dt beside the viscous fluxes
    if (I_.viscous) {
      res += 1 + 1;  // mu, amut
      if (I_.turb == 2 && NV == 6) res += I_.sa_fused ? 3 : 6;  // sa_pre, (tile | 3 fluxes + res), mu_finish
      else if (I_.turb == 3 && NV == 7) res += 11;
    }
    int lu = I_.lu_planes ? 2 * (I_.max_plane - 2) : (I_.lu_version == 5 ? 3 : (I_.lu_version == 4 && I_.lu_fused ? 1 : 2));
    int upd = 1 + 1 + (NV == 6 ? 3 : 0);
    int nbc = 0;
    for (int r = 0; r < I_.nround; r++) nbc += I_.bc_rounds[3 * r + 2] > 0;
    int bch = nbc + 2 + (A_.tot_halo > 0 ? (I_.nhlevel ? 2 * I_.nhlevel : 1) : 0) + (I_.xs_cells > 0) + (I_.xr_cells > 0);
    int n;
    if (I_.time_method == -1) return res + 1 + lu + upd + bch;  // one dual-time inner iteration
    if (I_.time_method == 0) n = res + lu + upd + bch;
    else if (I_.time_method == 1) n = 1 + res + upd + bch;
    else n = 1 + 3 * (res + upd + bch);
    if (NV >= 6) n += 1;
    return n;
  }

  void lu5_pack_geo(cudaStream_t st) override {
    if (I_.lus) k_lu_pack_geo<T><<<dim3(8, L_.ntiles), 256, 0, st>>>(A_, S_, L_.TJ, L_.TK);
  }

  void dual_init(cudaStream_t st) override { k_dual_init<T, NV><<<grid_of((long long)NV * A_.tot_box), 256, 0, st>>>(A_); }
  void dual_end(cudaStream_t st) override {
    k_dual_shift<T, NV><<<grid_of(A_.tot_cell), 256, 0, st>>>(A_);
    if (NV >= 6) k_vtkw<T, NV><<<grid_of(A_.tot_cell), 256, 0, st>>>(A_);
  }

  void init_flow(cudaStream_t st) override {
    k_init_flow<T, NV><<<grid_of(A_.tot_box), 256, 0, st>>>(A_);
    bc_halo(st);
  }

  void norms(cudaStream_t st, double* part, double* out, unsigned long long* nan_at) override {
    k_norms<T, NV><<<A_.ncchunk, 256, 0, st>>>(A_, part, nan_at);
    k_norms_combine<T><<<A_.nsolve, 128, 0, st>>>(A_, part, out);
  }

  void forces(cudaStream_t st, double* part) override {
    if (A_.nwchunk > 0) k_forces<T><<<A_.nwchunk, 256, 0, st>>>(A_, part);
  }

  void scatter_state(cudaStream_t st, int blk, const double* aos, long long box_b) override {
    k_scatter_state<T, NV><<<grid_of(box_b), 256, 0, st>>>(A_, blk, aos, box_b);
  }
  void gather_state(cudaStream_t st, int blk, double* aos, long long box_b) override {
    k_gather_state<T, NV><<<grid_of(box_b), 256, 0, st>>>(A_, blk, aos, box_b);
  }

 private:
  Arena<T> A_;
  RunInfo I_;
  LuArgs L_{};
  LuStream S_{};
  int ns_grid_[5] = {1, 1, 1, 1, 1};  // CTAs of k_ns_tile per instantiation (resident CTAs, at most the tiles)
  int sa_grid_ = 1;                 // CTAs of k_sa_tile
  cudaStream_t st2_ = nullptr;      // the second stream of a forked residual (RunInfo::res_streams)
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr, ev_mu_ = nullptr;
};

template <class T>
Runner* make_runner_t(const Arena<T>& A, const RunInfo& I) {
  if (I.nvar == 5) return new RunnerT<T, 5>(A, I);
  if (I.nvar == 6) return new RunnerT<T, 6>(A, I);
  if (I.nvar == 7) return new RunnerT<T, 7>(A, I);
  return nullptr;
}

}  // namespace ocfd
