/*
 * ocfd_ec_gpu.h -- C-ABI of the B200 (sm_100a) implementation of the OpenCFD-EC 3D v1.16a
 * per-iteration hot path: multi-block residual (MUSCL/WENO reconstruction, Roe/HLLC/AUSMPW/
 * Van Leer/Steger-Warming/HLL fluxes, central viscous fluxes, SA/SST sources), LU-SGS and RK3
 * updates, flow limiter, physical boundary conditions, block-interface halos, residual norms
 * and force integration.
 *
 * Plain C: pointers and sizes only, no C++ or torch types. Every entry point returns 0
 * (OCFD_OK) or a negative OCFD_ERR_* code; ocfd_last_error() returns a message for the last
 * failing call on a handle.
 *
 * Index conventions follow the reference (sub_modules.f90:20, sub_init.f90:444-541):
 *   a block with nx,ny,nz NODES has (nx-1)(ny-1)(nz-1) cells indexed 1..n-1; cell arrays carry
 *   LAP=4 ghost layers (1-LAP..n+LAP-1); all host arrays are Fortran column-major (first index
 *   fastest).  The conserved state at the boundary is the Fortran array
 *   U(NVAR, 1-LAP:nx+LAP-1, 1-LAP:ny+LAP-1, 1-LAP:nz+LAP-1) (sub_init.f90:469).
 *
 * Connectivity is the reference's internal .inc record: 21 ints per subface, in the field
 * order ib,ie,jb,je,kb,ke,bc,face,f_no, ib1,ie1,jb1,je1,kb1,ke1,nb1,face1,f_no1,L1,L2,L3
 * (sub_IO.f90:700-705; produced from Gridgen bc3d.inp by sub_convert_inp.f90:25-248).
 * Block numbers nb1 are 1-based like the reference.
 */
#ifndef OCFD_EC_GPU_H
#define OCFD_EC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define OCFD_ABI_VERSION 2

/* error codes */
#define OCFD_OK 0
#define OCFD_ERR_ARG (-1)         /* bad argument / unsupported option                       */
#define OCFD_ERR_CUDA (-2)        /* CUDA runtime error                                       */
#define OCFD_ERR_OOM (-3)         /* device allocation failed                                 */
#define OCFD_ERR_NAN (-4)         /* NaN in the residual (replaces the reference's `stop`,
                                     sub_time_advance.f90:358-365)                            */
#define OCFD_ERR_TIMEOUT (-5)     /* a bounded device-side wait gave up                       */
#define OCFD_ERR_UNSUPPORTED (-6) /* boundary type / model outside the implemented hot path  */
#define OCFD_ERR_NOSYM (-7)       /* a required symbol or library is missing                  */
#define OCFD_ERR_COMM (-8)        /* an exchange or all-reduce callback of a sharded handle failed */

/* numeric constants of the reference (sub_modules.f90:21-47) */
#define OCFD_SCHEME_UD1 0
#define OCFD_SCHEME_NND2 1
#define OCFD_SCHEME_UD3 2
#define OCFD_SCHEME_MUSCL2U 3
#define OCFD_SCHEME_MUSCL2C 4
#define OCFD_SCHEME_MUSCL3 5
#define OCFD_SCHEME_OMUSCL2 6
#define OCFD_SCHEME_WENO5 7
#define OCFD_SCHEME_UD5 8
#define OCFD_SCHEME_WENO7 9
#define OCFD_SCHEME_CD2 20
#define OCFD_SCHEME_NONE (-1)
#define OCFD_FLUX_STEGER_WARMING 1
#define OCFD_FLUX_HLL 2
#define OCFD_FLUX_HLLC 3
#define OCFD_FLUX_ROE 4
#define OCFD_FLUX_VAN_LEER 5
#define OCFD_FLUX_AUSM 6 /* dispatches to AUSMPW, as the reference does (sub_Residual.f90:326) */
#define OCFD_BC_WALL 2
#define OCFD_BC_SYMMETRY 3
#define OCFD_BC_FARFIELD 4
#define OCFD_BC_INFLOW 5
#define OCFD_BC_OUTFLOW 6
#define OCFD_BC_EXTRAPOLATE 401
#define OCFD_BC_INNER (-1)
#define OCFD_TIME_LU_SGS 0
#define OCFD_TIME_EULER1 1 /* explicit first-order Euler, sub_time_advance.f90:217-260 */
#define OCFD_TIME_RK3 3
#define OCFD_TIME_DUAL_LU_SGS (-1) /* dual time stepping, sub_time_advance.f90:126-202 */
#define OCFD_TURB_NONE 0
#define OCFD_TURB_SA 2
#define OCFD_TURB_SST 3

/* precision modes */
#define OCFD_PREC_FP64 0  /* plain FP64 everywhere (parity path)                               */
#define OCFD_PREC_MIXED 1 /* FP32 reconstruction/fluxes/sources/metrics/Res/dt/Lc/Lv;
                             FP64 state U, DU, LU-SGS diagonal + divide, norms, forces       */

/*
 * Flow and control parameters: the namelist &control_ec values of the reference
 * (sub_read_parameter.f90:114-129) AFTER set_const_para (sub_read_parameter.f90:371-429),
 * i.e. exactly the Fortran module variables of Global_Var once read_parameter returns:
 * aoa/aos/a_alfa/a_beta in radians, twall divided by t_inf, lpmin/lpmax divided by
 * gamma*Ma^2, cv/cp derived. ocfd_default_params() + ocfd_finalize_params() reproduce
 * set_default_parameter + set_const_para for callers that start from raw namelist values.
 */
typedef struct ocfd_params {
  int nvar;                   /* NVAR: 5 (laminar/Euler), 6 (SA), 7 (SST)                  */
  int iflag_scheme;           /* interior reconstruction scheme id                          */
  int bound_scheme;           /* scheme for faces < LAP from a physical boundary           */
  int iflag_flux;             /* flux id                                                     */
  int iflag_reconstruction;   /* 0 primitive, 1 conservative, 2 characteristic              */
  int iflag_turbulence_model; /* 0, 2 (SA) or 3 (SST)                                       */
  int time_method;            /* 0 LU-SGS, 1 explicit Euler, 3 RK3, -1 dual-time LU-SGS    */
  int if_viscous;             /* 0 Euler, 1 Navier-Stokes                                   */
  int iflag_local_dt;         /* 1 local time step, 0 global                               */
  int if_dtime_mesh;          /* 1: scale dt by the mesh-quality factor                    */
  int iflag_limit_flow;       /* 1: flow limiter after every update                        */
  int if_scheme_positivity;   /* 1: first-order fallback on negative rho/p after reconstr. */
  int cood_y_up;              /* 1: y axis up, 0: z axis up                                */
  int precision;              /* OCFD_PREC_FP64 or OCFD_PREC_MIXED                         */
  double ma, re, gamma, prl, prt, t_inf, twall, kt_inf, wt_inf;
  double aoa, aos, a_alfa, a_beta; /* radians                                               */
  double cfl, dt_global, dtmin, dtmax, w_lu, mut_max, p_outlet;
  double ldmin, ldmax, lpmin, lpmax, lumax, lsamax;
  double ref_s, ref_l, centroid[3];
  double cv, cp;
  double res_inner_limit;     /* dual time: inner-iteration residual target (Res_Inner_Limit) */
  int step_inner_limit;       /* dual time: inner iterations per physical step (Step_Inner_Limit) */
  int if_residual_smoothing;  /* 1: upwind implicit residual smoothing of Res(1:5) after the
                                 spectral radii (If_Residual_smoothing, sub_Residual.f90:111-113;
                                 Residual_smoothing, sub_time_acceleraction.f90:119-217)  */
} ocfd_params;

/* Opaque solver handle: all blocks of one case resident on one GPU. */
typedef struct ocfd_handle ocfd_handle;

/* ---- parameters --------------------------------------------------------------------- */

/* Defaults of set_default_parameter (sub_read_parameter.f90:30-106); raw (pre-set_const) form,
 * angles in degrees, twall in K. */
int ocfd_default_params(ocfd_params* p);
/* set_const_para (sub_read_parameter.f90:371-429): derives nvar, converts angles to radians,
 * twall/=t_inf, scales lpmin/lpmax, maps a_alfa/a_beta by cood_y_up, computes cv/cp. */
int ocfd_finalize_params(ocfd_params* p);

/* ---- lifetime ------------------------------------------------------------------------- */

/*
 * Creates a case on the current CUDA device (replaces the per-block part of Init,
 * sub_init.f90:7-54, for the hot path):
 *   nblk            number of blocks
 *   nijk[3*b..]     nodes nx,ny,nz of block b (b = 0..nblk-1)
 *   xyz[b]          node coordinates of block b, 3*nx*ny*nz doubles: x(1:nx,1:ny,1:nz) then y
 *                   then z, i fastest (the PLOT3D record read at sub_IO.f90:36-44)
 *   nsub[b]         subfaces of block b
 *   inc             concatenated .inc records, 21 ints per subface, blocks in order
 *   dw[b]           wall distance at cell centres ((nx-1)(ny-1)(nz-1) doubles) or NULL; when the
 *                   pointer array itself is NULL and a turbulence model is on, the distance is
 *                   computed on the device (sub_comput_dw.f90:43-101)
 * Geometry (coordinate ghosts sub_update_buffer_mpi.f90:230-512, metrics sub_geometry.f90:6-346,
 * mesh-quality dt factor sub_geometry.f90:361-515) is computed on the device.  The flow is set
 * to freestream (init_flow_zero, sub_init.f90:302-410) with BC + halo applied.
 * OCFD_ERR_ARG for a block with fewer than 2 nodes in a direction or whose ghost box
 * (nx+7)(ny+7)(nz+7) reaches 2^31 cells (the kernels index within a block in 32 bits).
 */
int ocfd_create(const ocfd_params* p, int nblk, const int* nijk, const double* const* xyz,
                const int* nsub, const int* inc, const double* const* dw, ocfd_handle** out);
int ocfd_destroy(ocfd_handle* h);
const char* ocfd_last_error(const ocfd_handle* h);

/* ---- state ---------------------------------------------------------------------------- */

/* Number of doubles in the Fortran U array of block b: NVAR*(nx+7)*(ny+7)*(nz+7). */
long long ocfd_state_size(const ocfd_handle* h, int blk);
/* Copy the Fortran-layout U(NVAR,1-LAP:n+LAP-1,...) of block blk to / from the device. */
int ocfd_set_state(ocfd_handle* h, int blk, const double* U);
int ocfd_get_state(ocfd_handle* h, int blk, double* U);
/* Re-initialise to freestream (Init_flow with Iflag_init=0, sub_init.f90:264-438). */
int ocfd_init_flow(ocfd_handle* h);

/* ---- the hot path --------------------------------------------------------------------- */

/*
 * nsteps calls of NS_Time_advance(1) (sub_time_advance.f90:6-23; the driver call at
 * opencfd_ec3d_v1.16a.f90:167): residual + LU-SGS (or the 3 RK3 stages, or one explicit Euler
 * stage U = Un + dt Res/vol for time_method = 1), U update, flow
 * limiter, BC, halo, vt/k/w clamps.  kstep and tt (may be NULL) receive the step counter and
 * time after the last step (tt advances by dt_global per step, sub_time_advance.f90:115).
 * Asynchronous on the device; the NaN check happens in ocfd_residual.  With time_method = -1 each
 * step is a physical time step of NS_Time_Dual_LU_SGS (sub_time_advance.f90:126-202): up to
 * step_inner_limit inner LU-SGS iterations on the physical-time residual, stopping when the largest
 * residual RMS (of every solve) is at most res_inner_limit; the call then waits for each inner
 * iteration's norms.
 */
int ocfd_advance(ocfd_handle* h, int nsteps, int* kstep, double* tt);

/* Comput_Residual_one_mesh (sub_Residual.f90:14-127) alone: the residual Res, the local time
 * step and, when with_lusgs != 0, the LU-SGS increment DU from the current state, without
 * updating U.  Used to check one residual evaluation in isolation. */
int ocfd_compute_residual(ocfd_handle* h, int with_lusgs);

/* comput_max_Res_onemesh (sub_time_advance.f90:330-380): FP64 max and RMS of the last
 * residual over all interior cells; arrays of 7 (entries >= NVAR are 0).  Returns
 * OCFD_ERR_NAN if any residual is NaN (the reference stops there). */
int ocfd_residual(ocfd_handle* h, double* res_max, double* res_rms);

/* comput_force (sub_Post.f90:4-265): ft[9] = pressure force (3), viscous force (3), moments
 * (3), normalised by 2/Ref_S and 2/(Ref_S Ref_L); cl, cd, cs projected by AoA / Cood_Y_UP. */
int ocfd_forces(ocfd_handle* h, double* ft, double* cl, double* cd, double* cs);

/* Number of bound-violation cells the limiter repaired on the last update of block blk and
 * the block's sticky IF_OverLimit flag (sub_limitflow.f90:82-171). */
int ocfd_limiter_status(ocfd_handle* h, int blk, int* n_limited, int* overlimit);

/* Debug / parity access to one per-block array, copied to host in the reference's index
 * ranges.  name: "Res" (NVAR,-1:n+1 interior used), "dt", "DU", "mu", "mu_t", "vol",
 * "dtime_mesh", "dw", "Si","Sj","Sk", "ni1".."nk3", "ix1".."kz0", "xc","yc","zc", "surf1".."surf6".
 * Layouts are given by ocfd_array_shape. */
int ocfd_array_shape(const ocfd_handle* h, int blk, const char* name, int* lo, int* hi, int* nv);
int ocfd_get_array(ocfd_handle* h, int blk, const char* name, double* out);

/* ---- batches of independent solves (no counterpart in the reference, which runs one case per
 *      MPI job; the batched form serves Mach/AoA sweeps and many meshes at once) ------------ */

/*
 * One handle holding nsolve independent cases: every kernel of a step covers the blocks of all
 * of them, so a step of the batch is one graph launch of the same kernels as a single case.
 *   ps[q]       parameters of solve q; all solves share NVAR (turbulence model), if_viscous,
 *               time_method and precision (OCFD_ERR_ARG otherwise); Mach, angles, Re, CFL,
 *               schemes, fluxes and limits may differ
 *   nblk[q]     blocks of solve q; blocks are numbered globally in solve order for every other
 *               argument and entry point (nijk, xyz, nsub, inc, dw, set/get_state, ...)
 *   inc         partner block numbers (nb1) are 1-based WITHIN the solve, exactly as each
 *               case's own .inc file has them
 * Wall distance is taken over the walls of each block's own solve.  ocfd_create is this call
 * with nsolve = 1.
 */
int ocfd_create_batch(const ocfd_params* ps, int nsolve, const int* nblk, const int* nijk,
                      const double* const* xyz, const int* nsub, const int* inc,
                      const double* const* dw, ocfd_handle** out);
/* Number of solves of the handle. */
int ocfd_nsolve(const ocfd_handle* h);
/* ocfd_residual for every solve: res_max / res_rms hold 7*nsolve doubles (solve-major). */
int ocfd_residual_all(ocfd_handle* h, double* res_max, double* res_rms);
/* ocfd_forces for every solve: ft holds 9*nsolve doubles, cl / cd / cs nsolve each (may be
 * NULL); each solve uses its own Ref_S, Ref_L, AoA and Cood_Y_UP. */
int ocfd_forces_all(ocfd_handle* h, double* ft, double* cl, double* cd, double* cs);
/*
 * Solve q of a batch starts over with new parameters on its own mesh (a new Mach number, angle,
 * Reynolds number, CFL, scheme, ...; the same NVAR, if_viscous, time_method and precision as the
 * other solves, OCFD_ERR_ARG otherwise): its constants are replaced, the arrays that carry history
 * between steps (mu, mu_t, the SST k / omega planes, the limiter flags) return to their state
 * after allocation, and its flow is set to the new freestream with BC, halo and corners on its
 * blocks, exactly as a new handle holding this case alone starts.  The other solves keep their
 * state, and the next ocfd_advance steps all of them together (the captured step graph stays
 * valid).  This is how a serving loop admits a new request into a free slot of a running batch.
 * Not for sharded handles or dual time (OCFD_ERR_UNSUPPORTED).  Synchronous.
 */
int ocfd_reset_solve(ocfd_handle* h, int q, const ocfd_params* p);
/* Upper estimate of the device bytes ocfd_create would allocate for these blocks and
 * parameters (admission control by HBM footprint); -1 on bad arguments.  No device call. */
long long ocfd_footprint(const ocfd_params* p, int nblk, const int* nijk);
/* ocfd_advance only queues work on the handle's stream; this waits for it to finish.  Driving
 * several handles from one host thread (advance each, then synchronize each) overlaps their
 * work on the device. */
int ocfd_synchronize(ocfd_handle* h);

/* ---- allocation-free monitoring (no counterpart in the reference) ------------------------ */

/*
 * ocfd_residual for solve 0 that allocates nothing, neither device nor host heap memory: for
 * callers that must not allocate inside their iteration loop (a driver whose device memory is
 * fully committed to resident solves, or a monitor that must not touch an allocator while the
 * solver runs).  Its error paths allocate nothing either: their messages are formatted on the
 * stack into the handle's preallocated error string.  Its scratch is one static device area per
 * device, shared by all handles of the process: at most 4096 norm chunks and 256 solves per
 * handle.  Every block's interior cells are cut into chunks of at most 8192 cells, so the limit is
 * 33,554,432 cells for large blocks and fewer for many small ones (256 solves of 17 small blocks
 * already make 4352 chunks); larger handles get OCFD_ERR_ARG with their chunk count in the
 * message (use ocfd_residual).  The first call on a device
 * looks the area up (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture.  Calls that overlap in time (other threads, other handles on the same
 * device) race on the shared area and must be serialised by the caller.  On a NaN it returns
 * OCFD_ERR_NAN without the cell location (ocfd_residual reports it).
 */
int ocfd_residual_static(ocfd_handle* h, double* res_max, double* res_rms);

/* ---- block-sharded solves: one case split over ranks by whole blocks ----------------------
 *
 * The reference's MPI mode (sub_partation_mpi.f90:126-158 assigns whole blocks to ranks;
 * Umessage_send_mpi / Umessage_recv_mpi, sub_update_buffer_mpi.f90:42-211, exchange the LAP ghost
 * layers of interfaces between blocks on different ranks; comput_max_Res_onemesh and comput_force
 * all-reduce their sums, sub_time_advance.f90:373-374, sub_Post.f90:202).  Every rank creates one
 * handle with the whole case description and owner[] (rank of each block); the handle holds only
 * the blocks with owner == rank, numbered 0.. in ascending global order (ocfd_part_blocks gives
 * the map), and ocfd_get_state / ocfd_set_state / ocfd_limiter_status / ocfd_get_array take
 * those local numbers.  Copies between the handle's own blocks stay on the device; copies to and
 * from other ranks go through two device buffers handed to comm->exchange once per halo update
 * (each step, each RK3 stage, each dual-time inner iteration, and at initialisation).
 * ocfd_create_part, ocfd_advance, ocfd_init_flow, ocfd_residual, ocfd_forces and ocfd_profile
 * are collective: every rank calls them in the same order.  Norms and forces are all-reduced
 * through comm->allreduce (RMS over the cells of the whole case; a NaN or a timed-out wait on
 * any rank is reported on all).  Single solve only; steps run without a CUDA graph; blocks must
 * be at least LAP (4) cells thick across interfaces between ranks (OCFD_ERR_UNSUPPORTED
 * otherwise), so that the exchange order cannot matter.
 */
typedef struct ocfd_comm {
  /* send[send_off[q] .. send_off[q+1]) goes to rank peers[q], recv[recv_off[q] .. recv_off[q+1])
   * comes from it; device pointers, offsets in doubles, npeer + 1 offsets each.  Called on the
   * handle's host thread after the pack kernel is queued on stream (a cudaStream_t); the transfer
   * is queued on that stream (NCCL send/recv) or complete when the call returns.  0 = ok. */
  int (*exchange)(void* user, void* stream, int npeer, const int* peers, const double* send, const long long* send_off,
                  double* recv, const long long* recv_off);
  /* in-place all-reduce of n host doubles over the ranks; op 0 = sum, 1 = max.  0 = ok. */
  int (*allreduce)(void* user, double* buf, int n, int op);
  void* user;
} ocfd_comm;

int ocfd_create_part(const ocfd_params* p, int nblk, const int* nijk, const double* const* xyz, const int* nsub,
                     const int* inc, const double* const* dw, const int* owner, int rank, const ocfd_comm* comm,
                     ocfd_handle** h);
/* The exchange plan of rank `rank` without creating anything (host only, no device call): returns
 * the number of peers (or an error code); when the pointers are not NULL, peers[npeer] and the
 * per-peer offsets send_off / recv_off[npeer + 1] in CELLS of the exchange buffers (NVAR doubles
 * per cell).  ocfd_create_part hands the exchange callback the same plan in doubles. */
int ocfd_part_plan(int nblk, const int* nijk, const int* nsub, const int* inc, const int* owner, int rank, int* peers,
                   long long* send_off, long long* recv_off);
/* Number of blocks the handle holds; their global (0-based) block numbers into global_ids when
 * it is not NULL.  A handle from ocfd_create holds every block (identity map). */
int ocfd_part_blocks(const ocfd_handle* h, int* global_ids);

/* Library build/ABI information: "ocfd-b200 <abi> sm_100a ..." */
const char* ocfd_version(void);

/* ---- measurement (no counterpart in the reference, which only prints wall time per step at
 *      opencfd_ec3d_v1.16a.f90:224-243) ----------------------------------------------------- */

/* The cudaStream_t (as void*) all work of the handle is queued on, so a caller can time it with
 * CUDA events or order its own work after it. */
void* ocfd_stream(ocfd_handle* h);
/* Runs nsteps steps phase by phase (outside the step graph) and accumulates the device time of
 * each phase in ms: [0] residual (primitives, turbulence, fluxes, assembly, dt), [1] LU-SGS lower
 * sweep, [2] LU-SGS upper sweep, [3] update + flow limiter + vt/k/w clamps, [4] BC + halo +
 * corners, [5] whole step.  phase_ms must hold 8 doubles. */
int ocfd_profile(ocfd_handle* h, int nsteps, double* phase_ms);
/* Kernel launches queued by one ocfd_advance step (all of them this library's own kernels). */
int ocfd_launches_per_step(ocfd_handle* h);
/* Columns per CTA tile (32 or 64) of the LU-SGS wavefront sweeps, and the wavefront kernel version
 * in use (3: inputs staged by element; 4: staged by 32-byte sector, helper warps off the step's
 * phases; 2: one thread per column).  ocfd_create times each tile width with versions 3 and 4 on
 * the new case (a few steps from freestream, before the state is initialised; the result does not
 * depend on the choice) and keeps the fastest; OCFD_LU_TC=32|64 fixes the width, OCFD_LU_V3=1 or
 * OCFD_LU_V4=1 the version, OCFD_NO_AUTOTUNE=1 takes the first candidate (64 columns if fixed,
 * else 32; version 4 unless fixed). */
int ocfd_lu_tile_width(const ocfd_handle* h);
int ocfd_lu_kernel_version(const ocfd_handle* h);
/* 1 when the two LU-SGS sweeps run as one launch: version 4 in which a block's upper sweep starts
 * as soon as its own lower sweep is done, while deeper blocks still run theirs (OCFD_LU_ONE_LAUNCH=1
 * puts it in version 4's place; same results, measured slower than the two launches once tiles are
 * taken longest first within a level).  ocfd_profile then reports the joint time as the lower
 * sweep's and 0 for the upper. */
int ocfd_lu_one_launch(const ocfd_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* OCFD_EC_GPU_H */
