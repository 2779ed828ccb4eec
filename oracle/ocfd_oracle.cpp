// ============================================================================================
// ORACLE -- TEST INFRASTRUCTURE ONLY.  Never linked into, called by, or shipped with the
// product library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load it, and only as the checker / CPU baseline.
//
// CPU FP64 restatement of the per-iteration hot path of OpenCFD-EC 3D v1.16a (Fortran 90):
// geometry + coordinate ghosts (sub_geometry.f90, sub_update_buffer_mpi.f90), wall distance
// (sub_comput_dw.f90), freestream init (sub_init.f90), residual (sub_Residual.f90,
// sub_scheme.f90, sub_flux_split.f90, sub_turbulence_SA.f90, sub_turbulence_SST.f90),
// spectral radii and local dt (sub_time_acceleraction.f90), LU-SGS (sub_LU_SGS.f90), RK3 and
// norms (sub_time_advance.f90), flow limiter (sub_limitflow.f90), boundary conditions
// (sub_boundary.f90), block-interface halo + corner averaging (sub_update_buffer_mpi.f90) and
// forces (sub_Post.f90).  Loops, index ranges and the order of every floating-point operation
// follow the Fortran source (left-to-right evaluation, x**n as the powi multiplication chain,
// single-precision literals such as 0.09 and 1.e-8 rounded to float first).
//
// PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures for this path and
// cannot be compiled here (no Fortran compiler in the image), so this restatement is checked
// only by self-made known answers (freestream preservation, flux consistency, polynomial
// exactness, LU-SGS schedule invariance, halo copy exactness) in tests/.
//
// One documented choice where the reference is undefined: sub_turbulence_SST.f90 reads f1 at
// faces i=nx / j=ny / k=nz (lines 187, 237, 286) where f1 was never set (uninitialised memory);
// this restatement uses f1 of the adjacent interior cell there.
//
// Build: g++ -O2 -ffp-contract=off -fopenmp -shared -fPIC (see oracle/Makefile).
// ============================================================================================
#include "../include/ocfd_ec_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

namespace orc {

// ---------- a small persistent thread pool standing in for the reference's !$OMP loops ----------
// (the image has no OpenMP runtime).  par_for(lo, hi, f) splits [lo, hi] into contiguous chunks,
// one per thread, like OMP's static schedule; f(k) must only write data owned by iteration k.
class Pool {
 public:
  static Pool& get() { static Pool p; return p; }
  int size() const { return (int)workers_.size() + 1; }
  void set_threads(int n) {
    stop();
    if (n < 1) n = 1;
    std::unique_lock<std::mutex> lk(m_);
    quit_ = false;
    // a worker starts at the current generation, so it only ever takes part in later runs
    const unsigned g0 = gen_;
    for (int t = 1; t < n; t++) workers_.emplace_back([this, t, g0] { loop(t, g0); });
  }
  template <class F>
  void run(int lo, int hi, F&& f) {
    int n = hi - lo + 1;
    if (n <= 0) return;
    int nt = size();
    if (nt == 1 || n < 2) { for (int k = lo; k <= hi; k++) f(k); return; }
    std::function<void(int)> job = [&](int tid) {
      int chunk = (n + nt - 1) / nt, a = lo + tid * chunk, b = std::min(hi, a + chunk - 1);
      for (int k = a; k <= b; k++) f(k);
    };
    {
      std::unique_lock<std::mutex> lk(m_);
      job_ = &job; pending_ = nt - 1; gen_++;
    }
    cv_.notify_all();
    job(0);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }
  ~Pool() { stop(); }

 private:
  Pool() {
    int n = (int)std::thread::hardware_concurrency();
    if (const char* e = std::getenv("OCFD_ORACLE_THREADS")) n = std::atoi(e);
    set_threads(n > 0 ? n : 1);
  }
  void stop() {
    { std::unique_lock<std::mutex> lk(m_); quit_ = true; gen_++; }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    workers_.clear();
  }
  void loop(int tid, unsigned seen) {
    for (;;) {
      std::function<void(int)>* job;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (quit_) return;
        job = job_;
      }
      if (!job) continue;
      (*job)(tid);
      std::unique_lock<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  std::function<void(int)>* job_ = nullptr;
  int pending_ = 0;
  unsigned gen_ = 0;
  bool quit_ = false;
};
template <class F>
static inline void par_for(int lo, int hi, F&& f) { Pool::get().run(lo, hi, f); }

constexpr int LAP = 4;
constexpr double Lim_Zero = 1.e-20;
constexpr double PI = 3.1415926535897932;

enum { S_UD1 = 0, S_NND2 = 1, S_UD3 = 2, S_MUSCL2U = 3, S_MUSCL2C = 4, S_MUSCL3 = 5, S_OMUSCL2 = 6,
       S_WENO5 = 7, S_UD5 = 8, S_WENO7 = 9, S_CD2 = 20 };
enum { F_SW = 1, F_HLL = 2, F_HLLC = 3, F_ROE = 4, F_VL = 5, F_AUSM = 6 };
enum { BC_Wall = 2, BC_Symmetry = 3, BC_Farfield = 4, BC_Inflow = 5, BC_Outflow = 6, BC_Extrap = 401 };

// x**n with integer n: the multiplication chain gfortran emits through __builtin_powi.
static inline double p2(double x) { return x * x; }
static inline double p3(double x) { return (x * x) * x; }
static inline double p4(double x) { double t = x * x; return t * t; }
static inline double p6(double x) { double t = (x * x) * x; return t * t; }

// ---------- arrays with Fortran lower bounds, first index fastest ---------------------------
struct A3 {
  int l0 = 0, l1 = 0, l2 = 0, n0 = 0, n1 = 0, n2 = 0;
  std::vector<double> v;
  void alloc(int a0, int b0, int a1, int b1, int a2, int b2, double init = 0.0) {
    l0 = a0; l1 = a1; l2 = a2; n0 = b0 - a0 + 1; n1 = b1 - a1 + 1; n2 = b2 - a2 + 1;
    v.assign((size_t)n0 * n1 * n2, init);
  }
  inline double& operator()(int i, int j, int k) {
    return v[(size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * (size_t)(k - l2))];
  }
};
struct A4 {  // (m, i, j, k), m = 1..nv fastest
  int nv = 0, l0 = 0, l1 = 0, l2 = 0, n0 = 0, n1 = 0, n2 = 0;
  std::vector<double> v;
  void alloc(int nv_, int a0, int b0, int a1, int b1, int a2, int b2, double init = 0.0) {
    nv = nv_; l0 = a0; l1 = a1; l2 = a2; n0 = b0 - a0 + 1; n1 = b1 - a1 + 1; n2 = b2 - a2 + 1;
    v.assign((size_t)nv * n0 * n1 * n2, init);
  }
  inline double& operator()(int m, int i, int j, int k) {
    return v[(size_t)(m - 1) + (size_t)nv * ((size_t)(i - l0) + (size_t)n0 * ((size_t)(j - l1) + (size_t)n1 * (size_t)(k - l2)))];
  }
};
struct I3 {
  int l0 = 1, l1 = 1, n0 = 0, n1 = 0;
  std::vector<int> v;
  void alloc(int a, int b, int c) { n0 = a; n1 = b; v.assign((size_t)a * b * c, 0); }
  inline int& operator()(int i, int j, int s) { return v[(size_t)(i - 1) + (size_t)n0 * ((size_t)(j - 1) + (size_t)n1 * (size_t)(s - 1))]; }
};

struct Sub {
  int ib, ie, jb, je, kb, ke, bc, face, f_no, ib1, ie1, jb1, je1, kb1, ke1, nb1, face1, f_no1, L1, L2, L3;
};

struct Block {
  int nx, ny, nz, no;
  std::vector<Sub> sub;
  A3 x, y, z, xc, yc, zc, vol, Si, Sj, Sk, ni1, ni2, ni3, nj1, nj2, nj3, nk1, nk2, nk3;
  A3 ix1, iy1, iz1, jx1, jy1, jz1, kx1, ky1, kz1, ix2, iy2, iz2, jx2, jy2, jz2, kx2, ky2, kz2;
  A3 ix3, iy3, iz3, jx3, jy3, jz3, kx3, ky3, kz3, ix0, iy0, iz0, jx0, jy0, jz0, kx0, ky0, kz0;
  A4 U, Un, Res, DU;
  A4 Un1;  // dual time: the state two physical steps back
  A3 dt, dw, mu, mu_t, dtime_mesh;
  A3 surf1, surf2, surf3, surf4, surf5, surf6;  // (n,n,3)
  I3 BcI, BcJ, BcK;
  int overlimit = 0, nlimited = 0;
};

struct Case {
  ocfd_params P;
  int NVAR;
  std::vector<Block> B;
  int Kstep = 0;
  double tt = 0.0;
  long long Num_Cell = 0;
  double Ralfa[3], Rbeta[3], Rgamma[3];
  std::string err;
  int threads = 0;
  int dual_started = 0;  // Comput_Residual_one_mesh's saved Iflag1 (sub_Residual.f90:25-33)
};

// per-block flow temporaries (Flow_Var module: d,uu,v,w,T,cc,p, Flux, Lci..Lvk)
struct Work {
  A3 d, uu, v, w, T, cc, p;
  A4 Flux;
  A3 Lci, Lcj, Lck, Lvi, Lvj, Lvk;
};

// ============================================================================================
// reconstruction schemes: sub_scheme.f90
// u[] holds u(1-LAP:LAP) = u(-3..4) at u[0..7]; U(k) = u[k+3]
// ============================================================================================
static inline double minmod(double a, double b) {  // sub_scheme.f90:281-292
  if (a * b <= 0.0) return 0.0;
  if (std::fabs(a) <= std::fabs(b)) return a;
  return b;
}
#define UU(k) u[(k) + 3]

static double weno5_L(const double* u) {  // sub_scheme.f90:101-119
  const double ep = 1.e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = 13.0 / 12.0 * p2(UU(0) - 2.0 * UU(1) + UU(2)) + 1.0 / 4.0 * p2(3.0 * UU(0) - 4.0 * UU(1) + UU(2));
  double S1 = 13.0 / 12.0 * p2(UU(-1) - 2.0 * UU(0) + UU(1)) + 1.0 / 4.0 * p2(UU(-1) - UU(1));
  double S2 = 13.0 / 12.0 * p2(UU(-2) - 2.0 * UU(-1) + UU(0)) + 1.0 / 4.0 * p2(UU(-2) - 4.0 * UU(-1) + 3.0 * UU(0));
  double a0 = C03 / p2(ep + S0), a1 = C13 / p2(ep + S1), a2 = C23 / p2(ep + S2);
  double am = a0 + a1 + a2;
  double q03 = 1.0 / 3.0 * UU(0) + 5.0 / 6.0 * UU(1) - 1.0 / 6.0 * UU(2);
  double q13 = -1.0 / 6.0 * UU(-1) + 5.0 / 6.0 * UU(0) + 1.0 / 3.0 * UU(1);
  double q23 = 1.0 / 3.0 * UU(-2) - 7.0 / 6.0 * UU(-1) + 11.0 / 6.0 * UU(0);
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
static double weno5_R(const double* u) {  // sub_scheme.f90:122-140
  const double ep = 1.e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = 13.0 / 12.0 * p2(UU(1) - 2.0 * UU(0) + UU(-1)) + 1.0 / 4.0 * p2(3.0 * UU(1) - 4.0 * UU(0) + UU(-1));
  double S1 = 13.0 / 12.0 * p2(UU(2) - 2.0 * UU(1) + UU(0)) + 1.0 / 4.0 * p2(UU(2) - UU(0));
  double S2 = 13.0 / 12.0 * p2(UU(3) - 2.0 * UU(2) + UU(1)) + 1.0 / 4.0 * p2(UU(3) - 4.0 * UU(2) + 3.0 * UU(1));
  double a0 = C03 / p2(ep + S0), a1 = C13 / p2(ep + S1), a2 = C23 / p2(ep + S2);
  double am = a0 + a1 + a2;
  double q03 = 1.0 / 3.0 * UU(1) + 5.0 / 6.0 * UU(0) - 1.0 / 6.0 * UU(-1);
  double q13 = -1.0 / 6.0 * UU(2) + 5.0 / 6.0 * UU(1) + 1.0 / 3.0 * UU(0);
  double q23 = 1.0 / 3.0 * UU(3) - 7.0 / 6.0 * UU(2) + 11.0 / 6.0 * UU(1);
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
// WENO7 coefficient set (sub_scheme.f90:151-166)
namespace w7 {
const double C0 = 1.0 / 35.0, C1 = 12.0 / 35.0, C2 = 18.0 / 35.0, C3 = 4.0 / 35.0;
const double a11 = -2.0 / 6.0, a12 = 9.0 / 6.0, a13 = -18.0 / 6.0, a14 = 11.0 / 6.0;
const double a21 = 1.0 / 6.0, a23 = 3.0 / 6.0, a24 = 2.0 / 6.0;
const double a31 = -2.0 / 6.0, a32 = -3.0 / 6.0, a34 = -1.0 / 6.0;
const double a41 = -11.0 / 6.0, a42 = 18.0 / 6.0, a43 = -9.0 / 6.0, a44 = 2.0 / 6.0;
const double b12 = 4.0, b13 = -5.0, b14 = 2.0, b22 = -2.0, b41 = 2.0, b42 = -5.0, b43 = 4.0, c12 = 3.0;
const double d12 = 13.0 / 12.0, d13 = 1043.0 / 960.0, d14 = 1.0 / 12.0;
const double e11 = -3.0 / 12.0, e12 = 13.0 / 12.0, e13 = -23.0 / 12.0, e14 = 25.0 / 12.0;
const double e21 = 1.0 / 12.0, e22 = -5.0 / 12.0, e23 = 13.0 / 12.0, e24 = 3.0 / 12.0;
const double e31 = -1.0 / 12.0, e32 = 7.0 / 12.0, e33 = 7.0 / 12.0, e34 = -1.0 / 12.0;
const double e41 = 3.0 / 12.0, e42 = 13.0 / 12.0, e43 = -5.0 / 12.0, e44 = 1.0 / 12.0;
const double ep = 1.e-8;
}  // namespace w7
static double weno7_core(double vm3, double vm2, double vm1, double v0, double v1, double v2, double v3) {
  using namespace w7;
  double S10 = a11 * vm3 + a12 * vm2 + a13 * vm1 + a14 * v0;
  double S11 = a21 * vm2 - vm1 + a23 * v0 + a24 * v1;
  double S12 = a31 * vm1 + a32 * v0 + v1 + a34 * v2;
  double S13 = a41 * v0 + a42 * v1 + a43 * v2 + a44 * v3;
  double S20 = -vm3 + b12 * vm2 + b13 * vm1 + b14 * v0;
  double S21 = vm1 + b22 * v0 + v1;
  double S22 = v0 + b22 * v1 + v2;
  double S23 = b41 * v0 + b42 * v1 + b43 * v2 - v3;
  double S30 = -vm3 + c12 * (vm2 - vm1) + v0;
  double S31 = -vm2 + c12 * (vm1 - v0) + v1;
  double S32 = -vm1 + c12 * (v0 - v1) + v2;
  double S33 = -v0 + c12 * (v1 - v2) + v3;
  double S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  double S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  double S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  double S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  double a0 = C0 / p2(ep + S0), a1 = C1 / p2(ep + S1), a2 = C2 / p2(ep + S2), a3 = C3 / p2(ep + S3);
  double am = a0 + a1 + a2 + a3;
  double q0 = e11 * vm3 + e12 * vm2 + e13 * vm1 + e14 * v0;
  double q1 = e21 * vm2 + e22 * vm1 + e23 * v0 + e24 * v1;
  double q2 = e31 * vm1 + e32 * v0 + e33 * v1 + e34 * v2;
  double q3 = e41 * v0 + e42 * v1 + e43 * v2 + e44 * v3;
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}
// weno7_L (sub_scheme.f90:144-206) uses v(-3..3); weno7_R (212-277) is the mirror with
// v(4),v(3),...,v(-2) in the roles of v(-3),...,v(3).
static double weno7_L(const double* u) { return weno7_core(UU(-3), UU(-2), UU(-1), UU(0), UU(1), UU(2), UU(3)); }
static double weno7_R(const double* u) { return weno7_core(UU(4), UU(3), UU(2), UU(1), UU(0), UU(-1), UU(-2)); }

static const double k2c = 1.0, k2u = -1.0, b2 = 2.0, k3 = 1.0 / 3.0, sep = 1.e-6;
static const double eta_om = (double)0.05f;  // `real(PRE_EC),parameter:: eta=0.05` (default-real literal)

static double scheme_fP(const double* u, int s) {  // sub_scheme.f90:6-53
  switch (s) {
    case S_CD2: return 0.5 * (UU(0) + UU(1));
    case S_UD1: return UU(0);
    case S_UD3: return (-UU(-1) + 5.0 * UU(0) + 2.0 * UU(1)) / 6.0;
    case S_NND2: return UU(0) + 0.5 * minmod(UU(0) - UU(-1), UU(1) - UU(0));
    case S_MUSCL2U:
      return UU(0) + 0.25 * ((1.0 - k2u) * minmod(UU(0) - UU(-1), b2 * (UU(1) - UU(0))) + (1.0 + k2u) * minmod(UU(1) - UU(0), b2 * (UU(0) - UU(-1))));
    case S_MUSCL2C:
      return UU(0) + 0.25 * ((1.0 - k2c) * minmod(UU(0) - UU(-1), b2 * (UU(1) - UU(0))) + (1.0 + k2c) * minmod(UU(1) - UU(0), b2 * (UU(0) - UU(-1))));
    case S_MUSCL3: {
      double up = UU(1) - UU(0), um = UU(0) - UU(-1);
      double s_ = (2.0 * up * um + sep) / (up * up + um * um + sep);
      return UU(0) + 0.25 * s_ * ((1.0 - k3 * s_) * um + (1.0 + k3 * s_) * up);
    }
    case S_OMUSCL2: {
      double r1 = (UU(0) - UU(-1) + sep) / (UU(1) - UU(0) + sep), r2 = (UU(1) - UU(0) + sep) / (UU(2) - UU(1) + sep);
      double f1 = (1.0 - eta_om) + (eta_om - 0.55) * 0.5 / r2 + (eta_om + 0.55) * 0.5 * r1;
      double f = std::max(0.0, std::min(std::min(2.0, f1), 2.0 * r1));
      return UU(0) + 0.5 * f * (UU(1) - UU(0));
    }
    case S_WENO5: return weno5_L(u);
    case S_WENO7: return weno7_L(u);
    case S_UD5: return (2.0 * UU(-2) - 13.0 * UU(-1) + 47.0 * UU(0) + 27.0 * UU(1) - 3.0 * UU(2)) / 60.0;
  }
  return 0.0;
}
static double scheme_fm(const double* u, int s) {  // sub_scheme.f90:55-96
  switch (s) {
    case S_CD2: return 0.5 * (UU(0) + UU(1));
    case S_UD1: return UU(1);
    case S_UD3: return (2.0 * UU(0) + 5.0 * UU(1) - UU(2)) / 6.0;
    case S_NND2: return UU(1) - 0.5 * minmod(UU(1) - UU(0), UU(2) - UU(1));
    case S_MUSCL2U:
      return UU(1) - 0.25 * ((1.0 - k2u) * minmod(UU(2) - UU(1), b2 * (UU(1) - UU(0))) + (1.0 + k2u) * minmod(UU(1) - UU(0), b2 * (UU(2) - UU(1))));
    case S_MUSCL2C:
      return UU(1) - 0.25 * ((1.0 - k2c) * minmod(UU(2) - UU(1), b2 * (UU(1) - UU(0))) + (1.0 + k2c) * minmod(UU(1) - UU(0), b2 * (UU(2) - UU(1))));
    case S_MUSCL3: {
      double up = UU(2) - UU(1), um = UU(1) - UU(0);
      double s_ = (2.0 * up * um + sep) / (up * up + um * um + sep);
      return UU(1) - 0.25 * s_ * ((1.0 - k3 * s_) * up + (1.0 + k3 * s_) * um);
    }
    case S_OMUSCL2: {
      double r1 = (UU(2) - UU(1) + sep) / (UU(1) - UU(0) + sep), r2 = (UU(1) - UU(0) + sep) / (UU(0) - UU(-1) + sep);
      double f1 = (1.0 - eta_om) + (eta_om - 0.55) * 0.5 / r2 + (eta_om + 0.55) * 0.5 * r1;
      double f = std::max(0.0, std::min(std::min(2.0, f1), 2.0 * r1));
      return UU(1) - 0.5 * f * (UU(1) - UU(0));
    }
    case S_WENO5: return weno5_R(u);
    case S_WENO7: return weno7_R(u);
    case S_UD5: return (-3.0 * UU(-1) + 27.0 * UU(0) + 47.0 * UU(1) - 13.0 * UU(2) + 2.0 * UU(3)) / 60.0;
  }
  return 0.0;
}
#undef UU

// U0[m][k] : m = 0..4 (d,u,v,w,p or conservative), k = 0..7 (stencil -3..4)
static void recon_original(double U0[5][8], double* UL, double* UR, int s) {  // sub_Residual.f90:1258-1268
  for (int m = 0; m < 5; m++) { UL[m] = scheme_fP(U0[m], s); UR[m] = scheme_fm(U0[m], s); }
}
static void recon_conservative(double U0[5][8], double* UL, double* UR, double gamma, int s) {  // 1271-1286
  double QL[5], QR[5];
  for (int m = 0; m < 5; m++) { QL[m] = scheme_fP(U0[m], s); QR[m] = scheme_fm(U0[m], s); }
  UL[0] = QL[0]; UL[1] = QL[1] / UL[0]; UL[2] = QL[2] / UL[0]; UL[3] = QL[3] / UL[0];
  UL[4] = (QL[4] - (UL[1] * QL[1] + UL[2] * QL[2] + UL[3] * QL[3]) * 0.5) * (gamma - 1.0);
  UR[0] = QR[0]; UR[1] = QR[1] / UR[0]; UR[2] = QR[2] / UR[0]; UR[3] = QR[3] / UR[0];
  UR[4] = (QR[4] - (UR[1] * QR[1] + UR[2] * QR[2] + UR[3] * QR[3]) * 0.5) * (gamma - 1.0);
}
static void recon_characteristic(double U0[5][8], double* UL, double* UR, double gamma, int s) {  // 1291-1347
  double Uh[5];
  for (int m = 0; m < 5; m++) Uh[m] = 0.5 * (U0[m][3] + U0[m][4]);
  double d1 = Uh[0], u1 = Uh[1] / d1, v1 = Uh[2] / d1, w1 = Uh[3] / d1;
  double p1 = (Uh[4] - (Uh[1] * u1 + Uh[2] * v1 + Uh[3] * w1) * 0.5) * (gamma - 1.0);
  double c1 = std::sqrt(gamma * p1 / d1);
  double V2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
  double tmp1 = (gamma - 1.0) / c1, tmp3 = (gamma - 1.0) / (c1 * c1), tmp5 = 1.0 / (2.0 * c1), tmp0 = 1.0 / tmp3;
  double S[5][5] = {{V2 - tmp0, -u1, -v1, -w1, 1.0},
                    {-v1, 0.0, 1.0, 0.0, 0.0},
                    {-w1, 0.0, 0.0, 1.0, 0.0},
                    {-u1 - V2 * tmp1, 1.0 + tmp1 * u1, tmp1 * v1, tmp1 * w1, -tmp1},
                    {-u1 + V2 * tmp1, 1.0 - tmp1 * u1, -tmp1 * v1, -tmp1 * w1, tmp1}};
  double S1[5][5] = {{-tmp3, 0.0, 0.0, -tmp5, tmp5},
                     {-tmp3 * u1, 0.0, 0.0, 0.5 - u1 * tmp5, 0.5 + u1 * tmp5},
                     {-tmp3 * v1, 1.0, 0.0, -v1 * tmp5, v1 * tmp5},
                     {-tmp3 * w1, 0.0, 1.0, -w1 * tmp5, w1 * tmp5},
                     {-tmp3 * V2, v1, w1, (c1 * u1 - V2 - tmp0) * tmp5, (c1 * u1 + V2 + tmp0) * tmp5}};
  double V0[5][8];
  for (int k = 0; k < 8; k++)
    for (int m = 0; m < 5; m++) {
      double acc = 0.0;
      for (int j = 0; j < 5; j++) acc = acc + S[m][j] * U0[j][k];
      V0[m][k] = acc;
    }
  double VL[5], VR[5], QL[5], QR[5];
  for (int m = 0; m < 5; m++) { VL[m] = scheme_fP(V0[m], s); VR[m] = scheme_fm(V0[m], s); }
  for (int m = 0; m < 5; m++) {
    QL[m] = 0.0; QR[m] = 0.0;
    for (int j = 0; j < 5; j++) { QL[m] = QL[m] + S1[m][j] * VL[j]; QR[m] = QR[m] + S1[m][j] * VR[j]; }
  }
  UL[0] = QL[0]; UL[1] = QL[1] / UL[0]; UL[2] = QL[2] / UL[0]; UL[3] = QL[3] / UL[0];
  UL[4] = (QL[4] - (UL[1] * QL[1] + UL[2] * QL[2] + UL[3] * QL[3]) * 0.5) * (gamma - 1.0);
  UR[0] = QR[0]; UR[1] = QR[1] / UR[0]; UR[2] = QR[2] / UR[0]; UR[3] = QR[3] / UR[0];
  UR[4] = (QR[4] - (UR[1] * QR[1] + UR[2] * QR[2] + UR[3] * QR[3]) * 0.5) * (gamma - 1.0);
}

// ============================================================================================
// 1-D fluxes: sub_flux_split.f90
// ============================================================================================
static void flux_hll_hllc(const double* QL, const double* QR, double* F, double gamma, int iflux) {  // 13-95
  double dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  double dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  double UL[5], UR[5], Fl[5], Fr[5], Fsl[5], Fsr[5];
  UL[0] = dl; UL[1] = dl * uul; UL[2] = dl * vvl; UL[3] = dl * wwl; UL[4] = pl / (gamma - 1.0) + dl * (uul * uul + vvl * vvl + wwl * wwl) * 0.5;
  UR[0] = dr; UR[1] = dr * uur; UR[2] = dr * vvr; UR[3] = dr * wwr; UR[4] = pr / (gamma - 1.0) + dr * (uur * uur + vvr * vvr + wwr * wwr) * 0.5;
  double al = std::sqrt(gamma * pl / dl), ar = std::sqrt(gamma * pr / dr);
  double p_pvrs = 0.5 * (pl + pr) - (uur - uul) * (dl + dr) * (al + ar) * 0.125;
  double p_star = std::max(0.0, p_pvrs);
  double qql, qqr;
  if (p_star <= pl) qql = 1.0; else qql = std::sqrt(1.0 + ((gamma + 1.0) / (2.0 * gamma)) * (p_star / pl - 1.0));
  if (p_star <= pr) qqr = 1.0; else qqr = std::sqrt(1.0 + ((gamma + 1.0) / (2.0 * gamma)) * (p_star / pr - 1.0));
  double Sl = uul - al * qql, Sr = uur + ar * qqr;
  Fl[0] = UL[1]; Fl[1] = UL[1] * uul + pl; Fl[2] = UL[2] * uul; Fl[3] = UL[3] * uul; Fl[4] = uul * (UL[4] + pl);
  Fr[0] = UR[1]; Fr[1] = UR[1] * uur + pr; Fr[2] = UR[2] * uur; Fr[3] = UR[3] * uur; Fr[4] = uur * (UR[4] + pr);
  if (iflux == F_HLL) {
    if (Sl >= 0) { for (int m = 0; m < 5; m++) F[m] = Fl[m]; }
    else if (Sr <= 0) { for (int m = 0; m < 5; m++) F[m] = Fr[m]; }
    else { for (int m = 0; m < 5; m++) F[m] = (Sr * Fl[m] - Sl * Fr[m] + Sl * Sr * (UR[m] - UL[m])) / (Sr - Sl); }
    return;
  }
  double S_star = (pr - pl + dl * uul * (Sl - uul) - dr * uur * (Sr - uur)) / (dl * (Sl - uul) - dr * (Sr - uur));
  double tmpl = dl * (Sl - uul) / (Sl - S_star), tmpr = dr * (Sr - uur) / (Sr - S_star);
  Fsl[0] = Fl[0] + Sl * (tmpl - UL[0]);
  Fsl[1] = Fl[1] + Sl * (tmpl * S_star - UL[1]);
  Fsl[2] = Fl[2] + Sl * (tmpl * vvl - UL[2]);
  Fsl[3] = Fl[3] + Sl * (tmpl * wwl - UL[3]);
  double tmp = UL[4] / dl + (S_star - uul) * (S_star + pl / (dl * (Sl - uul)));
  Fsl[4] = Fl[4] + Sl * (tmpl * tmp - UL[4]);
  Fsr[0] = Fr[0] + Sr * (tmpr - UR[0]);
  Fsr[1] = Fr[1] + Sr * (tmpr * S_star - UR[1]);
  Fsr[2] = Fr[2] + Sr * (tmpr * vvr - UR[2]);
  Fsr[3] = Fr[3] + Sr * (tmpr * vvr - UR[3]);  // the reference uses vvr here (line 67)
  tmp = UR[4] / dr + (S_star - uur) * (S_star + pr / (dr * (Sr - uur)));
  Fsr[4] = Fr[4] + Sr * (tmpr * tmp - UR[4]);
  const double* src;
  if (Sl >= 0) src = Fl; else if (Sr <= 0) src = Fr; else if (S_star >= 0) src = Fsl; else src = Fsr;
  for (int m = 0; m < 5; m++) F[m] = src[m];
}

static void flux_sw(const double* QL, const double* QR, double* F, double gamma) {  // 102-141
  double dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  double dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  double al = std::sqrt(gamma * pl / dl), ar = std::sqrt(gamma * pr / dr);
  double tmp1 = 2.0 * (gamma - 1.0), tmp3 = (3.0 - gamma) / (2.0 * (gamma - 1.0));
  double E1P = (uul + std::fabs(uul)) * 0.5, E2P = (uul - al + std::fabs(uul - al)) * 0.5, E3P = (uul + al + std::fabs(uul + al)) * 0.5;
  double tmp0 = dl / (2.0 * gamma), fp[5], fm[5];
  fp[0] = tmp0 * (tmp1 * E1P + E2P + E3P);
  fp[1] = tmp0 * (tmp1 * E1P * uul + E2P * (uul - al) + E3P * (uul + al));
  fp[2] = tmp0 * (tmp1 * E1P * vvl + E2P * vvl + E3P * vvl);
  fp[3] = tmp0 * (tmp1 * E1P * wwl + E2P * wwl + E3P * wwl);
  fp[4] = tmp0 * (E1P * (gamma - 1.0) * (uul * uul + vvl * vvl + wwl * wwl) + E2P * (p2(uul - al) + vvl * vvl + wwl * wwl) * 0.5 +
                  E3P * (p2(uul + al) + vvl * vvl + wwl * wwl) * 0.5 + tmp3 * al * al * (E2P + E3P));
  double E1M = (uur - std::fabs(uur)) * 0.5, E2M = (uur - ar - std::fabs(uur - ar)) * 0.5, E3M = (uur + ar - std::fabs(uur + ar)) * 0.5;
  tmp0 = dr / (2.0 * gamma);
  fm[0] = tmp0 * (tmp1 * E1M + E2M + E3M);
  fm[1] = tmp0 * (tmp1 * E1M * uur + E2M * (uur - ar) + E3M * (uur + ar));
  fm[2] = tmp0 * (tmp1 * E1M * vvr + E2M * vvr + E3M * vvr);
  fm[3] = tmp0 * (tmp1 * E1M * wwr + E2M * wwr + E3M * wwr);
  fm[4] = tmp0 * (E1M * (gamma - 1.0) * (uur * uur + vvr * vvr + wwr * wwr) + E2M * (p2(uur - ar) + vvr * vvr + wwr * wwr) * 0.5 +
                  E3M * (p2(uur + ar) + vvr * vvr + wwr * wwr) * 0.5 + tmp3 * ar * ar * (E2M + E3M));
  for (int m = 0; m < 5; m++) F[m] = fp[m] + fm[m];
}

static void flux_roe(const double* QL, const double* QR, double* F, double gamma) {  // 148-210
  const double delt = 0.1;
  const double e8 = (double)1.e-8f;  // `1.e-8` default-real literal (lines 195, 197)
  double dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  double dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  double hl = gamma * pl / ((gamma - 1.0) * dl) + 0.5 * (uul * uul + vvl * vvl + wwl * wwl);
  double hr = gamma * pr / ((gamma - 1.0) * dr) + 0.5 * (uur * uur + vvr * vvr + wwr * wwr);
  double UL[5], UR[5], Fl[5], Fr[5];
  UL[0] = dl; UL[1] = dl * uul; UL[2] = dl * vvl; UL[3] = dl * wwl; UL[4] = pl / (gamma - 1.0) + dl * (uul * uul + vvl * vvl + wwl * wwl) * 0.5;
  UR[0] = dr; UR[1] = dr * uur; UR[2] = dr * vvr; UR[3] = dr * wwr; UR[4] = pr / (gamma - 1.0) + dr * (uur * uur + vvr * vvr + wwr * wwr) * 0.5;
  Fl[0] = UL[1]; Fl[1] = UL[1] * uul + pl; Fl[2] = UL[2] * uul; Fl[3] = UL[3] * uul; Fl[4] = uul * (UL[4] + pl);
  Fr[0] = UR[1]; Fr[1] = UR[1] * uur + pr; Fr[2] = UR[2] * uur; Fr[3] = UR[3] * uur; Fr[4] = uur * (UR[4] + pr);
  double tmpp = std::sqrt(dr / dl);
  double avu = (uul + tmpp * uur) / (1.0 + tmpp);
  double avv = (vvl + tmpp * vvr) / (1.0 + tmpp);
  double avw = (wwl + tmpp * wwr) / (1.0 + tmpp);
  double avh = (hl + tmpp * hr) / (1.0 + tmpp);
  double ava = std::sqrt((gamma - 1.0) * (avh - 0.5 * (avu * avu + avv * avv + avw * avw)));
  double l1 = std::fabs(avu - ava), l2 = std::fabs(avu), l3 = std::fabs(avu + ava);
  if (l1 < delt) l1 = (p2(l1) + delt * delt) / (2.0 * delt);
  if (l2 < delt) l2 = (p2(l2) + delt * delt) / (2.0 * delt);
  if (l3 < delt) l3 = (p2(l3) + delt * delt) / (2.0 * delt);
  double arr1, arr2, arr3, arr4, arr5;
  arr2 = (UR[2] - UL[2]) / (avv + e8) - (dr - dl);
  arr3 = (UR[3] - UL[3]) / (avw + e8) - (dr - dl);
  arr4 = (gamma - 1.0) * ((dr - dl) * (avh - avu * avu - avv * avv - avw * avw) + avu * (UR[1] - UL[1]) + avv * (UR[2] - UL[2]) +
                          avw * (UR[3] - UL[3]) - (UR[4] - UL[4])) / (ava * ava);
  arr1 = ((avu + ava) * (dr - dl) - UR[1] + UL[1] - ava * arr4) / (2.0 * ava);
  arr5 = dr - dl - (arr1 + arr4);
  F[0] = 0.5 * (Fl[0] + Fr[0]) - 0.5 * (l1 * arr1 + l2 * arr4 + l3 * arr5);
  F[1] = 0.5 * (Fl[1] + Fr[1]) - 0.5 * (l1 * arr1 * (avu - ava) + l2 * arr4 * avu + l3 * arr5 * (avu + ava));
  F[2] = 0.5 * (Fl[2] + Fr[2]) - 0.5 * (l1 * arr1 * avv + l2 * arr2 * avv + l2 * arr4 * avv + l3 * arr5 * avv);
  F[3] = 0.5 * (Fl[3] + Fr[3]) - 0.5 * (l1 * arr1 * avw + l2 * arr3 * avw + l2 * arr4 * avw + l3 * arr5 * avw);
  F[4] = 0.5 * (Fl[4] + Fr[4]) - 0.5 * (l1 * arr1 * (avh - avu * ava) + l2 * arr2 * avv * avv + l2 * arr3 * avw * avw +
                                        l2 * arr4 * 0.5 * (avu * avu + avv * avv + avw * avw) + l3 * arr5 * (avh + avu * ava));
}

static void flux_vl(const double* QL, const double* QR, double* F, double gamma) {  // 217-275
  double dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  double dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  double al = std::sqrt(gamma * pl / dl), ar = std::sqrt(gamma * pr / dr);
  double Ml = uul / al, Mr = uur / ar, fp[5] = {0, 0, 0, 0, 0}, fm[5] = {0, 0, 0, 0, 0};
  if (Ml >= 1.0) {
    fp[0] = dl * uul; fp[1] = dl * uul * uul + pl; fp[2] = dl * uul * vvl; fp[3] = dl * uul * wwl;
    fp[4] = uul * (gamma * pl / (gamma - 1.0) + 0.5 * dl * (uul * uul + vvl * vvl + wwl * wwl));
  } else if (std::fabs(Ml) < 1.0) {
    double Mp = 0.25 * (1.0 + Ml) * (1.0 + Ml), tmp0 = dl * al * Mp;
    fp[0] = tmp0; fp[1] = tmp0 * ((gamma - 1.0) * uul + 2.0 * al) / gamma; fp[2] = tmp0 * vvl; fp[3] = tmp0 * wwl;
    fp[4] = tmp0 * (((gamma - 1.0) * uul + 2.0 * al) * ((gamma - 1.0) * uul + 2.0 * al) * 0.5 / (gamma * gamma - 1.0) + 0.5 * (vvl * vvl + wwl * wwl));
  }
  if (Mr >= 1.0) {
  } else if (std::fabs(Mr) < 1.0) {
    double Mm = -0.25 * (Mr - 1.0) * (Mr - 1.0), tmp0 = dr * ar * Mm;
    fm[0] = tmp0; fm[1] = tmp0 * ((gamma - 1.0) * uur - 2.0 * ar) / gamma; fm[2] = tmp0 * vvr; fm[3] = tmp0 * wwr;
    fm[4] = tmp0 * (((gamma - 1.0) * uur - 2.0 * ar) * ((gamma - 1.0) * uur - 2.0 * ar) * 0.5 / (gamma * gamma - 1.0) + 0.5 * (vvr * vvr + wwr * wwr));
  } else if (Mr <= -1.0) {
    fm[0] = dr * uur; fm[1] = dr * uur * uur + pr; fm[2] = dr * uur * vvr; fm[3] = dr * uur * wwr;
    fm[4] = uur * (gamma * pr / (gamma - 1.0) + 0.5 * dr * (uur * uur + vvr * vvr + wwr * wwr));
  }
  for (int m = 0; m < 5; m++) F[m] = fp[m] + fm[m];
}

static void flux_ausmpw(const double* QL, const double* QR, double* F, double gamma) {  // 356-442
  double dl = QL[0], uul = QL[1], vvl = QL[2], wwl = QL[3], pl = QL[4];
  double dr = QR[0], uur = QR[1], vvr = QR[2], wwr = QR[3], pr = QR[4];
  double hl = gamma * pl / ((gamma - 1.0) * dl) + 0.5 * (uul * uul + vvl * vvl + wwl * wwl);
  double hr = gamma * pr / ((gamma - 1.0) * dr) + 0.5 * (uur * uur + vvr * vvr + wwr * wwr);
  double al = std::sqrt(gamma * pl / dl), ar = std::sqrt(gamma * pr / dr);
  double a = 0.5 * (al + ar), Ml = uul / a, Mr = uur / a;
  double wpl = 1.0 - std::pow(std::min(pl / pr, pr / pl), 3.0);
  double plpl, plpr;
  if ((0.75 <= std::min(pl / pr, pr / pl)) && (1.0 > std::min(pl / pr, pr / pl))) plpl = 4.0 * std::min(pl / pr, pr / pl) - 3.0; else plpl = 0.0;
  if ((0.75 <= std::min(pr / pl, pl / pr)) && (1.0 > std::min(pr / pl, pl / pr))) plpr = 4.0 * std::min(pr / pl, pl / pr) - 3.0; else plpr = 0.0;
  double Pp5, Pm5;
  if (std::fabs(Ml) >= 1.0) Pp5 = 0.5 * (Ml + std::fabs(Ml)) / Ml;
  else Pp5 = 0.25 * (Ml + 1.0) * (Ml + 1.0) * (2.0 - Ml) + 3.0 * Ml * (Ml * Ml - 1.0) * (Ml * Ml - 1.0) / 16.0;
  if (std::fabs(Mr) >= 1.0) Pm5 = 0.5 * (Mr - std::fabs(Mr)) / Mr;
  else Pm5 = 0.25 * (Mr - 1.0) * (Mr - 1.0) * (2.0 + Mr) - 3.0 * Mr * (Mr * Mr - 1.0) * (Mr * Mr - 1.0) / 16.0;
  double p = pl * Pp5 + pr * Pm5;
  double Mp4, Mm4, fL, fR;
  if (std::fabs(Ml) >= 1.0) { Mp4 = 0.5 * (Ml + std::fabs(Ml)); fL = 0.0; }
  else {
    Mp4 = 0.25 * (Ml + 1.0) * (Ml + 1.0) + 0.125 * (Ml * Ml - 1.0) * (Ml * Ml - 1.0);
    fL = (pl / p - 1.0) * plpl * std::fabs(0.25 * (Ml + 1.0) * (Ml + 1.0)) * std::min(1.0, std::pow(std::sqrt(uul * uul + vvl * vvl + wwl * wwl) / a, 0.25));
  }
  if (std::fabs(Mr) >= 1.0) { Mm4 = 0.5 * (Mr - std::fabs(Mr)); fR = 0.0; }
  else {
    Mm4 = -0.25 * (Mr - 1.0) * (Mr - 1.0) - 0.125 * (Mr * Mr - 1.0) * (Mr * Mr - 1.0);
    fR = (pr / p - 1.0) * plpr * std::fabs(-0.25 * (Mr - 1.0) * (Mr - 1.0)) * std::min(1.0, std::pow(std::sqrt(uur * uur + vvr * vvr + wwr * wwr) / a, 0.25));
  }
  double M = Mp4 + Mm4, MLp, MRm;
  if (M >= 0.0) MLp = Mp4 + Mm4 - Mm4 * wpl * (1.0 + fR) + (fL * Mp4 + fR * Mm4); else MLp = Mp4 * wpl * (1.0 + fL);
  if (M < 0.0) MRm = Mp4 + Mm4 - Mp4 * wpl * (1.0 + fL) + (fL * Mp4 + fR * Mm4); else MRm = Mm4 * wpl * (1.0 + fR);
  double fp[5] = {dl, dl * uul, dl * vvl, dl * wwl, dl * hl};
  double fm[5] = {dr, dr * uur, dr * vvr, dr * wwr, dr * hr};
  F[0] = MLp * a * fp[0] + MRm * a * fm[0];
  F[1] = MLp * a * fp[1] + MRm * a * fm[1] + p;
  F[2] = MLp * a * fp[2] + MRm * a * fm[2];
  F[3] = MLp * a * fp[3] + MRm * a * fm[3];
  F[4] = MLp * a * fp[4] + MRm * a * fm[4];
}

static void flux_1d(const double* QL, const double* QR, double* F, double gamma, int iflux) {  // dispatch 320-330
  if (iflux == F_SW) flux_sw(QL, QR, F, gamma);
  else if (iflux == F_ROE) flux_roe(QL, QR, F, gamma);
  else if (iflux == F_VL) flux_vl(QL, QR, F, gamma);
  else if (iflux == F_AUSM) flux_ausmpw(QL, QR, F, gamma);
  else flux_hll_hllc(QL, QR, F, gamma, iflux);
}

// ============================================================================================
// setup: coordinate ghosts, geometry, mesh quality, BcI/J/K, wall distance, init
// ============================================================================================
static void coordinate_ghosts(Case& C) {  // sub_update_buffer_mpi.f90:230-512
  // interface copy (Coordinate_send_mpi 250-352): source = 1 interior node layer, target = 1 ghost layer
  for (size_t mb = 0; mb < C.B.size(); mb++) {
    Block& B = C.B[mb];
    for (const Sub& Bc : B.sub) {
      if (Bc.bc >= 0) continue;
      int kb[3] = {Bc.ib, Bc.jb, Bc.kb}, ke[3] = {Bc.ie, Bc.je, Bc.ke};
      int k = (Bc.face - 1) % 3;
      if (Bc.face <= 3) kb[k] = kb[k] + 1; else kb[k] = kb[k] - 1;
      ke[k] = kb[k];
      int kb1[3] = {Bc.ib1, Bc.jb1, Bc.kb1}, ke1[3] = {Bc.ie1, Bc.je1, Bc.ke1};
      k = (Bc.face1 - 1) % 3;
      if (Bc.face1 <= 3) kb1[k] = kb1[k] - 1; else kb1[k] = kb1[k] + 1;
      ke1[k] = kb1[k];
      int L[3] = {std::abs(Bc.L1), std::abs(Bc.L2), std::abs(Bc.L3)};
      int P[3] = {Bc.L1 >= 0 ? 1 : -1, Bc.L2 >= 0 ? 1 : -1, Bc.L3 >= 0 ? 1 : -1};
      int ks[3];
      for (int q = 0; q < 3; q++) ks[q] = P[q] > 0 ? kb[q] : ke[q];
      Block& B1 = C.B[Bc.nb1 - 1];
      for (int kk = kb1[2]; kk <= ke1[2]; kk++)
        for (int jj = kb1[1]; jj <= ke1[1]; jj++)
          for (int ii = kb1[0]; ii <= ke1[0]; ii++) {
            int ka[3] = {ii - kb1[0], jj - kb1[1], kk - kb1[2]};
            int i1 = ks[0] + ka[L[0] - 1] * P[0], j1 = ks[1] + ka[L[1] - 1] * P[1], k1 = ks[2] + ka[L[2] - 1] * P[2];
            B1.x(ii, jj, kk) = B.x(i1, j1, k1);
            B1.y(ii, jj, kk) = B.y(i1, j1, k1);
            B1.z(ii, jj, kk) = B.z(i1, j1, k1);
          }
    }
  }
  // physical boundaries: linear extrapolation (coordinate_boundary_and_corner 413-468)
  for (Block& B : C.B) {
    for (const Sub& Bc : B.sub) {
      if (Bc.bc < 0) continue;
      int i1 = Bc.ib, i2 = Bc.ie, j1 = Bc.jb, j2 = Bc.je, k1 = Bc.kb, k2 = Bc.ke;
      A3* X[3] = {&B.x, &B.y, &B.z};
      for (A3* a : X) {
        A3& x = *a;
        if (Bc.face == 1) { for (int k = k1; k <= k2; k++) for (int j = j1; j <= j2; j++) x(i1 - 1, j, k) = 2.0 * x(i1, j, k) - x(i1 + 1, j, k); }
        else if (Bc.face == 2) { for (int k = k1; k <= k2; k++) for (int i = i1; i <= i2; i++) x(i, j1 - 1, k) = 2.0 * x(i, j1, k) - x(i, j1 + 1, k); }
        else if (Bc.face == 3) { for (int j = j1; j <= j2; j++) for (int i = i1; i <= i2; i++) x(i, j, k1 - 1) = 2.0 * x(i, j, k1) - x(i, j, k1 + 1); }
        else if (Bc.face == 4) { for (int k = k1; k <= k2; k++) for (int j = j1; j <= j2; j++) x(i2 + 1, j, k) = 2.0 * x(i2, j, k) - x(i2 - 1, j, k); }
        else if (Bc.face == 5) { for (int k = k1; k <= k2; k++) for (int i = i1; i <= i2; i++) x(i, j2 + 1, k) = 2.0 * x(i, j2, k) - x(i, j2 - 1, k); }
        else if (Bc.face == 6) { for (int j = j1; j <= j2; j++) for (int i = i1; i <= i2; i++) x(i, j, k2 + 1) = 2.0 * x(i, j, k2) - x(i, j, k2 - 1); }
      }
    }
  }
  // edges and vertices (get_xyz_conner 476-512)
  for (Block& B : C.B) {
    int nx = B.nx, ny = B.ny, nz = B.nz;
    A3* X[3] = {&B.x, &B.y, &B.z};
    for (A3* a : X) {
      A3& x = *a;
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
      x(0, 0, 0) = (2.0 * (x(1, 0, 0) + x(0, 1, 0) + x(0, 0, 1)) - (x(1, 1, 0) + x(1, 0, 1) + x(0, 1, 1))) / 3.0;
      x(nx + 1, 0, 0) = (2.0 * (x(nx, 0, 0) + x(nx + 1, 1, 0) + x(nx + 1, 0, 1)) - (x(nx, 1, 0) + x(nx, 0, 1) + x(nx + 1, 1, 1))) / 3.0;
      x(0, ny + 1, 0) = (2.0 * (x(1, ny + 1, 0) + x(0, ny, 0) + x(0, ny + 1, 1)) - (x(1, ny, 0) + x(1, ny + 1, 1) + x(0, ny, 1))) / 3.0;
      x(nx + 1, ny + 1, 0) = (2.0 * (x(nx, ny + 1, 0) + x(nx + 1, ny, 0) + x(nx + 1, ny + 1, 1)) - (x(nx, ny, 0) + x(nx, ny + 1, 1) + x(nx + 1, ny, 1))) / 3.0;
      x(0, 0, nz + 1) = (2.0 * (x(1, 0, nz + 1) + x(0, 1, nz + 1) + x(0, 0, nz)) - (x(1, 1, nz + 1) + x(1, 0, nz) + x(0, 1, nz))) / 3.0;
      x(nx + 1, 0, nz + 1) = (2.0 * (x(nx, 0, nz + 1) + x(nx + 1, 1, nz + 1) + x(nx + 1, 0, nz)) - (x(nx, 1, nz + 1) + x(nx, 0, nz) + x(nx + 1, 1, nz))) / 3.0;
      x(0, ny + 1, nz + 1) = (2.0 * (x(1, ny + 1, nz + 1) + x(0, ny, nz + 1) + x(0, ny + 1, nz)) - (x(1, ny, nz + 1) + x(1, ny + 1, nz) + x(0, ny, nz))) / 3.0;
      x(nx + 1, ny + 1, nz + 1) = (2.0 * (x(nx, ny + 1, nz + 1) + x(nx + 1, ny, nz + 1) + x(nx + 1, ny + 1, nz)) - (x(nx, ny, nz + 1) + x(nx, ny + 1, nz) + x(nx + 1, ny, nz))) / 3.0;
    }
  }
}

static void jac9(double xi, double yi, double zi, double xj, double yj, double zj, double xk, double yk, double zk, double* o) {
  double Jac1 = xi * yj * zk + yi * zj * xk + zi * xj * yk - xi * zj * yk - yi * xj * zk - zi * yj * xk;
  if (std::fabs(Jac1) < Lim_Zero) Jac1 = Lim_Zero;
  double Jac = 1.0 / Jac1;
  o[0] = Jac * (yj * zk - zj * yk); o[1] = Jac * (zj * xk - xj * zk); o[2] = Jac * (xj * yk - yj * xk);
  o[3] = Jac * (yk * zi - zk * yi); o[4] = Jac * (zk * xi - xk * zi); o[5] = Jac * (xk * yi - yk * xi);
  o[6] = Jac * (yi * zj - zi * yj); o[7] = Jac * (zi * xj - xi * zj); o[8] = Jac * (xi * yj - yi * xj);
}

static void geometry(Block& B) {  // sub_geometry.f90:6-346
  int nx = B.nx, ny = B.ny, nz = B.nz;
  A3 Vi, Vj, Vk;
  Vi.alloc(1, nx, 1, ny, 1, nz); Vj.alloc(1, nx, 1, ny, 1, nz); Vk.alloc(1, nx, 1, ny, 1, nz);
  A3 &x = B.x, &y = B.y, &z = B.z;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        double t1x, t1y, t1z, t2x, t2y, t2z, s1x, s1y, s1z, ss, xa, ya, za;
        t1x = x(i, j + 1, k) - x(i, j, k + 1); t1y = y(i, j + 1, k) - y(i, j, k + 1); t1z = z(i, j + 1, k) - z(i, j, k + 1);
        t2x = x(i, j + 1, k + 1) - x(i, j, k); t2y = y(i, j + 1, k + 1) - y(i, j, k); t2z = z(i, j + 1, k + 1) - z(i, j, k);
        s1x = t1y * t2z - t1z * t2y; s1y = t1z * t2x - t1x * t2z; s1z = t1x * t2y - t1y * t2x;
        ss = std::sqrt(s1x * s1x + s1y * s1y + s1z * s1z);
        B.Si(i, j, k) = ss * 0.5;
        if (ss >= Lim_Zero) { B.ni1(i, j, k) = s1x / ss; B.ni2(i, j, k) = s1y / ss; B.ni3(i, j, k) = s1z / ss; }
        else { B.ni1(i, j, k) = 1.0; B.ni2(i, j, k) = 0.0; B.ni3(i, j, k) = 0.0; }
        xa = (x(i, j, k) + x(i, j + 1, k) + x(i, j, k + 1) + x(i, j + 1, k + 1)) * 0.25;
        ya = (y(i, j, k) + y(i, j + 1, k) + y(i, j, k + 1) + y(i, j + 1, k + 1)) * 0.25;
        za = (z(i, j, k) + z(i, j + 1, k) + z(i, j, k + 1) + z(i, j + 1, k + 1)) * 0.25;
        Vi(i, j, k) = (s1x * xa + s1y * ya + s1z * za) * 0.5;

        t1x = x(i + 1, j, k + 1) - x(i, j, k); t1y = y(i + 1, j, k + 1) - y(i, j, k); t1z = z(i + 1, j, k + 1) - z(i, j, k);
        t2x = x(i + 1, j, k) - x(i, j, k + 1); t2y = y(i + 1, j, k) - y(i, j, k + 1); t2z = z(i + 1, j, k) - z(i, j, k + 1);
        s1x = t1y * t2z - t1z * t2y; s1y = t1z * t2x - t1x * t2z; s1z = t1x * t2y - t1y * t2x;
        ss = std::sqrt(s1x * s1x + s1y * s1y + s1z * s1z);
        B.Sj(i, j, k) = ss * 0.5;
        if (ss >= Lim_Zero) { B.nj1(i, j, k) = s1x / ss; B.nj2(i, j, k) = s1y / ss; B.nj3(i, j, k) = s1z / ss; }
        else { B.nj1(i, j, k) = 1.0; B.nj2(i, j, k) = 0.0; B.nj3(i, j, k) = 0.0; }
        xa = (x(i, j, k) + x(i + 1, j, k) + x(i, j, k + 1) + x(i + 1, j, k + 1)) * 0.25;
        ya = (y(i, j, k) + y(i + 1, j, k) + y(i, j, k + 1) + y(i + 1, j, k + 1)) * 0.25;
        za = (z(i, j, k) + z(i + 1, j, k) + z(i, j, k + 1) + z(i + 1, j, k + 1)) * 0.25;
        Vj(i, j, k) = (s1x * xa + s1y * ya + s1z * za) * 0.5;

        t1x = x(i + 1, j + 1, k) - x(i, j, k); t1y = y(i + 1, j + 1, k) - y(i, j, k); t1z = z(i + 1, j + 1, k) - z(i, j, k);
        t2x = x(i, j + 1, k) - x(i + 1, j, k); t2y = y(i, j + 1, k) - y(i + 1, j, k); t2z = z(i, j + 1, k) - z(i + 1, j, k);
        s1x = t1y * t2z - t1z * t2y; s1y = t1z * t2x - t1x * t2z; s1z = t1x * t2y - t1y * t2x;
        ss = std::sqrt(s1x * s1x + s1y * s1y + s1z * s1z);
        B.Sk(i, j, k) = ss * 0.5;
        if (ss >= Lim_Zero) { B.nk1(i, j, k) = s1x / ss; B.nk2(i, j, k) = s1y / ss; B.nk3(i, j, k) = s1z / ss; }
        else { B.nk1(i, j, k) = 1.0; B.nk2(i, j, k) = 0.0; B.nk3(i, j, k) = 0.0; }
        xa = (x(i, j, k) + x(i + 1, j, k) + x(i, j + 1, k) + x(i + 1, j + 1, k)) * 0.25;
        ya = (y(i, j, k) + y(i + 1, j, k) + y(i, j + 1, k) + y(i + 1, j + 1, k)) * 0.25;
        za = (z(i, j, k) + z(i + 1, j, k) + z(i, j + 1, k) + z(i + 1, j + 1, k)) * 0.25;
        Vk(i, j, k) = (s1x * xa + s1y * ya + s1z * za) * 0.5;
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++)
        B.vol(i, j, k) = (Vi(i + 1, j, k) - Vi(i, j, k) + Vj(i, j + 1, k) - Vj(i, j, k) + Vk(i, j, k + 1) - Vk(i, j, k)) / 3.0;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        B.xc(i, j, k) = (x(i, j, k) + x(i, j + 1, k) + x(i, j, k + 1) + x(i, j + 1, k + 1) + x(i + 1, j, k) + x(i + 1, j + 1, k) + x(i + 1, j, k + 1) + x(i + 1, j + 1, k + 1)) * 0.125;
        B.yc(i, j, k) = (y(i, j, k) + y(i, j + 1, k) + y(i, j, k + 1) + y(i, j + 1, k + 1) + y(i + 1, j, k) + y(i + 1, j + 1, k) + y(i + 1, j, k + 1) + y(i + 1, j + 1, k + 1)) * 0.125;
        B.zc(i, j, k) = (z(i, j, k) + z(i, j + 1, k) + z(i, j, k + 1) + z(i, j + 1, k + 1) + z(i + 1, j, k) + z(i + 1, j + 1, k) + z(i + 1, j, k + 1) + z(i + 1, j + 1, k + 1)) * 0.125;
      }
  A3 &xc = B.xc, &yc = B.yc, &zc = B.zc;
  double o[9];
  // (I-1/2,J,K) family (110-175)
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++) {
        double xi = xc(i, j, k) - xc(i - 1, j, k), yi = yc(i, j, k) - yc(i - 1, j, k), zi = zc(i, j, k) - zc(i - 1, j, k);
        double xj1, yj1, zj1, xj2, yj2, zj2, xk1, yk1, zk1, xk2, yk2, zk2;
        if ((i == 1 || i == nx) && (j == 1 || j == ny - 1)) {
          xj1 = xc(i, j - 1, k); yj1 = yc(i, j - 1, k); zj1 = zc(i, j - 1, k);
          xj2 = xc(i, j + 1, k); yj2 = yc(i, j + 1, k); zj2 = zc(i, j + 1, k);
        } else {
          xj1 = 0.5 * (xc(i, j - 1, k) + xc(i - 1, j - 1, k)); yj1 = 0.5 * (yc(i, j - 1, k) + yc(i - 1, j - 1, k)); zj1 = 0.5 * (zc(i, j - 1, k) + zc(i - 1, j - 1, k));
          xj2 = 0.5 * (xc(i, j + 1, k) + xc(i - 1, j + 1, k)); yj2 = 0.5 * (yc(i, j + 1, k) + yc(i - 1, j + 1, k)); zj2 = 0.5 * (zc(i, j + 1, k) + zc(i - 1, j + 1, k));
        }
        if ((i == 1 || i == nx) && (k == 1 || k == nz - 1)) {
          xk1 = xc(i, j, k - 1); yk1 = yc(i, j, k - 1); zk1 = zc(i, j, k - 1);
          xk2 = xc(i, j, k + 1); yk2 = yc(i, j, k + 1); zk2 = zc(i, j, k + 1);
        } else {
          xk1 = 0.5 * (xc(i, j, k - 1) + xc(i - 1, j, k - 1)); yk1 = 0.5 * (yc(i, j, k - 1) + yc(i - 1, j, k - 1)); zk1 = 0.5 * (zc(i, j, k - 1) + zc(i - 1, j, k - 1));
          xk2 = 0.5 * (xc(i, j, k + 1) + xc(i - 1, j, k + 1)); yk2 = 0.5 * (yc(i, j, k + 1) + yc(i - 1, j, k + 1)); zk2 = 0.5 * (zc(i, j, k + 1) + zc(i - 1, j, k + 1));
        }
        double xj = 0.5 * (xj2 - xj1), yj = 0.5 * (yj2 - yj1), zj = 0.5 * (zj2 - zj1);
        double xk = 0.5 * (xk2 - xk1), yk = 0.5 * (yk2 - yk1), zk = 0.5 * (zk2 - zk1);
        jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, o);
        B.ix1(i, j, k) = o[0]; B.iy1(i, j, k) = o[1]; B.iz1(i, j, k) = o[2]; B.jx1(i, j, k) = o[3]; B.jy1(i, j, k) = o[4];
        B.jz1(i, j, k) = o[5]; B.kx1(i, j, k) = o[6]; B.ky1(i, j, k) = o[7]; B.kz1(i, j, k) = o[8];
      }
  // (I,J-1/2,K) family (180-242)
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double xj = xc(i, j, k) - xc(i, j - 1, k), yj = yc(i, j, k) - yc(i, j - 1, k), zj = zc(i, j, k) - zc(i, j - 1, k);
        double xi1, yi1, zi1, xi2, yi2, zi2, xk1, yk1, zk1, xk2, yk2, zk2;
        if ((j == 1 || j == ny) && (i == 1 || i == nx - 1)) {
          xi1 = xc(i - 1, j, k); yi1 = yc(i - 1, j, k); zi1 = zc(i - 1, j, k);
          xi2 = xc(i + 1, j, k); yi2 = yc(i + 1, j, k); zi2 = zc(i + 1, j, k);
        } else {
          xi1 = 0.5 * (xc(i - 1, j, k) + xc(i - 1, j - 1, k)); yi1 = 0.5 * (yc(i - 1, j, k) + yc(i - 1, j - 1, k)); zi1 = 0.5 * (zc(i - 1, j, k) + zc(i - 1, j - 1, k));
          xi2 = 0.5 * (xc(i + 1, j, k) + xc(i + 1, j - 1, k)); yi2 = 0.5 * (yc(i + 1, j, k) + yc(i + 1, j - 1, k)); zi2 = 0.5 * (zc(i + 1, j, k) + zc(i + 1, j - 1, k));
        }
        if ((j == 1 || j == ny) && (k == 1 || k == nz - 1)) {
          xk1 = xc(i, j, k - 1); yk1 = yc(i, j, k - 1); zk1 = zc(i, j, k - 1);
          xk2 = xc(i, j, k + 1); yk2 = yc(i, j, k + 1); zk2 = zc(i, j, k + 1);
        } else {
          xk1 = 0.5 * (xc(i, j, k - 1) + xc(i, j - 1, k - 1)); yk1 = 0.5 * (yc(i, j, k - 1) + yc(i, j - 1, k - 1)); zk1 = 0.5 * (zc(i, j, k - 1) + zc(i, j - 1, k - 1));
          xk2 = 0.5 * (xc(i, j, k + 1) + xc(i, j - 1, k + 1)); yk2 = 0.5 * (yc(i, j, k + 1) + yc(i, j - 1, k + 1)); zk2 = 0.5 * (zc(i, j, k + 1) + zc(i, j - 1, k + 1));
        }
        double xi = 0.5 * (xi2 - xi1), yi = 0.5 * (yi2 - yi1), zi = 0.5 * (zi2 - zi1);
        double xk = 0.5 * (xk2 - xk1), yk = 0.5 * (yk2 - yk1), zk = 0.5 * (zk2 - zk1);
        jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, o);
        B.ix2(i, j, k) = o[0]; B.iy2(i, j, k) = o[1]; B.iz2(i, j, k) = o[2]; B.jx2(i, j, k) = o[3]; B.jy2(i, j, k) = o[4];
        B.jz2(i, j, k) = o[5]; B.kx2(i, j, k) = o[6]; B.ky2(i, j, k) = o[7]; B.kz2(i, j, k) = o[8];
      }
  // (I,J,K-1/2) family (247-310)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double xk = xc(i, j, k) - xc(i, j, k - 1), yk = yc(i, j, k) - yc(i, j, k - 1), zk = zc(i, j, k) - zc(i, j, k - 1);
        double xi1, yi1, zi1, xi2, yi2, zi2, xj1, yj1, zj1, xj2, yj2, zj2;
        if ((k == 1 || k == nz) && (i == 1 || i == nx - 1)) {
          xi1 = xc(i - 1, j, k); yi1 = yc(i - 1, j, k); zi1 = zc(i - 1, j, k);
          xi2 = xc(i + 1, j, k); yi2 = yc(i + 1, j, k); zi2 = zc(i + 1, j, k);
        } else {
          xi1 = 0.5 * (xc(i - 1, j, k) + xc(i - 1, j, k - 1)); yi1 = 0.5 * (yc(i - 1, j, k) + yc(i - 1, j, k - 1)); zi1 = 0.5 * (zc(i - 1, j, k) + zc(i - 1, j, k - 1));
          xi2 = 0.5 * (xc(i + 1, j, k) + xc(i + 1, j, k - 1)); yi2 = 0.5 * (yc(i + 1, j, k) + yc(i + 1, j, k - 1)); zi2 = 0.5 * (zc(i + 1, j, k) + zc(i + 1, j, k - 1));
        }
        if ((k == 1 || k == nz) && (j == 1 || j == ny - 1)) {
          xj1 = xc(i, j - 1, k); yj1 = yc(i, j - 1, k); zj1 = zc(i, j - 1, k);
          xj2 = xc(i, j + 1, k); yj2 = yc(i, j + 1, k); zj2 = zc(i, j + 1, k);
        } else {
          xj1 = 0.5 * (xc(i, j - 1, k) + xc(i, j - 1, k - 1)); yj1 = 0.5 * (yc(i, j - 1, k) + yc(i, j - 1, k - 1)); zj1 = 0.5 * (zc(i, j - 1, k) + zc(i, j - 1, k - 1));
          xj2 = 0.5 * (xc(i, j + 1, k) + xc(i, j + 1, k - 1)); yj2 = 0.5 * (yc(i, j + 1, k) + yc(i, j + 1, k - 1)); zj2 = 0.5 * (zc(i, j + 1, k) + zc(i, j + 1, k - 1));
        }
        double xi = 0.5 * (xi2 - xi1), yi = 0.5 * (yi2 - yi1), zi = 0.5 * (zi2 - zi1);
        double xj = 0.5 * (xj2 - xj1), yj = 0.5 * (yj2 - yj1), zj = 0.5 * (zj2 - zj1);
        jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, o);
        B.ix3(i, j, k) = o[0]; B.iy3(i, j, k) = o[1]; B.iz3(i, j, k) = o[2]; B.jx3(i, j, k) = o[3]; B.jy3(i, j, k) = o[4];
        B.jz3(i, j, k) = o[5]; B.kx3(i, j, k) = o[6]; B.ky3(i, j, k) = o[7]; B.kz3(i, j, k) = o[8];
      }
  // cell-centre family (312-341)
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double xi = xc(i + 1, j, k) - xc(i - 1, j, k), yi = yc(i + 1, j, k) - yc(i - 1, j, k), zi = zc(i + 1, j, k) - zc(i - 1, j, k);
        double xj = xc(i, j + 1, k) - xc(i, j - 1, k), yj = yc(i, j + 1, k) - yc(i, j - 1, k), zj = zc(i, j + 1, k) - zc(i, j - 1, k);
        double xk = xc(i, j, k + 1) - xc(i, j, k - 1), yk = yc(i, j, k + 1) - yc(i, j, k - 1), zk = zc(i, j, k + 1) - zc(i, j, k - 1);
        jac9(xi, yi, zi, xj, yj, zj, xk, yk, zk, o);
        B.ix0(i, j, k) = o[0]; B.iy0(i, j, k) = o[1]; B.iz0(i, j, k) = o[2]; B.jx0(i, j, k) = o[3]; B.jy0(i, j, k) = o[4];
        B.jz0(i, j, k) = o[5]; B.kx0(i, j, k) = o[6]; B.ky0(i, j, k) = o[7]; B.kz0(i, j, k) = o[8];
      }
}

static void mesh_quality(Block& B) {  // sub_geometry.f90:361-444 (the dt factor only)
  A3 &xc = B.xc, &yc = B.yc, &zc = B.zc;
  for (int k = 1; k <= B.nz - 1; k++)
    for (int j = 1; j <= B.ny - 1; j++)
      for (int i = 1; i <= B.nx - 1; i++) {
        double fl1 = std::sqrt(p2(xc(i, j, k) - xc(i - 1, j, k)) + p2(yc(i, j, k) - yc(i - 1, j, k)) + p2(zc(i, j, k) - zc(i - 1, j, k))) /
                     std::sqrt(p2(xc(i, j, k) - xc(i + 1, j, k)) + p2(yc(i, j, k) - yc(i + 1, j, k)) + p2(zc(i, j, k) - zc(i + 1, j, k)));
        double fl2 = std::sqrt(p2(xc(i, j, k) - xc(i, j - 1, k)) + p2(yc(i, j, k) - yc(i, j - 1, k)) + p2(zc(i, j, k) - zc(i, j - 1, k))) /
                     std::sqrt(p2(xc(i, j, k) - xc(i, j + 1, k)) + p2(yc(i, j, k) - yc(i, j + 1, k)) + p2(zc(i, j, k) - zc(i, j + 1, k)));
        double fl3 = std::sqrt(p2(xc(i, j, k) - xc(i, j, k - 1)) + p2(yc(i, j, k) - yc(i, j, k - 1)) + p2(zc(i, j, k) - zc(i, j, k - 1))) /
                     std::sqrt(p2(xc(i, j, k) - xc(i, j, k + 1)) + p2(yc(i, j, k) - yc(i, j, k + 1)) + p2(zc(i, j, k) - zc(i, j, k + 1)));
        if (fl1 < 1.0) fl1 = 1.0 / fl1;
        if (fl2 < 1.0) fl2 = 1.0 / fl2;
        if (fl3 < 1.0) fl3 = 1.0 / fl3;
        double fl = std::max(std::max(fl1, fl2), fl3);
        double x1, x2, y1, y2, z1, z2, ft1, ft2, ft3;
        x1 = xc(i, j, k) - xc(i - 1, j, k); x2 = xc(i + 1, j, k) - xc(i, j, k);
        y1 = yc(i, j, k) - yc(i - 1, j, k); y2 = yc(i + 1, j, k) - yc(i, j, k);
        z1 = zc(i, j, k) - zc(i - 1, j, k); z2 = zc(i + 1, j, k) - zc(i, j, k);
        ft1 = (x1 * x2 + y1 * y2 + z1 * z2) / std::sqrt((x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2));
        x1 = xc(i, j, k) - xc(i, j - 1, k); x2 = xc(i, j + 1, k) - xc(i, j, k);
        y1 = yc(i, j, k) - yc(i, j - 1, k); y2 = yc(i, j + 1, k) - yc(i, j, k);
        z1 = zc(i, j, k) - zc(i, j - 1, k); z2 = zc(i, j + 1, k) - zc(i, j, k);
        ft2 = (x1 * x2 + y1 * y2 + z1 * z2) / std::sqrt((x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2));
        x1 = xc(i, j, k) - xc(i, j, k - 1); x2 = xc(i, j, k + 1) - xc(i, j, k);
        y1 = yc(i, j, k) - yc(i, j, k - 1); y2 = yc(i, j, k + 1) - yc(i, j, k);
        z1 = zc(i, j, k) - zc(i, j, k - 1); z2 = zc(i, j, k + 1) - zc(i, j, k);
        ft3 = (x1 * x2 + y1 * y2 + z1 * z2) / std::sqrt((x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2));
        double ft = std::min(1.0, 1.0 * std::min(std::min(ft1, ft2), ft3));
        ft = std::acos(ft);
        double Af = 0.9 * std::exp(-4.0 * p2(fl - 1.0)) + 0.1;
        double Aa = 0.9 * std::exp(-p2(4.0 / 3.1415926535 * ft)) + 0.1;
        B.dtime_mesh(i, j, k) = std::min(Af, Aa);
      }
}

static void set_BcK(Block& B) {  // sub_init.f90:545-577
  std::fill(B.BcI.v.begin(), B.BcI.v.end(), 0);
  std::fill(B.BcJ.v.begin(), B.BcJ.v.end(), 0);
  std::fill(B.BcK.v.begin(), B.BcK.v.end(), 0);
  for (const Sub& Bc : B.sub) {
    if (Bc.bc < 0) continue;
    int s = Bc.face <= 3 ? 1 : 2;
    if (Bc.face == 1 || Bc.face == 4) { for (int k = Bc.kb; k <= Bc.ke - 1; k++) for (int j = Bc.jb; j <= Bc.je - 1; j++) B.BcI(j, k, s) = 1; }
    if (Bc.face == 2 || Bc.face == 5) { for (int k = Bc.kb; k <= Bc.ke - 1; k++) for (int i = Bc.ib; i <= Bc.ie - 1; i++) B.BcJ(i, k, s) = 1; }
    if (Bc.face == 3 || Bc.face == 6) { for (int j = Bc.jb; j <= Bc.je - 1; j++) for (int i = Bc.ib; i <= Bc.ie - 1; i++) B.BcK(i, j, s) = 1; }
  }
}

static void wall_distance(Case& C) {  // sub_comput_dw.f90:43-168
  std::vector<double> Xw;
  for (Block& B : C.B)
    for (const Sub& Bc : B.sub)
      if (Bc.bc == BC_Wall)
        for (int k = Bc.kb; k <= Bc.ke; k++)
          for (int j = Bc.jb; j <= Bc.je; j++)
            for (int i = Bc.ib; i <= Bc.ie; i++) { Xw.push_back(B.x(i, j, k)); Xw.push_back(B.y(i, j, k)); Xw.push_back(B.z(i, j, k)); }
  size_t Nw = Xw.size() / 3;
  for (Block& B : C.B) {
    int nx = B.nx, ny = B.ny, nz = B.nz;
    A3 dis;
    dis.alloc(1, nx, 1, ny, 1, nz);
    par_for(1, nz, [&](int k) {
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          double dmin = 1.e8;
          for (size_t q = 0; q < Nw; q++) {
            double d1 = std::sqrt(p2(B.x(i, j, k) - Xw[3 * q]) + p2(B.y(i, j, k) - Xw[3 * q + 1]) + p2(B.z(i, j, k) - Xw[3 * q + 2]));
            if (d1 < dmin) dmin = d1;
          }
          dis(i, j, k) = dmin;
        }
    });
    for (int k = 1; k <= nz - 1; k++)
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++)
          B.dw(i, j, k) = (dis(i, j, k) + dis(i, j + 1, k) + dis(i, j, k + 1) + dis(i, j + 1, k + 1) + dis(i + 1, j, k) + dis(i + 1, j + 1, k) +
                           dis(i + 1, j, k + 1) + dis(i + 1, j + 1, k + 1)) * 0.125;
  }
}

// ============================================================================================
// boundary conditions: sub_boundary.f90
// ============================================================================================
static void wall_bound(const Case& C, int NV, Block& B, int i1, int j1, int k1, int i2, int j2, int k2, double mu1, double dw) {  // 405-454
  const ocfd_params& P = C.P;
  const double beta1_SST = 0.075;
  double gamma = P.gamma, Ma = P.ma;
  double U1[7], Ug[7];
  for (int m = 0; m < NV; m++) U1[m] = B.U(m + 1, i1, j1, k1);
  if (P.twall > 0.0) {
    double d1 = U1[0], uu1 = U1[1] / d1, v1 = U1[2] / d1, w1 = U1[3] / d1;
    double p1 = (U1[4] - 0.5 * d1 * (uu1 * uu1 + v1 * v1 + w1 * w1)) * (gamma - 1.0);
    double T1 = gamma * Ma * Ma * p1 / d1;
    double p2_ = p1, T2 = 2.0 * P.twall - T1;
    if (T2 < 0.5 * T1) T2 = 0.5 * T1;
    double uu2 = -uu1, v2 = -v1, w2 = -w1;
    double d2 = gamma * Ma * Ma * p2_ / T2;
    Ug[0] = d2; Ug[1] = d2 * uu2; Ug[2] = d2 * v2; Ug[3] = d2 * w2;
    Ug[4] = p2_ / (gamma - 1.0) + 0.5 * d2 * (uu2 * uu2 + v2 * v2 + w2 * w2);
  } else {
    Ug[0] = U1[0]; Ug[1] = -U1[1]; Ug[2] = -U1[2]; Ug[3] = -U1[3]; Ug[4] = U1[4];
  }
  if (NV == 6) Ug[5] = 0.0;
  else if (NV == 7) {
    double wt = 60.0 * mu1 / (U1[0] * beta1_SST * p2(dw) * P.re);
    Ug[5] = -U1[5];
    Ug[6] = (U1[0] + Ug[0]) * wt - U1[6];
  }
  for (int m = 0; m < NV; m++) B.U(m + 1, i2, j2, k2) = Ug[m];
}

static void boundary_wall(Case& C, Block& B, const Sub& Bc) {  // 87-147
  int NV = C.NVAR;
  if (Bc.face == 1) { for (int k = Bc.kb; k <= Bc.ke - 1; k++) for (int j = Bc.jb; j <= Bc.je - 1; j++) wall_bound(C, NV, B, 1, j, k, 0, j, k, B.mu(1, j, k), B.dw(1, j, k)); }
  else if (Bc.face == 4) { int ie = Bc.ie; for (int k = Bc.kb; k <= Bc.ke - 1; k++) for (int j = Bc.jb; j <= Bc.je - 1; j++) wall_bound(C, NV, B, ie - 1, j, k, ie, j, k, B.mu(ie - 1, j, k), B.dw(ie - 1, j, k)); }
  else if (Bc.face == 2) { for (int k = Bc.kb; k <= Bc.ke - 1; k++) for (int i = Bc.ib; i <= Bc.ie - 1; i++) wall_bound(C, NV, B, i, 1, k, i, 0, k, B.mu(i, 1, k), B.dw(i, 1, k)); }
  else if (Bc.face == 5) { int je = Bc.je; for (int k = Bc.kb; k <= Bc.ke - 1; k++) for (int i = Bc.ib; i <= Bc.ie - 1; i++) wall_bound(C, NV, B, i, je - 1, k, i, je, k, B.mu(i, je - 1, k), B.dw(i, je - 1, k)); }
  else if (Bc.face == 3) { for (int j = Bc.jb; j <= Bc.je - 1; j++) for (int i = Bc.ib; i <= Bc.ie - 1; i++) wall_bound(C, NV, B, i, j, 1, i, j, 0, B.mu(i, j, 1), B.dw(i, j, 1)); }
  else if (Bc.face == 6) { int ke = Bc.ke; for (int j = Bc.jb; j <= Bc.je - 1; j++) for (int i = Bc.ib; i <= Bc.ie - 1; i++) wall_bound(C, NV, B, i, j, ke - 1, i, j, ke, B.mu(i, j, ke - 1), B.dw(i, j, ke - 1)); }
}

static void boundary_farfield(Case& C, Block& B, const Sub& Bc, int Flag) {  // 152-283
  const ocfd_params& P = C.P;
  const int FLAG_OUTLET = 1, FLAG_INLET = 2;
  double gamma = P.gamma;
  double d_inf = 1.0, u_inf = std::cos(P.a_alfa) * std::cos(P.a_beta), v_inf = std::sin(P.a_alfa) * std::cos(P.a_beta), w_inf = std::sin(P.a_beta);
  double p_inf = 1.0 / (gamma * P.ma * P.ma);
  int NV = C.NVAR;
  for (int k = Bc.kb; k <= Bc.ke; k++)
    for (int j = Bc.jb; j <= Bc.je; j++)
      for (int i = Bc.ib; i <= Bc.ie; i++) {
        int i1 = i, j1 = j, k1 = k, i2 = i, j2 = j, k2 = k;
        double n1, n2, n3;
        if (Bc.face == 1) { i2 = i - 1; n1 = -B.ni1(i, j, k); n2 = -B.ni2(i, j, k); n3 = -B.ni3(i, j, k); }
        else if (Bc.face == 2) { j2 = j - 1; n1 = -B.nj1(i, j, k); n2 = -B.nj2(i, j, k); n3 = -B.nj3(i, j, k); }
        else if (Bc.face == 3) { k2 = k - 1; n1 = -B.nk1(i, j, k); n2 = -B.nk2(i, j, k); n3 = -B.nk3(i, j, k); }
        else if (Bc.face == 4) { i1 = i - 1; n1 = B.ni1(i, j, k); n2 = B.ni2(i, j, k); n3 = B.ni3(i, j, k); }
        else if (Bc.face == 5) { j1 = j - 1; n1 = B.nj1(i, j, k); n2 = B.nj2(i, j, k); n3 = B.nj3(i, j, k); }
        else { k1 = k - 1; n1 = B.nk1(i, j, k); n2 = B.nk2(i, j, k); n3 = B.nk3(i, j, k); }
        double d1 = B.U(1, i1, j1, k1), u1 = B.U(2, i1, j1, k1) / d1, v1 = B.U(3, i1, j1, k1) / d1, w1 = B.U(4, i1, j1, k1) / d1;
        double p1 = (B.U(5, i1, j1, k1) - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1)) * (gamma - 1.0);
        double c1 = std::sqrt(gamma * p1 / d1);
        double d2, u2, v2, w2, p2_, Ma_n = 0.0;
        if (Flag == FLAG_OUTLET) { d2 = d1; u2 = u1; v2 = v1; w2 = w1; p2_ = p1; }
        else if (Flag == FLAG_INLET) { d2 = d_inf; u2 = u_inf; v2 = v_inf; w2 = w_inf; p2_ = p_inf; }
        else {
          if (P.p_outlet <= -1.0) Ma_n = (u_inf * n1 + v_inf * n2 + w_inf * n3) * P.ma;
          else Ma_n = (u1 * n1 + v1 * n2 + w1 * n3) / c1;
          if (Ma_n > 1.0) { d2 = d1; u2 = u1; v2 = v1; w2 = w1; p2_ = p1; }
          else if (Ma_n > -1.e-6) {
            if (P.p_outlet > 0.0) {
              double pb = P.p_outlet, db = d1 + (pb - p1) / (c1 * c1);
              double ub = u1 + (p1 - pb) / (d1 * c1) * n1, vb = v1 + (p1 - pb) / (d1 * c1) * n2, wb = w1 + (p1 - pb) / (d1 * c1) * n3;
              p2_ = 2.0 * pb - p1; d2 = 2.0 * db - d1; u2 = 2.0 * ub - u1; v2 = 2.0 * vb - v1; w2 = 2.0 * wb - w1;
            } else { d2 = d1; u2 = u1; v2 = v1; w2 = w1; p2_ = p1; }
          } else if (Ma_n > -1.0) {
            double pb = 0.5 * (p1 + p_inf - d1 * c1 * ((u_inf - u1) * n1 + (v_inf - v1) * n2 + (w_inf - w1) * n3));
            double db = d_inf + (pb - p_inf) / (c1 * c1);
            double ub = u_inf - (p_inf - pb) / (d1 * c1) * n1, vb = v_inf - (p_inf - pb) / (d1 * c1) * n2, wb = w_inf - (p_inf - pb) / (d1 * c1) * n3;
            p2_ = 2.0 * pb - p1; d2 = 2.0 * db - d1; u2 = 2.0 * ub - u1; v2 = 2.0 * vb - v1; w2 = 2.0 * wb - w1;
          } else { d2 = d_inf; u2 = u_inf; v2 = v_inf; w2 = w_inf; p2_ = p_inf; }
        }
        B.U(1, i2, j2, k2) = d2; B.U(2, i2, j2, k2) = d2 * u2; B.U(3, i2, j2, k2) = d2 * v2; B.U(4, i2, j2, k2) = d2 * w2;
        B.U(5, i2, j2, k2) = p2_ / (gamma - 1.0) + 0.5 * d2 * (u2 * u2 + v2 * v2 + w2 * w2);
        if (Ma_n > 0.0 || Flag == FLAG_OUTLET) {
          if (NV == 6) B.U(6, i2, j2, k2) = B.U(6, i1, j1, k1);
          else if (NV == 7) { B.U(6, i2, j2, k2) = B.U(6, i1, j1, k1); B.U(7, i2, j2, k2) = B.U(7, i1, j1, k1); }
        } else {
          if (NV == 6) B.U(6, i2, j2, k2) = 5.0;
          else if (NV == 7) { B.U(6, i2, j2, k2) = d_inf * P.kt_inf; B.U(7, i2, j2, k2) = d_inf * P.wt_inf; }
        }
      }
}

static void boundary_symmetry(Case& C, Block& B, const Sub& Bc) {  // 291-373
  int NV = C.NVAR;
  if (Bc.face == 1 || Bc.face == 4) {
    int i, i1, i2;
    if (Bc.face == 1) { i = Bc.ib; i1 = Bc.ib; i2 = Bc.ib - 1; } else { i = Bc.ie; i1 = Bc.ie - 1; i2 = Bc.ie; }
    for (int k = Bc.kb; k <= Bc.ke - 1; k++)
      for (int j = Bc.jb; j <= Bc.je - 1; j++) {
        for (int m = 1; m <= NV; m++) B.U(m, i2, j, k) = B.U(m, i1, j, k);
        double n1 = B.ni1(i, j, k), n2 = B.ni2(i, j, k), n3 = B.ni3(i, j, k);
        double Vn = B.U(2, i1, j, k) * n1 + B.U(3, i1, j, k) * n2 + B.U(4, i1, j, k) * n3;
        B.U(2, i2, j, k) = B.U(2, i2, j, k) - 2.0 * Vn * n1;
        B.U(3, i2, j, k) = B.U(3, i2, j, k) - 2.0 * Vn * n2;
        B.U(4, i2, j, k) = B.U(4, i2, j, k) - 2.0 * Vn * n3;
      }
  } else if (Bc.face == 2 || Bc.face == 5) {
    int j, j1, j2;
    if (Bc.face == 2) { j = Bc.jb; j1 = Bc.jb; j2 = Bc.jb - 1; } else { j = Bc.je; j1 = Bc.je - 1; j2 = Bc.je; }
    for (int k = Bc.kb; k <= Bc.ke - 1; k++)
      for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
        for (int m = 1; m <= NV; m++) B.U(m, i, j2, k) = B.U(m, i, j1, k);
        double n1 = B.nj1(i, j, k), n2 = B.nj2(i, j, k), n3 = B.nj3(i, j, k);
        double Vn = B.U(2, i, j1, k) * n1 + B.U(3, i, j1, k) * n2 + B.U(4, i, j1, k) * n3;
        B.U(2, i, j2, k) = B.U(2, i, j2, k) - 2.0 * Vn * n1;
        B.U(3, i, j2, k) = B.U(3, i, j2, k) - 2.0 * Vn * n2;
        B.U(4, i, j2, k) = B.U(4, i, j2, k) - 2.0 * Vn * n3;
      }
  } else {
    int k, k1, k2;
    if (Bc.face == 3) { k = Bc.kb; k1 = Bc.kb; k2 = Bc.kb - 1; } else { k = Bc.ke; k1 = Bc.ke - 1; k2 = Bc.ke; }
    for (int j = Bc.jb; j <= Bc.je - 1; j++)
      for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
        for (int m = 1; m <= NV; m++) B.U(m, i, j, k2) = B.U(m, i, j, k1);
        double n1 = B.nk1(i, j, k), n2 = B.nk2(i, j, k), n3 = B.nk3(i, j, k);
        double Vn = B.U(2, i, j, k1) * n1 + B.U(3, i, j, k1) * n2 + B.U(4, i, j, k1) * n3;
        B.U(2, i, j, k2) = B.U(2, i, j, k2) - 2.0 * Vn * n1;
        B.U(3, i, j, k2) = B.U(3, i, j, k2) - 2.0 * Vn * n2;
        B.U(4, i, j, k2) = B.U(4, i, j, k2) - 2.0 * Vn * n3;
      }
  }
}

static void boundary_extrapolate(Case& C, Block& B, const Sub& Bc) {  // 458-504
  for (int k = Bc.kb; k <= Bc.ke; k++)
    for (int j = Bc.jb; j <= Bc.je; j++)
      for (int i = Bc.ib; i <= Bc.ie; i++) {
        int i1 = i, j1 = j, k1 = k, i2 = i, j2 = j, k2 = k;
        if (Bc.face == 1) i2 = i - 1; else if (Bc.face == 2) j2 = j - 1; else if (Bc.face == 3) k2 = k - 1;
        else if (Bc.face == 4) i1 = i - 1; else if (Bc.face == 5) j1 = j - 1; else k1 = k - 1;
        for (int m = 1; m <= C.NVAR; m++) B.U(m, i2, j2, k2) = B.U(m, i1, j1, k1);
      }
}

static int boundary_all(Case& C) {  // Boundary_condition_onemesh 6-80 (non-turbomachinery branch)
  for (Block& B : C.B)
    for (const Sub& Bc : B.sub) {
      if (Bc.bc <= 0) continue;
      if (Bc.bc == BC_Wall && C.P.if_viscous == 1) boundary_wall(C, B, Bc);
      else if (Bc.bc == BC_Farfield) boundary_farfield(C, B, Bc, 0);
      else if (Bc.bc == BC_Inflow) boundary_farfield(C, B, Bc, 2);
      else if (Bc.bc == BC_Outflow) boundary_farfield(C, B, Bc, 1);
      else if (Bc.bc == BC_Symmetry || (Bc.bc == BC_Wall && C.P.if_viscous == 0)) boundary_symmetry(C, B, Bc);
      else if (Bc.bc == BC_Extrap) boundary_extrapolate(C, B, Bc);
      else { C.err = "unsupported boundary condition " + std::to_string(Bc.bc); return OCFD_ERR_UNSUPPORTED; }
    }
  return 0;
}

// ============================================================================================
// halo: sub_update_buffer_mpi.f90:42-211, 515-549
// ============================================================================================
static void halo(Case& C) {
  int NV = C.NVAR;
  for (size_t mb = 0; mb < C.B.size(); mb++) {
    Block& B = C.B[mb];
    for (const Sub& Bc : B.sub) {
      if (Bc.bc >= 0) continue;
      int kb[3] = {Bc.ib, Bc.jb, Bc.kb}, ke[3] = {Bc.ie - 1, Bc.je - 1, Bc.ke - 1};
      int k = (Bc.face - 1) % 3;
      if (Bc.face > 3) kb[k] = kb[k] - LAP;
      ke[k] = kb[k] + LAP - 1;
      int kb1[3] = {Bc.ib1, Bc.jb1, Bc.kb1}, ke1[3] = {Bc.ie1 - 1, Bc.je1 - 1, Bc.ke1 - 1};
      k = (Bc.face1 - 1) % 3;
      if (Bc.face1 <= 3) kb1[k] = kb1[k] - LAP;
      ke1[k] = kb1[k] + LAP - 1;
      int L[3] = {std::abs(Bc.L1), std::abs(Bc.L2), std::abs(Bc.L3)};
      int P[3] = {Bc.L1 >= 0 ? 1 : -1, Bc.L2 >= 0 ? 1 : -1, Bc.L3 >= 0 ? 1 : -1};
      int ks[3];
      for (int q = 0; q < 3; q++) ks[q] = P[q] > 0 ? kb[q] : ke[q];
      Block& B1 = C.B[Bc.nb1 - 1];
      // the whole copy goes through a buffer first (Usend, 97-111), then into the target (126-134):
      // a source range that reaches ghost cells sees the values before this copy
      std::vector<double> Usend;
      Usend.reserve((size_t)NV * (ke1[0] - kb1[0] + 1) * (ke1[1] - kb1[1] + 1) * (ke1[2] - kb1[2] + 1));
      for (int kk = kb1[2]; kk <= ke1[2]; kk++)
        for (int jj = kb1[1]; jj <= ke1[1]; jj++)
          for (int ii = kb1[0]; ii <= ke1[0]; ii++) {
            int ka[3] = {ii - kb1[0], jj - kb1[1], kk - kb1[2]};
            int i1 = ks[0] + ka[L[0] - 1] * P[0], j1 = ks[1] + ka[L[1] - 1] * P[1], k1 = ks[2] + ka[L[2] - 1] * P[2];
            for (int m = 1; m <= NV; m++) Usend.push_back(B.U(m, i1, j1, k1));
          }
      size_t q = 0;
      for (int kk = kb1[2]; kk <= ke1[2]; kk++)
        for (int jj = kb1[1]; jj <= ke1[1]; jj++)
          for (int ii = kb1[0]; ii <= ke1[0]; ii++)
            for (int m = 1; m <= NV; m++) B1.U(m, ii, jj, kk) = Usend[q++];
    }
  }
  for (Block& B : C.B) {  // get_U_conner 515-549
    int nx = B.nx, ny = B.ny, nz = B.nz;
    A4& U = B.U;
    for (int m = 1; m <= NV; m++) {
      for (int k = 1; k <= nz - 1; k++) {
        U(m, 0, 0, k) = (U(m, 1, 0, k) + U(m, 0, 1, k)) * 0.5;
        U(m, nx, 0, k) = (U(m, nx - 1, 0, k) + U(m, nx, 1, k)) * 0.5;
        U(m, 0, ny, k) = (U(m, 1, ny, k) + U(m, 0, ny - 1, k)) * 0.5;
        U(m, nx, ny, k) = (U(m, nx - 1, ny, k) + U(m, nx, ny - 1, k)) * 0.5;
      }
      for (int j = 1; j <= ny - 1; j++) {
        U(m, 0, j, 0) = (U(m, 1, j, 0) + U(m, 0, j, 1)) * 0.5;
        U(m, nx, j, 0) = (U(m, nx - 1, j, 0) + U(m, nx, j, 1)) * 0.5;
        U(m, 0, j, nz) = (U(m, 1, j, nz) + U(m, 0, j, nz - 1)) * 0.5;
        U(m, nx, j, nz) = (U(m, nx - 1, j, nz) + U(m, nx, j, nz - 1)) * 0.5;
      }
      for (int i = 1; i <= nx - 1; i++) {
        U(m, i, 0, 0) = (U(m, i, 1, 0) + U(m, i, 0, 1)) * 0.5;
        U(m, i, ny, 0) = (U(m, i, ny - 1, 0) + U(m, i, ny, 1)) * 0.5;
        U(m, i, 0, nz) = (U(m, i, 1, nz) + U(m, i, 0, nz - 1)) * 0.5;
        U(m, i, ny, nz) = (U(m, i, ny - 1, nz) + U(m, i, ny, nz - 1)) * 0.5;
      }
      U(m, 0, 0, 0) = (2.0 * (U(m, 1, 0, 0) + U(m, 0, 1, 0) + U(m, 0, 0, 1)) - (U(m, 1, 1, 0) + U(m, 1, 0, 1) + U(m, 0, 1, 1))) / 3.0;
      U(m, nx, 0, 0) = (2.0 * (U(m, nx - 1, 0, 0) + U(m, nx, 1, 0) + U(m, nx, 0, 1)) - (U(m, nx - 1, 1, 0) + U(m, nx - 1, 0, 1) + U(m, nx, 1, 1))) / 3.0;
      U(m, 0, ny, 0) = (2.0 * (U(m, 1, ny, 0) + U(m, 0, ny - 1, 0) + U(m, 0, ny, 1)) - (U(m, 1, ny - 1, 0) + U(m, 1, ny, 1) + U(m, 0, ny - 1, 1))) / 3.0;
      U(m, nx, ny, 0) = (2.0 * (U(m, nx - 1, ny, 0) + U(m, nx, ny - 1, 0) + U(m, nx, ny, 1)) - (U(m, nx - 1, ny - 1, 0) + U(m, nx - 1, ny, 1) + U(m, nx, ny - 1, 1))) / 3.0;
      U(m, 0, 0, nz) = (2.0 * (U(m, 1, 0, nz) + U(m, 0, 1, nz) + U(m, 0, 0, nz - 1)) - (U(m, 1, 1, nz) + U(m, 1, 0, nz - 1) + U(m, 0, 1, nz - 1))) / 3.0;
      U(m, nx, 0, nz) = (2.0 * (U(m, nx - 1, 0, nz) + U(m, nx, 1, nz) + U(m, nx, 0, nz - 1)) - (U(m, nx - 1, 1, nz) + U(m, nx - 1, 0, nz - 1) + U(m, nx, 1, nz - 1))) / 3.0;
      U(m, 0, ny, nz) = (2.0 * (U(m, 1, ny, nz) + U(m, 0, ny - 1, nz) + U(m, 0, ny, nz - 1)) - (U(m, 1, ny - 1, nz) + U(m, 1, ny, nz - 1) + U(m, 0, ny - 1, nz - 1))) / 3.0;
      U(m, nx, ny, nz) = (2.0 * (U(m, nx - 1, ny, nz) + U(m, nx, ny - 1, nz) + U(m, nx, ny, nz - 1)) - (U(m, nx - 1, ny - 1, nz) + U(m, nx - 1, ny, nz - 1) + U(m, nx, ny - 1, nz - 1))) / 3.0;
    }
  }
}

// ============================================================================================
// residual: sub_Residual.f90
// ============================================================================================
static void limit_vt(Case& C, Block& B) {  // sub_time_advance.f90:410-443
  if (C.NVAR == 6) {
    for (int k = 0; k <= B.nz; k++) for (int j = 0; j <= B.ny; j++) for (int i = 0; i <= B.nx; i++) if (B.U(6, i, j, k) < 0.0) B.U(6, i, j, k) = 0.0;
  } else if (C.NVAR == 7) {
    for (int k = 0; k <= B.nz; k++) for (int j = 0; j <= B.ny; j++) for (int i = 0; i <= B.nx; i++) {
      if (B.U(6, i, j, k) < 0.0) B.U(6, i, j, k) = 0.0;
      if (B.U(7, i, j, k) < 0.0) B.U(7, i, j, k) = 0.0;
    }
  }
}

static void comput_duvtpc(Case& C, Block& B, Work& W) {  // sub_Residual.f90:1417-1456
  double gamma = C.P.gamma, Ma = C.P.ma, Cv = C.P.cv;
  double p00 = 1.0 / (gamma * Ma * Ma);
  int nx = B.nx, ny = B.ny, nz = B.nz;
  par_for(1 - LAP, nz + LAP - 1, [&](int k) {
    for (int j = 1 - LAP; j <= ny + LAP - 1; j++)
      for (int i = 1 - LAP; i <= nx + LAP - 1; i++) {
        double d = B.U(1, i, j, k);
        double uu = B.U(2, i, j, k) / d, v = B.U(3, i, j, k) / d, w = B.U(4, i, j, k) / d;
        double T = (B.U(5, i, j, k) - 0.5 * d * (uu * uu + v * v + w * w)) / (Cv * d);
        W.d(i, j, k) = d; W.uu(i, j, k) = uu; W.v(i, j, k) = v; W.w(i, j, k) = w; W.T(i, j, k) = T;
        W.p(i, j, k) = p00 * d * T;
        W.cc(i, j, k) = std::sqrt(T) / Ma;
      }
  });
}

static void get_viscous(Case& C, Block& B, Work& W) {  // 1355-1383
  double Tsb = 110.4 / C.P.t_inf, Re = C.P.re;
  int nx = B.nx, ny = B.ny, nz = B.nz;
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double T = W.T(i, j, k);
        B.mu(i, j, k) = 1.0 / Re * (1.0 + Tsb) * std::sqrt(p3(T)) / (Tsb + T);
      }
  for (int k = 1; k <= nz - 1; k++) for (int j = 1; j <= ny - 1; j++) { B.mu(0, j, k) = B.mu(1, j, k); B.mu(nx, j, k) = B.mu(nx - 1, j, k); }
  for (int k = 1; k <= nz - 1; k++) for (int i = 1; i <= nx - 1; i++) { B.mu(i, 0, k) = B.mu(i, 1, k); B.mu(i, ny, k) = B.mu(i, ny - 1, k); }
  for (int j = 1; j <= ny - 1; j++) for (int i = 1; i <= nx - 1; i++) { B.mu(i, j, 0) = B.mu(i, j, 1); B.mu(i, j, nz) = B.mu(i, j, nz - 1); }
}

static void amut_boundary(Block& B) {  // sub_turbulence_SA.f90:282-368
  for (const Sub& Bc : B.sub) {
    if (Bc.bc != BC_Wall) continue;
    int ib = Bc.ib, ie = Bc.ie, jb = Bc.jb, je = Bc.je, kb = Bc.kb, ke = Bc.ke;
    if (Bc.face == 1) { for (int k = kb; k <= ke - 1; k++) for (int j = jb; j <= je - 1; j++) B.mu_t(0, j, k) = -B.mu_t(1, j, k); }
    else if (Bc.face == 4) { for (int k = kb; k <= ke - 1; k++) for (int j = jb; j <= je - 1; j++) B.mu_t(ie, j, k) = -B.mu_t(ie - 1, j, k); }
    else if (Bc.face == 2) { for (int k = kb; k <= ke - 1; k++) for (int i = ib; i <= ie - 1; i++) B.mu_t(i, 0, k) = -B.mu_t(i, 1, k); }
    else if (Bc.face == 5) { for (int k = kb; k <= ke - 1; k++) for (int i = ib; i <= ie - 1; i++) B.mu_t(i, je, k) = -B.mu_t(i, je - 1, k); }
    else if (Bc.face == 3) { for (int j = jb; j <= je - 1; j++) for (int i = ib; i <= ie - 1; i++) B.mu_t(i, j, 0) = -B.mu_t(i, j, 1); }
    else if (Bc.face == 6) { for (int j = jb; j <= je - 1; j++) for (int i = ib; i <= ie - 1; i++) B.mu_t(i, j, ke) = -B.mu_t(i, j, ke - 1); }
  }
}

static void limit_mut(Case& C, Block& B) {  // sub_Residual.f90:1387-1408
  double MUT_MAX = C.P.mut_max;
  for (int k = 0; k <= B.nz; k++)
    for (int j = 0; j <= B.ny; j++)
      for (int i = 0; i <= B.nx; i++) {
        if (B.mu_t(i, j, k) < 0.0) B.mu_t(i, j, k) = 0.0;
        if (MUT_MAX >= 0.0 && B.mu_t(i, j, k) > MUT_MAX * B.mu(i, j, k)) B.mu_t(i, j, k) = MUT_MAX * B.mu(i, j, k);
      }
  amut_boundary(B);
}

// SA constants (sub_turbulence_SA.f90:18-20)
namespace sa {
const double sigma = 2.0 / 3.0, Cv1 = 7.1, Cb1 = 0.1355, Cb2 = 0.622, kap = 0.41;
const double Cw1 = Cb1 / (kap * kap) + (1.0 + Cb2) / sigma, Cw2 = 0.3, Cw3 = 2.0, Ct3 = 1.2, Ct4 = 0.5;
const double Cv1_3 = 357.91099999999994; // Cv1**3 folded at compile time: correctly rounded 7.1d0**3
const double Cw3_6 = 64.0;
}  // namespace sa

static void turbulence_SA(Case& C, Block& B, Work& W) {  // sub_turbulence_SA.f90:8-273
  using namespace sa;
  double Re = C.P.re;
  int nx = B.nx, ny = B.ny, nz = B.nz;
  A3 vt, Fluxv, Fluxv2;
  vt.alloc(0, nx, 0, ny, 0, nz); Fluxv.alloc(1, nx, 1, ny, 1, nz); Fluxv2.alloc(1, nx, 1, ny, 1, nz);
  A3 &d = W.d, &uu = W.uu, &v = W.v, &w = W.w;
  for (int k = 0; k <= nz; k++) for (int j = 0; j <= ny; j++) for (int i = 0; i <= nx; i++) B.mu(i, j, k) = B.mu(i, j, k) * Re;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        vt(i, j, k) = B.U(6, i, j, k);
        double X = d(i, j, k) * vt(i, j, k) / B.mu(i, j, k);
        double fv1 = p3(X) / (p3(X) + Cv1_3);
        B.mu_t(i, j, k) = fv1 * d(i, j, k) * vt(i, j, k);
      }
  limit_mut(C, B);
  const double c0 = 0.5 * (1.0 + Cb2) / sigma;
  // i direction
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++) {
        double s1x = B.ni1(i, j, k), s1y = B.ni2(i, j, k), s1z = B.ni3(i, j, k);
        double vti = vt(i, j, k) - vt(i - 1, j, k);
        double vtj = 0.25 * (vt(i, j + 1, k) - vt(i, j - 1, k) + vt(i - 1, j + 1, k) - vt(i - 1, j - 1, k));
        double vtk = 0.25 * (vt(i, j, k + 1) - vt(i, j, k - 1) + vt(i - 1, j, k + 1) - vt(i - 1, j, k - 1));
        double ix = B.ix1(i, j, k), iy = B.iy1(i, j, k), iz = B.iz1(i, j, k), jx = B.jx1(i, j, k), jy = B.jy1(i, j, k), jz = B.jz1(i, j, k);
        double kx = B.kx1(i, j, k), ky = B.ky1(i, j, k), kz = B.kz1(i, j, k);
        double vtx = vti * ix + vtj * jx + vtk * kx, vty = vti * iy + vtj * jy + vtk * ky, vtz = vti * iz + vtj * jz + vtk * kz;
        double v0 = c0 * (vt(i, j, k) + B.mu(i, j, k) / d(i, j, k) + vt(i - 1, j, k) + B.mu(i - 1, j, k) / d(i - 1, j, k));
        double vn1 = uu(i - 1, j, k) * s1x + v(i - 1, j, k) * s1y + w(i - 1, j, k) * s1z;
        double vn2 = uu(i, j, k) * s1x + v(i, j, k) * s1y + w(i, j, k) * s1z;
        double vfi = 0.5 * ((vn1 + std::fabs(vn1)) * vt(i - 1, j, k) + (vn2 - std::fabs(vn2)) * vt(i, j, k));
        Fluxv(i, j, k) = (-vfi + v0 / Re * (vtx * s1x + vty * s1y + vtz * s1z)) * B.Si(i, j, k);
        Fluxv2(i, j, k) = (vtx * s1x + vty * s1y + vtz * s1z) * B.Si(i, j, k);
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double v0 = (vt(i, j, k) + B.mu(i, j, k) / d(i, j, k)) * Cb2 / sigma;
        B.Res(6, i, j, k) = Fluxv(i + 1, j, k) - Fluxv(i, j, k) - v0 / Re * (Fluxv2(i + 1, j, k) - Fluxv2(i, j, k));
      }
  // j direction
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double s1x = B.nj1(i, j, k), s1y = B.nj2(i, j, k), s1z = B.nj3(i, j, k);
        double vti = 0.25 * (vt(i + 1, j, k) - vt(i - 1, j, k) + vt(i + 1, j - 1, k) - vt(i - 1, j - 1, k));
        double vtj = vt(i, j, k) - vt(i, j - 1, k);
        double vtk = 0.25 * (vt(i, j, k + 1) - vt(i, j, k - 1) + vt(i, j - 1, k + 1) - vt(i, j - 1, k - 1));
        double ix = B.ix2(i, j, k), iy = B.iy2(i, j, k), iz = B.iz2(i, j, k), jx = B.jx2(i, j, k), jy = B.jy2(i, j, k), jz = B.jz2(i, j, k);
        double kx = B.kx2(i, j, k), ky = B.ky2(i, j, k), kz = B.kz2(i, j, k);
        double vtx = vti * ix + vtj * jx + vtk * kx, vty = vti * iy + vtj * jy + vtk * ky, vtz = vti * iz + vtj * jz + vtk * kz;
        double v0 = c0 * (vt(i, j, k) + B.mu(i, j, k) / d(i, j, k) + vt(i, j - 1, k) + B.mu(i, j - 1, k) / d(i, j - 1, k));
        double vn1 = uu(i, j - 1, k) * s1x + v(i, j - 1, k) * s1y + w(i, j - 1, k) * s1z;
        double vn2 = uu(i, j, k) * s1x + v(i, j, k) * s1y + w(i, j, k) * s1z;
        double vfi = 0.5 * ((vn1 + std::fabs(vn1)) * vt(i, j - 1, k) + (vn2 - std::fabs(vn2)) * vt(i, j, k));
        Fluxv(i, j, k) = (-vfi + v0 / Re * (vtx * s1x + vty * s1y + vtz * s1z)) * B.Sj(i, j, k);
        Fluxv2(i, j, k) = (vtx * s1x + vty * s1y + vtz * s1z) * B.Sj(i, j, k);
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double v0 = (vt(i, j, k) + B.mu(i, j, k) / d(i, j, k)) * Cb2 / sigma;
        B.Res(6, i, j, k) = B.Res(6, i, j, k) + Fluxv(i, j + 1, k) - Fluxv(i, j, k) - v0 / Re * (Fluxv2(i, j + 1, k) - Fluxv2(i, j, k));
      }
  // k direction
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double s1x = B.nk1(i, j, k), s1y = B.nk2(i, j, k), s1z = B.nk3(i, j, k);
        double vti = 0.25 * (vt(i + 1, j, k) - vt(i - 1, j, k) + vt(i + 1, j, k - 1) - vt(i - 1, j, k - 1));
        double vtj = 0.25 * (vt(i, j + 1, k) - vt(i, j - 1, k) + vt(i, j + 1, k - 1) - vt(i, j - 1, k - 1));
        double vtk = vt(i, j, k) - vt(i, j, k - 1);
        double ix = B.ix3(i, j, k), iy = B.iy3(i, j, k), iz = B.iz3(i, j, k), jx = B.jx3(i, j, k), jy = B.jy3(i, j, k), jz = B.jz3(i, j, k);
        double kx = B.kx3(i, j, k), ky = B.ky3(i, j, k), kz = B.kz3(i, j, k);
        double vtx = vti * ix + vtj * jx + vtk * kx, vty = vti * iy + vtj * jy + vtk * ky, vtz = vti * iz + vtj * jz + vtk * kz;
        double v0 = c0 * (vt(i, j, k) + B.mu(i, j, k) / d(i, j, k) + vt(i, j, k - 1) + B.mu(i, j, k - 1) / d(i, j, k - 1));
        double vn1 = uu(i, j, k - 1) * s1x + v(i, j, k - 1) * s1y + w(i, j, k - 1) * s1z;
        double vn2 = uu(i, j, k) * s1x + v(i, j, k) * s1y + w(i, j, k) * s1z;
        double vfi = 0.5 * ((vn1 + std::fabs(vn1)) * vt(i, j, k - 1) + (vn2 - std::fabs(vn2)) * vt(i, j, k));
        Fluxv(i, j, k) = (-vfi + v0 / Re * (vtx * s1x + vty * s1y + vtz * s1z)) * B.Sk(i, j, k);
        Fluxv2(i, j, k) = (vtx * s1x + vty * s1y + vtz * s1z) * B.Sk(i, j, k);
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double v0 = (vt(i, j, k) + B.mu(i, j, k) / d(i, j, k)) * Cb2 / sigma;
        B.Res(6, i, j, k) = B.Res(6, i, j, k) + Fluxv(i, j, k + 1) - Fluxv(i, j, k) - v0 / Re * (Fluxv2(i, j, k + 1) - Fluxv2(i, j, k));
      }
  // source (180-254)
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double ui = uu(i + 1, j, k) - uu(i - 1, j, k), vi = v(i + 1, j, k) - v(i - 1, j, k), wi = w(i + 1, j, k) - w(i - 1, j, k);
        double uj = uu(i, j + 1, k) - uu(i, j - 1, k), vj = v(i, j + 1, k) - v(i, j - 1, k), wj = w(i, j + 1, k) - w(i, j - 1, k);
        double uk = uu(i, j, k + 1) - uu(i, j, k - 1), vk = v(i, j, k + 1) - v(i, j, k - 1), wk = w(i, j, k + 1) - w(i, j, k - 1);
        double ix = B.ix0(i, j, k), iy = B.iy0(i, j, k), iz = B.iz0(i, j, k), jx = B.jx0(i, j, k), jy = B.jy0(i, j, k), jz = B.jz0(i, j, k);
        double kx = B.kx0(i, j, k), ky = B.ky0(i, j, k), kz = B.kz0(i, j, k);
        double ux = ui * ix + uj * jx + uk * kx, vx = vi * ix + vj * jx + vk * kx, wx = wi * ix + wj * jx + wk * kx;
        double uy = ui * iy + uj * jy + uk * ky, vy = vi * iy + vj * jy + vk * ky, wy = wi * iy + wj * jy + wk * ky;
        double uz = ui * iz + uj * jz + uk * kz, vz = vi * iz + vj * jz + vk * kz, wz = wi * iz + wj * jz + wk * kz;
        double S = std::sqrt(p2(wy - vz) + p2(uz - wx) + p2(vx - uy));
        double vt0 = vt(i, j, k), dw = B.dw(i, j, k);
        double X = d(i, j, k) * vt0 / B.mu(i, j, k);
        double fv1 = p3(X) / (p3(X) + Cv1_3);
        double fv2 = 1.0 - X / (1.0 + X * fv1);
        double ft2 = Ct3 * std::exp(-(Ct4 * X * X));
        double S1 = std::max(S + fv2 * vt0 / (Re * p2(kap * dw)), 0.0);
        double r = std::min(vt0 / (Re * S1 * kap * kap * dw * dw), 10.0);
        double g = r + Cw2 * (p6(r) - r);
        double fw = g * std::pow((1.0 + Cw3_6) / (p6(g) + Cw3_6), 1.0 / 6.0);
        double Q3 = Cb1 * ((1 - ft2) * fv2 + ft2) / (kap * kap) - Cw1 * fw;
        double Q_SA = Cb1 * (1.0 - ft2) * S1 * vt0 + Q3 * p2(vt0 / dw) / Re;
        B.Res(6, i, j, k) = B.Res(6, i, j, k) + Q_SA * B.vol(i, j, k);
      }
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) { B.mu(i, j, k) = B.mu(i, j, k) / Re; B.mu_t(i, j, k) = B.mu_t(i, j, k) / Re; }
}

namespace sst {  // sub_turbulence_SST.f90:20-22
const double sigma_k1 = 0.85, sigma_w1 = 0.5, beta1 = 0.075, Cw1 = 0.533, sigma_k2 = 1.0, sigma_w2 = 0.856, beta2 = 0.0828, Cw2 = 0.440;
const double a1 = 0.31, betas = 0.09;
const double c009 = (double)0.09f;  // `0.09` default-real literal (lines 108, 120)
}  // namespace sst

static void turbulence_SST(Case& C, Block& B, Work& W) {  // sub_turbulence_SST.f90:7-348
  using namespace sst;
  double Re = C.P.re;
  int nx = B.nx, ny = B.ny, nz = B.nz;
  A3 Kt, Wt, Fluxk, Fluxw, f1;
  Kt.alloc(0, nx, 0, ny, 0, nz); Wt.alloc(0, nx, 0, ny, 0, nz);
  Fluxk.alloc(1, nx, 1, ny, 1, nz); Fluxw.alloc(1, nx, 1, ny, 1, nz); f1.alloc(1, nx, 1, ny, 1, nz);
  A3 &d = W.d, &uu = W.uu, &v = W.v, &w = W.w;
  for (int k = 0; k <= nz; k++) for (int j = 0; j <= ny; j++) for (int i = 0; i <= nx; i++) B.mu(i, j, k) = B.mu(i, j, k) * Re;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) { Kt(i, j, k) = B.U(6, i, j, k) / B.U(1, i, j, k); Wt(i, j, k) = B.U(7, i, j, k) / B.U(1, i, j, k); }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double ui = uu(i + 1, j, k) - uu(i - 1, j, k), vi = v(i + 1, j, k) - v(i - 1, j, k), wi = w(i + 1, j, k) - w(i - 1, j, k);
        double Kti = Kt(i + 1, j, k) - Kt(i - 1, j, k), wti = Wt(i + 1, j, k) - Wt(i - 1, j, k);
        double uj = uu(i, j + 1, k) - uu(i, j - 1, k), vj = v(i, j + 1, k) - v(i, j - 1, k), wj = w(i, j + 1, k) - w(i, j - 1, k);
        double Ktj = Kt(i, j + 1, k) - Kt(i, j - 1, k), wtj = Wt(i, j + 1, k) - Wt(i, j - 1, k);
        double uk = uu(i, j, k + 1) - uu(i, j, k - 1), vk = v(i, j, k + 1) - v(i, j, k - 1), wk = w(i, j, k + 1) - w(i, j, k - 1);
        double Ktk = Kt(i, j, k + 1) - Kt(i, j, k - 1), wtk = Wt(i, j, k + 1) - Wt(i, j, k - 1);
        double ix = B.ix0(i, j, k), iy = B.iy0(i, j, k), iz = B.iz0(i, j, k), jx = B.jx0(i, j, k), jy = B.jy0(i, j, k), jz = B.jz0(i, j, k);
        double kx = B.kx0(i, j, k), ky = B.ky0(i, j, k), kz = B.kz0(i, j, k);
        double ux = ui * ix + uj * jx + uk * kx, vx = vi * ix + vj * jx + vk * kx, wx = wi * ix + wj * jx + wk * kx;
        double Ktx = Kti * ix + Ktj * jx + Ktk * kx, wtx = wti * ix + wtj * jx + wtk * kx;
        double uy = ui * iy + uj * jy + uk * ky, vy = vi * iy + vj * jy + vk * ky, wy = wi * iy + wj * jy + wk * ky;
        double Kty = Kti * iy + Ktj * jy + Ktk * ky, wty = wti * iy + wtj * jy + wtk * ky;
        double uz = ui * iz + uj * jz + uk * kz, vz = vi * iz + vj * jz + vk * kz, wz = wi * iz + wj * jz + wk * kz;
        double Ktz = Kti * iz + Ktj * jz + Ktk * kz, wtz = wti * iz + wtj * jz + wtk * kz;
        (void)ux; (void)vy; (void)wz;
        double omega = std::sqrt(p2(wy - vz) + p2(uz - wx) + p2(vx - uy));
        double dw = B.dw(i, j, k), K = Kt(i, j, k), Wv = Wt(i, j, k), dd = d(i, j, k), mu = B.mu(i, j, k);
        double arg2 = std::max(2.0 * std::sqrt(std::fabs(K)) / (c009 * Wv * dw * Re), 500.0 * mu / (dd * Wv * p2(dw) * Re * Re));
        double f2 = std::tanh(p2(arg2));
        B.mu_t(i, j, k) = a1 * dd * K / std::max(a1 * Wv, f2 * std::fabs(omega) / Re);
        double Kws = 2.0 * (Ktx * wtx + Kty * wty + Ktz * wtz) * dd * sigma_w2 / (Wv + 1.e-20);
        double CD_kw = std::max(Kws, 1.e-20);
        double arg3 = std::max(std::sqrt(std::fabs(K)) / (c009 * Wv * dw * Re), 500.0 * mu / (dd * Wv * p2(dw) * Re * Re));
        double arg1 = std::min(arg3, 4.0 * dd * sigma_w2 * K / (CD_kw * p2(dw)));
        f1(i, j, k) = std::tanh(p4(arg1));
        double Pk = B.mu_t(i, j, k) * omega * omega;
        double Pk0 = Pk;
        double Qk = Pk0 / Re - Re * betas * dd * Wv * K;
        double Cw_SST = f1(i, j, k) * Cw1 + (1.0 - f1(i, j, k)) * Cw2;
        double beta_SST = f1(i, j, k) * beta1 + (1.0 - f1(i, j, k)) * beta2;
        double Qw = Cw_SST * dd * omega * omega / Re - Re * beta_SST * dd * p2(Wv) + (1.0 - f1(i, j, k)) * Kws / Re;
        B.Res(6, i, j, k) = Qk * B.vol(i, j, k);
        B.Res(7, i, j, k) = Qw * B.vol(i, j, k);
      }
  // f1 on the faces i=nx, j=ny, k=nz: undefined in the reference; take the adjacent interior cell.
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++)
        if (i == nx || j == ny || k == nz) f1(i, j, k) = f1(std::min(i, nx - 1), std::min(j, ny - 1), std::min(k, nz - 1));
  // mu_t ghosts: copy of the neighbours over the whole (-1:n+1) extent, in this order (170-175)
  for (int k = -1; k <= nz + 1; k++) for (int j = -1; j <= ny + 1; j++) { B.mu_t(0, j, k) = B.mu_t(1, j, k); }
  for (int k = -1; k <= nz + 1; k++) for (int j = -1; j <= ny + 1; j++) { B.mu_t(nx, j, k) = B.mu_t(nx - 1, j, k); }
  for (int k = -1; k <= nz + 1; k++) for (int i = -1; i <= nx + 1; i++) { B.mu_t(i, 0, k) = B.mu_t(i, 1, k); }
  for (int k = -1; k <= nz + 1; k++) for (int i = -1; i <= nx + 1; i++) { B.mu_t(i, ny, k) = B.mu_t(i, ny - 1, k); }
  for (int j = -1; j <= ny + 1; j++) for (int i = -1; i <= nx + 1; i++) { B.mu_t(i, j, 0) = B.mu_t(i, j, 1); }
  for (int j = -1; j <= ny + 1; j++) for (int i = -1; i <= nx + 1; i++) { B.mu_t(i, j, nz) = B.mu_t(i, j, nz - 1); }
  amut_boundary(B);
  // i direction
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++) {
        double sk = f1(i, j, k) * sigma_k1 + (1.0 - f1(i, j, k)) * sigma_k2;
        double sw = f1(i, j, k) * sigma_w1 + (1.0 - f1(i, j, k)) * sigma_w2;
        double muk = (B.mu(i - 1, j, k) + B.mu(i, j, k) + sk * (B.mu_t(i - 1, j, k) + B.mu_t(i, j, k))) * 0.5 / Re;
        double muw = (B.mu(i - 1, j, k) + B.mu(i, j, k) + sw * (B.mu_t(i - 1, j, k) + B.mu_t(i, j, k))) * 0.5 / Re;
        double s1x = B.ni1(i, j, k), s1y = B.ni2(i, j, k), s1z = B.ni3(i, j, k);
        double Kti = Kt(i, j, k) - Kt(i - 1, j, k), Wti = Wt(i, j, k) - Wt(i - 1, j, k);
        double Ktj = 0.25 * (Kt(i, j + 1, k) - Kt(i, j - 1, k) + Kt(i - 1, j + 1, k) - Kt(i - 1, j - 1, k));
        double Wtj = 0.25 * (Wt(i, j + 1, k) - Wt(i, j - 1, k) + Wt(i - 1, j + 1, k) - Wt(i - 1, j - 1, k));
        double Ktk = 0.25 * (Kt(i, j, k + 1) - Kt(i, j, k - 1) + Kt(i - 1, j, k + 1) - Kt(i - 1, j, k - 1));
        double Wtk = 0.25 * (Wt(i, j, k + 1) - Wt(i, j, k - 1) + Wt(i - 1, j, k + 1) - Wt(i - 1, j, k - 1));
        double ix = B.ix1(i, j, k), iy = B.iy1(i, j, k), iz = B.iz1(i, j, k), jx = B.jx1(i, j, k), jy = B.jy1(i, j, k), jz = B.jz1(i, j, k);
        double kx = B.kx1(i, j, k), ky = B.ky1(i, j, k), kz = B.kz1(i, j, k);
        double ktx = Kti * ix + Ktj * jx + Ktk * kx, wtx = Wti * ix + Wtj * jx + Wtk * kx;
        double kty = Kti * iy + Ktj * jy + Ktk * ky, wty = Wti * iy + Wtj * jy + Wtk * ky;
        double ktz = Kti * iz + Ktj * jz + Ktk * kz, wtz = Wti * iz + Wtj * jz + Wtk * kz;
        double vn1 = uu(i - 1, j, k) * s1x + v(i - 1, j, k) * s1y + w(i - 1, j, k) * s1z;
        double vn2 = uu(i, j, k) * s1x + v(i, j, k) * s1y + w(i, j, k) * s1z;
        double kfi = 0.5 * ((vn1 + std::fabs(vn1)) * Kt(i - 1, j, k) + (vn2 - std::fabs(vn2)) * Kt(i, j, k));
        double wfi = 0.5 * ((vn1 + std::fabs(vn1)) * Wt(i - 1, j, k) + (vn2 - std::fabs(vn2)) * Wt(i, j, k));
        Fluxk(i, j, k) = (-kfi + muk * (ktx * s1x + kty * s1y + ktz * s1z)) * B.Si(i, j, k);
        Fluxw(i, j, k) = (-wfi + muw * (wtx * s1x + wty * s1y + wtz * s1z)) * B.Si(i, j, k);
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        B.Res(6, i, j, k) = B.Res(6, i, j, k) + Fluxk(i + 1, j, k) - Fluxk(i, j, k);
        B.Res(7, i, j, k) = B.Res(7, i, j, k) + Fluxw(i + 1, j, k) - Fluxw(i, j, k);
      }
  // j direction
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double sk = f1(i, j, k) * sigma_k1 + (1.0 - f1(i, j, k)) * sigma_k2;
        double sw = f1(i, j, k) * sigma_w1 + (1.0 - f1(i, j, k)) * sigma_w2;
        double muk = (B.mu(i, j - 1, k) + B.mu(i, j, k) + sk * (B.mu_t(i, j - 1, k) + B.mu_t(i, j, k))) * 0.5 / Re;
        double muw = (B.mu(i, j - 1, k) + B.mu(i, j, k) + sw * (B.mu_t(i, j - 1, k) + B.mu_t(i, j, k))) * 0.5 / Re;
        double s1x = B.nj1(i, j, k), s1y = B.nj2(i, j, k), s1z = B.nj3(i, j, k);
        double kti = 0.25 * (Kt(i + 1, j, k) - Kt(i - 1, j, k) + Kt(i + 1, j - 1, k) - Kt(i - 1, j - 1, k));
        double ktj = Kt(i, j, k) - Kt(i, j - 1, k);
        double ktk = 0.25 * (Kt(i, j, k + 1) - Kt(i, j, k - 1) + Kt(i, j - 1, k + 1) - Kt(i, j - 1, k - 1));
        double wti = 0.25 * (Wt(i + 1, j, k) - Wt(i - 1, j, k) + Wt(i + 1, j - 1, k) - Wt(i - 1, j - 1, k));
        double wtj = Wt(i, j, k) - Wt(i, j - 1, k);
        double wtk = 0.25 * (Wt(i, j, k + 1) - Wt(i, j, k - 1) + Wt(i, j - 1, k + 1) - Wt(i, j - 1, k - 1));
        double ix = B.ix2(i, j, k), iy = B.iy2(i, j, k), iz = B.iz2(i, j, k), jx = B.jx2(i, j, k), jy = B.jy2(i, j, k), jz = B.jz2(i, j, k);
        double kx = B.kx2(i, j, k), ky = B.ky2(i, j, k), kz = B.kz2(i, j, k);
        double ktx = kti * ix + ktj * jx + ktk * kx, kty = kti * iy + ktj * jy + ktk * ky, ktz = kti * iz + ktj * jz + ktk * kz;
        double wtx = wti * ix + wtj * jx + wtk * kx, wty = wti * iy + wtj * jy + wtk * ky, wtz = wti * iz + wtj * jz + wtk * kz;
        double vn1 = uu(i, j - 1, k) * s1x + v(i, j - 1, k) * s1y + w(i, j - 1, k) * s1z;
        double vn2 = uu(i, j, k) * s1x + v(i, j, k) * s1y + w(i, j, k) * s1z;
        double kfi = 0.5 * ((vn1 + std::fabs(vn1)) * Kt(i, j - 1, k) + (vn2 - std::fabs(vn2)) * Kt(i, j, k));
        double wfi = 0.5 * ((vn1 + std::fabs(vn1)) * Wt(i, j - 1, k) + (vn2 - std::fabs(vn2)) * Wt(i, j, k));
        Fluxk(i, j, k) = (-kfi + muk * (ktx * s1x + kty * s1y + ktz * s1z)) * B.Sj(i, j, k);
        Fluxw(i, j, k) = (-wfi + muw * (wtx * s1x + wty * s1y + wtz * s1z)) * B.Sj(i, j, k);
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        B.Res(6, i, j, k) = B.Res(6, i, j, k) + Fluxk(i, j + 1, k) - Fluxk(i, j, k);
        B.Res(7, i, j, k) = B.Res(7, i, j, k) + Fluxw(i, j + 1, k) - Fluxw(i, j, k);
      }
  // k direction
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        double sk = f1(i, j, k) * sigma_k1 + (1.0 - f1(i, j, k)) * sigma_k2;
        double sw = f1(i, j, k) * sigma_w1 + (1.0 - f1(i, j, k)) * sigma_w2;
        double muk = (B.mu(i, j, k - 1) + B.mu(i, j, k) + sk * (B.mu_t(i, j, k - 1) + B.mu_t(i, j, k))) * 0.5 / Re;
        double muw = (B.mu(i, j, k - 1) + B.mu(i, j, k) + sw * (B.mu_t(i, j, k - 1) + B.mu_t(i, j, k))) * 0.5 / Re;
        double s1x = B.nk1(i, j, k), s1y = B.nk2(i, j, k), s1z = B.nk3(i, j, k);
        double kti = 0.25 * (Kt(i + 1, j, k) - Kt(i - 1, j, k) + Kt(i + 1, j, k - 1) - Kt(i - 1, j, k - 1));
        double ktj = 0.25 * (Kt(i, j + 1, k) - Kt(i, j - 1, k) + Kt(i, j + 1, k - 1) - Kt(i, j - 1, k - 1));
        double ktk = Kt(i, j, k) - Kt(i, j, k - 1);
        double wti = 0.25 * (Wt(i + 1, j, k) - Wt(i - 1, j, k) + Wt(i + 1, j, k - 1) - Wt(i - 1, j, k - 1));
        double wtj = 0.25 * (Wt(i, j + 1, k) - Wt(i, j - 1, k) + Wt(i, j + 1, k - 1) - Wt(i, j - 1, k - 1));
        double wtk = Wt(i, j, k) - Wt(i, j, k - 1);
        double ix = B.ix3(i, j, k), iy = B.iy3(i, j, k), iz = B.iz3(i, j, k), jx = B.jx3(i, j, k), jy = B.jy3(i, j, k), jz = B.jz3(i, j, k);
        double kx = B.kx3(i, j, k), ky = B.ky3(i, j, k), kz = B.kz3(i, j, k);
        double ktx = kti * ix + ktj * jx + ktk * kx, kty = kti * iy + ktj * jy + ktk * ky, ktz = kti * iz + ktj * jz + ktk * kz;
        double wtx = wti * ix + wtj * jx + wtk * kx, wty = wti * iy + wtj * jy + wtk * ky, wtz = wti * iz + wtj * jz + wtk * kz;
        double vn1 = uu(i, j, k - 1) * s1x + v(i, j, k - 1) * s1y + w(i, j, k - 1) * s1z;
        double vn2 = uu(i, j, k) * s1x + v(i, j, k) * s1y + w(i, j, k) * s1z;
        double kfi = 0.5 * ((vn1 + std::fabs(vn1)) * Kt(i, j, k - 1) + (vn2 - std::fabs(vn2)) * Kt(i, j, k));
        double wfi = 0.5 * ((vn1 + std::fabs(vn1)) * Wt(i, j, k - 1) + (vn2 - std::fabs(vn2)) * Wt(i, j, k));
        Fluxk(i, j, k) = (-kfi + muk * (ktx * s1x + kty * s1y + ktz * s1z)) * B.Sk(i, j, k);
        Fluxw(i, j, k) = (-wfi + muw * (wtx * s1x + wty * s1y + wtz * s1z)) * B.Sk(i, j, k);
      }
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        B.Res(6, i, j, k) = B.Res(6, i, j, k) + Fluxk(i, j, k + 1) - Fluxk(i, j, k);
        B.Res(7, i, j, k) = B.Res(7, i, j, k) + Fluxw(i, j, k + 1) - Fluxw(i, j, k);
      }
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) { B.mu(i, j, k) = B.mu(i, j, k) / Re; B.mu_t(i, j, k) = B.mu_t(i, j, k) / Re; }
}

// inviscid face flux (common body of flux_inviscous_i/j/k, sub_Residual.f90:222-337)
// dir: 0=i, 1=j, 2=k; (i,j,k) is the face index, stencil cells along dir from face-4 to face+3
static void face_inviscid(Case& C, Block& B, Work& W, int dir, int i, int j, int k, int Scheme, double* Fout) {
  const ocfd_params& P = C.P;
  double gamma = P.gamma;
  double s1x, s1y, s1z, t1x, t1y, t1z, S;
  if (dir == 0) {
    s1x = B.ni1(i, j, k); s1y = B.ni2(i, j, k); s1z = B.ni3(i, j, k); S = B.Si(i, j, k);
    t1x = B.x(i, j + 1, k) - B.x(i, j, k + 1); t1y = B.y(i, j + 1, k) - B.y(i, j, k + 1); t1z = B.z(i, j + 1, k) - B.z(i, j, k + 1);
  } else if (dir == 1) {
    s1x = B.nj1(i, j, k); s1y = B.nj2(i, j, k); s1z = B.nj3(i, j, k); S = B.Sj(i, j, k);
    t1x = B.x(i + 1, j, k + 1) - B.x(i, j, k); t1y = B.y(i + 1, j, k + 1) - B.y(i, j, k); t1z = B.z(i + 1, j, k + 1) - B.z(i, j, k);
  } else {
    s1x = B.nk1(i, j, k); s1y = B.nk2(i, j, k); s1z = B.nk3(i, j, k); S = B.Sk(i, j, k);
    t1x = B.x(i + 1, j + 1, k) - B.x(i, j, k); t1y = B.y(i + 1, j + 1, k) - B.y(i, j, k); t1z = B.z(i + 1, j + 1, k) - B.z(i, j, k);
  }
  double t10 = 1.0 / (std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z));
  double s2x = t1x * t10, s2y = t1y * t10, s2z = t1z * t10;
  double s3x = s1y * s2z - s1z * s2y, s3y = s1z * s2x - s1x * s2z, s3z = s1x * s2y - s1y * s2x;
  int di = dir == 0, dj = dir == 1, dk = dir == 2;
  double U0[5][8], UL[5], UR[5];
  int rec = P.iflag_reconstruction;
  for (int q = 0; q < 8; q++) {
    int s = q - LAP;  // cell offset -4..3 from the face
    int ii = i + s * di, jj = j + s * dj, kk = k + s * dk;
    if (rec == 0) { U0[0][q] = W.d(ii, jj, kk); U0[1][q] = W.uu(ii, jj, kk); U0[2][q] = W.v(ii, jj, kk); U0[3][q] = W.w(ii, jj, kk); U0[4][q] = W.p(ii, jj, kk); }
    else { for (int m = 0; m < 5; m++) U0[m][q] = B.U(m + 1, ii, jj, kk); }
  }
  if (rec == 0) recon_original(U0, UL, UR, Scheme);
  else if (rec == 1) recon_conservative(U0, UL, UR, gamma, Scheme);
  else recon_characteristic(U0, UL, UR, gamma, Scheme);
  if (P.if_scheme_positivity == 1) {
    if (UL[0] <= Lim_Zero || UL[4] <= Lim_Zero) {
      int ii = i - di, jj = j - dj, kk = k - dk;
      UL[0] = W.d(ii, jj, kk); UL[1] = W.uu(ii, jj, kk); UL[2] = W.v(ii, jj, kk); UL[3] = W.w(ii, jj, kk); UL[4] = W.p(ii, jj, kk);
    }
    if (UR[0] <= Lim_Zero || UR[4] <= Lim_Zero) {
      UR[0] = W.d(i, j, k); UR[1] = W.uu(i, j, k); UR[2] = W.v(i, j, k); UR[3] = W.w(i, j, k); UR[4] = W.p(i, j, k);
    }
  }
  double QL[5], QR[5], F0[5];
  QL[0] = UL[0]; QL[1] = UL[1] * s1x + UL[2] * s1y + UL[3] * s1z; QL[2] = UL[1] * s2x + UL[2] * s2y + UL[3] * s2z;
  QL[3] = UL[1] * s3x + UL[2] * s3y + UL[3] * s3z; QL[4] = UL[4];
  QR[0] = UR[0]; QR[1] = UR[1] * s1x + UR[2] * s1y + UR[3] * s1z; QR[2] = UR[1] * s2x + UR[2] * s2y + UR[3] * s2z;
  QR[3] = UR[1] * s3x + UR[2] * s3y + UR[3] * s3z; QR[4] = UR[4];
  flux_1d(QL, QR, F0, gamma, P.iflag_flux);
  Fout[0] = -F0[0] * S;
  Fout[1] = -(F0[1] * s1x + F0[2] * s2x + F0[3] * s3x) * S;
  Fout[2] = -(F0[1] * s1y + F0[2] * s2y + F0[3] * s3y) * S;
  Fout[3] = -(F0[1] * s1z + F0[2] * s2z + F0[3] * s3z) * S;
  Fout[4] = -F0[4] * S;
}

static void flux_inviscid(Case& C, Block& B, Work& W, int dir) {  // flux_inviscous_i/j/k
  int nx = B.nx, ny = B.ny, nz = B.nz, NV = C.NVAR;
  std::fill(W.Flux.v.begin(), W.Flux.v.end(), 0.0);
  int n1 = dir == 0 ? nx : nx - 1, n2 = dir == 1 ? ny : ny - 1, n3 = dir == 2 ? nz : nz - 1;
  int nd = dir == 0 ? nx : (dir == 1 ? ny : nz);
  par_for(1, n3, [&](int k) {
    for (int j = 1; j <= n2; j++)
      for (int i = 1; i <= n1; i++) {
        int Scheme = C.P.iflag_scheme;
        int idx = dir == 0 ? i : (dir == 1 ? j : k);
        int lo, hi;
        if (dir == 0) { lo = B.BcI(j, k, 1); hi = B.BcI(j, k, 2); }
        else if (dir == 1) { lo = B.BcJ(i, k, 1); hi = B.BcJ(i, k, 2); }
        else { lo = B.BcK(i, j, 1); hi = B.BcK(i, j, 2); }
        if (lo == 1) { if (idx == 1) Scheme = S_CD2; else if (idx < LAP) Scheme = C.P.bound_scheme; }
        if (hi == 1) { if (idx == nd) Scheme = S_CD2; else if (idx > nd - LAP + 1) Scheme = C.P.bound_scheme; }
        if (B.overlimit == 1) Scheme = S_UD1;
        double F[5];
        face_inviscid(C, B, W, dir, i, j, k, Scheme, F);
        for (int m = 0; m < 5; m++) W.Flux(m + 1, i, j, k) = F[m];
      }
  });
  if (dir == 2) {  // physical k-faces: central flux of averaged primitives (666-689)
    double gamma = C.P.gamma;
    for (const Sub& Bc : B.sub) {
      if (Bc.bc > 0 && (Bc.face == 3 || Bc.face == 6)) {
        int k = Bc.kb;
        for (int j = Bc.jb; j <= Bc.je - 1; j++)
          for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
            double d0 = (W.d(i, j, k) + W.d(i, j, k - 1)) * 0.5, uu0 = (W.uu(i, j, k) + W.uu(i, j, k - 1)) * 0.5;
            double v0 = (W.v(i, j, k) + W.v(i, j, k - 1)) * 0.5, w0 = (W.w(i, j, k) + W.w(i, j, k - 1)) * 0.5;
            double p0 = (W.p(i, j, k) + W.p(i, j, k - 1)) * 0.5;
            double E0 = p0 / (gamma - 1.0) + d0 * (uu0 * uu0 + v0 * v0 + w0 * w0) * 0.5;
            double un = uu0 * B.nk1(i, j, k) + v0 * B.nk2(i, j, k) + w0 * B.nk3(i, j, k);
            W.Flux(1, i, j, k) = -d0 * un * B.Sk(i, j, k);
            W.Flux(2, i, j, k) = -(d0 * un * uu0 + p0 * B.nk1(i, j, k)) * B.Sk(i, j, k);
            W.Flux(3, i, j, k) = -(d0 * un * v0 + p0 * B.nk2(i, j, k)) * B.Sk(i, j, k);
            W.Flux(4, i, j, k) = -(d0 * un * w0 + p0 * B.nk3(i, j, k)) * B.Sk(i, j, k);
            W.Flux(5, i, j, k) = -(E0 + p0) * un * B.Sk(i, j, k);
          }
      }
    }
  }
  (void)NV;
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++)
        for (int m = 1; m <= 5; m++) {
          if (dir == 0) B.Res(m, i, j, k) = W.Flux(m, i + 1, j, k) - W.Flux(m, i, j, k);
          else if (dir == 1) B.Res(m, i, j, k) = B.Res(m, i, j, k) + W.Flux(m, i, j + 1, k) - W.Flux(m, i, j, k);
          else B.Res(m, i, j, k) = B.Res(m, i, j, k) + W.Flux(m, i, j, k + 1) - W.Flux(m, i, j, k);
        }
}

// viscous face flux (flux_viscous_i/j/k bodies, sub_Residual.f90:755-854, 936-1032, 1116-1212)
static void flux_viscous(Case& C, Block& B, Work& W, int dir) {
  int nx = B.nx, ny = B.ny, nz = B.nz;
  const double tmp1 = 4.0 / 3.0, tmp2 = 2.0 / 3.0;
  double Cp = C.P.cp, PrL = C.P.prl, PrT = C.P.prt;
  A3 &uu = W.uu, &v = W.v, &w = W.w, &T = W.T;
  if (B.overlimit == 1) {
    if (dir == 0) for (int k = 1; k <= nz - 1; k++) for (int j = 1; j <= ny - 1; j++) for (int c = 1; c <= 3; c++) { B.surf1(j, k, c) = 0.0; B.surf4(j, k, c) = 0.0; }
    if (dir == 1) for (int k = 1; k <= nz - 1; k++) for (int i = 1; i <= nx - 1; i++) for (int c = 1; c <= 3; c++) { B.surf2(i, k, c) = 0.0; B.surf5(i, k, c) = 0.0; }
    if (dir == 2) for (int j = 1; j <= ny - 1; j++) for (int i = 1; i <= nx - 1; i++) for (int c = 1; c <= 3; c++) { B.surf3(i, j, c) = 0.0; B.surf6(i, j, c) = 0.0; }
    return;
  }
  int n1 = dir == 0 ? nx : nx - 1, n2 = dir == 1 ? ny : ny - 1, n3 = dir == 2 ? nz : nz - 1;
  par_for(1, n3, [&](int k) {
    for (int j = 1; j <= n2; j++)
      for (int i = 1; i <= n1; i++) {
        double s1x, s1y, s1z, S;
        double ui, vi, wi, Ti, uj, vj, wj, Tj, uk, vk, wk, Tk;
        double ix, iy, iz, jx, jy, jz, kx, ky, kz;
        int im = i, jm = j, km = k;  // the other cell of the face
        if (dir == 0) {
          im = i - 1;
          s1x = B.ni1(i, j, k); s1y = B.ni2(i, j, k); s1z = B.ni3(i, j, k); S = B.Si(i, j, k);
          ui = uu(i, j, k) - uu(i - 1, j, k); vi = v(i, j, k) - v(i - 1, j, k); wi = w(i, j, k) - w(i - 1, j, k); Ti = T(i, j, k) - T(i - 1, j, k);
          double uj1, vj1, wj1, Tj1, uj2, vj2, wj2, Tj2, uk1, vk1, wk1, Tk1, uk2, vk2, wk2, Tk2;
          if ((i == 1 || i == nx) && (j == 1 || j == ny - 1)) { uj1 = vj1 = wj1 = Tj1 = uj2 = vj2 = wj2 = Tj2 = 0.0; }
          else {
            uj1 = 0.5 * (uu(i, j - 1, k) + uu(i - 1, j - 1, k)); vj1 = 0.5 * (v(i, j - 1, k) + v(i - 1, j - 1, k));
            wj1 = 0.5 * (w(i, j - 1, k) + w(i - 1, j - 1, k)); Tj1 = 0.5 * (T(i, j - 1, k) + T(i - 1, j - 1, k));
            uj2 = 0.5 * (uu(i, j + 1, k) + uu(i - 1, j + 1, k)); vj2 = 0.5 * (v(i, j + 1, k) + v(i - 1, j + 1, k));
            wj2 = 0.5 * (w(i, j + 1, k) + w(i - 1, j + 1, k)); Tj2 = 0.5 * (T(i, j + 1, k) + T(i - 1, j + 1, k));
          }
          if ((i == 1 || i == nx) && (k == 1 || k == nz - 1)) { uk1 = vk1 = wk1 = Tk1 = uk2 = vk2 = wk2 = Tk2 = 0.0; }
          else {
            uk1 = 0.5 * (uu(i, j, k - 1) + uu(i - 1, j, k - 1)); vk1 = 0.5 * (v(i, j, k - 1) + v(i - 1, j, k - 1));
            wk1 = 0.5 * (w(i, j, k - 1) + w(i - 1, j, k - 1)); Tk1 = 0.5 * (T(i, j, k - 1) + T(i - 1, j, k - 1));
            uk2 = 0.5 * (uu(i, j, k + 1) + uu(i - 1, j, k + 1)); vk2 = 0.5 * (v(i, j, k + 1) + v(i - 1, j, k + 1));
            wk2 = 0.5 * (w(i, j, k + 1) + w(i - 1, j, k + 1)); Tk2 = 0.5 * (T(i, j, k + 1) + T(i - 1, j, k + 1));
          }
          uj = 0.5 * (uj2 - uj1); vj = 0.5 * (vj2 - vj1); wj = 0.5 * (wj2 - wj1); Tj = 0.5 * (Tj2 - Tj1);
          uk = 0.5 * (uk2 - uk1); vk = 0.5 * (vk2 - vk1); wk = 0.5 * (wk2 - wk1); Tk = 0.5 * (Tk2 - Tk1);
          ix = B.ix1(i, j, k); iy = B.iy1(i, j, k); iz = B.iz1(i, j, k); jx = B.jx1(i, j, k); jy = B.jy1(i, j, k); jz = B.jz1(i, j, k);
          kx = B.kx1(i, j, k); ky = B.ky1(i, j, k); kz = B.kz1(i, j, k);
        } else if (dir == 1) {
          jm = j - 1;
          s1x = B.nj1(i, j, k); s1y = B.nj2(i, j, k); s1z = B.nj3(i, j, k); S = B.Sj(i, j, k);
          uj = uu(i, j, k) - uu(i, j - 1, k); vj = v(i, j, k) - v(i, j - 1, k); wj = w(i, j, k) - w(i, j - 1, k); Tj = T(i, j, k) - T(i, j - 1, k);
          double ui1, vi1, wi1, Ti1, ui2, vi2, wi2, Ti2, uk1, vk1, wk1, Tk1, uk2, vk2, wk2, Tk2;
          if ((j == 1 || j == ny) && (i == 1 || i == nx - 1)) { ui1 = vi1 = wi1 = Ti1 = ui2 = vi2 = wi2 = Ti2 = 0.0; }
          else {
            ui1 = 0.5 * (uu(i - 1, j, k) + uu(i - 1, j - 1, k)); vi1 = 0.5 * (v(i - 1, j, k) + v(i - 1, j - 1, k));
            wi1 = 0.5 * (w(i - 1, j, k) + w(i - 1, j - 1, k)); Ti1 = 0.5 * (T(i - 1, j, k) + T(i - 1, j - 1, k));
            ui2 = 0.5 * (uu(i + 1, j, k) + uu(i + 1, j - 1, k)); vi2 = 0.5 * (v(i + 1, j, k) + v(i + 1, j - 1, k));
            wi2 = 0.5 * (w(i + 1, j, k) + w(i + 1, j - 1, k)); Ti2 = 0.5 * (T(i + 1, j, k) + T(i + 1, j - 1, k));
          }
          if ((j == 1 || j == ny) && (k == 1 || k == nz - 1)) { uk1 = vk1 = wk1 = Tk1 = uk2 = vk2 = wk2 = Tk2 = 0.0; }
          else {
            uk1 = 0.5 * (uu(i, j, k - 1) + uu(i, j - 1, k - 1)); vk1 = 0.5 * (v(i, j, k - 1) + v(i, j - 1, k - 1));
            wk1 = 0.5 * (w(i, j, k - 1) + w(i, j - 1, k - 1)); Tk1 = 0.5 * (T(i, j, k - 1) + T(i, j - 1, k - 1));
            uk2 = 0.5 * (uu(i, j, k + 1) + uu(i, j - 1, k + 1)); vk2 = 0.5 * (v(i, j, k + 1) + v(i, j - 1, k + 1));
            wk2 = 0.5 * (w(i, j, k + 1) + w(i, j - 1, k + 1)); Tk2 = 0.5 * (T(i, j, k + 1) + T(i, j - 1, k + 1));
          }
          ui = 0.5 * (ui2 - ui1); vi = 0.5 * (vi2 - vi1); wi = 0.5 * (wi2 - wi1); Ti = 0.5 * (Ti2 - Ti1);
          uk = 0.5 * (uk2 - uk1); vk = 0.5 * (vk2 - vk1); wk = 0.5 * (wk2 - wk1); Tk = 0.5 * (Tk2 - Tk1);
          ix = B.ix2(i, j, k); iy = B.iy2(i, j, k); iz = B.iz2(i, j, k); jx = B.jx2(i, j, k); jy = B.jy2(i, j, k); jz = B.jz2(i, j, k);
          kx = B.kx2(i, j, k); ky = B.ky2(i, j, k); kz = B.kz2(i, j, k);
        } else {
          km = k - 1;
          s1x = B.nk1(i, j, k); s1y = B.nk2(i, j, k); s1z = B.nk3(i, j, k); S = B.Sk(i, j, k);
          uk = uu(i, j, k) - uu(i, j, k - 1); vk = v(i, j, k) - v(i, j, k - 1); wk = w(i, j, k) - w(i, j, k - 1); Tk = T(i, j, k) - T(i, j, k - 1);
          double ui1, vi1, wi1, Ti1, ui2, vi2, wi2, Ti2, uj1, vj1, wj1, Tj1, uj2, vj2, wj2, Tj2;
          if ((k == 1 || k == nz) && (i == 1 || i == nx - 1)) { ui1 = vi1 = wi1 = Ti1 = ui2 = vi2 = wi2 = Ti2 = 0.0; }
          else {
            ui1 = 0.5 * (uu(i - 1, j, k) + uu(i - 1, j, k - 1)); vi1 = 0.5 * (v(i - 1, j, k) + v(i - 1, j, k - 1));
            wi1 = 0.5 * (w(i - 1, j, k) + w(i - 1, j, k - 1)); Ti1 = 0.5 * (T(i - 1, j, k) + T(i - 1, j, k - 1));
            ui2 = 0.5 * (uu(i + 1, j, k) + uu(i + 1, j, k - 1)); vi2 = 0.5 * (v(i + 1, j, k) + v(i + 1, j, k - 1));
            wi2 = 0.5 * (w(i + 1, j, k) + w(i + 1, j, k - 1)); Ti2 = 0.5 * (T(i + 1, j, k) + T(i + 1, j, k - 1));
          }
          if ((k == 1 || k == nz) && (j == 1 || j == ny - 1)) { uj1 = vj1 = wj1 = Tj1 = uj2 = vj2 = wj2 = Tj2 = 0.0; }
          else {
            uj1 = 0.5 * (uu(i, j - 1, k) + uu(i, j - 1, k - 1)); vj1 = 0.5 * (v(i, j - 1, k) + v(i, j - 1, k - 1));
            wj1 = 0.5 * (w(i, j - 1, k) + w(i, j - 1, k - 1)); Tj1 = 0.5 * (T(i, j - 1, k) + T(i, j - 1, k - 1));
            uj2 = 0.5 * (uu(i, j + 1, k) + uu(i, j + 1, k - 1)); vj2 = 0.5 * (v(i, j + 1, k) + v(i, j + 1, k - 1));
            wj2 = 0.5 * (w(i, j + 1, k) + w(i, j + 1, k - 1)); Tj2 = 0.5 * (T(i, j + 1, k) + T(i, j + 1, k - 1));
          }
          ui = 0.5 * (ui2 - ui1); vi = 0.5 * (vi2 - vi1); wi = 0.5 * (wi2 - wi1); Ti = 0.5 * (Ti2 - Ti1);
          uj = 0.5 * (uj2 - uj1); vj = 0.5 * (vj2 - vj1); wj = 0.5 * (wj2 - wj1); Tj = 0.5 * (Tj2 - Tj1);
          ix = B.ix3(i, j, k); iy = B.iy3(i, j, k); iz = B.iz3(i, j, k); jx = B.jx3(i, j, k); jy = B.jy3(i, j, k); jz = B.jz3(i, j, k);
          kx = B.kx3(i, j, k); ky = B.ky3(i, j, k); kz = B.kz3(i, j, k);
        }
        double ux = ui * ix + uj * jx + uk * kx, vx = vi * ix + vj * jx + vk * kx, wx = wi * ix + wj * jx + wk * kx, Tx = Ti * ix + Tj * jx + Tk * kx;
        double uy = ui * iy + uj * jy + uk * ky, vy = vi * iy + vj * jy + vk * ky, wy = wi * iy + wj * jy + wk * ky, Ty = Ti * iy + Tj * jy + Tk * ky;
        double uz = ui * iz + uj * jz + uk * kz, vz = vi * iz + vj * jz + vk * kz, wz = wi * iz + wj * jz + wk * kz, Tz = Ti * iz + Tj * jz + Tk * kz;
        double mu0 = 0.5 * (B.mu(i, j, k) + B.mu_t(i, j, k) + B.mu(im, jm, km) + B.mu_t(im, jm, km));
        double k0 = 0.5 * Cp * (B.mu(i, j, k) / PrL + B.mu_t(i, j, k) / PrT + B.mu(im, jm, km) / PrL + B.mu_t(im, jm, km) / PrT);
        double s11 = mu0 * (tmp1 * ux - tmp2 * (vy + wz)), s12 = mu0 * (uy + vx), s13 = mu0 * (uz + wx);
        double s22 = mu0 * (tmp1 * vy - tmp2 * (ux + wz)), s23 = mu0 * (vz + wy), s33 = mu0 * (tmp1 * wz - tmp2 * (ux + vy));
        double u1 = (uu(i, j, k) + uu(im, jm, km)) * 0.5, v1 = (v(i, j, k) + v(im, jm, km)) * 0.5, w1 = (w(i, j, k) + w(im, jm, km)) * 0.5;
        double E1 = u1 * s11 + v1 * s12 + w1 * s13 + k0 * Tx;
        double E2 = u1 * s12 + v1 * s22 + w1 * s23 + k0 * Ty;
        double E3 = u1 * s13 + v1 * s23 + w1 * s33 + k0 * Tz;
        W.Flux(2, i, j, k) = (s11 * s1x + s12 * s1y + s13 * s1z) * S;
        W.Flux(3, i, j, k) = (s12 * s1x + s22 * s1y + s23 * s1z) * S;
        W.Flux(4, i, j, k) = (s13 * s1x + s23 * s1y + s33 * s1z) * S;
        W.Flux(5, i, j, k) = (E1 * s1x + E2 * s1y + E3 * s1z) * S;
      }
  });
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++)
        for (int m = 2; m <= 5; m++) {
          if (dir == 0) B.Res(m, i, j, k) = B.Res(m, i, j, k) + W.Flux(m, i + 1, j, k) - W.Flux(m, i, j, k);
          else if (dir == 1) B.Res(m, i, j, k) = B.Res(m, i, j, k) + W.Flux(m, i, j + 1, k) - W.Flux(m, i, j, k);
          else B.Res(m, i, j, k) = B.Res(m, i, j, k) + W.Flux(m, i, j, k + 1) - W.Flux(m, i, j, k);
        }
  if (dir == 0) for (int k = 1; k <= nz - 1; k++) for (int j = 1; j <= ny - 1; j++) for (int c = 1; c <= 3; c++) { B.surf1(j, k, c) = W.Flux(c + 1, 1, j, k); B.surf4(j, k, c) = W.Flux(c + 1, nx, j, k); }
  if (dir == 1) for (int k = 1; k <= nz - 1; k++) for (int i = 1; i <= nx - 1; i++) for (int c = 1; c <= 3; c++) { B.surf2(i, k, c) = W.Flux(c + 1, i, 1, k); B.surf5(i, k, c) = W.Flux(c + 1, i, ny, k); }
  if (dir == 2) for (int j = 1; j <= ny - 1; j++) for (int i = 1; i <= nx - 1; i++) for (int c = 1; c <= 3; c++) { B.surf3(i, j, c) = W.Flux(c + 1, i, j, 1); B.surf6(i, j, c) = W.Flux(c + 1, i, j, nz); }
}

static void comput_Lijk(Case& C, Block& B, Work& W) {  // sub_time_acceleraction.f90:7-56
  double gamma = C.P.gamma, PrL = C.P.prl, Prt = C.P.prt;
  const double four3 = (double)(4.0f / 3.0f);  // `4./3.` default-real
  for (int k = 1; k <= B.nz - 1; k++)
    for (int j = 1; j <= B.ny - 1; j++)
      for (int i = 1; i <= B.nx - 1; i++) {
        double D0;
        if (C.P.if_viscous == 1) D0 = std::max(gamma, four3) / W.d(i, j, k) * (B.mu(i, j, k) / PrL + B.mu_t(i, j, k) / Prt);
        else D0 = 0.0;
        double vol1 = 1.0 / B.vol(i, j, k);
        double uu = W.uu(i, j, k), v = W.v(i, j, k), w = W.w(i, j, k), cc = W.cc(i, j, k);
        double un = 0.5 * (uu * (B.ni1(i, j, k) + B.ni1(i + 1, j, k)) + v * (B.ni2(i, j, k) + B.ni2(i + 1, j, k)) + w * (B.ni3(i, j, k) + B.ni3(i + 1, j, k)));
        double S0 = (B.Si(i, j, k) + B.Si(i + 1, j, k)) * 0.5;
        W.Lci(i, j, k) = (std::fabs(un) + cc) * S0; W.Lvi(i, j, k) = D0 * S0 * S0 * vol1;
        un = 0.5 * (uu * (B.nj1(i, j, k) + B.nj1(i, j + 1, k)) + v * (B.nj2(i, j, k) + B.nj2(i, j + 1, k)) + w * (B.nj3(i, j, k) + B.nj3(i, j + 1, k)));
        S0 = (B.Sj(i, j, k) + B.Sj(i, j + 1, k)) * 0.5;
        W.Lcj(i, j, k) = (std::fabs(un) + cc) * S0; W.Lvj(i, j, k) = D0 * S0 * S0 * vol1;
        un = 0.5 * (uu * (B.nk1(i, j, k) + B.nk1(i, j, k + 1)) + v * (B.nk2(i, j, k) + B.nk2(i, j, k + 1)) + w * (B.nk3(i, j, k) + B.nk3(i, j, k + 1)));
        S0 = (B.Sk(i, j, k) + B.Sk(i, j, k + 1)) * 0.5;
        W.Lck(i, j, k) = (std::fabs(un) + cc) * S0; W.Lvk(i, j, k) = D0 * S0 * S0 * vol1;
      }
}

static void comput_dt(Case& C, Block& B, Work& W) {  // sub_time_acceleraction.f90:61-112
  const ocfd_params& P = C.P;
  double dt_fac = B.overlimit == 0 ? 1.0 : 0.1, Cc = 1.0;
  for (int k = 1; k <= B.nz - 1; k++)
    for (int j = 1; j <= B.ny - 1; j++)
      for (int i = 1; i <= B.nx - 1; i++) {
        if (P.iflag_local_dt == 1) {
          double dt = dt_fac * P.cfl * B.vol(i, j, k) / (W.Lci(i, j, k) + W.Lcj(i, j, k) + W.Lck(i, j, k) + Cc * (W.Lvi(i, j, k) + W.Lvj(i, j, k) + W.Lvk(i, j, k)));
          if (P.if_dtime_mesh == 1) dt = dt * B.dtime_mesh(i, j, k);
          if (dt > P.dtmax) dt = P.dtmax;
          if (dt < P.dtmin) dt = P.dtmin;
          B.dt(i, j, k) = dt;
        } else B.dt(i, j, k) = P.dt_global;
      }
}

// tridiagonal (sub_time_acceleraction.f90:222-241): a(i) Rs(i-1) + b(i) Rs(i) + c(i) Rs(i+1) = R(i) on
// i = 2..n-1 with the end values held, Rs(1) = R(1), Rs(n) = R(n); arrays 1-based (element 0 unused)
static void tridiagonal(int n, const double* a, const double* b, const double* c, const double* R, double* Rs) {
  std::vector<double> P(n + 1), Q(n + 1);
  P[1] = 0.0; Q[1] = R[1];
  P[n] = 0.0; Q[n] = R[n];
  for (int i = 2; i <= n; i++) {
    double tmp = 1.0 / (a[i] * P[i - 1] + b[i]);
    P[i] = -c[i] * tmp;
    Q[i] = (R[i] - a[i] * Q[i - 1]) * tmp;
  }
  Rs[n] = R[n];
  Rs[1] = R[1];
  for (int i = n - 1; i >= 2; i--) Rs[i] = P[i] * Rs[i + 1] + Q[i];
}

// upwind implicit residual smoothing (Residual_smoothing, sub_time_acceleraction.f90:119-217): per
// line in i, then j, then k, coefficients from the spectral-radius ratio ei = min(1, L_d/L_a, L_d/L_b)
// and the cell's normal Mach number on the averaged face normal; Res(1:5) only
static void residual_smoothing(Case& C, Block& B, Work& W) {
  (void)C;
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const double epsl = 1.0;
  const int nmax = std::max(nx, std::max(ny, nz)) + 1;
  std::vector<double> as(nmax), bs(nmax), cs(nmax), R(nmax), Rs(nmax);
  auto coef = [&](int q, double ei, double Mn) {
    if (Mn > 1.0) { as[q] = -ei; bs[q] = 1.0 + ei; cs[q] = 0.0; }
    else if (Mn < -1.0) { as[q] = 0.0; bs[q] = 1.0 + ei; cs[q] = -ei; }
    else { as[q] = -ei; bs[q] = 1.0 + 2.0 * ei; cs[q] = -ei; }
  };
  for (int k = 1; k <= nz - 1; k++)  // i direction, 131-156
    for (int j = 1; j <= ny - 1; j++) {
      for (int i = 1; i <= nx - 1; i++) {
        double ei = epsl * std::min(std::min(1.0, W.Lci(i, j, k) / W.Lcj(i, j, k)), W.Lci(i, j, k) / W.Lck(i, j, k));
        double Mn = 0.5 * (W.uu(i, j, k) * (B.ni1(i, j, k) + B.ni1(i + 1, j, k)) + W.v(i, j, k) * (B.ni2(i, j, k) + B.ni2(i + 1, j, k)) +
                           W.w(i, j, k) * (B.ni3(i, j, k) + B.ni3(i + 1, j, k))) / W.cc(i, j, k);
        coef(i, ei, Mn);
      }
      for (int m = 1; m <= 5; m++) {
        for (int i = 1; i <= nx - 1; i++) R[i] = B.Res(m, i, j, k);
        tridiagonal(nx - 1, as.data(), bs.data(), cs.data(), R.data(), Rs.data());
        for (int i = 1; i <= nx - 1; i++) B.Res(m, i, j, k) = Rs[i];
      }
    }
  for (int k = 1; k <= nz - 1; k++)  // j direction, 159-184
    for (int i = 1; i <= nx - 1; i++) {
      for (int j = 1; j <= ny - 1; j++) {
        double ei = epsl * std::min(std::min(1.0, W.Lcj(i, j, k) / W.Lci(i, j, k)), W.Lcj(i, j, k) / W.Lck(i, j, k));
        double Mn = 0.5 * (W.uu(i, j, k) * (B.nj1(i, j, k) + B.nj1(i, j + 1, k)) + W.v(i, j, k) * (B.nj2(i, j, k) + B.nj2(i, j + 1, k)) +
                           W.w(i, j, k) * (B.nj3(i, j, k) + B.nj3(i, j + 1, k))) / W.cc(i, j, k);
        coef(j, ei, Mn);
      }
      for (int m = 1; m <= 5; m++) {
        for (int j = 1; j <= ny - 1; j++) R[j] = B.Res(m, i, j, k);
        tridiagonal(ny - 1, as.data(), bs.data(), cs.data(), R.data(), Rs.data());
        for (int j = 1; j <= ny - 1; j++) B.Res(m, i, j, k) = Rs[j];
      }
    }
  for (int j = 1; j <= ny - 1; j++)  // k direction, 186-213
    for (int i = 1; i <= nx - 1; i++) {
      for (int k = 1; k <= nz - 1; k++) {
        double ei = epsl * std::min(std::min(1.0, W.Lck(i, j, k) / W.Lci(i, j, k)), W.Lck(i, j, k) / W.Lcj(i, j, k));
        double Mn = 0.5 * (W.uu(i, j, k) * (B.nk1(i, j, k) + B.nk1(i, j, k + 1)) + W.v(i, j, k) * (B.nk2(i, j, k) + B.nk2(i, j, k + 1)) +
                           W.w(i, j, k) * (B.nk3(i, j, k) + B.nk3(i, j, k + 1))) / W.cc(i, j, k);
        coef(k, ei, Mn);
      }
      for (int m = 1; m <= 5; m++) {
        for (int k = 1; k <= nz - 1; k++) R[k] = B.Res(m, i, j, k);
        tridiagonal(nz - 1, as.data(), bs.data(), cs.data(), R.data(), Rs.data());
        for (int k = 1; k <= nz - 1; k++) B.Res(m, i, j, k) = Rs[k];
      }
    }
}

static void comput_DFn(int NV, double* DF, const double* U, const double* DU, double n1, double n2, double n3, double gamma) {  // sub_LU_SGS.f90:135-157
  double U2[7];
  for (int m = 0; m < NV; m++) U2[m] = U[m] + DU[m];
  double un1 = (U[1] * n1 + U[2] * n2 + U[3] * n3) / U[0];
  double p1 = (gamma - 1.0) * (U[4] - 0.5 * (p2(U[1]) + p2(U[2]) + p2(U[3])) / U[0]);
  double un2 = (U2[1] * n1 + U2[2] * n2 + U2[3] * n3) / U2[0];
  double pp2 = (gamma - 1.0) * (U2[4] - 0.5 * (p2(U2[1]) + p2(U2[2]) + p2(U2[3])) / U2[0]);
  DF[0] = U2[0] * un2 - U[0] * un1;
  DF[1] = (U2[1] * un2 + pp2 * n1) - (U[1] * un1 + p1 * n1);
  DF[2] = (U2[2] * un2 + pp2 * n2) - (U[2] * un1 + p1 * n2);
  DF[3] = (U2[3] * un2 + pp2 * n3) - (U[3] * un1 + p1 * n3);
  DF[4] = (U2[4] + pp2) * un2 - (U[4] + p1) * un1;
  if (NV >= 6) DF[5] = U2[5] * un2 - U[5] * un1;
  if (NV == 7) DF[6] = U2[6] * un2 - U[6] * un1;
}

static void du_LU_SGS(Case& C, Block& B, Work& W, double Sfac1 = 0.0) {  // sub_LU_SGS.f90:4-129
  int NV = C.NVAR, nx = B.nx, ny = B.ny, nz = B.nz;
  double gamma = C.P.gamma, w_LU = C.P.w_lu;
  int visc = C.P.if_viscous;
  for (int plane = 3; plane <= nx + ny + nz - 3; plane++) {
    par_for(1, nz - 1, [&](int k) {
      for (int j = 1; j <= ny - 1; j++) {
        int i = plane - k - j;
        if (i < 1 || i > nx - 1) continue;
        double alfa[7], dui[7], duj[7], duk[7], DF[7], Uv[7], DUv[7];
        double a0 = B.vol(i, j, k) / B.dt(i, j, k) + w_LU * (W.Lci(i, j, k) + W.Lcj(i, j, k) + W.Lck(i, j, k));
        for (int m = 0; m < NV; m++) alfa[m] = a0;
        if (visc == 1) {
          for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + 2.0 * (W.Lvi(i, j, k) + W.Lvj(i, j, k) + W.Lvk(i, j, k));
          if (NV == 6) alfa[5] = alfa[5] + (W.Lvi(i, j, k) + W.Lvj(i, j, k) + W.Lvk(i, j, k));
        }
        if (C.P.time_method == -1) for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + Sfac1 * B.vol(i, j, k);  // line 39
        if (i != 1) {
          for (int m = 0; m < NV; m++) { Uv[m] = B.U(m + 1, i - 1, j, k); DUv[m] = B.DU(m + 1, i - 1, j, k); }
          comput_DFn(NV, DF, Uv, DUv, B.ni1(i, j, k), B.ni2(i, j, k), B.ni3(i, j, k), gamma);
          for (int m = 0; m < NV; m++) {
            dui[m] = 0.5 * (DF[m] * B.Si(i, j, k) + w_LU * W.Lci(i - 1, j, k) * DUv[m]);
            if (visc == 1) dui[m] = dui[m] + W.Lvi(i - 1, j, k) * DUv[m];
          }
        } else for (int m = 0; m < NV; m++) dui[m] = 0.0;
        if (j != 1) {
          for (int m = 0; m < NV; m++) { Uv[m] = B.U(m + 1, i, j - 1, k); DUv[m] = B.DU(m + 1, i, j - 1, k); }
          comput_DFn(NV, DF, Uv, DUv, B.nj1(i, j, k), B.nj2(i, j, k), B.nj3(i, j, k), gamma);
          for (int m = 0; m < NV; m++) {
            duj[m] = 0.5 * (DF[m] * B.Sj(i, j, k) + w_LU * W.Lcj(i, j - 1, k) * DUv[m]);
            if (visc == 1) duj[m] = duj[m] + W.Lvj(i, j - 1, k) * DUv[m];
          }
        } else for (int m = 0; m < NV; m++) duj[m] = 0.0;
        if (k != 1) {
          for (int m = 0; m < NV; m++) { Uv[m] = B.U(m + 1, i, j, k - 1); DUv[m] = B.DU(m + 1, i, j, k - 1); }
          comput_DFn(NV, DF, Uv, DUv, B.nk1(i, j, k), B.nk2(i, j, k), B.nk3(i, j, k), gamma);
          for (int m = 0; m < NV; m++) {
            duk[m] = 0.5 * (DF[m] * B.Sk(i, j, k) + w_LU * W.Lck(i, j, k - 1) * DUv[m]);
            if (visc == 1) duk[m] = duk[m] + W.Lvk(i, j, k - 1) * DUv[m];
          }
        } else for (int m = 0; m < NV; m++) duk[m] = 0.0;
        for (int m = 0; m < NV; m++) B.DU(m + 1, i, j, k) = (B.Res(m + 1, i, j, k) + dui[m] + duj[m] + duk[m]) / alfa[m];
      }
    });
  }
  for (int plane = nx + ny + nz - 3; plane >= 3; plane--) {
    par_for(1, nz - 1, [&](int k) {
      for (int j = ny - 1; j >= 1; j--) {
        int i = plane - k - j;
        if (i < 1 || i > nx - 1) continue;
        double alfa[7], dui[7], duj[7], duk[7], DF[7], Uv[7], DUv[7];
        double a0 = B.vol(i, j, k) / B.dt(i, j, k) + w_LU * (W.Lci(i, j, k) + W.Lcj(i, j, k) + W.Lck(i, j, k));
        for (int m = 0; m < NV; m++) alfa[m] = a0;
        if (visc == 1) {
          for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + 2.0 * (W.Lvi(i, j, k) + W.Lvj(i, j, k) + W.Lvk(i, j, k));
          if (NV == 6) alfa[5] = alfa[5] + W.Lvi(i, j, k) + W.Lvj(i, j, k) + W.Lvk(i, j, k);
        }
        if (C.P.time_method == -1) for (int m = 0; m < NV; m++) alfa[m] = alfa[m] + Sfac1 * B.vol(i, j, k);  // line 92
        if (i != nx - 1) {
          for (int m = 0; m < NV; m++) { Uv[m] = B.U(m + 1, i + 1, j, k); DUv[m] = B.DU(m + 1, i + 1, j, k); }
          comput_DFn(NV, DF, Uv, DUv, B.ni1(i, j, k), B.ni2(i, j, k), B.ni3(i, j, k), gamma);
          for (int m = 0; m < NV; m++) {
            dui[m] = -(0.5 * (DF[m] * B.Si(i + 1, j, k) - w_LU * W.Lci(i + 1, j, k) * DUv[m]));
            if (visc == 1) dui[m] = dui[m] + W.Lvi(i + 1, j, k) * DUv[m];
          }
        } else for (int m = 0; m < NV; m++) dui[m] = 0.0;
        if (j != ny - 1) {
          for (int m = 0; m < NV; m++) { Uv[m] = B.U(m + 1, i, j + 1, k); DUv[m] = B.DU(m + 1, i, j + 1, k); }
          comput_DFn(NV, DF, Uv, DUv, B.nj1(i, j, k), B.nj2(i, j, k), B.nj3(i, j, k), gamma);
          for (int m = 0; m < NV; m++) {
            duj[m] = -(0.5 * (DF[m] * B.Sj(i, j + 1, k) - w_LU * W.Lcj(i, j + 1, k) * DUv[m]));
            if (visc == 1) duj[m] = duj[m] + W.Lvj(i, j + 1, k) * DUv[m];
          }
        } else for (int m = 0; m < NV; m++) duj[m] = 0.0;
        if (k != nz - 1) {
          for (int m = 0; m < NV; m++) { Uv[m] = B.U(m + 1, i, j, k + 1); DUv[m] = B.DU(m + 1, i, j, k + 1); }
          comput_DFn(NV, DF, Uv, DUv, B.nk1(i, j, k), B.nk2(i, j, k), B.nk3(i, j, k), gamma);
          for (int m = 0; m < NV; m++) {
            duk[m] = -(0.5 * (DF[m] * B.Sk(i, j, k + 1) - w_LU * W.Lck(i, j, k + 1) * DUv[m]));
            if (visc == 1) duk[m] = duk[m] + W.Lvk(i, j, k + 1) * DUv[m];
          }
        } else for (int m = 0; m < NV; m++) duk[m] = 0.0;
        for (int m = 0; m < NV; m++) B.DU(m + 1, i, j, k) = B.DU(m + 1, i, j, k) + (dui[m] + duj[m] + duk[m]) / alfa[m];
      }
    });
  }
}

static int residual_block(Case& C, Block& B, bool lusgs, double Sfac = 0.0, double Sfac1 = 0.0) {  // Comput_Residual_one_mesh body, sub_Residual.f90:45-124
  Work W;
  int nx = B.nx, ny = B.ny, nz = B.nz;
  W.d.alloc(1 - LAP, nx + LAP - 1, 1 - LAP, ny + LAP - 1, 1 - LAP, nz + LAP - 1);
  W.uu = W.d; W.v = W.d; W.w = W.d; W.T = W.d; W.cc = W.d; W.p = W.d;
  W.Flux.alloc(C.NVAR, 1, nx, 1, ny, 1, nz);
  W.Lci.alloc(1, nx, 1, ny, 1, nz); W.Lcj = W.Lci; W.Lck = W.Lci; W.Lvi = W.Lci; W.Lvj = W.Lci; W.Lvk = W.Lci;
  limit_vt(C, B);
  comput_duvtpc(C, B, W);
  if (C.P.if_viscous == 1) {  // Residual, 134-178
    get_viscous(C, B, W);
    if (C.P.iflag_turbulence_model == 2) turbulence_SA(C, B, W);
    else if (C.P.iflag_turbulence_model == 3) turbulence_SST(C, B, W);
    else std::fill(B.mu_t.v.begin(), B.mu_t.v.end(), 0.0);
    limit_mut(C, B);
  }
  flux_inviscid(C, B, W, 0);
  flux_inviscid(C, B, W, 1);
  flux_inviscid(C, B, W, 2);
  if (C.P.if_viscous == 1) { flux_viscous(C, B, W, 0); flux_viscous(C, B, W, 1); flux_viscous(C, B, W, 2); }
  if (C.P.time_method == -1) {  // physical-time derivative of the dual-time scheme (sub_Residual.f90:94-104)
    for (int k = 1; k <= nz - 1; k++)
      for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++)
          for (int m = 1; m <= C.NVAR; m++)
            B.Res(m, i, j, k) = B.Res(m, i, j, k) - (3.0 * B.U(m, i, j, k) - 4.0 * B.Un(m, i, j, k) + B.Un1(m, i, j, k)) * B.vol(i, j, k) * Sfac;
  }
  comput_Lijk(C, B, W);
  if (C.P.if_residual_smoothing == 1) residual_smoothing(C, B, W);  // sub_Residual.f90:111-113
  comput_dt(C, B, W);
  if (lusgs) du_LU_SGS(C, B, W, Sfac1);
  return 0;
}

// ============================================================================================
// limiter, time advance, norms, forces
// ============================================================================================
static void limit_flow_U(Case& C, Block& B) {  // sub_limitflow.f90:24-176
  const ocfd_params& P = C.P;
  double gamma = P.gamma;
  int nx = B.nx, ny = B.ny, nz = B.nz;
  A3 d1, u1, v1, w1, p1;
  d1.alloc(1, nx - 1, 1, ny - 1, 1, nz - 1); u1 = d1; v1 = d1; w1 = d1; p1 = d1;
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        d1(i, j, k) = B.U(1, i, j, k);
        u1(i, j, k) = B.U(2, i, j, k) / d1(i, j, k); v1(i, j, k) = B.U(3, i, j, k) / d1(i, j, k); w1(i, j, k) = B.U(4, i, j, k) / d1(i, j, k);
        p1(i, j, k) = (B.U(5, i, j, k) - 0.5 * d1(i, j, k) * (u1(i, j, k) * u1(i, j, k) + v1(i, j, k) * v1(i, j, k) + w1(i, j, k) * w1(i, j, k))) * (gamma - 1.0);
      }
  auto bad = [&](int i, int j, int k) {
    return d1(i, j, k) < P.ldmin || p1(i, j, k) < P.lpmin || d1(i, j, k) > P.ldmax || p1(i, j, k) > P.lpmax || std::fabs(u1(i, j, k)) > P.lumax ||
           std::fabs(v1(i, j, k)) > P.lumax || std::fabs(w1(i, j, k)) > P.lumax;
  };
  int Nneg = 0;
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        if (!bad(i, j, k)) continue;
        Nneg++;
        double d0 = 0, u0 = 0, v0 = 0, w0 = 0, p0 = 0;
        int kn = 0;
        for (int ka = -1; ka <= 1; ka++)
          for (int ja = -1; ja <= 1; ja++)
            for (int ia = -1; ia <= 1; ia++) {
              int k1 = k + ka, j1 = j + ja, i1 = i + ia;
              if (i1 > 0 && i1 < nx && j1 > 0 && j1 < ny && k1 > 0 && k1 < nz) {
                if (!bad(i1, j1, k1)) { d0 += d1(i1, j1, k1); u0 += u1(i1, j1, k1); v0 += v1(i1, j1, k1); w0 += w1(i1, j1, k1); p0 += p1(i1, j1, k1); kn++; }
              }
            }
        if (kn == 0) {
          d0 = d1(i, j, k); u0 = u1(i, j, k); v0 = v1(i, j, k); w0 = w1(i, j, k); p0 = p1(i, j, k);
          if (d0 < P.ldmin) d0 = P.ldmin;
          if (d0 > P.ldmax) d0 = P.ldmax;
          if (p0 < P.lpmin) p0 = P.lpmin;
          if (p0 > P.lpmax) p0 = P.lpmax;
          if (std::fabs(u0) > P.lumax) u0 = std::copysign(P.lumax, u0);
          if (std::fabs(v0) > P.lumax) v0 = std::copysign(P.lumax, v0);
          if (std::fabs(w0) > P.lumax) w0 = std::copysign(P.lumax, w0);
        } else {
          double sn1 = 1.0 / (kn);
          d0 = d0 * sn1; u0 = u0 * sn1; v0 = v0 * sn1; w0 = w0 * sn1; p0 = p0 * sn1;
        }
        B.U(1, i, j, k) = d0; B.U(2, i, j, k) = d0 * u0; B.U(3, i, j, k) = d0 * v0; B.U(4, i, j, k) = d0 * w0;
        B.U(5, i, j, k) = p0 / (gamma - 1.0) + 0.5 * d0 * (u0 * u0 + v0 * v0 + w0 * w0);
      }
  B.nlimited = Nneg;
  if (Nneg > 0) B.overlimit = 1;
}

static void limit_flow_SA(Case& C, Block& B) {  // sub_limitflow.f90:182-231 (serial loop order)
  const double SAmin = 1.e-8;
  double LSAmax = C.P.lsamax;
  int nx = B.nx, ny = B.ny, nz = B.nz;
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        if (B.U(6, i, j, k) < SAmin) B.U(6, i, j, k) = SAmin;
        if (B.U(6, i, j, k) > LSAmax) {
          double s0 = 0.0;
          int kn = 0;
          for (int ka = -1; ka <= 1; ka++)
            for (int ja = -1; ja <= 1; ja++)
              for (int ia = -1; ia <= 1; ia++) {
                int k1 = k + ka, j1 = j + ja, i1 = i + ia;
                if (i1 > 0 && i1 < nx && j1 > 0 && j1 < ny && k1 > 0 && k1 < nz)
                  if (B.U(6, i1, j1, k1) >= SAmin && B.U(6, i1, j1, k1) <= LSAmax) { s0 = s0 + B.U(6, i1, j1, k1); kn++; }
              }
          if (kn == 0) B.U(6, i, j, k) = LSAmax; else B.U(6, i, j, k) = s0 / kn;
        }
      }
}

static void limit_flow(Case& C) {
  for (Block& B : C.B) limit_flow_U(C, B);
  if (C.NVAR == 6) for (Block& B : C.B) limit_flow_SA(C, B);
}

static void force_vt_kw(Case& C) {  // sub_time_advance.f90:27-61
  for (Block& B : C.B)
    for (int k = 1; k <= B.nz - 1; k++)
      for (int j = 1; j <= B.ny - 1; j++)
        for (int i = 1; i <= B.nx - 1; i++) {
          if (C.NVAR >= 6 && B.U(6, i, j, k) < 0) B.U(6, i, j, k) = 1.e-10;
          if (C.NVAR == 7 && B.U(7, i, j, k) < 0) B.U(7, i, j, k) = 1.e-10;
        }
}

static void set_Un(Case& C) {  // Set_Un, sub_time_advance.f90:635-656
  for (Block& B : C.B)
    for (int k = -1; k <= B.nz + 1; k++)
      for (int j = -1; j <= B.ny + 1; j++)
        for (int i = -1; i <= B.nx + 1; i++)
          for (int m = 1; m <= C.NVAR; m++) B.Un(m, i, j, k) = B.U(m, i, j, k);
}

static int advance_lusgs(Case& C) {  // sub_time_advance.f90:75-118
  int NV = C.NVAR;
  set_Un(C);  // before limit_vt clamps U6/U7 in place: the update below uses the unclamped copy
  for (Block& B : C.B) residual_block(C, B, true);
  for (Block& B : C.B)
    for (int k = 1; k <= B.nz - 1; k++)
      for (int j = 1; j <= B.ny - 1; j++)
        for (int i = 1; i <= B.nx - 1; i++)
          for (int m = 1; m <= NV; m++) B.U(m, i, j, k) = B.Un(m, i, j, k) + B.DU(m, i, j, k);
  if (C.P.iflag_limit_flow == 1) limit_flow(C);
  int rc = boundary_all(C);
  if (rc) return rc;
  halo(C);
  C.tt = C.tt + C.P.dt_global;
  C.Kstep = C.Kstep + 1;
  return 0;
}

static int advance_euler1(Case& C) {  // NS_Time_advance_1Euler, sub_time_advance.f90:217-260
  int NV = C.NVAR;
  set_Un(C);
  for (Block& B : C.B) residual_block(C, B, false);
  for (Block& B : C.B)
    for (int k = 1; k <= B.nz - 1; k++)
      for (int j = 1; j <= B.ny - 1; j++)
        for (int i = 1; i <= B.nx - 1; i++)
          for (int m = 1; m <= NV; m++) {
            double du = B.Res(m, i, j, k) / B.vol(i, j, k);
            B.U(m, i, j, k) = B.Un(m, i, j, k) + B.dt(i, j, k) * du;
          }
  if (C.P.iflag_limit_flow == 1) limit_flow(C);
  int rc = boundary_all(C);
  if (rc) return rc;
  halo(C);
  C.tt = C.tt + C.P.dt_global;
  C.Kstep = C.Kstep + 1;
  return 0;
}

static int advance_rk3(Case& C) {  // sub_time_advance.f90:265-326
  int NV = C.NVAR;
  set_Un(C);
  for (int KRK = 0; KRK < 3; KRK++) {
    for (Block& B : C.B) residual_block(C, B, false);
    for (Block& B : C.B)
      for (int k = 1; k <= B.nz - 1; k++)
        for (int j = 1; j <= B.ny - 1; j++)
          for (int i = 1; i <= B.nx - 1; i++)
            for (int m = 1; m <= NV; m++) {
              double du = B.Res(m, i, j, k) / B.vol(i, j, k);
              B.U(m, i, j, k) = C.Ralfa[KRK] * B.Un(m, i, j, k) + C.Rgamma[KRK] * B.U(m, i, j, k) + B.dt(i, j, k) * C.Rbeta[KRK] * du;
            }
    if (C.P.iflag_limit_flow == 1) limit_flow(C);
    int rc = boundary_all(C);
    if (rc) return rc;
    halo(C);
  }
  C.tt = C.tt + C.P.dt_global;
  C.Kstep = C.Kstep + 1;
  return 0;
}

static int norms(Case& C, double* rmax, double* rrms);

// Sfac, Sfac1 of one Comput_Residual_one_mesh call: the first call of the run uses the
// first-order values, every later call the second-order ones (sub_Residual.f90:25-33)
static void dual_factors(Case& C, double& Sfac, double& Sfac1) {
  const double dt = C.P.dt_global;
  if (C.dual_started == 0) { C.dual_started = 1; Sfac = 1.0 / (3.0 * dt); Sfac1 = 1.0 / dt; }
  else { Sfac = 1.0 / (2.0 * dt); Sfac1 = 3.0 / (2.0 * dt); }
}

static void dual_init(Case& C) {  // Init_flow, sub_init.f90:278-296
  for (Block& B : C.B)
    for (int k = -1; k <= B.nz + 1; k++)
      for (int j = -1; j <= B.ny + 1; j++)
        for (int i = -1; i <= B.nx + 1; i++)
          for (int m = 1; m <= C.NVAR; m++) { B.Un(m, i, j, k) = B.U(m, i, j, k); B.Un1(m, i, j, k) = B.U(m, i, j, k); }
}

static int advance_dual(Case& C) {  // NS_Time_Dual_LU_SGS, sub_time_advance.f90:126-202
  int NV = C.NVAR;
  for (int kt = 1; kt <= C.P.step_inner_limit; kt++) {
    double Sfac, Sfac1;
    dual_factors(C, Sfac, Sfac1);
    for (Block& B : C.B) residual_block(C, B, true, Sfac, Sfac1);
    for (Block& B : C.B)
      for (int k = 1; k <= B.nz - 1; k++)
        for (int j = 1; j <= B.ny - 1; j++)
          for (int i = 1; i <= B.nx - 1; i++)
            for (int m = 1; m <= NV; m++) B.U(m, i, j, k) = B.U(m, i, j, k) + B.DU(m, i, j, k);
    if (C.P.iflag_limit_flow == 1) limit_flow(C);
    int rc = boundary_all(C);
    if (rc) return rc;
    halo(C);
    double rmax[7], rrms[7];
    rc = norms(C, rmax, rrms);
    if (rc) return rc;
    double max_res = rrms[0];
    for (int m = 0; m < NV; m++) max_res = std::max(max_res, rrms[m]);
    if (max_res <= C.P.res_inner_limit) break;
  }
  for (Block& B : C.B)
    for (int k = 1; k <= B.nz - 1; k++)
      for (int j = 1; j <= B.ny - 1; j++)
        for (int i = 1; i <= B.nx - 1; i++)
          for (int m = 1; m <= NV; m++) { B.Un1(m, i, j, k) = B.Un(m, i, j, k); B.Un(m, i, j, k) = B.U(m, i, j, k); }
  C.tt = C.tt + C.P.dt_global;
  C.Kstep = C.Kstep + 1;
  return 0;
}

static int advance(Case& C) {  // NS_Time_advance, sub_time_advance.f90:6-23
  int rc;
  if (C.P.time_method == 0) rc = advance_lusgs(C);
  else if (C.P.time_method == 1) rc = advance_euler1(C);
  else if (C.P.time_method == 3) rc = advance_rk3(C);
  else if (C.P.time_method == -1) rc = advance_dual(C);
  else { C.err = "time method not supported"; return OCFD_ERR_UNSUPPORTED; }
  if (rc) return rc;
  force_vt_kw(C);
  return 0;
}

static void init_flow(Case& C) {  // init_flow_zero (external flow, freestream), sub_init.f90:302-410
  double gamma = C.P.gamma, Ma = C.P.ma;
  double d0 = 1.0, p0 = 1.0 / (gamma * Ma * Ma);
  double u0 = std::cos(C.P.a_alfa) * std::cos(C.P.a_beta), v0 = std::sin(C.P.a_alfa) * std::cos(C.P.a_beta), w0 = std::sin(C.P.a_beta);
  for (Block& B : C.B)
    for (int k = 1 - LAP; k <= B.nz + LAP - 1; k++)
      for (int j = 1 - LAP; j <= B.ny + LAP - 1; j++)
        for (int i = 1 - LAP; i <= B.nx + LAP - 1; i++) {
          B.U(1, i, j, k) = d0; B.U(2, i, j, k) = d0 * u0; B.U(3, i, j, k) = d0 * v0; B.U(4, i, j, k) = d0 * w0;
          B.U(5, i, j, k) = p0 / (gamma - 1.0) + 0.5 * d0 * (u0 * u0 + v0 * v0 + w0 * w0);
          if (C.NVAR == 6) B.U(6, i, j, k) = 5.0;
          else if (C.NVAR == 7) { B.U(6, i, j, k) = 10.0 * C.P.kt_inf; B.U(7, i, j, k) = C.P.wt_inf; }
        }
  boundary_all(C);
  halo(C);
}

static int norms(Case& C, double* rmax, double* rrms) {  // comput_max_Res_onemesh, sub_time_advance.f90:330-380
  for (int m = 0; m < 7; m++) { rmax[m] = 0.0; rrms[m] = 0.0; }
  for (Block& B : C.B)
    for (int k = 1; k <= B.nz - 1; k++)
      for (int j = 1; j <= B.ny - 1; j++)
        for (int i = 1; i <= B.nx - 1; i++)
          for (int m = 1; m <= C.NVAR; m++) {
            double Res = B.Res(m, i, j, k);
            if (std::isnan(Res)) {
              char buf[160];
              snprintf(buf, sizeof buf, "NaN in residual: block %d i,j,k,m = %d %d %d %d", B.no, i, j, k, m);
              C.err = buf;
              return OCFD_ERR_NAN;
            }
            rmax[m - 1] = std::max(rmax[m - 1], std::fabs(Res));
            rrms[m - 1] = rrms[m - 1] + Res * Res;
          }
  for (int m = 0; m < C.NVAR; m++) rrms[m] = std::sqrt(rrms[m] / (double)C.Num_Cell);
  return 0;
}

static void forces(Case& C, double* Ft0, double* cl, double* cd, double* cs) {  // comput_force, sub_Post.f90:4-265
  double gamma = C.P.gamma, p_inf = 1.0 / (gamma * C.P.ma * C.P.ma);
  const double* cen = C.P.centroid;
  double Ft[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (Block& B : C.B) {
    double Px = 0, Py = 0, Pz = 0, Cfx = 0, Cfy = 0, Cfz = 0, Mx = 0, My = 0, Mz = 0;
    int nx = B.nx, ny = B.ny, nz = B.nz;
    auto pres = [&](int i, int j, int k) {
      return (gamma - 1.0) * (B.U(5, i, j, k) - (p2(B.U(2, i, j, k)) + p2(B.U(3, i, j, k)) + p2(B.U(4, i, j, k))) / B.U(1, i, j, k));
    };
    auto acc = [&](double Pw, double n1, double n2, double n3, double sf1, double sf2, double sf3, double sgn, double xc, double yc, double zc) {
      Px = Px + Pw * n1; Py = Py + Pw * n2; Pz = Pz + Pw * n3;
      if (sgn > 0) { Cfx = Cfx + sf1; Cfy = Cfy + sf2; Cfz = Cfz + sf3; }
      else { Cfx = Cfx - sf1; Cfy = Cfy - sf2; Cfz = Cfz - sf3; }
      double fx0 = sgn > 0 ? Pw * n1 + sf1 : Pw * n1 - sf1;
      double fy0 = sgn > 0 ? Pw * n2 + sf2 : Pw * n2 - sf2;
      double fz0 = sgn > 0 ? Pw * n3 + sf3 : Pw * n3 - sf3;
      Mx = Mx + (yc * fz0 - zc * fy0);
      My = My + (zc * fx0 - xc * fz0);
      Mz = Mz + (xc * fy0 - yc * fx0);
    };
    for (const Sub& Bc : B.sub) {
      if (Bc.bc != BC_Wall) continue;
      if (Bc.face == 1) {
        for (int k = Bc.kb; k <= Bc.ke - 1; k++)
          for (int j = Bc.jb; j <= Bc.je - 1; j++) {
            double pw1 = pres(1, j, k), pw2 = pres(0, j, k);
            double Pw = -(0.5 * (pw1 + pw2) - p_inf) * B.Si(1, j, k);
            acc(Pw, B.ni1(1, j, k), B.ni2(1, j, k), B.ni3(1, j, k), B.surf1(j, k, 1), B.surf1(j, k, 2), B.surf1(j, k, 3), 1.0,
                (B.xc(1, j, k) + B.xc(0, j, k)) * 0.5 - cen[0], (B.yc(1, j, k) + B.yc(0, j, k)) * 0.5 - cen[1], (B.zc(1, j, k) + B.zc(0, j, k)) * 0.5 - cen[2]);
          }
      } else if (Bc.face == 2) {
        for (int k = Bc.kb; k <= Bc.ke - 1; k++)
          for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
            double pw1 = pres(i, 1, k), pw2 = pres(i, 0, k);
            double Pw = -(0.5 * (pw1 + pw2) - p_inf) * B.Sj(i, 1, k);
            acc(Pw, B.nj1(i, 1, k), B.nj2(i, 1, k), B.nj3(i, 1, k), B.surf2(i, k, 1), B.surf2(i, k, 2), B.surf2(i, k, 3), 1.0,
                (B.xc(i, 1, k) + B.xc(i, 0, k)) * 0.5 - cen[0], (B.yc(i, 1, k) + B.yc(i, 0, k)) * 0.5 - cen[1], (B.zc(i, 1, k) + B.zc(i, 0, k)) * 0.5 - cen[2]);
          }
      } else if (Bc.face == 3) {
        for (int j = Bc.jb; j <= Bc.je - 1; j++)
          for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
            double pw1 = pres(i, j, 1), pw2 = pres(i, j, 0);
            double Pw = -(0.5 * (pw1 + pw2) - p_inf) * B.Sk(i, j, 1);
            acc(Pw, B.nk1(i, j, 1), B.nk2(i, j, 1), B.nk3(i, j, 1), B.surf3(i, j, 1), B.surf3(i, j, 2), B.surf3(i, j, 3), 1.0,
                (B.xc(i, j, 1) + B.xc(i, j, 0)) * 0.5 - cen[0], (B.yc(i, j, 1) + B.yc(i, j, 0)) * 0.5 - cen[1], (B.zc(i, j, 1) + B.zc(i, j, 0)) * 0.5 - cen[2]);
          }
      } else if (Bc.face == 4) {
        for (int k = Bc.kb; k <= Bc.ke - 1; k++)
          for (int j = Bc.jb; j <= Bc.je - 1; j++) {
            double pw1 = pres(nx - 1, j, k), pw2 = pres(nx, j, k);
            double Pw = (0.5 * (pw1 + pw2) - p_inf) * B.Si(nx, j, k);
            acc(Pw, B.ni1(nx, j, k), B.ni2(nx, j, k), B.ni3(nx, j, k), B.surf4(j, k, 1), B.surf4(j, k, 2), B.surf4(j, k, 3), -1.0,
                (B.xc(nx - 1, j, k) + B.xc(nx, j, k)) * 0.5 - cen[0], (B.yc(nx - 1, j, k) + B.yc(nx, j, k)) * 0.5 - cen[1], (B.zc(nx - 1, j, k) + B.zc(nx, j, k)) * 0.5 - cen[2]);
          }
      } else if (Bc.face == 5) {
        for (int k = Bc.kb; k <= Bc.ke - 1; k++)
          for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
            double pw1 = pres(i, ny - 1, k), pw2 = pres(i, ny, k);
            double Pw = (0.5 * (pw1 + pw2) - p_inf) * B.Sj(i, ny, k);
            acc(Pw, B.nj1(i, ny, k), B.nj2(i, ny, k), B.nj3(i, ny, k), B.surf5(i, k, 1), B.surf5(i, k, 2), B.surf5(i, k, 3), -1.0,
                (B.xc(i, ny - 1, k) + B.xc(i, ny, k)) * 0.5 - cen[0], (B.yc(i, ny - 1, k) + B.yc(i, ny, k)) * 0.5 - cen[1], (B.zc(i, ny - 1, k) + B.zc(i, ny, k)) * 0.5 - cen[2]);
          }
      } else if (Bc.face == 6) {
        for (int j = Bc.jb; j <= Bc.je - 1; j++)
          for (int i = Bc.ib; i <= Bc.ie - 1; i++) {
            double pw1 = pres(i, j, nz - 1), pw2 = pres(i, j, nz);
            double Pw = (0.5 * (pw1 + pw2) - p_inf) * B.Sk(i, j, nz);
            acc(Pw, B.nk1(i, j, nz), B.nk2(i, j, nz), B.nk3(i, j, nz), B.surf6(i, j, 1), B.surf6(i, j, 2), B.surf6(i, j, 3), -1.0,
                (B.xc(i, j, nz - 1) + B.xc(i, j, nz)) * 0.5 - cen[0], (B.yc(i, j, nz - 1) + B.yc(i, j, nz)) * 0.5 - cen[1], (B.zc(i, j, nz - 1) + B.zc(i, j, nz)) * 0.5 - cen[2]);
          }
      }
    }
    Ft[0] = Ft[0] + Px; Ft[1] = Ft[1] + Py; Ft[2] = Ft[2] + Pz;
    Ft[3] = Ft[3] + Cfx; Ft[4] = Ft[4] + Cfy; Ft[5] = Ft[5] + Cfz;
    Ft[6] = Ft[6] + Mx; Ft[7] = Ft[7] + My; Ft[8] = Ft[8] + Mz;
  }
  for (int q = 0; q < 6; q++) Ft0[q] = 2.0 * Ft[q] / C.P.ref_s;
  for (int q = 6; q < 9; q++) Ft0[q] = 2.0 * Ft[q] / (C.P.ref_s * C.P.ref_l);
  double Fx = Ft0[0] + Ft0[3], Fy = Ft0[1] + Ft0[4], Fz = Ft0[2] + Ft0[5];
  double AoA = C.P.aoa;
  if (C.P.cood_y_up == 1) { *cl = Fy * std::cos(AoA) - Fx * std::sin(AoA); *cd = Fx * std::cos(AoA) + Fy * std::sin(AoA); *cs = Fz; }
  else { *cl = Fz * std::cos(AoA) - Fx * std::sin(AoA); *cd = Fx * std::cos(AoA) + Fz * std::sin(AoA); *cs = Fy; }
}

static int nvar_of(const ocfd_params& p) {
  int tm = p.if_viscous == 0 ? 0 : p.iflag_turbulence_model;
  return tm == 2 || tm == 21 ? 6 : (tm == 3 ? 7 : 5);
}

}  // namespace orc

// ============================================================================================
// C entry points (oracle_*), mirroring include/ocfd_ec_gpu.h
// ============================================================================================
using namespace orc;

extern "C" {

// host threads of the oracle's loop pool (OCFD_ORACLE_THREADS or all hardware threads at load);
// returns the count in use
int oracle_set_threads(int n) {
  orc::Pool::get().set_threads(n);
  return orc::Pool::get().size();
}
int oracle_threads() { return orc::Pool::get().size(); }

int oracle_create(const ocfd_params* p, int nblk, const int* nijk, const double* const* xyz, const int* nsub, const int* inc,
                  const double* const* dw, void** out) {
  if (!p || nblk <= 0 || !nijk || !xyz || !nsub || !inc || !out) return OCFD_ERR_ARG;
  Case* C = new Case();
  C->P = *p;
  C->NVAR = nvar_of(*p);
  C->Ralfa[0] = 1.0; C->Ralfa[1] = 3.0 / 4.0; C->Ralfa[2] = 1.0 / 3.0;
  C->Rbeta[0] = 1.0; C->Rbeta[1] = 1.0 / 4.0; C->Rbeta[2] = 2.0 / 3.0;
  C->Rgamma[0] = 0.0; C->Rgamma[1] = 1.0 / 4.0; C->Rgamma[2] = 2.0 / 3.0;
  C->B.resize(nblk);
  const int* q = inc;
  int NV = C->NVAR;
  for (int b = 0; b < nblk; b++) {
    Block& B = C->B[b];
    int nx = nijk[3 * b], ny = nijk[3 * b + 1], nz = nijk[3 * b + 2];
    B.nx = nx; B.ny = ny; B.nz = nz; B.no = b + 1;
    for (int s = 0; s < nsub[b]; s++, q += 21) {
      Sub S;
      int* f = &S.ib;
      for (int t = 0; t < 21; t++) f[t] = q[t];
      B.sub.push_back(S);
    }
    C->Num_Cell += (long long)(nx - 1) * (ny - 1) * (nz - 1);
    A3* nodes[3] = {&B.x, &B.y, &B.z};
    for (int c = 0; c < 3; c++) {
      nodes[c]->alloc(0, nx + 1, 0, ny + 1, 0, nz + 1);
      const double* src = xyz[b] + (size_t)c * nx * ny * nz;
      for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) (*nodes[c])(i, j, k) = src[(i - 1) + (size_t)nx * ((j - 1) + (size_t)ny * (k - 1))];
    }
    B.xc.alloc(1 - LAP, nx + LAP - 1, 1 - LAP, ny + LAP - 1, 1 - LAP, nz + LAP - 1); B.yc = B.xc; B.zc = B.xc;
    B.vol.alloc(1, nx - 1, 1, ny - 1, 1, nz - 1);
    A3* fm[] = {&B.Si, &B.Sj, &B.Sk, &B.ni1, &B.ni2, &B.ni3, &B.nj1, &B.nj2, &B.nj3, &B.nk1, &B.nk2, &B.nk3,
                &B.ix1, &B.iy1, &B.iz1, &B.jx1, &B.jy1, &B.jz1, &B.kx1, &B.ky1, &B.kz1, &B.ix2, &B.iy2, &B.iz2, &B.jx2, &B.jy2, &B.jz2, &B.kx2, &B.ky2, &B.kz2,
                &B.ix3, &B.iy3, &B.iz3, &B.jx3, &B.jy3, &B.jz3, &B.kx3, &B.ky3, &B.kz3, &B.ix0, &B.iy0, &B.iz0, &B.jx0, &B.jy0, &B.jz0, &B.kx0, &B.ky0, &B.kz0};
    for (A3* a : fm) a->alloc(1, nx, 1, ny, 1, nz);
    B.U.alloc(NV, 1 - LAP, nx + LAP - 1, 1 - LAP, ny + LAP - 1, 1 - LAP, nz + LAP - 1, 0.0);
    for (int k = 1 - LAP; k <= nz + LAP - 1; k++)  // allocate-time fill (sub_init.f90:518-525)
      for (int j = 1 - LAP; j <= ny + LAP - 1; j++)
        for (int i = 1 - LAP; i <= nx + LAP - 1; i++) {
          B.U(1, i, j, k) = 1.0; B.U(5, i, j, k) = 1.0;
          if (NV == 6) B.U(6, i, j, k) = 1.0;
          else if (NV == 7) { B.U(6, i, j, k) = 0.0; B.U(7, i, j, k) = 1.0; }
        }
    B.Un.alloc(NV, -1, nx + 1, -1, ny + 1, -1, nz + 1);
    if (p->time_method == -1) B.Un1.alloc(NV, -1, nx + 1, -1, ny + 1, -1, nz + 1);
    B.Res.alloc(NV, -1, nx + 1, -1, ny + 1, -1, nz + 1);
    B.DU.alloc(NV, -1, nx + 1, -1, ny + 1, -1, nz + 1);
    B.dt.alloc(-1, nx + 1, -1, ny + 1, -1, nz + 1);
    B.dw.alloc(1, nx - 1, 1, ny - 1, 1, nz - 1);
    B.dtime_mesh.alloc(1, nx - 1, 1, ny - 1, 1, nz - 1, 1.0);
    B.mu.alloc(-1, nx + 1, -1, ny + 1, -1, nz + 1, 1.0 / p->re);
    B.mu_t.alloc(-1, nx + 1, -1, ny + 1, -1, nz + 1, 0.0);
    B.surf1.alloc(1, ny, 1, nz, 1, 3); B.surf4 = B.surf1;
    B.surf2.alloc(1, nx, 1, nz, 1, 3); B.surf5 = B.surf2;
    B.surf3.alloc(1, nx, 1, ny, 1, 3); B.surf6 = B.surf3;
    B.BcI.alloc(ny - 1, nz - 1, 2); B.BcJ.alloc(nx - 1, nz - 1, 2); B.BcK.alloc(nx - 1, ny - 1, 2);
  }
  coordinate_ghosts(*C);
  for (Block& B : C->B) { geometry(B); set_BcK(B); }
  if (C->NVAR > 5) {
    if (dw && dw[0]) {
      for (int b = 0; b < nblk; b++) {
        Block& B = C->B[b];
        for (int k = 1; k <= B.nz - 1; k++) for (int j = 1; j <= B.ny - 1; j++) for (int i = 1; i <= B.nx - 1; i++)
          B.dw(i, j, k) = dw[b][(i - 1) + (size_t)(B.nx - 1) * ((j - 1) + (size_t)(B.ny - 1) * (k - 1))];
      }
    } else wall_distance(*C);
  }
  for (Block& B : C->B) mesh_quality(B);
  init_flow(*C);
  if (C->P.time_method == -1) dual_init(*C);
  *out = C;
  return 0;
}

int oracle_destroy(void* h) { delete (Case*)h; return 0; }
const char* oracle_last_error(void* h) { return h ? ((Case*)h)->err.c_str() : "null handle"; }

int oracle_advance(void* h, int nsteps, int* kstep, double* tt) {
  Case* C = (Case*)h;
  for (int s = 0; s < nsteps; s++) { int rc = advance(*C); if (rc) return rc; }
  if (kstep) *kstep = C->Kstep;
  if (tt) *tt = C->tt;
  return 0;
}

// Comput_Residual_one_mesh only (sub_Residual.f90:14-127): Res, dt (and DU if lusgs) from the
// current state, no update.
int oracle_compute_residual(void* h, int lusgs) {
  Case* C = (Case*)h;
  double Sfac = 0.0, Sfac1 = 0.0;
  if (C->P.time_method == -1) dual_factors(*C, Sfac, Sfac1);
  for (Block& B : C->B) residual_block(*C, B, lusgs != 0, Sfac, Sfac1);
  return 0;
}

int oracle_init_flow(void* h) {
  Case* C = (Case*)h;
  C->Kstep = 0; C->tt = 0.0;
  init_flow(*C);
  if (C->P.time_method == -1) dual_init(*C);
  return 0;
}

int oracle_residual(void* h, double* rmax, double* rrms) { return norms(*(Case*)h, rmax, rrms); }

int oracle_forces(void* h, double* ft, double* cl, double* cd, double* cs) { forces(*(Case*)h, ft, cl, cd, cs); return 0; }

long long oracle_state_size(void* h, int b) {
  Case* C = (Case*)h;
  Block& B = C->B[b];
  return (long long)C->NVAR * (B.nx + 7) * (B.ny + 7) * (B.nz + 7);
}
int oracle_get_state(void* h, int b, double* U) { Block& B = ((Case*)h)->B[b]; std::memcpy(U, B.U.v.data(), B.U.v.size() * 8); return 0; }
int oracle_set_state(void* h, int b, const double* U) {
  Case* C = (Case*)h;
  Block& B = C->B[b];
  std::memcpy(B.U.v.data(), U, B.U.v.size() * 8);
  if (C->P.time_method == -1)  // a restart sets both earlier time levels too (Init_flow, sub_init.f90:278-296)
    for (int k = -1; k <= B.nz + 1; k++)
      for (int j = -1; j <= B.ny + 1; j++)
        for (int i = -1; i <= B.nx + 1; i++)
          for (int m = 1; m <= C->NVAR; m++) { B.Un(m, i, j, k) = B.U(m, i, j, k); B.Un1(m, i, j, k) = B.U(m, i, j, k); }
  return 0;
}

int oracle_limiter_status(void* h, int b, int* n, int* ov) { Block& B = ((Case*)h)->B[b]; *n = B.nlimited; *ov = B.overlimit; return 0; }

static A3* named3(Block& B, const std::string& s) {
  struct E { const char* n; A3 Block::*p; };
  static const E tab[] = {{"vol", &Block::vol}, {"dt", &Block::dt}, {"dw", &Block::dw}, {"mu", &Block::mu}, {"mu_t", &Block::mu_t}, {"dtime_mesh", &Block::dtime_mesh},
                          {"Si", &Block::Si}, {"Sj", &Block::Sj}, {"Sk", &Block::Sk}, {"ni1", &Block::ni1}, {"ni2", &Block::ni2}, {"ni3", &Block::ni3},
                          {"nj1", &Block::nj1}, {"nj2", &Block::nj2}, {"nj3", &Block::nj3}, {"nk1", &Block::nk1}, {"nk2", &Block::nk2}, {"nk3", &Block::nk3},
                          {"ix1", &Block::ix1}, {"iy1", &Block::iy1}, {"iz1", &Block::iz1}, {"jx1", &Block::jx1}, {"jy1", &Block::jy1}, {"jz1", &Block::jz1},
                          {"kx1", &Block::kx1}, {"ky1", &Block::ky1}, {"kz1", &Block::kz1}, {"ix2", &Block::ix2}, {"iy2", &Block::iy2}, {"iz2", &Block::iz2},
                          {"jx2", &Block::jx2}, {"jy2", &Block::jy2}, {"jz2", &Block::jz2}, {"kx2", &Block::kx2}, {"ky2", &Block::ky2}, {"kz2", &Block::kz2},
                          {"ix3", &Block::ix3}, {"iy3", &Block::iy3}, {"iz3", &Block::iz3}, {"jx3", &Block::jx3}, {"jy3", &Block::jy3}, {"jz3", &Block::jz3},
                          {"kx3", &Block::kx3}, {"ky3", &Block::ky3}, {"kz3", &Block::kz3}, {"ix0", &Block::ix0}, {"iy0", &Block::iy0}, {"iz0", &Block::iz0},
                          {"jx0", &Block::jx0}, {"jy0", &Block::jy0}, {"jz0", &Block::jz0}, {"kx0", &Block::kx0}, {"ky0", &Block::ky0}, {"kz0", &Block::kz0},
                          {"xc", &Block::xc}, {"yc", &Block::yc}, {"zc", &Block::zc}, {"x", &Block::x}, {"y", &Block::y}, {"z", &Block::z},
                          {"surf1", &Block::surf1}, {"surf2", &Block::surf2}, {"surf3", &Block::surf3}, {"surf4", &Block::surf4}, {"surf5", &Block::surf5}, {"surf6", &Block::surf6}};
  for (const E& e : tab) if (s == e.n) return &(B.*(e.p));
  return nullptr;
}

// shape in Fortran bounds: lo[3], hi[3], nv (1 for 3-D arrays)
int oracle_array_shape(void* h, int b, const char* name, int* lo, int* hi, int* nv) {
  Block& B = ((Case*)h)->B[b];
  std::string s(name);
  if (s == "Res" || s == "DU" || s == "U") {
    A4& a = s == "Res" ? B.Res : (s == "DU" ? B.DU : B.U);
    lo[0] = a.l0; lo[1] = a.l1; lo[2] = a.l2; hi[0] = a.l0 + a.n0 - 1; hi[1] = a.l1 + a.n1 - 1; hi[2] = a.l2 + a.n2 - 1; *nv = a.nv;
    return 0;
  }
  A3* a = named3(B, s);
  if (!a) return OCFD_ERR_ARG;
  lo[0] = a->l0; lo[1] = a->l1; lo[2] = a->l2; hi[0] = a->l0 + a->n0 - 1; hi[1] = a->l1 + a->n1 - 1; hi[2] = a->l2 + a->n2 - 1; *nv = 1;
  return 0;
}
int oracle_get_array(void* h, int b, const char* name, double* out) {
  Block& B = ((Case*)h)->B[b];
  std::string s(name);
  if (s == "Res" || s == "DU" || s == "U") {
    A4& a = s == "Res" ? B.Res : (s == "DU" ? B.DU : B.U);
    std::memcpy(out, a.v.data(), a.v.size() * 8);
    return 0;
  }
  A3* a = named3(B, s);
  if (!a) return OCFD_ERR_ARG;
  std::memcpy(out, a->v.data(), a->v.size() * 8);
  return 0;
}

// Single-face flux and single-stencil reconstruction, exposed for unit known-answer tests.
int oracle_flux_1d(const double* QL, const double* QR, double* F, double gamma, int iflux) { flux_1d(QL, QR, F, gamma, iflux); return 0; }
int oracle_scheme(const double* u8, int scheme, double* uL, double* uR) { *uL = scheme_fP(u8, scheme); *uR = scheme_fm(u8, scheme); return 0; }

}  // extern "C"
