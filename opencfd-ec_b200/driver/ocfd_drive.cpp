// ocfd_drive: a compiled caller of libocfd_b200.so that runs a case the way the reference's main
// program does (opencfd_ec3d_v1.16a.f90): parameters from set_default_parameter plus the
// namelist values given on the command line, then set_const_para (ocfd_default_params,
// ocfd_finalize_params); the mesh from Mesh3d.dat (read_main_mesh, sub_IO.f90:4-93, Fortran
// unformatted records); the connectivity from bc3d.inc (read_inc, sub_IO.f90:656-743, the text
// layout convert_inp_inc writes, sub_convert_inp.f90:103-114); then the time loop of lines
// 163-202: NS_Time_advance(1) each step (ocfd_advance), comput_force + output_Res every
// Kstep_show steps (ocfd_forces, ocfd_residual), output_flow every Kstep_save steps and at the end
// (ocfd_get_state, then flow3d.dat + Step_mess.dat in the reference's layout, sub_IO.f90:350-484).
//
// It uses only include/ocfd_ec_gpu.h: this is the call sequence a Fortran driver makes through
// the ISO_C_BINDING module.
//
//   ocfd_drive <case dir> steps=N [show=1] [save=0] [out=<dir>] [name=value ...]
//   ocfd_drive <case dir> --check          (read the files, print what was read; no device call)
//
// Each show step prints one line: "step K tt res_max[0..6] res_rms[0..6] ft[0..8] cl cd cs",
// numbers with 17 significant digits.  Exit status: 0, or the library's error code (negated).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ocfd_ec_gpu.h"

namespace {

// one record of a gfortran sequential unformatted file (4-byte length markers)
bool read_record(FILE* f, std::vector<char>& buf) {
  int32_t n = 0, m = 0;
  if (std::fread(&n, 4, 1, f) != 1 || n < 0) return false;
  buf.resize((size_t)n);
  if (n && std::fread(buf.data(), 1, (size_t)n, f) != (size_t)n) return false;
  if (std::fread(&m, 4, 1, f) != 1 || m != n) return false;
  return true;
}
bool write_record(FILE* f, const void* p, size_t n) {
  const int32_t m = (int32_t)n;
  return std::fwrite(&m, 4, 1, f) == 1 && (n == 0 || std::fwrite(p, 1, n, f) == n) && std::fwrite(&m, 4, 1, f) == 1;
}

struct Mesh {
  int nb = 0;
  std::vector<int> nijk;                 // nx, ny, nz per block
  std::vector<std::vector<double>> xyz;  // per block: x, y, z planes, i fastest
};

// read_main_mesh: Num_Block; (NI, NJ, NK) of every block; per block x, y, z
bool read_mesh3d(const std::string& path, Mesh& M) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::vector<char> r;
  bool ok = read_record(f, r) && r.size() == 4;
  if (ok) {
    std::memcpy(&M.nb, r.data(), 4);
    ok = M.nb > 0 && read_record(f, r) && r.size() == (size_t)12 * M.nb;
  }
  if (ok) {
    M.nijk.resize(3 * (size_t)M.nb);
    std::memcpy(M.nijk.data(), r.data(), r.size());
    for (int b = 0; ok && b < M.nb; b++) {
      const size_t np = (size_t)M.nijk[3 * b] * M.nijk[3 * b + 1] * M.nijk[3 * b + 2];
      ok = read_record(f, r) && r.size() == 3 * np * 8;
      if (ok) {
        M.xyz.emplace_back(3 * np);
        std::memcpy(M.xyz.back().data(), r.data(), r.size());
      }
    }
  }
  std::fclose(f);
  return ok;
}

// read_inc: a title line; NB; per block "nx ny nz", a label line, Nsub, then per subface the
// 9 + 12 integers of its two lines
bool read_inc(const std::string& path, const Mesh& M, std::vector<int>& nsub, std::vector<int>& inc) {
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  char line[4096];
  bool ok = std::fgets(line, sizeof line, f) != nullptr;
  int nb = 0;
  ok = ok && std::fscanf(f, "%d", &nb) == 1 && nb == M.nb;
  for (int b = 0; ok && b < nb; b++) {
    int nx, ny, nz, ns;
    ok = std::fscanf(f, "%d %d %d", &nx, &ny, &nz) == 3 && nx == M.nijk[3 * b] && ny == M.nijk[3 * b + 1] && nz == M.nijk[3 * b + 2];
    ok = ok && std::fgets(line, sizeof line, f) && std::fgets(line, sizeof line, f);  // rest of the line, label line
    ok = ok && std::fscanf(f, "%d", &ns) == 1 && ns >= 0;
    if (!ok) break;
    nsub.push_back(ns);
    for (int s = 0; ok && s < ns; s++)
      for (int q = 0; ok && q < 21; q++) {
        int v;
        ok = std::fscanf(f, "%d", &v) == 1;
        inc.push_back(v);
      }
  }
  std::fclose(f);
  return ok;
}

// namelist-style overrides: the raw values of set_default_parameter's variables, before set_const_para
bool set_param(ocfd_params& p, const std::string& key, const std::string& val) {
  struct I { const char* n; int* v; };
  struct D { const char* n; double* v; };
  const I ints[] = {{"nvar", &p.nvar}, {"iflag_scheme", &p.iflag_scheme}, {"bound_scheme", &p.bound_scheme}, {"iflag_flux", &p.iflag_flux},
                    {"iflag_reconstruction", &p.iflag_reconstruction}, {"iflag_turbulence_model", &p.iflag_turbulence_model},
                    {"time_method", &p.time_method}, {"if_viscous", &p.if_viscous}, {"iflag_local_dt", &p.iflag_local_dt},
                    {"if_dtime_mesh", &p.if_dtime_mesh}, {"iflag_limit_flow", &p.iflag_limit_flow},
                    {"if_scheme_positivity", &p.if_scheme_positivity}, {"cood_y_up", &p.cood_y_up}, {"precision", &p.precision},
                    {"step_inner_limit", &p.step_inner_limit}, {"if_residual_smoothing", &p.if_residual_smoothing}};
  const D dbls[] = {{"ma", &p.ma}, {"re", &p.re}, {"gamma", &p.gamma}, {"prl", &p.prl}, {"prt", &p.prt}, {"t_inf", &p.t_inf},
                    {"twall", &p.twall}, {"kt_inf", &p.kt_inf}, {"wt_inf", &p.wt_inf}, {"aoa", &p.aoa}, {"aos", &p.aos},
                    {"cfl", &p.cfl}, {"dt_global", &p.dt_global}, {"dtmin", &p.dtmin}, {"dtmax", &p.dtmax}, {"w_lu", &p.w_lu},
                    {"mut_max", &p.mut_max}, {"p_outlet", &p.p_outlet}, {"ldmin", &p.ldmin}, {"ldmax", &p.ldmax},
                    {"lpmin", &p.lpmin}, {"lpmax", &p.lpmax}, {"lumax", &p.lumax}, {"lsamax", &p.lsamax}, {"ref_s", &p.ref_s},
                    {"ref_l", &p.ref_l}, {"res_inner_limit", &p.res_inner_limit}};
  for (const I& e : ints)
    if (key == e.n) { *e.v = std::atoi(val.c_str()); return true; }
  for (const D& e : dbls)
    if (key == e.n) { *e.v = std::strtod(val.c_str(), nullptr); return true; }
  if (key == "centroid_x" || key == "centroid_y" || key == "centroid_z") {
    p.centroid[key.back() - 'x'] = std::strtod(val.c_str(), nullptr);
    return true;
  }
  return false;
}

// output_flow: per block one record of d, u, v, w, T on cells 0..n (sub_IO.f90:404-423), and the
// step counter file; the state comes from ocfd_get_state in the Fortran layout U(NV, -3:n+3, ...)
bool write_flow(const std::string& dir, ocfd_handle* h, const Mesh& M, const ocfd_params& p, int kstep, double tt) {
  FILE* f = std::fopen((dir + "/flow3d.dat").c_str(), "wb");
  if (!f) return false;
  const int NV = p.nvar;
  const double cv = 1.0 / (p.gamma * (p.gamma - 1.0) * p.ma * p.ma);
  bool ok = true;
  for (int b = 0; ok && b < M.nb; b++) {
    const int nx = M.nijk[3 * b], ny = M.nijk[3 * b + 1], nz = M.nijk[3 * b + 2];
    const long long NX = nx + 7, NY = ny + 7;
    std::vector<double> U((size_t)ocfd_state_size(h, b));
    ok = ocfd_get_state(h, b, U.data()) == OCFD_OK;
    const size_t nc = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    std::vector<double> out(5 * nc);
    size_t q = 0;
    for (int k = 0; ok && k <= nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++, q++) {
          const double* u = &U[(size_t)NV * ((i + 3) + NX * ((j + 3) + NY * (k + 3)))];
          const double d = u[0], uu = u[1] / d, v = u[2] / d, w = u[3] / d;
          out[q] = d; out[nc + q] = uu; out[2 * nc + q] = v; out[3 * nc + q] = w;
          out[4 * nc + q] = (u[4] - 0.5 * d * (uu * uu + v * v + w * w)) / (cv * d);
        }
    ok = ok && write_record(f, out.data(), out.size() * 8);
  }
  std::fclose(f);
  FILE* s = std::fopen((dir + "/Step_mess.dat").c_str(), "w");
  if (!s) return false;
  std::fprintf(s, " %d %.17g\n ---time Step, time ----\n", kstep, tt);
  std::fclose(s);
  return ok;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <case dir> steps=N [show=1] [save=0] [out=<dir>] [name=value ...] | --check\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  ocfd_params p;
  ocfd_default_params(&p);
  int steps = 0, show = 1, save = 0;
  bool check = false;
  std::string out = dir;
  for (int a = 2; a < argc; a++) {
    std::string s = argv[a];
    if (s == "--check") { check = true; continue; }
    const size_t e = s.find('=');
    if (e == std::string::npos) { std::fprintf(stderr, "bad argument %s\n", s.c_str()); return 2; }
    const std::string k = s.substr(0, e), v = s.substr(e + 1);
    if (k == "steps") steps = std::atoi(v.c_str());
    else if (k == "show") show = std::atoi(v.c_str());
    else if (k == "save") save = std::atoi(v.c_str());
    else if (k == "out") out = v;
    else if (!set_param(p, k, v)) { std::fprintf(stderr, "unknown parameter %s\n", k.c_str()); return 2; }
  }
  Mesh M;
  if (!read_mesh3d(dir + "/Mesh3d.dat", M)) { std::fprintf(stderr, "cannot read %s/Mesh3d.dat\n", dir.c_str()); return 3; }
  std::vector<int> nsub, inc;
  if (!read_inc(dir + "/bc3d.inc", M, nsub, inc)) { std::fprintf(stderr, "cannot read %s/bc3d.inc\n", dir.c_str()); return 3; }
  if (check) {
    std::printf("blocks %d\n", M.nb);
    for (int b = 0; b < M.nb; b++) std::printf("block %d %d %d %d nsub %d\n", b + 1, M.nijk[3 * b], M.nijk[3 * b + 1], M.nijk[3 * b + 2], nsub[b]);
    std::printf("inc");
    for (int v : inc) std::printf(" %d", v);
    std::printf("\n");
    double sx = 0.0;
    for (const auto& x : M.xyz)
      for (double v : x) sx += v;
    std::printf("xyz_sum %.17g\n", sx);
    return 0;
  }
  if (int rc = ocfd_finalize_params(&p)) return -rc;
  std::vector<const double*> xyz;
  for (const auto& x : M.xyz) xyz.push_back(x.data());
  ocfd_handle* h = nullptr;
  int rc = ocfd_create(&p, M.nb, M.nijk.data(), xyz.data(), nsub.data(), inc.data(), nullptr, &h);
  if (rc) { std::fprintf(stderr, "ocfd_create: %d\n", rc); return -rc; }
  int kstep = 0;
  double tt = 0.0;
  while (kstep < steps) {
    if ((rc = ocfd_advance(h, 1, &kstep, &tt))) break;
    if (show > 0 && kstep % show == 0) {
      double rmax[7], rrms[7], ft[9], cl = 0, cd = 0, cs = 0;
      if ((rc = ocfd_forces(h, ft, &cl, &cd, &cs))) break;
      if ((rc = ocfd_residual(h, rmax, rrms))) break;
      std::printf("step %d %.17g", kstep, tt);
      for (double v : rmax) std::printf(" %.17g", v);
      for (double v : rrms) std::printf(" %.17g", v);
      for (double v : ft) std::printf(" %.17g", v);
      std::printf(" %.17g %.17g %.17g\n", cl, cd, cs);
    }
    if (save > 0 && kstep % save == 0 && !write_flow(out, h, M, p, kstep, tt)) { rc = OCFD_ERR_ARG; break; }
  }
  if (!rc && !write_flow(out, h, M, p, kstep, tt)) rc = OCFD_ERR_ARG;
  if (rc) std::fprintf(stderr, "stopped at step %d: %s (%d)\n", kstep, ocfd_last_error(h), rc);
  ocfd_destroy(h);
  return rc ? -rc : 0;
}
