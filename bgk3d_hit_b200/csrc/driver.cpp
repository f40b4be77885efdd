// bgk3d_hit: the reference program's main loop (SRC/bgk3d_HIT.F90:74-146)
// as a C++ executable over the library's C-ABI.
//
//   bgk3d_hit [bgk.input] [--precision fp64|fp32|fp16] [--scheme two_lattice|aa]
//             [--init tgv|tgv_faithful] [--out DIR] [--device N]
//
// Reads the namelist &parameters (SRC/input.F90:41-47: lx, ly, lz, u0, svisc,
// itfin, itsave, ivtim, icheck, cteS; proc_x = proc_y = proc_z = 1), runs
// boundaries -> col_MC -> diagnostic for itime = 1..itfin with the icheck gate
// (SRC/diagnostic.F90:37), and writes:
//   diagno.dat       (fort.70, format(i8,5(e14.6,1x)), SRC/diagno.F90:137,152)
//   dissipation.dat  (fort.71, format(i8,4(e14.6,1x)), SRC/dissipation.F90:265-278)
//   tec_{xy,xz,yz}.00000.<itime>.vtk at itime 0 and every ivtim steps
//   restart.<itime>.bin every itsave steps
//   bgk.perf and the GLUPS line of finalize (SRC/finalize.F90:83-97):
//   lx*ly*lz*(itfin - itstart)/(loop seconds * 1e9).
// Exit status 0 on success, 1 on a library error (its message on stderr).
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>

#include "bgk3d.h"

namespace {

// Fortran Ew.d edit descriptor with d = 6, w = 14 (0.ddddddE+ee).
std::string fortran_e(double x) {
  char buf[64];
  if (!std::isfinite(x)) {
    std::snprintf(buf, sizeof(buf), "%14s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
    return buf;
  }
  if (x == 0.0) {
    std::snprintf(buf, sizeof(buf), "%14s", "0.000000E+00");
    return buf;
  }
  char s[32];
  std::snprintf(s, sizeof(s), "%.5E", std::fabs(x));  // d.dddddE+ee
  const int e = std::atoi(s + 8) + 1;
  char m[16];
  std::snprintf(m, sizeof(m), "%c%.5s", s[0], s + 2);  // six significant digits
  char body[32];
  std::snprintf(body, sizeof(body), "%s0.%sE%c%02d", x < 0 ? "-" : "", m, e < 0 ? '-' : '+', std::abs(e));
  std::snprintf(buf, sizeof(buf), "%14s", body);
  return buf;
}

std::map<std::string, std::string> read_namelist(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  std::string t = ss.str();
  std::string low = t;
  for (char& c : low) c = (char)std::tolower((unsigned char)c);
  const size_t a = low.find("&parameters");
  if (a == std::string::npos) throw std::runtime_error("no &parameters group in " + path);
  const size_t b = low.find('/', a);
  std::string body = low.substr(a + 11, b == std::string::npos ? std::string::npos : b - a - 11);
  // tokens "key = value" with separators , newline tab and optional spaces
  std::string flat;
  for (char c : body) {
    if (c == '=') flat += " = ";
    else if (c == ',' || c == '\n' || c == '\r' || c == '\t') flat += ' ';
    else flat += c;
  }
  std::map<std::string, std::string> kv;
  std::istringstream in(flat);
  std::string prev, cur, key;
  bool expect_value = false;
  while (in >> cur) {
    if (cur == "=") {
      key = prev;
      expect_value = true;
    } else if (expect_value) {
      for (char& c : cur)
        if (c == 'd') c = 'e';  // Fortran double-precision exponent
      kv[key] = cur;
      expect_value = false;
    }
    prev = cur;
  }
  return kv;
}

int fail(const char* where) {
  std::fprintf(stderr, "bgk3d_hit: %s: %s\n", where, bgk_last_error());
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::string input = "bgk.input", out = ".", precision = "fp64", scheme = "two_lattice", init = "tgv_faithful";
  int device = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "bgk3d_hit: %s needs a value\n", a.c_str());
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--precision") precision = next();
    else if (a == "--scheme") scheme = next();
    else if (a == "--init") init = next();
    else if (a == "--out") out = next();
    else if (a == "--device") device = std::atoi(next().c_str());
    else if (a == "-h" || a == "--help") {
      std::printf("usage: bgk3d_hit [bgk.input] [--precision fp64|fp32|fp16] [--scheme two_lattice|aa] "
                  "[--init tgv|tgv_faithful] [--out DIR] [--device N]\n");
      return 0;
    } else input = a;
  }
  std::map<std::string, std::string> nl;
  try {
    nl = read_namelist(input);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "bgk3d_hit: %s\n", e.what());
    return 2;
  }
  auto geti = [&](const char* k, int d) { return nl.count(k) ? (int)std::strtod(nl[k].c_str(), nullptr) : d; };
  auto getd = [&](const char* k, double d) { return nl.count(k) ? std::strtod(nl[k].c_str(), nullptr) : d; };
  if (geti("proc_x", 1) != 1 || geti("proc_y", 1) != 1 || geti("proc_z", 1) != 1) {
    std::fprintf(stderr, "bgk3d_hit: one box per process (proc_x = proc_y = proc_z = 1)\n");
    return 2;
  }
  bgk_params p;
  bgk_params_default(&p);
  p.lx = geti("lx", 64);
  p.ly = geti("ly", p.lx);
  p.lz = geti("lz", p.lx);
  p.u0 = getd("u0", 0.05);
  p.svisc = getd("svisc", 0.01);
  p.icheck = geti("icheck", 10);
  p.les_cs = getd("ctes", 0.0);
  p.device = device;
  p.precision = precision == "fp32" ? BGK_FP32DEV : precision == "fp16" ? BGK_FP16DEV : BGK_FP64;
  p.scheme = scheme == "aa" ? BGK_AA : BGK_TWO_LATTICE;
  p.mode = init == "tgv" ? BGK_CORRECTED : BGK_FAITHFUL;
  const int itfin = geti("itfin", 100), itstart = 1;
  const int ivtim = geti("ivtim", 0), itsave = geti("itsave", 0);

  bgk_ctx* ctx = nullptr;
  if (bgk_create(&p, &ctx)) return fail("bgk_create");
  if (bgk_init_tgv(ctx)) return fail("bgk_init_tgv");
  const std::string d70 = out + "/diagno.dat", d71 = out + "/dissipation.dat";
  FILE* f70 = std::fopen(d70.c_str(), "w");
  FILE* f71 = std::fopen(d71.c_str(), "w");
  if (!f70 || !f71) {
    std::fprintf(stderr, "bgk3d_hit: cannot write into %s\n", out.c_str());
    return 2;
  }
  auto slices = [&](int it) {
    return bgk_vtk(ctx, it, 1, p.lz / 2, out.c_str()) || bgk_vtk(ctx, it, 2, p.ly / 2, out.c_str()) ||
           bgk_vtk(ctx, it, 3, p.lx / 2, out.c_str());
  };
  if (ivtim > 0 && slices(0)) return fail("bgk_vtk");
  if (bgk_synchronize(ctx)) return fail("bgk_synchronize");
  const auto t0 = std::chrono::steady_clock::now();
  for (int itime = itstart; itime <= itfin; ++itime) {
    if (bgk_boundaries(ctx, itime)) return fail("bgk_boundaries");
    if (bgk_col_mc(ctx, itime)) return fail("bgk_col_mc");
    bgk_diag d;
    const int rc = bgk_diagnostic(ctx, itime, &d);
    if (rc < 0) return fail("bgk_diagnostic");
    if (rc == BGK_OK) {
      std::fprintf(f70, "%8d", itime);
      for (double v : {d.ux_mean, d.uy_mean, d.uz_mean, d.rho_mean, d.ke_mean})
        std::fprintf(f70, "%s ", fortran_e(v).c_str());
      std::fprintf(f70, "\n");
      std::fprintf(f71, "%8d", itime);
      for (double v : {d.t, d.tke_norm, d.diss}) std::fprintf(f71, "%s ", fortran_e(v).c_str());
      std::fprintf(f71, "\n");
      std::fflush(f70);
      std::fflush(f71);
      if (ivtim > 0 && itime % ivtim == 0 && slices(itime)) return fail("bgk_vtk");
    }
    if (itsave > 0 && itime % itsave == 0) {
      char name[64];
      std::snprintf(name, sizeof(name), "/restart.%08d.bin", itime);
      if (bgk_save(ctx, (out + name).c_str())) return fail("bgk_save");
    }
  }
  if (bgk_synchronize(ctx)) return fail("bgk_synchronize");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::fclose(f70);
  std::fclose(f71);
  const double glups = (double)p.lx * p.ly * p.lz * (double)(itfin - itstart) / (secs * 1e9);
  FILE* perf = std::fopen((out + "/bgk.perf").c_str(), "w");
  if (perf) {
    std::fprintf(perf, "time loop (s)  %14.6f\nGLUPS          %14.6f\n", secs, glups);
    std::fclose(perf);
  }
  std::printf("INFO: loop %.6f s, GLUPS %.6f (lx*ly*lz*(itfin-itstart)/(t*1e9))\n", secs, glups);
  bgk_destroy(ctx);
  return 0;
}
