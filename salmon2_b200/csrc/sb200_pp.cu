// sb200_pp.cu -- host side: Kleinman-Bylander tables of s_pp_grid and the
// local pseudopotential from pseudopotential files with one projector per
// angular momentum (Yabana-Bertsch `_rps.dat` 'KY', ABINIT format 1 `.pspnc`,
// the ABINIT tables' FHI `.fhi`, FHI98PP `.cpi`), the set-up that produces the
// tables the propagation path consumes (no device code).
//
//   read_ps_KY                    src/atom/pp/input_pp.f90:288-341
//   read_ps_abinit                src/atom/pp/input_pp.f90:343-400
//   read_ps_abinitfhi             src/atom/pp/input_pp.f90:402-496
//   read_ps_fhi                   src/atom/pp/input_pp.f90:614-684
//   format by file name (init_pp) src/atom/pp/salmon_pp.f90:66-100
//   input_pp (radial domain,
//     KB norms)                   src/atom/pp/input_pp.f90:96-193
//   making_ps_without_masking     src/atom/pp/input_pp.f90:1111-1240
//   init_ps: calc_nps / calc_jxyz src/atom/pp/prep_pp.f90:22-372
//            set_lma / calc_uv    src/atom/pp/prep_pp.f90:374-525
//   calc_Vpsl_isolated            src/atom/pp/prep_pp.f90:550-620
//   calc_Vpsl_periodic            src/atom/pp/prep_pp.f90:798-974
//   spline (natural cubic)        src/math/salmon_math.f90:500-584
//   Ylm                           src/math/salmon_math.f90:386-426
//
// The radial KB function of angular momentum l is
//   udv_l(r) = (v_l(r) - v_lloc(r)) u_l(r) sqrt((2l+1)/4pi) / r^(l+1) / anorm_l,
//   anorm_l^2 = |int u_l^2 (v_l - v_lloc) dr| (trapezoid on the file's grid),
// interpolated at each sphere point by a natural cubic spline over the points
// r < rps (rps = max of the file's cut-off radii) and multiplied by the
// polynomial Ylm(x, y, z) of the point's offset from the atom; rinv_uvu =
// sign(anorm_l^2) hvol.  Projectors with anorm_l^2 = 0 (the local l) are left
// out.  Vpsl of an isolated grid: the local channel v_lloc interpolated
// linearly at each point's distance from every atom (beyond the file's grid,
// -Zps / r) and summed over the atoms; of a periodic grid: the form factors of
// the local channel and the structure sum, transformed back to the grid.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sb200_internal.cuh"

namespace sb200 {
namespace {

constexpr double PP_PI = 3.141592653589793;
constexpr double AU_LENGTH_AA = 0.52917721067;  // src/io/inputoutput.f90:27
constexpr double AU_ENERGY_EV = 27.21138505;    // src/io/inputoutput.f90:26

struct PsElement {
  int mr = 0, mlps = 0, lref = 0, nrps = 0, nrmax = 0;
  double step = 0.0, zps = 0.0, rps = 0.0;
  std::vector<double> rad;                  // rad[i - 1] = (i - 1) step, i = 1..nrmax
  std::vector<std::vector<double>> vpp;     // [l][0..nrmax]
  std::vector<std::vector<double>> upp;     // [l][0..nrmax]
  std::vector<double> anorm;
  std::vector<int> inorm;
  std::vector<std::vector<double>> sa, sb, sc, sd;  // spline of udv_l on rad[0..nrps-1]
};

double ylm_poly(double x, double y, double z, int l, int m) {
  const double r2 = x * x + y * y + z * z;
  if (l == 0) return 1.0;
  if (l == 1) return m == -1 ? -y : (m == 0 ? z : -x);
  if (l == 2) {
    switch (m) {
      case -2: return std::sqrt(3.0) * x * y;
      case -1: return -std::sqrt(3.0) * y * z;
      case 0: return (3.0 * z * z - r2) / 2.0;
      case 1: return -std::sqrt(3.0) * x * z;
      default: return std::sqrt(3.0 / 4.0) * (x * x - y * y);
    }
  }
  switch (m) {  // l = 3
    case -3: return -std::sqrt(5.0 / 8.0) * y * (3 * x * x - y * y);
    case -2: return std::sqrt(15.0) * x * y * z;
    case -1: return -std::sqrt(3.0 / 8.0) * y * (5.0 * z * z - r2);
    case 0: return z * (5.0 * z * z - 3 * r2) / 2.0;
    case 1: return -std::sqrt(3.0 / 8.0) * x * (5.0 * z * z - r2);
    case 2: return std::sqrt(15.0 / 4.0) * z * (x * x - y * y);
    default: return -std::sqrt(5.0 / 8.0) * x * (x * x - 3.0 * y * y);
  }
}

// natural cubic spline through (xn[i], yn[i]), i < np: on interval i
// y = a (x - xn_i)^3 + b (x - xn_i)^2 + c (x - xn_i) + d; the second
// derivatives from the tridiagonal system (Thomas algorithm)
void natural_spline(const std::vector<double>& xn, const std::vector<double>& yn, int np, std::vector<double>& a,
                    std::vector<double>& b, std::vector<double>& c, std::vector<double>& d) {
  const int n = np - 2;
  std::vector<double> dx(np - 1), dy(np - 1), u(np, 0.0);
  for (int i = 0; i < np - 1; ++i) {
    dx[i] = xn[i + 1] - xn[i];
    dy[i] = yn[i + 1] - yn[i];
  }
  if (n > 0) {
    std::vector<double> diag(n + 1), up(n + 1), rhs(n + 1);
    for (int i = 1; i <= n; ++i) {
      diag[i] = 2.0 * (dx[i] + dx[i - 1]);
      up[i] = dx[i];
      rhs[i] = 6.0 * (dy[i] / dx[i] - dy[i - 1] / dx[i - 1]);
    }
    for (int i = 2; i <= n; ++i) {  // forward elimination (sub-diagonal dx[i-1])
      const double w = dx[i - 1] / diag[i - 1];
      diag[i] -= w * up[i - 1];
      rhs[i] -= w * rhs[i - 1];
    }
    u[n] = rhs[n] / diag[n];
    for (int i = n - 1; i >= 1; --i) u[i] = (rhs[i] - up[i] * u[i + 1]) / diag[i];
  }
  a.assign(np - 1, 0.0);
  b.assign(np - 1, 0.0);
  c.assign(np - 1, 0.0);
  d.assign(np - 1, 0.0);
  for (int i = 0; i < np - 1; ++i) {
    b[i] = 0.5 * u[i];
    a[i] = (u[i + 1] - 2.0 * b[i]) / (6.0 * dx[i]);
    d[i] = yn[i];
    c[i] = dy[i] / dx[i] - dx[i] * (u[i + 1] + 2.0 * u[i]) / 6.0;
  }
}

// Fortran list-directed input, line by line: every read statement starts at a
// new record (line) and drops what is left of the last line it used; values
// are separated by blanks or commas; D exponents are accepted.
class ListReader {
 public:
  explicit ListReader(FILE* f) : f_(f) {}
  bool skip_record() { return next_line(); }
  bool read(double* v, int n) {
    int got = 0;
    while (got < n) {
      if (!next_line()) return false;
      size_t i = 0;
      while (got < n) {
        while (i < line_.size() && (line_[i] == ' ' || line_[i] == '\t' || line_[i] == ',' || line_[i] == '\r')) ++i;
        if (i >= line_.size()) break;
        size_t j = i;
        while (j < line_.size() && line_[j] != ' ' && line_[j] != '\t' && line_[j] != ',' && line_[j] != '\r') ++j;
        std::string tok = line_.substr(i, j - i);
        for (char& ch : tok)
          if (ch == 'D' || ch == 'd') ch = 'E';
        char* end = nullptr;
        const double x = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str()) return false;
        v[got++] = x;
        i = j;
      }
    }
    return true;
  }

 private:
  bool next_line() {
    line_.clear();
    int ch = std::fgetc(f_);
    if (ch == EOF) return false;
    while (ch != EOF && ch != '\n') {
      line_.push_back((char)ch);
      ch = std::fgetc(f_);
    }
    return true;
  }
  FILE* f_;
  std::string line_;
};

// read_ps_KY (input_pp.f90:288-341): Angstrom / eV file, linear radial grid
int read_ky(const char* path, int nrmax, PsElement& e, std::vector<double>& rrc) {
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(SB200_ERR_INVALID_ARG, std::string("cannot open pseudopotential file ") + path);
  double rzps = 0.0;
  int ok = std::fscanf(f, "%d %lf %d %lf", &e.mr, &e.step, &e.mlps, &rzps) == 4;
  if (!ok || e.mr < 2 || e.mlps < 0 || e.mlps > 3 || e.step <= 0.0) {
    std::fclose(f);
    return set_error(SB200_ERR_INVALID_ARG, std::string("not a Yabana-Bertsch (KY) file: ") + path);
  }
  e.zps = (double)(int)(rzps + 1e-10);
  int irpc = 0;
  rrc.assign(e.mlps + 1, 0.0);
  ok = std::fscanf(f, "%d", &irpc) == 1;
  for (int l = 0; l <= e.mlps && ok; ++l) ok = std::fscanf(f, "%lf", &rrc[l]) == 1;
  const int nr = nrmax > e.mr ? nrmax : e.mr;
  const int nl = e.mlps + 1;
  e.vpp.assign(nl, std::vector<double>(nr + 1, 0.0));
  e.upp.assign(nl, std::vector<double>(nr + 1, 0.0));
  for (int i = 0; i <= e.mr && ok; ++i) {
    double r, rho;
    ok = std::fscanf(f, "%lf %lf", &r, &rho) == 2;
    for (int l = 0; l < nl && ok; ++l) ok = std::fscanf(f, "%lf", &e.vpp[l][i]) == 1;
  }
  for (int i = 0; i <= e.mr && ok; ++i) {
    double r;
    ok = std::fscanf(f, "%lf", &r) == 1;
    for (int l = 0; l < nl && ok; ++l) ok = std::fscanf(f, "%lf", &e.upp[l][i]) == 1;
  }
  std::fclose(f);
  if (!ok) return set_error(SB200_ERR_INVALID_ARG, std::string("truncated KY file: ") + path);
  // atomic units (read_ps_KY)
  e.step /= AU_LENGTH_AA;
  for (int l = 0; l < nl; ++l) {
    rrc[l] /= AU_LENGTH_AA;
    for (int i = 0; i <= e.mr; ++i) {
      e.vpp[l][i] /= AU_ENERGY_EV;
      e.upp[l][i] *= std::sqrt(AU_LENGTH_AA);
    }
  }
  e.rad.resize(nrmax + 1);
  for (int i = 1; i <= nrmax + 1; ++i) e.rad[i - 1] = (i - 1) * e.step;
  return SB200_OK;
}

// read_ps_abinit (input_pp.f90:343-400): ABINIT format 1 (Troullier-Martins,
// .pspnc), Hartree atomic units; rad(i + 1) = 100 (i / (mmax - 1) + 0.01)^5 - 1e-8
int read_abinit(const char* path, int nrmax, PsElement& e, std::vector<double>& rrc) {
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(SB200_ERR_INVALID_ARG, std::string("cannot open pseudopotential file ") + path);
  ListReader in(f);
  double v[6];
  bool ok = in.skip_record() && in.read(v, 3);
  if (ok) e.zps = (double)(int)(v[1] + 1e-10);
  ok = ok && in.read(v, 6);
  const int mmax = ok ? (int)v[4] : 0;
  if (ok) {
    e.mlps = (int)v[2];
    e.mr = mmax - 1;
  }
  if (!ok || e.mlps < 0 || e.mlps > 3 || e.mr < 2 || e.mr > 50000) {
    std::fclose(f);
    return set_error(SB200_ERR_INVALID_ARG, std::string("not an ABINIT (.pspnc) file: ") + path);
  }
  rrc.assign(e.mlps + 1, 0.0);
  for (int ll = 0; ll <= e.mlps && ok; ++ll) {
    ok = in.read(v, 5);  // l, e99.0, e99.9, nproj, rcpsp
    if (ok) rrc[ll] = v[4];
    ok = ok && in.read(v, 4);  // rms, ekb1, ekb2, epsatm
  }
  ok = ok && in.read(v, 3);  // rchrg, fchrg, qchrg
  const int nr = nrmax > e.mr ? nrmax : e.mr;
  const int nl = e.mlps + 1;
  e.vpp.assign(nl, std::vector<double>(nr + 1, 0.0));
  e.upp.assign(nl, std::vector<double>(nr + 1, 0.0));
  for (int pass = 0; pass < 2 && ok; ++pass) {
    std::vector<std::vector<double>>& t = pass == 0 ? e.vpp : e.upp;
    for (int ll = 0; ll <= e.mlps && ok; ++ll) {
      ok = in.skip_record();
      for (int i = 1; i <= (e.mr + 1) / 3 && ok; ++i) {
        ok = in.read(v, 3);
        for (int j = 0; j < 3 && ok; ++j) t[ll][3 * (i - 1) + j] = v[j];
      }
    }
  }
  std::fclose(f);
  if (!ok) return set_error(SB200_ERR_INVALID_ARG, std::string("truncated ABINIT file: ") + path);
  e.rad.resize(nrmax + 1);
  for (int i = 0; i <= nrmax; ++i) {
    const double x = (double)i / (double)(mmax - 1) + 1.0e-2;
    e.rad[i] = 1.0e2 * (x * x * x * x * x) - 1.0e-8;
  }
  return SB200_OK;
}

// read_ps_fhi (input_pp.f90:614-684, FHI98PP .cpi) and read_ps_abinitfhi
// (:402-496, the FHI files of the ABINIT tables, .fhi: seven header lines
// first, then an optional core-correction block): Hartree atomic units,
// logarithmic grid given point by point (upp(i) and vpp(i) at rad(i + 1)),
// rad(1) = 0, upp(0) = 0, vpp(0) extrapolated linearly; the grid continued
// by the common ratio; rrc(l) the largest radius where v_l differs from
// another channel by more than 1e-10.  The core-correction block is read past
// (its radii replace the grid's, as the reference reads them); nonlinear core
// correction itself is not part of this path.
int read_fhi(const char* path, int nrmax, PsElement& e, std::vector<double>& rrc, bool abinit) {
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(SB200_ERR_INVALID_ARG, std::string("cannot open pseudopotential file ") + path);
  ListReader in(f);
  double v[4];
  bool ok = true;
  if (abinit)
    for (int i = 0; i < 7 && ok; ++i) ok = in.skip_record();
  ok = ok && in.read(v, 2);
  if (ok) {
    e.zps = (double)(int)(v[0] + 1e-10);
    e.mlps = (int)v[1] - 1;
  }
  if (!ok || e.mlps < 0 || e.mlps > 3) {
    std::fclose(f);
    return set_error(SB200_ERR_INVALID_ARG, std::string("not an FHI pseudopotential file: ") + path);
  }
  for (int i = 0; i < 10 && ok; ++i) ok = in.read(v, 1);
  const int nl = e.mlps + 1;
  std::vector<int> mr_l(nl, 0);
  std::vector<double> step_l(nl, 0.0);
  e.rad.assign(nrmax + 1, 0.0);
  for (int l = 0; l <= e.mlps && ok; ++l) {
    ok = in.read(v, 2);
    if (!ok) break;
    mr_l[l] = (int)v[0];
    step_l[l] = v[1];
    if (mr_l[l] < 3 || mr_l[l] > 50000) {
      ok = false;
      break;
    }
    if ((int)e.vpp.size() < nl) {
      const int nr = nrmax > mr_l[l] ? nrmax : mr_l[l];
      e.vpp.assign(nl, std::vector<double>(nr + 1, 0.0));
      e.upp.assign(nl, std::vector<double>(nr + 1, 0.0));
      if ((int)e.rad.size() < nr + 2) e.rad.resize(nr + 2, 0.0);
    }
    if (mr_l[l] > (int)e.vpp[l].size() - 1) {
      ok = false;
      break;
    }
    for (int i = 1; i <= mr_l[l] && ok; ++i) {
      ok = in.read(v, 4);
      if (ok) {
        e.rad[i] = v[1];  // rad(i + 1)
        e.upp[l][i] = v[2];
        e.vpp[l][i] = v[3];
      }
    }
    if (!ok) break;
    e.rad[0] = 0.0;
    e.upp[l][0] = 0.0;
    e.vpp[l][0] = e.vpp[l][1] - (e.vpp[l][2] - e.vpp[l][1]) / (e.rad[2] - e.rad[1]) * e.rad[1];
  }
  if (ok && abinit)  // core-correction block, to the end of the file if present
    for (int i = 1; i <= mr_l[0]; ++i) {
      if (!in.read(v, 4)) break;
      e.rad[i] = v[0];
    }
  std::fclose(f);
  if (!ok) return set_error(SB200_ERR_INVALID_ARG, std::string("truncated FHI pseudopotential file: ") + path);
  for (int l = 1; l <= e.mlps; ++l)
    if (mr_l[l] != mr_l[0]) return set_error(SB200_ERR_INVALID_ARG, "FHI file: radial grids of different lengths");
  double smin = step_l[0], smax = step_l[0];
  for (int l = 1; l <= e.mlps; ++l) {
    smin = step_l[l] < smin ? step_l[l] : smin;
    smax = step_l[l] > smax ? step_l[l] : smax;
  }
  if (smax - smin >= 1e-14) return set_error(SB200_ERR_INVALID_ARG, "FHI file: radial grids of different ratios");
  e.mr = mr_l[0];
  e.step = smin;
  const int iend = abinit ? nrmax - 1 : nrmax;
  for (int i = e.mr + 1; i <= iend; ++i) e.rad[i] = e.rad[i - 1] * e.step;  // rad(i + 1) = rad(i) step
  rrc.assign(nl, 0.0);
  for (int l = 0; l <= e.mlps; ++l) {
    double best = -1.0;
    for (int ll = 0; ll <= e.mlps; ++ll) {
      double rm = -1.0;
      for (int i = e.mr; i >= 1; --i)
        if (std::fabs(e.vpp[l][i] - e.vpp[ll][i]) > 1e-10) {
          rm = e.rad[i + 1];  // rad(i + 2)
          break;
        }
      best = rm > best ? rm : best;
    }
    rrc[l] = best;
  }
  return SB200_OK;
}

// Masking of the radial KB functions (yn_psmask = 'y'; alpha_mask,
// gamma_mask, eta_mask), process-wide as the reference's input variables.
struct PsMask {
  int on = 0;
  double alpha = 0.8, gamma = 1.8, eta = 15.0;  // the reference's defaults (inputoutput.f90:680-682)
};
PsMask g_psmask;

// x j_l(x), the Riccati-Bessel function, and its derivative: the closed forms
// in sin / cos, and below x = 0.1 the Taylor series the reference uses
// (xjl / dxjl, salmon_math.f90:289-383), l = 0..3
double xjl(double x, int l) {
  if (x < 0.1) {
    const double x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x, x6 = x3 * x3, x7 = x6 * x, x8 = x4 * x4,
                 x9 = x8 * x;
    switch (l) {
      case 0: return x - x3 / 6.0 + x5 / 120.0 - x7 / 5040.0 + x9 / 362880.0;
      case 1: return (2.0 / 6.0) * x2 - (2.0 / 60.0) * x4 + (1.0 / 840.0) * x6 - (2.0 / 90720.0) * x8;
      case 2: return (4.0 / 60.0) * x3 - (4.0 / 840.0) * x5 + (2.0 / 15120.0) * x7 - (2.0 / 997920.0) * x9;
      default: return (8.0 / 840.0) * x4 - (8.0 / 15120.0) * x6 + (4.0 / 332640.0) * x8;
    }
  }
  const double s = std::sin(x), c = std::cos(x);
  switch (l) {
    case 0: return s;
    case 1: return (1.0 / x) * s - c;
    case 2: return (3.0 / (x * x) - 1.0) * s - (3.0 / x) * c;
    default: return (15.0 / (x * x * x) - 6.0 / x) * s - (15.0 / (x * x) - 1.0) * c;
  }
}

// lowest eigenpair's vector of the symmetric n x n matrix a (row-major,
// overwritten) by cyclic Jacobi rotations (the reference calls LAPACK dsyev);
// its sign is arbitrary
void lowest_eigenvector(std::vector<double>& a, int n, std::vector<double>& vec) {
  std::vector<double> v((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double x = a[(size_t)i * n + j] * a[(size_t)i * n + j];
        tot += x;
        if (i != j) off += x;
      }
    if (off <= 1e-30 * tot) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = cs * akp - sn * akq;
          a[(size_t)k * n + q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = cs * apk - sn * aqk;
          a[(size_t)q * n + k] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = cs * vkp - sn * vkq;
          v[(size_t)k * n + q] = sn * vkp + cs * vkq;
        }
      }
  }
  int lo = 0;
  for (int i = 1; i < n; ++i)
    if (a[(size_t)i * n + i] < a[(size_t)lo * n + lo]) lo = i;
  vec.resize(n);
  for (int i = 0; i < n; ++i) vec[i] = v[(size_t)i * n + lo];
}

// make_mask_function (input_pp.f90:1437-1542): the normalized mask on x in
// (0, 1] as the lowest eigenvector of the M = 200 concentration matrix
// (sin((x_i + x_j) eta) / (x_i + x_j) - sin((x_i - x_j) eta) / (x_i - x_j),
// diagonal sin(2 x_i eta) / (2 x_i) + M pi - eta), divided by x and by its
// value extrapolated to x = 0; its sine transform on k = pi, 2 pi, ..., M pi;
// back on the radial grid r / rps for i = 2..nrps, the first and last points
// extrapolated linearly.  rmask[i - 1] = mask(rad(i)).
void make_mask(const PsElement& e, double eta, std::vector<double>& rmask) {
  const int M = 200;
  std::vector<double> x(M), mat((size_t)M * M), nm(M), k(M), nmk(M, 0.0);
  for (int i = 0; i < M; ++i) x[i] = (double)(i + 1) / (double)M;
  for (int i = 0; i < M; ++i) {
    const double xp = 2.0 * x[i];
    mat[(size_t)i * M + i] = std::sin(xp * eta) / xp + (double)M * PP_PI - eta;
    for (int j = i + 1; j < M; ++j) {
      const double a = x[i] + x[j], b = x[i] - x[j];
      const double m = std::sin(a * eta) / a - std::sin(b * eta) / b;
      mat[(size_t)i * M + j] = m;
      mat[(size_t)j * M + i] = m;
    }
  }
  std::vector<double> u;
  lowest_eigenvector(mat, M, u);
  const double n0 = 3.0 * u[0] / x[0] - 3.0 * u[1] / x[1] + u[2] / x[2];
  for (int i = 0; i < M; ++i) nm[i] = u[i] / x[i] / n0;
  for (int i = 0; i < M; ++i) k[i] = PP_PI * (double)(i + 1);
  const double dx = x[1] - x[0];
  for (int i = 0; i < M; ++i) {
    double acc = 0.0;
    for (int j = 0; j < M; ++j) {
      const double kx = k[i] * x[j];
      acc = acc + nm[j] * kx * std::sin(kx);
    }
    nmk[i] = acc * dx / (k[i] * k[i]);
  }
  const int nrps = e.nrps;
  rmask.assign(nrps, 0.0);
  const double dk = k[1] - k[0];
  for (int i = 2; i <= nrps; ++i) {
    double acc = 0.0;
    for (int j = 0; j < M; ++j) {
      const double kx = k[j] * e.rad[i - 1] / e.rps;
      acc = acc + nmk[j] * kx * std::sin(kx);
    }
    rmask[i - 1] = (2.0 / PP_PI) * acc * dk * e.rps * e.rps / (e.rad[i - 1] * e.rad[i - 1]);
  }
  rmask[0] = rmask[1] - (rmask[2] - rmask[1]) / (e.rad[2] - e.rad[1]) * (e.rad[1] - e.rad[0]);
  const int i1 = nrps - 2, i2 = nrps - 1, i3 = nrps;
  rmask[i3 - 1] = rmask[i2 - 1] + (rmask[i2 - 1] - rmask[i1 - 1]) / (e.rad[i2 - 1] - e.rad[i1 - 1]) *
                                      (e.rad[i3 - 1] - e.rad[i2 - 1]);
}

// ps_masking (input_pp.f90:1302-1434) and the table part of
// making_ps_with_masking (:848-1016) for one-projector channels: the cut-off
// widened to gamma_mask rps (snapped to the next grid point), uv_l = u_l
// (v_l - v_lloc) divided by the mask, its Bessel transform (trapezoid on the
// file's grid) on nkmax = 1000 points up to alpha_mask pi / max(h), the
// transform back (trapezoid in k) times 2 / pi and the mask, then
// sqrt((2l+1)/4pi) / r^(l+1); uvm[l][i] = uv_l at rad(i + 1), i = 0..nrps-1.
int mask_element(PsElement& e, double hmax, std::vector<std::vector<double>>& uvm) {
  const PsMask& m = g_psmask;
  e.rps = m.gamma * e.rps;
  int i = 1;
  for (; i <= (int)e.rad.size(); ++i)
    if (e.rad[i - 1] > e.rps) break;
  if (i > e.mr - 2) return set_error(SB200_ERR_INVALID_ARG, "masked cut-off gamma_mask rps beyond the file's grid");
  e.nrps = i;
  e.rps = e.rad[e.nrps - 1];
  std::vector<double> mask;
  make_mask(e, m.eta, mask);
  const int mr = e.mr, nl = e.mlps + 1;
  std::vector<std::vector<double>> uv(nl, std::vector<double>(mr + 1, 0.0));
  for (int l = 0; l < nl; ++l) {
    for (int k = 0; k <= mr; ++k) uv[l][k] = e.upp[l][k] * (e.vpp[l][k] - e.vpp[e.lref][k]);
    for (int k = 0; k < e.nrps; ++k) uv[l][k] = uv[l][k] / mask[k];
  }
  const int nkmax = 1000;
  const double kmax = m.alpha * PP_PI / hmax;
  std::vector<double> radk(nkmax);
  for (int q = 0; q < nkmax; ++q) radk[q] = kmax * ((double)q / (double)(nkmax - 1));
  std::vector<std::vector<double>> wk(nl, std::vector<double>(nkmax, 0.0));
  for (int q = 0; q < nkmax; ++q)
    for (int j = 1; j <= mr - 1; ++j) {
      const double kr1 = radk[q] * e.rad[j - 1], kr2 = radk[q] * e.rad[j], dr = e.rad[j] - e.rad[j - 1];
      for (int l = 0; l < nl; ++l)
        wk[l][q] = wk[l][q] + 0.5 * (xjl(kr1, l) * uv[l][j - 1] + xjl(kr2, l) * uv[l][j]) * dr;
    }
  for (int l = 0; l < nl; ++l) std::fill(uv[l].begin(), uv[l].end(), 0.0);
  for (int q = 0; q < nkmax - 1; ++q)
    for (int j = 1; j <= mr; ++j) {
      const double kr1 = radk[q] * e.rad[j - 1], kr2 = radk[q + 1] * e.rad[j - 1], dk = radk[q + 1] - radk[q];
      for (int l = 0; l < nl; ++l)
        uv[l][j - 1] = uv[l][j - 1] + 0.5 * (xjl(kr1, l) * wk[l][q] + xjl(kr2, l) * wk[l][q + 1]) * dk;
    }
  for (int l = 0; l < nl; ++l) {
    uv[l][mr] = 2.0 * uv[l][mr - 1] - uv[l][mr - 2];
    for (int k = 0; k <= mr; ++k) uv[l][k] = (2.0 / PP_PI) * uv[l][k];
    for (int k = 0; k < e.nrps; ++k) uv[l][k] = uv[l][k] * mask[k];
    const double cst = std::sqrt((2.0 * l + 1.0) / (4.0 * PP_PI));
    for (int k = 1; k <= mr; ++k) uv[l][k] = uv[l][k] * cst / std::pow(e.rad[k], l + 1);
    uv[l][0] = 2.0 * uv[l][1] - uv[l][2];
  }
  uvm.swap(uv);
  return SB200_OK;
}

// input_pp's common part (input_pp.f90:93-193) and making_ps_without_masking
// (:1111-1240) for an element read by one of the readers above
int finish_element(PsElement& e, const std::vector<double>& rrc, int lmax_ps, int lloc, int nrmax, double hmax) {
  e.nrmax = nrmax;
  if (lmax_ps >= 0) {
    if (lmax_ps > e.mlps) return set_error(SB200_ERR_INVALID_ARG, "Lmax_ps above the file's angular momenta");
    e.mlps = lmax_ps;
  }
  if (lloc < 0 || lloc > e.mlps) return set_error(SB200_ERR_INVALID_ARG, "Lloc_ps must be in 0..Lmax_ps");
  e.lref = lloc;
  if ((int)e.rad.size() < e.mr + 2 || (int)e.rad.size() < nrmax + 1)
    return set_error(SB200_ERR_INVALID_ARG, "pseudopotential file's radial grid longer than the set-up's arrays");
  const int nr = (int)e.vpp[0].size() - 1;
  // beyond the file's grid: -Zps / r (input_pp.f90:96-102; the array index i
  // takes rad(i) here although vpp(i) otherwise stands for rad(i + 1))
  for (int i = e.mr + 1; i <= nrmax && i <= nr; ++i)
    for (int l = 0; l <= e.mlps; ++l) {
      if (e.rad[i - 1] > 0.0) e.vpp[l][i] = -e.zps / e.rad[i - 1];
      e.upp[l][i] = 0.0;
    }
  double rps = 0.0;
  for (int l = 0; l <= e.mlps; ++l) rps = rrc[l] > rps ? rrc[l] : rps;
  if (!(rps > 0.0)) return set_error(SB200_ERR_INVALID_ARG, "pseudopotential without a cut-off radius");
  e.rps = rps;
  int i = 1;
  for (; i <= nrmax; ++i)
    if (e.rad[i - 1] > e.rps) break;
  e.nrps = i;
  if (e.nrps >= nrmax) return set_error(SB200_ERR_INVALID_ARG, "pseudopotential cut-off beyond the radial grid");
  // KB norms (input_pp.f90:179-193), trapezoid on rad
  e.anorm.assign(e.mlps + 1, 0.0);
  e.inorm.assign(e.mlps + 1, 0);
  for (int l = 0; l <= e.mlps; ++l) {
    double s = 0.0;
    for (int k = 1; k <= e.mr - 1; ++k) {
      const double r1 = e.rad[k] - e.rad[k - 1];
      s = s + (e.upp[l][k] * e.upp[l][k] * (e.vpp[l][k] - e.vpp[e.lref][k]) +
               e.upp[l][k - 1] * e.upp[l][k - 1] * (e.vpp[l][k - 1] - e.vpp[e.lref][k - 1])) *
                  r1;
    }
    s = 0.5 * s;
    e.inorm[l] = 1;
    if (s < 0.0) {
      s = -s;
      e.inorm[l] = -1;
    }
    if (std::fabs(s) < 1e-10) e.inorm[l] = 0;
    e.anorm[l] = std::sqrt(s);
  }
  std::vector<std::vector<double>> uvm;  // masked udv_l before the norm (yn_psmask = 'y')
  if (g_psmask.on) {
    const int r = mask_element(e, hmax, uvm);
    if (r != SB200_OK) return r;
  } else {
    // making_ps_without_masking: radial functions / r^(l+1), then the KB tables
    for (int l = 0; l <= e.mlps; ++l) {
      for (int k = 1; k <= e.mr; ++k)
        e.upp[l][k] = e.upp[l][k] * std::sqrt((2 * l + 1.0) / (4 * PP_PI)) / std::pow(e.rad[k], l + 1);
      e.upp[l][0] = e.upp[l][1];
    }
  }
  e.sa.assign(e.mlps + 1, {});
  e.sb.assign(e.mlps + 1, {});
  e.sc.assign(e.mlps + 1, {});
  e.sd.assign(e.mlps + 1, {});
  std::vector<double> xn(e.rad.begin(), e.rad.begin() + e.nrps), yn(e.nrps);
  for (int l = 0; l <= e.mlps; ++l) {
    for (int k = 1; k <= e.nrps; ++k) {
      yn[k - 1] = g_psmask.on ? uvm[l][k - 1] : (e.vpp[l][k - 1] - e.vpp[e.lref][k - 1]) * e.upp[l][k - 1];
      if (e.inorm[l] != 0) yn[k - 1] = yn[k - 1] / e.anorm[l];
    }
    natural_spline(xn, yn, e.nrps, e.sa[l], e.sb[l], e.sc[l], e.sd[l]);
  }
  return SB200_OK;
}

bool ends_with(const std::string& s, const char* suffix) {
  const size_t n = std::strlen(suffix);
  return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

// one element: the reader of its format, then input_pp's common part.
// force_ky: the file is read as 'KY' whatever its name; otherwise the format
// follows the file name as init_pp does (salmon_pp.f90:66-100): _rps.dat KY,
// .pspnc ABINIT, .fhi ABINITFHI, .cpi FHI.
int read_element(const char* path, bool force_ky, int lmax_ps, int lloc, int nrmax, double hmax, PsElement& e) {
  const std::string name(path);
  std::vector<double> rrc;
  int r;
  if (force_ky || ends_with(name, "_rps.dat")) {
    r = read_ky(path, nrmax, e, rrc);
  } else if (ends_with(name, ".pspnc")) {
    r = read_abinit(path, nrmax, e, rrc);
  } else if (ends_with(name, ".fhi")) {
    r = read_fhi(path, nrmax, e, rrc, true);
  } else if (ends_with(name, ".cpi")) {
    r = read_fhi(path, nrmax, e, rrc, false);
  } else if (ends_with(name, ".psp8") || ends_with(name, ".vps") || ends_with(name, ".upf") ||
             ends_with(name, ".UPF")) {
    return set_error(SB200_ERR_UNSUPPORTED,
                     "pseudopotentials with several projectors per l or given beta projectors (psp8, vps, upf) "
                     "are not supported: " + name);
  } else {
    return set_error(SB200_ERR_INVALID_ARG, "unknown pseudopotential file format: " + name);
  }
  if (r != SB200_OK) return r;
  return finish_element(e, rrc, lmax_ps, lloc, nrmax, hmax);
}

int init_ps_impl(bool force_ky, int nelem, const char* const* files, const int* lmax_ps, const int* lloc_ps,
                 int periodic, const int num[3], const int is[3], const double hgs[3], double hvol, int natom,
                 const int* kion, const double* Rion, int* nps, int* nlma, int* mps, int* jxyz, double* rxyz,
                 double* uv, int* ia_tbl, double* rinv_uvu, double* Vpsl) {
  if (nelem < 1 || !files || !lloc_ps || !num || !is || !hgs || natom < 0 || (natom > 0 && (!kion || !Rion)) ||
      !nps || !nlma)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_init_ps: null or inconsistent argument");
  const int nrmax = periodic ? 3000 : 20000;  // read_pslfile, salmon_pp.f90:34-38
  std::vector<PsElement> el(nelem);
  const double hgs_max = hgs[0] > hgs[1] ? (hgs[0] > hgs[2] ? hgs[0] : hgs[2]) : (hgs[1] > hgs[2] ? hgs[1] : hgs[2]);
  for (int k = 0; k < nelem; ++k) {
    if (!files[k]) return set_error(SB200_ERR_INVALID_ARG, "null pseudopotential file name");
    const int r = read_element(files[k], force_ky, lmax_ps ? lmax_ps[k] : -1, lloc_ps[k], nrmax, hgs_max, el[k]);
    if (r != SB200_OK) return r;
  }
  for (int a = 0; a < natom; ++a)
    if (kion[a] < 1 || kion[a] > nelem) return set_error(SB200_ERR_INVALID_ARG, "kion out of 1..nelem");
  const int ie[3] = {is[0] + num[0] - 1, is[1] + num[1] - 1, is[2] + num[2] - 1};
  const double al[3] = {num[0] * hgs[0], num[1] * hgs[1], num[2] * hgs[2]};
  double rshift[3];
  for (int d = 0; d < 3; ++d) rshift[d] = periodic ? -hgs[d] : ((num[d] % 2 == 1) ? 0.0 : -0.5 * hgs[d]);
  // periodic images (init_ps, prep_pp.f90:86-112, cuboid cell)
  double rps_max = 0.0, hmax = 0.0;
  for (int k = 0; k < nelem; ++k) rps_max = el[k].rps > rps_max ? el[k].rps : rps_max;
  for (int d = 0; d < 3; ++d) hmax = hgs[d] > hmax ? hgs[d] : hmax;
  rps_max = rps_max + 1.5 * hmax + 1e-2;
  int nc[3] = {0, 0, 0};
  if (periodic)
    for (int d = 0; d < 3; ++d) {
      double mn = 1e300, mx = -1e300;
      for (int a = 0; a < natom; ++a) {
        mn = Rion[3 * a + d] < mn ? Rion[3 * a + d] : mn;
        mx = Rion[3 * a + d] > mx ? Rion[3 * a + d] : mx;
      }
      nc[d] = (mn + 2.0 * al[d] > al[d] + rps_max && mx - 2.0 * al[d] < -rps_max) ? 1 : 2;
    }
  // sphere points (calc_nps / calc_jxyz): images j1, j2, j3, then z, y, x
  std::vector<std::vector<int>> pj(natom);
  std::vector<std::vector<double>> pr(natom);
  for (int a = 0; a < natom; ++a) {
    const PsElement& e = el[kion[a] - 1];
    for (int j1 = -nc[0]; j1 <= nc[0]; ++j1) {
      const double x1 = Rion[3 * a] + j1 * al[0];
      if (x1 <= is[0] * hgs[0] - rps_max || x1 >= ie[0] * hgs[0] + rps_max) continue;
      for (int j2 = -nc[1]; j2 <= nc[1]; ++j2) {
        const double x2 = Rion[3 * a + 1] + j2 * al[1];
        if (x2 <= is[1] * hgs[1] - rps_max || x2 >= ie[1] * hgs[1] + rps_max) continue;
        for (int j3 = -nc[2]; j3 <= nc[2]; ++j3) {
          const double x3 = Rion[3 * a + 2] + j3 * al[2];
          if (x3 <= is[2] * hgs[2] - rps_max || x3 >= ie[2] * hgs[2] + rps_max) continue;
          for (int i3 = is[2]; i3 <= ie[2]; ++i3)
            for (int i2 = is[1]; i2 <= ie[1]; ++i2)
              for (int i1 = is[0]; i1 <= ie[0]; ++i1) {
                const double x = i1 * hgs[0] + rshift[0] - x1, y = i2 * hgs[1] + rshift[1] - x2,
                             z = i3 * hgs[2] + rshift[2] - x3;
                const double r = std::sqrt(x * x + y * y + z * z);
                if (r < e.rps + 1e-12) {
                  pj[a].insert(pj[a].end(), {i1, i2, i3});
                  pr[a].insert(pr[a].end(), {x, y, z});
                }
              }
        }
      }
    }
  }
  int np = 0, nl = 0;
  for (int a = 0; a < natom; ++a) {
    const int m = (int)pj[a].size() / 3;
    np = m > np ? m : np;
    const PsElement& e = el[kion[a] - 1];
    for (int l = 0; l <= e.mlps; ++l)
      if (e.inorm[l] != 0) nl += 2 * l + 1;
  }
  const bool fill = mps && jxyz && rxyz && uv && ia_tbl && rinv_uvu;
  if (fill && (*nps < np || *nlma < nl))
    return set_error(SB200_ERR_INVALID_ARG, "sb200_init_ps: output arrays smaller than *nps, *nlma");
  if (!fill) {
    *nps = np;
    *nlma = nl;
  } else {
    const int NPS = *nps, NLMA = *nlma;
    std::memset(jxyz, 0, sizeof(int) * 3 * (size_t)NPS * natom);
    std::memset(rxyz, 0, sizeof(double) * 3 * (size_t)NPS * natom);
    std::memset(uv, 0, sizeof(double) * (size_t)NPS * NLMA);
    int lma = 0;
    for (int a = 0; a < natom; ++a) {
      const PsElement& e = el[kion[a] - 1];
      const int m = (int)pj[a].size() / 3;
      mps[a] = m;
      for (int j = 0; j < m; ++j)
        for (int c = 0; c < 3; ++c) {
          jxyz[c + 3 * ((size_t)j + (size_t)NPS * a)] = pj[a][3 * j + c];
          rxyz[c + 3 * ((size_t)j + (size_t)NPS * a)] = pr[a][3 * j + c];
        }
      // calc_uv: spline at each sphere point, times Ylm of its offset
      const int lma0 = lma;
      for (int l = 0; l <= e.mlps; ++l) {
        if (e.inorm[l] == 0) continue;
        for (int mm = -l; mm <= l; ++mm) {
          ia_tbl[lma] = a + 1;
          rinv_uvu[lma] = (double)e.inorm[l] * hvol;
          ++lma;
        }
      }
      for (int j = 0; j < m; ++j) {
        const double x = pr[a][3 * j], y = pr[a][3 * j + 1], z = pr[a][3 * j + 2];
        const double r = std::sqrt(x * x + y * y + z * z) + 1e-50;
        int ir = 1;
        for (; ir <= e.nrps; ++ir)
          if (e.rad[ir - 1] > r) break;
        const int intr = ir - 1;  // 1-based interval: rad(intr) <= r < rad(intr + 1)
        if (intr < 1 || intr >= e.nrps) return set_error(SB200_ERR_INVALID_ARG, "sphere point outside the radial grid");
        const double xx = r - e.rad[intr - 1];
        int col = lma0;
        for (int l = 0; l <= e.mlps; ++l) {
          if (e.inorm[l] == 0) continue;
          const int s = intr - 1;
          const double uvr = e.sa[l][s] * xx * xx * xx + e.sb[l][s] * xx * xx + e.sc[l][s] * xx + e.sd[l][s];
          for (int mm = -l; mm <= l; ++mm) uv[(size_t)j + (size_t)NPS * col++] = uvr * ylm_poly(x, y, z, l, mm);
        }
      }
    }
  }
  if (Vpsl && periodic) {
    // calc_Vpsl_periodic (prep_pp.f90:798-974, transforms without FFTE): per
    // element the form factor of the local channel minus the Coulomb tail,
    // zVG(G) = 4 pi sum_i sin(|G| r1) / |G| (r1 vloc_av + Zps) dr (G = 0:
    // 4 pi sum_i (r1^2 vloc_av + r1 Zps) dr, midpoints r1), the structure sum
    // V(G) = sum_a (zVG(G) - 4 pi / G^2 Zps) e^{-i G.R_a} / det A, then the
    // inverse transforms along z, y, x with egz / egy / egx
    // (initialization.f90:700-784); Vpsl = the real part.
    const int n0 = num[0], n1 = num[1], n2 = num[2];
    const long npts = (long)n0 * n1 * n2;
    const double detA = al[0] * al[1] * al[2];
    auto fold = [](int m, int n) { return (m - (n + 1) / 2 >= 0) ? m - n : m; };  // ix-1 -> folded index
    std::vector<double> vre(npts, 0.0), vim(npts, 0.0);
    std::vector<std::vector<double>> zvg(nelem);
    for (int kz = 0; kz < n2; ++kz)
      for (int ky = 0; ky < n1; ++ky)
        for (int kx = 0; kx < n0; ++kx) {
          const long q = kx + (long)n0 * (ky + (long)n1 * kz);
          const double g[3] = {fold(kx, n0) * 2.0 * PP_PI / al[0], fold(ky, n1) * 2.0 * PP_PI / al[1],
                               fold(kz, n2) * 2.0 * PP_PI / al[2]};
          const double G2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
          const bool gzero = kx == 0 && ky == 0 && kz == 0;
          const double coef = gzero ? 0.0 : 4.0 * PP_PI / G2;
          const double gsq = std::sqrt(G2);
          double sr = 0.0, si = 0.0;
          for (int a = 0; a < natom; ++a) {
            const PsElement& e = el[kion[a] - 1];
            double zv = 0.0;
            for (int i2 = 2; i2 <= e.nrps; ++i2) {  // vloctbl(i) = vpp(i - 1, lref), i = 1..nrps
              const double r1 = 0.5 * (e.rad[i2 - 1] + e.rad[i2 - 2]);
              const double dr = e.rad[i2 - 1] - e.rad[i2 - 2];
              const double vav = 0.5 * (e.vpp[e.lref][i2 - 1] + e.vpp[e.lref][i2 - 2]);
              if (gzero) zv = zv + 4.0 * PP_PI * (r1 * r1 * vav + r1 * e.zps) * dr;
              else zv = zv + 4.0 * PP_PI * std::sin(gsq * r1) / gsq * (r1 * vav + e.zps) * dr;
            }
            const double gd = g[0] * Rion[3 * a] + g[1] * Rion[3 * a + 1] + g[2] * Rion[3 * a + 2];
            const double er = std::cos(gd) / detA, ei = -std::sin(gd) / detA;
            const double w = zv - coef * e.zps;
            sr = sr + w * er;
            si = si + w * ei;
          }
          vre[q] = sr;
          vim[q] = si;
        }
    // inverse transforms: z, then y, then x (each output the ordered sum over the axis)
    auto pass = [&](int axis) {
      const int n = axis == 0 ? n0 : axis == 1 ? n1 : n2;
      std::vector<double> ore(npts), oim(npts);
      for (int iz = 0; iz < n2; ++iz)
        for (int iy = 0; iy < n1; ++iy)
          for (int ix = 0; ix < n0; ++ix) {
            const int out_i = axis == 0 ? ix : axis == 1 ? iy : iz;
            double re = 0.0, im = 0.0;
            for (int k = 0; k < n; ++k) {
              const long q = axis == 0 ? k + (long)n0 * (iy + (long)n1 * iz)
                                       : axis == 1 ? ix + (long)n0 * (k + (long)n1 * iz)
                                                   : ix + (long)n0 * (iy + (long)n1 * k);
              const double ang = 2.0 * PP_PI * (double)((long)out_i * k) / (double)n;
              const double tr = std::cos(ang), ti = std::sin(ang);
              re = re + (tr * vre[q] - ti * vim[q]);
              im = im + (tr * vim[q] + ti * vre[q]);
            }
            const long p = ix + (long)n0 * (iy + (long)n1 * iz);
            ore[p] = re;
            oim[p] = im;
          }
      vre.swap(ore);
      vim.swap(oim);
    };
    pass(2);
    pass(1);
    pass(0);
    for (long p = 0; p < npts; ++p) Vpsl[p] = vre[p];
  } else if (Vpsl) {  // calc_Vpsl_isolated: linear interpolation of the local channel
    const long npts = (long)num[0] * num[1] * num[2];
    for (long p = 0; p < npts; ++p) Vpsl[p] = 0.0;
    for (int a = 0; a < natom; ++a) {
      const PsElement& e = el[kion[a] - 1];
      for (int iz = 0; iz < num[2]; ++iz)
        for (int iy = 0; iy < num[1]; ++iy)
          for (int ix = 0; ix < num[0]; ++ix) {
            const int g[3] = {ix + is[0], iy + is[1], iz + is[2]};
            double d2 = 0.0;
            for (int d = 0; d < 3; ++d) {
              const double c = (num[d] % 2 == 1) ? g[d] * hgs[d] : (g[d] - 0.5) * hgs[d];
              const double t = c - Rion[3 * a + d];
              d2 += t * t;
            }
            const double r = std::sqrt(d2) + 1e-50;
            int imin = 1, imax = e.nrmax;  // bisection (prep_pp.f90:1013-1035)
            while (imax - imin > 1) {
              const int in = (imin + imax) / 2;
              if (r > e.rad[in - 1]) imin = in;
              else imax = in;
            }
            const int intr = imin;
            const double ratio1 = (r - e.rad[intr - 1]) / (e.rad[intr] - e.rad[intr - 1]), ratio2 = 1.0 - ratio1;
            double& v = Vpsl[ix + (long)num[0] * (iy + (long)num[1] * iz)];
            v = v + ratio1 * e.vpp[e.lref][intr] + ratio2 * e.vpp[e.lref][intr - 1];
          }
    }
  }
  return SB200_OK;
}

}  // namespace
}  // namespace sb200

using namespace sb200;

extern "C" int sb200_init_ps_ky(int nelem, const char* const* files, const int* lmax_ps, const int* lloc_ps,
                                int periodic, const int num[3], const int is[3], const double hgs[3], double hvol,
                                int natom, const int* kion, const double* Rion, int* nps, int* nlma, int* mps,
                                int* jxyz, double* rxyz, double* uv, int* ia_tbl, double* rinv_uvu,
                                double* Vpsl) {
  return init_ps_impl(true, nelem, files, lmax_ps, lloc_ps, periodic, num, is, hgs, hvol, natom, kion, Rion, nps,
                      nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl);
}

extern "C" int sb200_init_ps(int nelem, const char* const* files, const int* lmax_ps, const int* lloc_ps,
                             int periodic, const int num[3], const int is[3], const double hgs[3], double hvol,
                             int natom, const int* kion, const double* Rion, int* nps, int* nlma, int* mps,
                             int* jxyz, double* rxyz, double* uv, int* ia_tbl, double* rinv_uvu, double* Vpsl) {
  return init_ps_impl(false, nelem, files, lmax_ps, lloc_ps, periodic, num, is, hgs, hvol, natom, kion, Rion, nps,
                      nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl);
}

extern "C" int sb200_set_psmask(int yn_psmask, double alpha_mask, double gamma_mask, double eta_mask) {
  if (yn_psmask != 0 && yn_psmask != 1) return set_error(SB200_ERR_INVALID_ARG, "yn_psmask is 0 or 1");
  if (yn_psmask && !(alpha_mask > 0.0 && gamma_mask >= 1.0 && eta_mask > 0.0))
    return set_error(SB200_ERR_INVALID_ARG, "alpha_mask > 0, gamma_mask >= 1 and eta_mask > 0 are required");
  g_psmask.on = yn_psmask;
  if (yn_psmask) {
    g_psmask.alpha = alpha_mask;
    g_psmask.gamma = gamma_mask;
    g_psmask.eta = eta_mask;
  }
  return SB200_OK;
}
