// salmon_oracle_scf.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the
// per-step potential update of the self-consistent RT path: the PZ-LDA
// exchange-correlation potential, the periodic Hartree potential by separable
// discrete Fourier transforms, and update_vlocal.  Plain restatements of the
// reference's Fortran, loop and summation order kept; the product library never
// links or calls this file.
//
// Parity status: unpinned against reference outputs (the Fortran reference
// cannot be compiled here); pinned by analytic known answers in
// tests/test_oracle_scf.py (uniform-gas exchange, the potential as the density
// derivative of the energy density, sampled plane waves through the Poisson
// solver, charge neutrality).
#include <cmath>
#include <vector>

#include "salmon_oracle.h"

namespace {

const double PI = 3.141592653589793;

// PZxc, src/xc/builtin_pz.f90:51-83 (Perdew-Zunger 1981 parametrisation of the
// Ceperley-Alder correlation energy plus Slater exchange).
void pzxc(double trho, double* exc, double* dexc_drho) {
  const double gammaU = -0.1423, beta1U = 1.0529, beta2U = 0.3334, AU = 0.0311, BU = -0.048, CU = 0.002,
               DU = -0.0116;
  const double cst = 0.75 * std::pow(3.0 / (2.0 * PI), 2.0 / 3.0);
  const double ttrho = trho + 1e-10;
  const double rs = std::pow(3.0 / (4.0 * PI * ttrho), 1.0 / 3.0);
  double e = -cst / rs;
  double de = e / (3.0 * ttrho);
  if (rs > 1.0) {
    const double rssq = std::sqrt(rs);
    const double den = 1.0 + beta1U * rssq + beta2U * rs;
    e = e + gammaU / den;
    de = de + gammaU * (0.5 * beta1U * rssq + beta2U * rs) / (3.0 * ttrho) / (den * den);
  } else {
    const double rsln = std::log(rs);
    e = e + AU * rsln + BU + CU * rs * rsln + DU * rs;
    de = de - rs / (3.0 * ttrho) * (AU / rs + CU * (rsln + 1.0) + DU);
  }
  *exc = e;
  *dexc_drho = de;
}

// Index folding of fg%coef, initialization.f90:700-702: m = ix-1 in 0..n-1
// maps to m - n when m >= (n+1)/2 (Fortran sign(1, m - (n+1)/2) = +1 there).
int fold(int m, int n) { return (m - (n + 1) / 2 >= 0) ? m - n : m; }

}  // namespace

extern "C" {

// exchange_correlation for nspin = 1 with xc = 'PZ' (src/xc/salmon_xc.f90:86-254,
// calc_xc :770-806, exc_cor_pz builtin_pz.f90:23-47): rho_s = rho*0.5,
// trho = 2*rho_s, Vxc = e_xc + trho*de_xc/drho, E_xc = hvol * sum(e_xc*trho)
// summed with x fastest.
void sbo_exc_cor_pz(long n, const double* rho, double hvol, double* vxc, double* E_xc) {
  std::vector<double> eexc(n);
#pragma omp parallel for
  for (long i = 0; i < n; ++i) {
    const double rho_s = rho[i] * 0.5;
    const double trho = 2.0 * rho_s;
    double e, de;
    pzxc(trho, &e, &de);
    eexc[i] = e * trho;
    vxc[i] = e + trho * de;
  }
  double tot = 0.0;
  for (long i = 0; i < n; ++i) tot = tot + eexc[i];
  *E_xc = tot * hvol;
}

// fg%coef = 4 pi / |G|^2 (0 at G = 0) on the (kx, ky, kz) grid, x fastest,
// initialization.f90:690-724, with brl = primitive_b (3x3, column j = b_j).
void sbo_poisson_coef(const int num[3], const double brl[9], double* coef) {
  for (int kz = 0; kz < num[2]; ++kz)
    for (int ky = 0; ky < num[1]; ++ky)
      for (int kx = 0; kx < num[0]; ++kx) {
        const long p = kx + (long)num[0] * (ky + (long)num[1] * kz);
        const int iix = fold(kx, num[0]), iiy = fold(ky, num[1]), iiz = fold(kz, num[2]);
        double g[3];
        for (int d = 0; d < 3; ++d)
          g[d] = (double)iix * brl[d + 0] + (double)iiy * brl[d + 3] + (double)iiz * brl[d + 6];
        const double G2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
        coef[p] = (kx == 0 && ky == 0 && kz == 0) ? 0.0 : 4.0 * PI / G2;
      }
}

// egx(k, i) = exp(i 2 pi (i-1)(k-1) / n), initialization.f90:752-776; stored
// [k][i] as interleaved (re, im).  The conjugate table is its complex conjugate.
void sbo_dft_table(int n, double* eg) {
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) {
      const double a = 2.0 * PI * (double)(i * k) / (double)n;
      eg[2 * ((long)k * n + i)] = std::cos(a);
      eg[2 * ((long)k * n + i) + 1] = std::sin(a);
    }
}

// poisson_ft, src/poisson/poisson_periodic.f90:23-242 (one process): forward
// transforms along z, y, x with the conjugate tables, division by the number of
// grid points, multiplication by fg%coef, inverse transforms along z, y, x;
// Vh = real part.  rho, vh: (nx, ny, nz) interior, x fastest.
void sbo_poisson_ft(const int num[3], const double brl[9], const double* rho, double* vh) {
  const int nx = num[0], ny = num[1], nz = num[2];
  const long n = (long)nx * ny * nz;
  std::vector<double> coef(n), egx(2L * nx * nx), egy(2L * ny * ny), egz(2L * nz * nz);
  sbo_poisson_coef(num, brl, coef.data());
  sbo_dft_table(nx, egx.data());
  sbo_dft_table(ny, egy.data());
  sbo_dft_table(nz, egz.data());
  std::vector<double> a(2 * n), b(2 * n);
  auto at = [&](int x, int y, int z) { return (long)x + (long)nx * (y + (long)ny * z); };
  // one pass: out(k along axis) = sum_j T(k, j) * in(j along axis); conj picks
  // egXc (forward) or egX (inverse; egX(k, j) is symmetric in k, j)
  auto pass = [&](const double* in, bool in_real, double* out, int axis, bool conj) {
    const int na = axis == 0 ? nx : axis == 1 ? ny : nz;
    const double* T = axis == 0 ? egx.data() : axis == 1 ? egy.data() : egz.data();
    const double sg = conj ? -1.0 : 1.0;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const int k = axis == 0 ? x : axis == 1 ? y : z;
          double re = 0.0, im = 0.0;
          for (int j = 0; j < na; ++j) {
            const long q = axis == 0 ? at(j, y, z) : axis == 1 ? at(x, j, z) : at(x, y, j);
            const double tr = T[2 * ((long)k * na + j)], ti = sg * T[2 * ((long)k * na + j) + 1];
            const double vr = in_real ? in[q] : in[2 * q], vi = in_real ? 0.0 : in[2 * q + 1];
            re = re + (tr * vr - ti * vi);
            im = im + (tr * vi + ti * vr);
          }
          const long p = at(x, y, z);
          out[2 * p] = re;
          out[2 * p + 1] = im;
        }
  };
  pass(rho, true, a.data(), 2, true);
  pass(a.data(), false, b.data(), 1, true);
  pass(b.data(), false, a.data(), 0, true);
  for (long p = 0; p < n; ++p) {
    const double re = a[2 * p] / (double)n, im = a[2 * p + 1] / (double)n;
    a[2 * p] = coef[p] * re;
    a[2 * p + 1] = coef[p] * im;
  }
  pass(a.data(), false, b.data(), 2, false);
  pass(b.data(), false, a.data(), 1, false);
  pass(a.data(), false, b.data(), 0, false);
  for (long p = 0; p < n; ++p) vh[p] = b[2 * p];
}

// poisson_isolated_ft, src/poisson/poisson_isolated.f90:692-836 (one process),
// with the tables of init_reciprocal_grid_isolated_ft (src/common/initialization.f90:
// 823-1077): rho placed in the corner of a doubled (2nx, 2ny, 2nz) box of zeros,
// forward transforms along z, y, x of size 2n, division by 8 nx ny nz,
// multiplication by 4 pi / |G|^2 of the doubled cell (G = fold(k) b_d / 2,
// G = 0 dropped), inverse transforms along z, y, x, Vh = real part on the
// original nx x ny x nz corner.  Only the corner rows that carry data are formed
// and only those summed, as the reference's loop bounds do.  The reference's
// tables repeat the first n columns in the second n (egx(k, i + n) = egx(k, i));
// those columns only ever multiply the zero half, so the plain exp(2 pi i j k / 2n)
// is used for all j.  brl: primitive_b (3x3, diagonal for this box).
void sbo_poisson_isolated_ft(const int num[3], const double brl[9], const double* rho, double* vh) {
  const int n0[3] = {num[0], num[1], num[2]};
  const int m[3] = {2 * num[0], 2 * num[1], 2 * num[2]};
  const long M = (long)m[0] * m[1] * m[2];
  std::vector<double> eg[3];
  for (int d = 0; d < 3; ++d) {
    eg[d].resize(2L * m[d] * m[d]);
    sbo_dft_table(m[d], eg[d].data());
  }
  std::vector<double> a(2 * M, 0.0), b(2 * M, 0.0);
  auto at = [&](int x, int y, int z) { return (long)x + (long)m[0] * (y + (long)m[1] * z); };
  // one pass over the box [0,bx) x [0,by) x [0,bz) of outputs, summing the
  // first nsum inputs along `axis`
  auto pass = [&](const double* in, double* out, int axis, bool conj, int bx, int by, int bz, int nsum) {
    const double* T = eg[axis].data();
    const int na = m[axis];
    const double sg = conj ? -1.0 : 1.0;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < bz; ++z)
      for (int y = 0; y < by; ++y)
        for (int x = 0; x < bx; ++x) {
          const int k = axis == 0 ? x : axis == 1 ? y : z;
          double re = 0.0, im = 0.0;
          for (int j = 0; j < nsum; ++j) {
            const long q = axis == 0 ? at(j, y, z) : axis == 1 ? at(x, j, z) : at(x, y, j);
            const double tr = T[2 * ((long)k * na + j)], ti = sg * T[2 * ((long)k * na + j) + 1];
            const double vr = in[2 * q], vi = in[2 * q + 1];
            re = re + (tr * vr - ti * vi);
            im = im + (tr * vi + ti * vr);
          }
          const long p = at(x, y, z);
          out[2 * p] = re;
          out[2 * p + 1] = im;
        }
  };
  for (int z = 0; z < n0[2]; ++z)
    for (int y = 0; y < n0[1]; ++y)
      for (int x = 0; x < n0[0]; ++x) a[2 * at(x, y, z)] = rho[x + (long)n0[0] * (y + (long)n0[1] * z)];
  pass(a.data(), b.data(), 2, true, n0[0], n0[1], m[2], n0[2]);
  pass(b.data(), a.data(), 1, true, n0[0], m[1], m[2], n0[1]);
  pass(a.data(), b.data(), 0, true, m[0], m[1], m[2], n0[0]);
  const double ntot = 8.0 * n0[0] * n0[1] * n0[2];
  for (int z = 0; z < m[2]; ++z)
    for (int y = 0; y < m[1]; ++y)
      for (int x = 0; x < m[0]; ++x) {
        const long p = at(x, y, z);
        const int ix = fold(x, m[0]), iy = fold(y, m[1]), iz = fold(z, m[2]);
        const double g0 = (double)ix * brl[0] / 2.0, g1 = (double)iy * brl[4] / 2.0, g2 = (double)iz * brl[8] / 2.0;
        const double G2 = g0 * g0 + g1 * g1 + g2 * g2;
        const double cf = (ix == 0 && iy == 0 && iz == 0) ? 0.0 : 4.0 * PI / G2;
        b[2 * p] = cf * (b[2 * p] / ntot);
        b[2 * p + 1] = cf * (b[2 * p + 1] / ntot);
      }
  pass(b.data(), a.data(), 2, false, m[0], m[1], n0[2], m[2]);
  pass(a.data(), b.data(), 1, false, m[0], n0[1], n0[2], m[1]);
  pass(b.data(), a.data(), 0, false, n0[0], n0[1], n0[2], m[0]);
  for (int z = 0; z < n0[2]; ++z)
    for (int y = 0; y < n0[1]; ++y)
      for (int x = 0; x < n0[0]; ++x) vh[x + (long)n0[0] * (y + (long)n0[1] * z)] = a[2 * at(x, y, z)];
}

// update_vlocal, src/common/hamiltonian.f90:813-843: V_local(is) = Vpsl + Vh + Vxc(is).
void sbo_update_vlocal(long n, int nspin, const double* vpsl, const double* vh, const double* vxc, double* vloc) {
  for (int is = 0; is < nspin; ++is)
    for (long i = 0; i < n; ++i) vloc[is * n + i] = vpsl[i] + vh[i] + vxc[is * n + i];
}

}  // extern "C"
