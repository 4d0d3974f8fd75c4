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

// PZxc_sp, src/xc/builtin_pz_sp.f90:43-95: Slater exchange with the spin
// interpolation f(zeta) = ((1+zeta)^(4/3) + (1-zeta)^(4/3) - 2) / (2^(4/3) - 2)
// between the unpolarised (U) and polarised (P) Perdew-Zunger 1981 correlation
// fits; vxc_s(js) for js = up (sign +1), down (-1).
void pzxc_sp(double trho, const double trho_s[2], double* exc_out, double vxc_s[2]) {
  const double gammaU = -0.1423, gammaP = -0.0843, beta1U = 1.0529, beta2U = 0.3334, beta1P = 1.3981,
               beta2P = 0.2611, AU = 0.0311, BU = -0.048, CU = 0.002, DU = -0.0116, AP = 0.01555, BP = -0.0269,
               CP = 0.0007, DP = -0.0048;
  const double sgn[2] = {1.0, -1.0};
  const double rs = std::pow(3.0 / (4.0 * PI * trho), 1.0 / 3.0);
  const double zeta = (trho_s[0] - trho_s[1]) / trho;
  const double fden = std::pow(2.0, 4.0 / 3.0) - 2.0;
  const double sf = (std::pow(1.0 + zeta, 4.0 / 3.0) + std::pow(1.0 - zeta, 4.0 / 3.0) - 2.0) / fden;
  const double dsf = 4.0 / 3.0 * (std::pow(1.0 + zeta, 1.0 / 3.0) - std::pow(1.0 - zeta, 1.0 / 3.0)) / fden;
  const double cx = 3.0 / 4.0 * std::pow(3.0 / (2 * PI), 2.0 / 3.0);
  const double a = -std::pow(2.0, 1.0 / 3.0) + 1.0;
  double exc = -cx / rs + a * cx / rs * sf;
  for (int js = 0; js < 2; ++js)
    vxc_s[js] = exc - 1.0 / 3.0 * cx / rs + 1.0 / 3.0 * a * cx / rs * sf + a * cx / rs * (sgn[js] - zeta) * dsf;
  double ecu, ecp, vcu, vcp;
  if (rs > 1.0) {
    const double q = std::sqrt(rs);
    const double du = 1.0 + beta1U * q + beta2U * rs, dp = 1.0 + beta1P * q + beta2P * rs;
    ecu = gammaU / du;
    ecp = gammaP / dp;
    vcu = gammaU * (1.0 + 7.0 / 6.0 * beta1U * q + 4.0 / 3.0 * beta2U * rs) / (du * du);
    vcp = gammaP * (1.0 + 7.0 / 6.0 * beta1P * q + 4.0 / 3.0 * beta2P * rs) / (dp * dp);
  } else {
    const double l = std::log(rs);
    ecu = AU * l + BU + CU * rs * l + DU * rs;
    ecp = AP * l + BP + CP * rs * l + DP * rs;
    vcu = AU * l + (BU - AU / 3.0) + 2.0 / 3.0 * CU * rs * l + (2.0 * DU - CU) / 3.0 * rs;
    vcp = AP * l + (BP - AP / 3.0) + 2.0 / 3.0 * CP * rs * l + (2.0 * DP - CP) / 3.0 * rs;
  }
  exc = exc + ecu + sf * (ecp - ecu);
  for (int js = 0; js < 2; ++js) vxc_s[js] = vxc_s[js] + vcu + sf * (vcp - vcu) + (ecp - ecu) * (sgn[js] - zeta) * dsf;
  *exc_out = exc;
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

// exchange_correlation for nspin = 2 with xc = 'PZ' (exc_cor_pz_sp,
// builtin_pz_sp.f90:23-40): rho_s(n, 2), trho = rho_up + rho_dn + 1e-20,
// trho_s = rho_s + 5e-21, vxc_s(n, 2), E_xc = hvol * sum(e_xc trho) summed
// with x fastest.
void sbo_exc_cor_pz_sp(long n, const double* rho_s, double hvol, double* vxc_s, double* E_xc) {
  std::vector<double> eexc(n);
#pragma omp parallel for
  for (long i = 0; i < n; ++i) {
    const double trho = rho_s[i] + rho_s[n + i] + 1e-20;
    const double ts[2] = {rho_s[i] + 5e-21, rho_s[n + i] + 5e-21};
    double e, v[2];
    pzxc_sp(trho, ts, &e, v);
    eexc[i] = e * trho;
    vxc_s[i] = v[0];
    vxc_s[n + i] = v[1];
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


// ---- poisson_isolated_cg with the multipole boundary ---------------------------
//
// poisson_isolated_cg (src/poisson/poisson_isolated.f90:30-221, one process),
// laplacian_poisson (:223-257) and poisson_boundary (:259-690), with the pole
// tables of make_corr_pole (src/poisson/init_poisson.f90:23-219) and the face
// halos of set_ig_bound (:223-299).  Grid from the sbo_system (is:ie, hgs,
// coef_lap0, coef_lap); rho and vh interior arrays (x fastest); vh is the start
// value on entry and the solution on exit.  layout 1: one pole at the origin;
// 2: one pole per atom over its nearest grid points; 3: box cells of about
// 8 A with their charge centroid as centre.  *iterations is poisson%iterVh
// (maxiter + 1 when not converged).
void sbo_poisson_isolated_cg(const sbo_system* s, const double* rho, double* vh, int layout, int lmax,
                             const double* rion, int natom, const int npole_xyz[3], double threshold,
                             int maxiter, int* iterations) {
  const int ND = 4;
  const int nx = s->ie[0] - s->is[0] + 1, ny = s->ie[1] - s->is[1] + 1, nz = s->ie[2] - s->is[2] + 1;
  const long N = (long)nx * ny * nz;
  const int px = nx + 2 * ND, py = ny + 2 * ND, pz = nz + 2 * ND;
  const long P = (long)px * py * pz;
  auto pa = [&](int x, int y, int z) {  // padded index of interior offsets (x, y, z) in [-4, n + 4)
    return (long)(x + ND) + px * ((long)(y + ND) + py * (long)(z + ND));
  };
  auto ri = [&](int x, int y, int z) { return (long)x + nx * ((long)y + (long)ny * z); };
  auto coord = [&](int d, int i) {  // i: global index
    return (s->lg_num[d] % 2 == 1) ? (double)i * s->hgs[d] : ((double)i - 0.5) * s->hgs[d];
  };
  const double hvol = s->hvol;
  const int nlm = (lmax + 1) * (lmax + 1);
  // ---- poles: centres, point lists and multipole moments (poisson_boundary)
  std::vector<std::vector<long>> pts;  // interior offsets per pole, in z, y, x loop order
  std::vector<double> cen;             // 3 per pole
  std::vector<int> itrho;
  if (layout == 1) {
    pts.resize(1);
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) pts[0].push_back(ri(x, y, z));
    cen.assign(3, 0.0);
    itrho.assign(1, 1);
  } else if (layout == 2) {
    pts.resize(natom);
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          double rmin = 1e6;
          int amin = 0;
          for (int a = 0; a < natom; ++a) {
            const double dx = coord(0, x + s->is[0]) - rion[3 * a], dy = coord(1, y + s->is[1]) - rion[3 * a + 1],
                         dz = coord(2, z + s->is[2]) - rion[3 * a + 2];
            const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (r < rmin) {
              rmin = r;
              amin = a;
            }
          }
          pts[amin].push_back(ri(x, y, z));
        }
    cen.assign(rion, rion + 3 * natom);
    itrho.assign(natom, 1);
  } else {
    const int n1 = npole_xyz[0], n2 = npole_xyz[1], n3 = npole_xyz[2];
    const int ncell = n1 * n2 * n3;
    pts.resize(ncell);
    for (int j3 = 0; j3 < n3; ++j3)
      for (int j2 = 0; j2 < n2; ++j2)
        for (int j1 = 0; j1 < n1; ++j1) {
          const int ib = j1 + n1 * (j2 + n2 * j3);
          for (int z = j3 * nz / n3; z <= (j3 + 1) * nz / n3 - 1; ++z)
            for (int y = j2 * ny / n2; y <= (j2 + 1) * ny / n2 - 1; ++y)
              for (int x = j1 * nx / n1; x <= (j1 + 1) * nx / n1 - 1; ++x) pts[ib].push_back(ri(x, y, z));
        }
    cen.assign(3 * (size_t)ncell, 0.0);
    itrho.assign(ncell, 0);
    for (int c = 0; c < ncell; ++c) {
      double nd[4] = {0, 0, 0, 0};
      for (long q : pts[c]) {
        const int x = (int)(q % nx), y = (int)((q / nx) % ny), z = (int)(q / ((long)nx * ny));
        nd[0] = nd[0] + rho[q] * coord(0, x + s->is[0]);
        nd[1] = nd[1] + rho[q] * coord(1, y + s->is[1]);
        nd[2] = nd[2] + rho[q] * coord(2, z + s->is[2]);
        nd[3] = nd[3] + rho[q];
      }
      if (nd[3] * hvol >= 1e-12) {
        itrho[c] = 1;
        for (int d = 0; d < 3; ++d) cen[3 * c + d] = nd[d] / nd[3];
      }
    }
  }
  const int npole = (int)pts.size();
  std::vector<double> rholm((size_t)npole * nlm, 0.0);
  for (int c = 0; c < npole; ++c) {
    if (!itrho[c]) continue;
    for (int lm = 0; lm < nlm; ++lm) {
      int l = 0;
      while ((l + 1) * (l + 1) <= lm) ++l;
      double acc = 0.0;
      for (long q : pts[c]) {
        const int x = (int)(q % nx), y = (int)((q / nx) % ny), z = (int)(q / ((long)nx * ny));
        const double xx = coord(0, x + s->is[0]) - cen[3 * c], yy = coord(1, y + s->is[1]) - cen[3 * c + 1],
                     zz = coord(2, z + s->is[2]) - cen[3 * c + 2];
        const double rr = std::sqrt(xx * xx + yy * yy + zz * zz) + 1e-50;
        double rl = 1.0;
        for (int i = 0; i < l; ++i) rl *= rr;
        acc = acc + rl * sbo_ylm(xx / rr, yy / rr, zz / rr, lm) * rho[q] * hvol;
      }
      rholm[(size_t)c * nlm + lm] = acc;
    }
  }
  // ---- CG (pk carries the boundary values in its face halos for the first Laplacian)
  std::vector<double> pk(P, 0.0), zk(P, 0.0), rlap(N, 0.0);
  auto boundary = [&](int gx, int gy, int gz) {  // global indices of a halo point
    double v = 0.0;
    for (int c = 0; c < npole; ++c) {
      if (!itrho[c]) continue;
      const double xx = coord(0, gx) - cen[3 * c], yy = coord(1, gy) - cen[3 * c + 1], zz = coord(2, gz) - cen[3 * c + 2];
      const double rinv = 1.0 / (std::sqrt(xx * xx + yy * yy + zz * zz) + 1e-50);
      double sum1 = 0.0, rp = rinv;
      int lcur = 0;
      for (int lm = 0; lm < nlm; ++lm) {
        int l = 0;
        while ((l + 1) * (l + 1) <= lm) ++l;
        if (l != lcur) {
          rp *= rinv;
          lcur = l;
        }
        sum1 = sum1 + sbo_ylm(xx * rinv, yy * rinv, zz * rinv, lm) * rp * rholm[(size_t)c * nlm + lm];
      }
      v = v + sum1;
    }
    return v;
  };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int h = 0; h < ND; ++h) {
        pk[pa(-ND + h, y, z)] = boundary(s->is[0] - ND + h, y + s->is[1], z + s->is[2]);
        pk[pa(nx + h, y, z)] = boundary(s->ie[0] + 1 + h, y + s->is[1], z + s->is[2]);
      }
  for (int z = 0; z < nz; ++z)
    for (int h = 0; h < ND; ++h)
      for (int x = 0; x < nx; ++x) {
        pk[pa(x, -ND + h, z)] = boundary(x + s->is[0], s->is[1] - ND + h, z + s->is[2]);
        pk[pa(x, ny + h, z)] = boundary(x + s->is[0], s->ie[1] + 1 + h, z + s->is[2]);
      }
  for (int h = 0; h < ND; ++h)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        pk[pa(x, y, -ND + h)] = boundary(x + s->is[0], y + s->is[1], s->is[2] - ND + h);
        pk[pa(x, y, nz + h)] = boundary(x + s->is[0], y + s->is[1], s->ie[2] + 1 + h);
      }
  const double lap0 = s->coef_lap0;
  const double* lt = s->coef_lap;  // lapt(i, d) at lt[i + 4 d]
  auto laplacian = [&]() {
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const long c = pa(x, y, z);
          const long sx = 1, sy = px, sz = (long)px * py;
          double t = 0.0;
          t = lt[0] * (pk[c + sx] + pk[c - sx]);
          t = t + lt[1] * (pk[c + 2 * sx] + pk[c - 2 * sx]);
          t = t + lt[2] * (pk[c + 3 * sx] + pk[c - 3 * sx]);
          t = t + lt[3] * (pk[c + 4 * sx] + pk[c - 4 * sx]);
          t = t + lt[4] * (pk[c + sy] + pk[c - sy]);
          t = t + lt[5] * (pk[c + 2 * sy] + pk[c - 2 * sy]);
          t = t + lt[6] * (pk[c + 3 * sy] + pk[c - 3 * sy]);
          t = t + lt[7] * (pk[c + 4 * sy] + pk[c - 4 * sy]);
          t = t + lt[8] * (pk[c + sz] + pk[c - sz]);
          t = t + lt[9] * (pk[c + 2 * sz] + pk[c - 2 * sz]);
          t = t + lt[10] * (pk[c + 3 * sz] + pk[c - 3 * sz]);
          t = t + lt[11] * (pk[c + 4 * sz] + pk[c - 4 * sz]);
          rlap[ri(x, y, z)] = -2.0 * lap0 * pk[c] + t;
        }
  };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        pk[pa(x, y, z)] = vh[ri(x, y, z)];
        zk[pa(x, y, z)] = -4.0 * PI * rho[ri(x, y, z)];
      }
  laplacian();
  std::fill(pk.begin(), pk.end(), 0.0);
  double sum1 = 0.0;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long c = pa(x, y, z);
        zk[c] = zk[c] - rlap[ri(x, y, z)];
        pk[c] = zk[c];
        sum1 = sum1 + zk[c] * zk[c] * hvol;
      }
  int iter = 1;
  for (; iter <= maxiter; ++iter) {
    laplacian();
    double tot = 0.0;
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) tot = tot + zk[pa(x, y, z)] * rlap[ri(x, y, z)];
    const double ak = sum1 / tot / hvol;
    double z2 = 0.0;
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const long c = pa(x, y, z), r = ri(x, y, z);
          vh[r] = vh[r] + ak * pk[c];
          zk[c] = zk[c] - ak * rlap[r];
          z2 = z2 + zk[c] * zk[c];
        }
    const double sum2 = z2 * hvol;
    if (std::fabs(sum2) < threshold * (double)N) break;
    const double ck = sum2 / sum1;
    sum1 = sum2;
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const long c = pa(x, y, z);
          pk[c] = zk[c] + ck * pk[c];
        }
  }
  *iterations = iter;
}

// Ylm of src/math/salmon_math.f90:386-426 (real harmonics with the normalisation
// sqrt(4 pi / (2l + 1)) r^l Y_lm, as polynomials of x, y, z), lm = l^2 + l + m.
double sbo_ylm(double x, double y, double z, int lm) {
  const double r2 = x * x + y * y + z * z;
  switch (lm) {
    case 0: return 1.0;
    case 1: return -y;
    case 2: return z;
    case 3: return -x;
    case 4: return std::sqrt(3.0) * x * y;
    case 5: return -std::sqrt(3.0) * y * z;
    case 6: return (3.0 * z * z - r2) / 2.0;
    case 7: return -std::sqrt(3.0) * x * z;
    case 8: return std::sqrt(3.0 / 4.0) * (x * x - y * y);
    case 9: return -std::sqrt(5.0 / 8.0) * y * (3 * x * x - y * y);
    case 10: return std::sqrt(15.0) * x * y * z;
    case 11: return -std::sqrt(3.0 / 8.0) * y * (5.0 * z * z - r2);
    case 12: return z * (5.0 * z * z - 3 * r2) / 2.0;
    case 13: return -std::sqrt(3.0 / 8.0) * x * (5.0 * z * z - r2);
    case 14: return std::sqrt(15.0 / 4.0) * z * (x * x - y * y);
    case 15: return -std::sqrt(5.0 / 8.0) * x * (x * x - 3.0 * y * y);
    case 16: return std::sqrt(35.0) / 2.0 * x * y * (x * x - y * y);
    case 17: return -std::sqrt(35.0 / 8.0) * y * z * (3.0 * x * x - y * y);
    case 18: return std::sqrt(5.0) / 2.0 * x * y * (7.0 * z * z - r2);
    case 19: return -std::sqrt(5.0 / 8.0) * y * z * (7.0 * z * z - 3.0 * r2);
    case 20: return (35.0 * z * z * z * z - 30.0 * z * z * r2 + 3.0 * r2 * r2) / 8.0;
    case 21: return -std::sqrt(5.0 / 8.0) * x * z * (7.0 * z * z - 3.0 * r2);
    case 22: return std::sqrt(5.0) / 4.0 * (7.0 * z * z - r2) * (x * x - y * y);
    case 23: return -std::sqrt(35.0 / 8.0) * x * z * (x * x - 3.0 * y * y);
    case 24: return std::sqrt(35.0) / 8.0 * (x * x * x * x + y * y * y * y - 6.0 * x * x * y * y);
    default: return 0.0;
  }
}

}  // extern "C"
