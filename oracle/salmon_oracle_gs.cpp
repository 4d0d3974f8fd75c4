// salmon_oracle_gs.cpp -- ground-state pieces of the CPU oracle (test
// infrastructure only): the band-by-band preconditioned CG of gscg_rwf, the
// low-pass preconditioner, classical Gram-Schmidt (real and complex) and the
// real subspace diagonalisation.  Same layout conventions as salmon_oracle.cpp;
// real orbitals are rwf(x,y,z,ispin,io,ik=1) with the reference's array bounds.
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "salmon_oracle.h"

namespace {

struct G {
  const sbo_system* s;
  long nxa, nya, vol;
  explicit G(const sbo_system* s_) : s(s_) {
    nxa = s->ie_array[0] - s->is_array[0] + 1;
    nya = s->ie_array[1] - s->is_array[1] + 1;
    vol = nxa * nya * (s->ie_array[2] - s->is_array[2] + 1);
  }
  long a(int ix, int iy, int iz) const {
    return (ix - s->is_array[0]) + nxa * ((iy - s->is_array[1]) + nya * (long)(iz - s->is_array[2]));
  }
  int X(int j) const { return s->idx[j - (s->is[0] - 4)]; }
  int Y(int j) const { return s->idy[j - (s->is[1] - 4)]; }
  int Z(int j) const { return s->idz[j - (s->is[2] - 4)]; }
  long norb() const { return (long)s->nspin * s->no; }
  // orbital block of (ispin, io) for ik = 1 (1-based)
  long orb(int ispin, int io) const { return (ispin - 1) + (long)s->nspin * (io - 1); }
};

template <typename F>
void for_interior(const sbo_system* s, F f) {
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) f(ix, iy, iz);
}

// inner_product, conjugate_gradient.f90:384-425: rbox(ispin,io) = hvol*sum x*y
void inner_product(const sbo_system* s, const G& g, const double* x, const double* y, double* out) {
#pragma omp parallel for collapse(2)
  for (int io = 1; io <= s->no; ++io)
    for (int is = 1; is <= s->nspin; ++is) {
      const long o = g.orb(is, io);
      const double* a = x + g.vol * o;
      const double* b = y + g.vol * o;
      double sum0 = 0.0;
      for_interior(s, [&](int ix, int iy, int iz) {
        const long p = g.a(ix, iy, iz);
        sum0 = sum0 + a[p] * b[p];
      });
      out[o] = sum0 * s->hvol;
    }
}

// Jacobi eigensolver for a symmetric n x n matrix (column-major); eigenvalues
// ascending with their column eigenvectors, as dsyev('V','U') returns them.
void jacobi_eigh(int n, std::vector<double> A, double* evals, double* evecs) {
  std::vector<double> V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  auto at = [&](int i, int j) -> double& { return A[(size_t)j * n + i]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < j; ++i) off += at(i, j) * at(i, j);
    if (off < 1e-30) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = at(p, q);
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (at(q, q) - at(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = at(k, p), akq = at(k, q);
          at(k, p) = c * akp - sn * akq;
          at(k, q) = sn * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = at(p, k), aqk = at(q, k);
          at(p, k) = c * apk - sn * aqk;
          at(q, k) = sn * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
          V[(size_t)p * n + k] = c * vkp - sn * vkq;
          V[(size_t)q * n + k] = sn * vkp + c * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (at(ord[j], ord[j]) < at(ord[i], ord[i])) std::swap(ord[i], ord[j]);
  for (int i = 0; i < n; ++i) {
    evals[i] = at(ord[i], ord[i]);
    // sign convention: largest-magnitude component positive
    int im = 0;
    for (int k = 1; k < n; ++k)
      if (std::fabs(V[(size_t)ord[i] * n + k]) > std::fabs(V[(size_t)ord[i] * n + im])) im = k;
    const double sg = V[(size_t)ord[i] * n + im] < 0 ? -1.0 : 1.0;
    for (int k = 0; k < n; ++k) evecs[(size_t)i * n + k] = sg * V[(size_t)ord[i] * n + k];
  }
}

}  // namespace

extern "C" {

// dstencil_preconditioning, preconditioning.f90:25-77 (low-pass filter,
// 2nd-order Laplacian), applied to every orbital of the block.
void sbo_precond_real(const sbo_system* s, const double* gk, double* pre_gk, double alpha) {
  G g(s);
  const double omega = 2.0 * (1.0 - alpha);
  const double h0 = s->hgs[0], h1 = s->hgs[1], h2 = s->hgs[2];
  const double d = -0.5 * ((-2.0) / (h0 * h0) + (-2.0) / (h1 * h1) + (-2.0) / (h2 * h2));
  const long norb = g.norb();
  for (long o = 0; o < norb; ++o) {
    const double* t = gk + g.vol * o;
    double* h = pre_gk + g.vol * o;
#pragma omp parallel for collapse(2)
    for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
      for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          const double c = t[g.a(ix, iy, iz)];
          const double v = (t[g.a(g.X(ix + 1), iy, iz)] - 2.0 * c + t[g.a(g.X(ix - 1), iy, iz)]) / (h0 * h0) +
                           (t[g.a(ix, g.Y(iy + 1), iz)] - 2.0 * c + t[g.a(ix, g.Y(iy - 1), iz)]) / (h1 * h1) +
                           (t[g.a(ix, iy, g.Z(iz + 1))] - 2.0 * c + t[g.a(ix, iy, g.Z(iz - 1))]) / (h2 * h2);
          h[g.a(ix, iy, iz)] = omega / d * (2.0 * c - omega / d * (-0.5 * v));
        }
  }
}

// gscg_rwf, conjugate_gradient.f90:21-466 (real orbitals, one k, im = 1).
// work holds 7 orbital blocks: xk, hxk, pk, gk, pre_gk, pko, hwf.
// esp_out(nspin*no) receives the final <xk|H|xk> (Rayleigh quotients).
void sbo_gscg_rwf(const sbo_system* s, int ncg, double* psi, double* work, int precondition, double alpha_pre,
                  double* esp_out) {
  G g(s);
  const long n = g.vol * g.norb();
  const long norb = g.norb();
  double *xk = work, *hxk = work + n, *pk = work + 2 * n, *gk = work + 3 * n, *pre = work + 4 * n,
         *pko = work + 5 * n, *hwf = work + 6 * n;
  std::memset(work, 0, sizeof(double) * 7 * n);
  std::vector<double> sum(norb), xkxk(norb), xkHxk(norb), xkHpk(norb), pkHpk(norb), gkgk(norb), uk(norb),
      ev(norb), cx(norb), cp(norb), zs(norb);
  auto each = [&](auto f) {
#pragma omp parallel for
    for (long o = 0; o < norb; ++o) {
      for_interior(s, [&](int ix, int iy, int iz) { f(o, g.vol * o + g.a(ix, iy, iz)); });
    }
  };
  each([&](long, long p) { xk[p] = psi[p]; });
  sbo_hpsi_real(s, xk, hxk);
  inner_product(s, g, xk, hxk, xkHxk.data());
  for (int iter = 1; iter <= ncg; ++iter) {
    each([&](long o, long p) { gk[p] = hxk[p] - xkHxk[o] * xk[p]; });
    if (precondition) {
      sbo_precond_real(s, gk, pre, alpha_pre);
      inner_product(s, g, pre, gk, sum.data());
    } else {
      inner_product(s, g, gk, gk, sum.data());
    }
    if (iter == 1) {
      for (long o = 0; o < norb; ++o) uk[o] = 0.0;
    } else {
      for (long o = 0; o < norb; ++o) uk[o] = (std::fabs(gkgk[o]) > 1e-16) ? sum[o] / gkgk[o] : 0.0;
    }
    if (precondition) each([&](long o, long p) { pk[p] = pre[p] + uk[o] * pk[p]; });
    else each([&](long o, long p) { pk[p] = gk[p] + uk[o] * pk[p]; });
    gkgk = sum;
    inner_product(s, g, xk, pk, zs.data());
    each([&](long o, long p) { pko[p] = pk[p] - zs[o] * xk[p]; });
    inner_product(s, g, pko, pko, sum.data());
    each([&](long o, long p) { pko[p] = pko[p] / std::sqrt(sum[o]); });
    sbo_hpsi_real(s, pko, hwf);
    inner_product(s, g, xk, hwf, xkHpk.data());
    inner_product(s, g, pko, hwf, pkHpk.data());
    for (long o = 0; o < norb; ++o) {
      ev[o] = 0.5 * ((xkHxk[o] + pkHpk[o]) -
                     std::sqrt((xkHxk[o] - pkHpk[o]) * (xkHxk[o] - pkHpk[o]) + 4.0 * std::fabs(xkHpk[o]) * std::fabs(xkHpk[o])));
      if (std::fabs(ev[o] - xkHxk[o]) > 1e-16) {
        cx[o] = xkHpk[o] / (ev[o] - xkHxk[o]);
        cp[o] = 1.0 / std::sqrt(1.0 + std::fabs(cx[o]) * std::fabs(cx[o]));
        cx[o] = cx[o] * cp[o];
      } else {
        cx[o] = 1.0;
        cp[o] = 0.0;
      }
    }
    each([&](long o, long p) {
      xk[p] = cx[o] * xk[p] + cp[o] * pko[p];
      hxk[p] = cx[o] * hxk[p] + cp[o] * hwf[p];
    });
    inner_product(s, g, xk, hxk, xkHxk.data());
    inner_product(s, g, xk, xk, xkxk.data());
    each([&](long o, long p) {
      if (1e-16 < std::fabs(xkxk[o]) && std::fabs(xkxk[o]) <= 1e30) psi[p] = xk[p] / std::sqrt(xkxk[o]);
    });
  }
  if (esp_out)
    for (long o = 0; o < norb; ++o) esp_out[o] = xkHxk[o] / xkxk[o];
}

// gram_schmidt_col_real8, gram_schmidt_orth.f90:59-230 (classical GS: all
// coefficients from the original vector, then one subtraction).
void sbo_gram_schmidt_real(const sbo_system* s, double* psi) {
  G g(s);
  std::vector<double> wf1(g.vol), exc(g.vol);
  for (int is = 1; is <= s->nspin; ++is)
    for (int io1 = 1; io1 <= s->no; ++io1) {
      double* w1 = psi + g.vol * g.orb(is, io1);
      std::memcpy(wf1.data(), w1, sizeof(double) * g.vol);
      std::vector<double> coeff(s->no, 0.0);
      for (int io2 = 1; io2 < io1; ++io2) {
        const double* w2 = psi + g.vol * g.orb(is, io2);
        double p = 0.0;
        for_interior(s, [&](int ix, int iy, int iz) { p = p + w2[g.a(ix, iy, iz)] * wf1[g.a(ix, iy, iz)]; });
        coeff[io2 - 1] = p * s->hvol;
      }
      std::fill(exc.begin(), exc.end(), 0.0);
      for (int io2 = 1; io2 < io1; ++io2) {
        const double* w2 = psi + g.vol * g.orb(is, io2);
        for_interior(s, [&](int ix, int iy, int iz) {
          const long p = g.a(ix, iy, iz);
          exc[p] = coeff[io2 - 1] * w2[p] + exc[p];
        });
      }
      for_interior(s, [&](int ix, int iy, int iz) {
        const long p = g.a(ix, iy, iz);
        wf1[p] = -1.0 * exc[p] + wf1[p];
      });
      double nrm = 0.0;
      for_interior(s, [&](int ix, int iy, int iz) { nrm = nrm + wf1[g.a(ix, iy, iz)] * wf1[g.a(ix, iy, iz)]; });
      nrm = nrm * s->hvol;
      const double sc = 1.0 / std::sqrt(nrm);
      for_interior(s, [&](int ix, int iy, int iz) { w1[g.a(ix, iy, iz)] = sc * wf1[g.a(ix, iy, iz)]; });
    }
}

// gram_schmidt_col_complex8, gram_schmidt_orth.f90:1069-1242, per (ik, ispin).
void sbo_gram_schmidt_complex(const sbo_system* s, double* psi_d) {
  G g(s);
  typedef std::complex<double> zc;
  zc* psi = reinterpret_cast<zc*>(psi_d);
  std::vector<zc> wf1(g.vol), exc(g.vol);
  for (int ik = 1; ik <= s->nk; ++ik)
    for (int is = 1; is <= s->nspin; ++is)
      for (int io1 = 1; io1 <= s->no; ++io1) {
        auto O = [&](int io) { return (is - 1) + (long)s->nspin * ((io - 1) + (long)s->no * (ik - 1)); };
        zc* w1 = psi + g.vol * O(io1);
        std::copy(w1, w1 + g.vol, wf1.begin());
        std::vector<zc> coeff(s->no, zc(0, 0));
        for (int io2 = 1; io2 < io1; ++io2) {
          const zc* w2 = psi + g.vol * O(io2);
          zc p(0, 0);
          for_interior(s, [&](int ix, int iy, int iz) { p = p + std::conj(w2[g.a(ix, iy, iz)]) * wf1[g.a(ix, iy, iz)]; });
          coeff[io2 - 1] = p * s->hvol;
        }
        std::fill(exc.begin(), exc.end(), zc(0, 0));
        for (int io2 = 1; io2 < io1; ++io2) {
          const zc* w2 = psi + g.vol * O(io2);
          for_interior(s, [&](int ix, int iy, int iz) {
            const long p = g.a(ix, iy, iz);
            exc[p] = coeff[io2 - 1] * w2[p] + exc[p];
          });
        }
        for_interior(s, [&](int ix, int iy, int iz) {
          const long p = g.a(ix, iy, iz);
          wf1[p] = -exc[p] + wf1[p];
        });
        double nrm = 0.0;
        for_interior(s, [&](int ix, int iy, int iz) { nrm = nrm + std::norm(wf1[g.a(ix, iy, iz)]); });
        nrm = nrm * s->hvol;
        const double sc = 1.0 / std::sqrt(nrm);
        for_interior(s, [&](int ix, int iy, int iz) { w1[g.a(ix, iy, iz)] = sc * wf1[g.a(ix, iy, iz)]; });
      }
}

// ssdg_rwf, subspace_diagonalization.f90:62-238 (single orbital domain), with
// a Jacobi eigensolver in place of LAPACK dsyev.  work: one orbital block.
void sbo_subspace_diag_real(const sbo_system* s, double* psi, double* work, double* evals) {
  G g(s);
  const int no = s->no;
  double* shpsi = work;
  sbo_hpsi_real(s, psi, shpsi);
  for (int is = 1; is <= s->nspin; ++is) {
    std::vector<double> mat((size_t)no * no), evec((size_t)no * no);
#pragma omp parallel for collapse(2)
    for (int io1 = 1; io1 <= no; ++io1)
      for (int io2 = 1; io2 <= no; ++io2) {
        const double* a = psi + g.vol * g.orb(is, io1);
        const double* b = shpsi + g.vol * g.orb(is, io2);
        double c = 0.0;
        for_interior(s, [&](int ix, int iy, int iz) { c = c + a[g.a(ix, iy, iz)] * b[g.a(ix, iy, iz)]; });
        mat[(size_t)(io2 - 1) * no + (io1 - 1)] = c * s->hvol;
      }
    // symmetrise (dsyev reads the upper triangle only)
    for (int j = 0; j < no; ++j)
      for (int i = j + 1; i < no; ++i) mat[(size_t)j * no + i] = mat[(size_t)i * no + j];
    jacobi_eigh(no, mat, evals + (size_t)(is - 1) * no, evec.data());
    // shpsi(io1) = sum_io2 evec(io2, io1) psi(io2); then normalise into psi
    std::vector<double> out((size_t)g.vol * no, 0.0);
#pragma omp parallel for
    for (int io1 = 1; io1 <= no; ++io1) {
      double* o1 = out.data() + g.vol * (io1 - 1);
      for (int io2 = 1; io2 <= no; ++io2) {
        const double e = evec[(size_t)(io1 - 1) * no + (io2 - 1)];
        const double* p2 = psi + g.vol * g.orb(is, io2);
        for_interior(s, [&](int ix, int iy, int iz) {
          const long p = g.a(ix, iy, iz);
          o1[p] = o1[p] + e * p2[p];
        });
      }
      double r = 0.0;
      for_interior(s, [&](int ix, int iy, int iz) { r = r + o1[g.a(ix, iy, iz)] * o1[g.a(ix, iy, iz)]; });
      const double sc = std::sqrt(r * s->hvol);
      for (long p = 0; p < g.vol; ++p) o1[p] = o1[p] / sc;
    }
    for (int io1 = 1; io1 <= no; ++io1)
      std::memcpy(psi + g.vol * g.orb(is, io1), out.data() + g.vol * (io1 - 1), sizeof(double) * g.vol);
  }
}

void sbo_inner_product_real(const sbo_system* s, const double* x, const double* y, double* out) {
  G g(s);
  inner_product(s, g, x, y, out);
}

}  // extern "C"
