// salmon_oracle.cpp -- CPU oracle (test infrastructure only) for the SALMON
// RT-TDDFT propagation hot path.  Each function restates one reference routine
// (SALMON v2.2.0 file:line cited at the function) with the same loop nesting
// and summation order, on the reference's own array layout.  See
// salmon_oracle.h for the parity status.
#include "salmon_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> zc_t;

namespace {

constexpr int Nd = 4;

struct Idx {
  const sbo_system* s;
  long nxa, nya, nza, vol;
  long nx, ny, nz;
  explicit Idx(const sbo_system* s_) : s(s_) {
    nxa = s->ie_array[0] - s->is_array[0] + 1;
    nya = s->ie_array[1] - s->is_array[1] + 1;
    nza = s->ie_array[2] - s->is_array[2] + 1;
    vol = nxa * nya * nza;
    nx = s->ie[0] - s->is[0] + 1;
    ny = s->ie[1] - s->is[1] + 1;
    nz = s->ie[2] - s->is[2] + 1;
  }
  // offset of (ix,iy,iz) inside one orbital block (Fortran bounds)
  inline long a(int ix, int iy, int iz) const {
    return (ix - s->is_array[0]) + nxa * ((iy - s->is_array[1]) + nya * (long)(iz - s->is_array[2]));
  }
  // offset inside an interior-shaped (is:ie) scalar field
  inline long r(int ix, int iy, int iz) const {
    return (ix - s->is[0]) + nx * ((iy - s->is[1]) + ny * (long)(iz - s->is[2]));
  }
  inline int X(int j) const { return s->idx[j - (s->is[0] - Nd)]; }
  inline int Y(int j) const { return s->idy[j - (s->is[1] - Nd)]; }
  inline int Z(int j) const { return s->idz[j - (s->is[2] - Nd)]; }
  // orbital block index of (ispin, io, ik), all 1-based
  inline long orb(int ispin, int io, int ik) const {
    return (ispin - 1) + (long)s->nspin * ((io - 1) + (long)s->no * (ik - 1));
  }
  long norb() const { return (long)s->nspin * s->no * s->nk; }
};

inline zc_t ld(const double* p, long off) { return zc_t(p[2 * off], p[2 * off + 1]); }
inline void st(double* p, long off, zc_t v) { p[2 * off] = v.real(); p[2 * off + 1] = v.imag(); }

// Fortran complex*complex is (ac-bd, ad+bc); std::complex operator* on gcc may
// take the C99 Annex G NaN-recovery path, which only differs for inf/nan.
inline zc_t cmul(zc_t a, zc_t b) {
  return zc_t(a.real() * b.real() - a.imag() * b.imag(),
              a.real() * b.imag() + a.imag() * b.real());
}
inline zc_t rmul(double r, zc_t a) { return zc_t(r * a.real(), r * a.imag()); }
// abs(z)**2 as the reference evaluates it (hypot, then square)
inline double abs2(zc_t a) { double h = std::hypot(a.real(), a.imag()); return h * h; }

// One orbital of the 25-point complex stencil.
// zstencil_core/typical/seq.f90:17-127 (and omp.f90:22-164 when rgrid-parallel).
void zstencil_one(const sbo_system* s, const Idx& I, const double* tpsi, double* htpsi,
                  const double* V, double lap0, const double* lapt, const double* nabt,
                  bool omp_grid) {
  const int zs = s->is[2], ze = s->ie[2], ys = s->is[1], ye = s->ie[1];
  const int xs = s->is[0], xe = s->ie[0];
#pragma omp parallel for collapse(2) if (omp_grid)
  for (int iz = zs; iz <= ze; ++iz)
    for (int iy = ys; iy <= ye; ++iy)
      for (int ix = xs; ix <= xe; ++ix) {
        zc_t t[8];
        // x: t(1..8) = psi(x+4 .. x+1, x-1 .. x-4)
        t[0] = ld(tpsi, I.a(I.X(ix + 4), iy, iz));
        t[1] = ld(tpsi, I.a(I.X(ix + 3), iy, iz));
        t[2] = ld(tpsi, I.a(I.X(ix + 2), iy, iz));
        t[3] = ld(tpsi, I.a(I.X(ix + 1), iy, iz));
        t[4] = ld(tpsi, I.a(I.X(ix - 1), iy, iz));
        t[5] = ld(tpsi, I.a(I.X(ix - 2), iy, iz));
        t[6] = ld(tpsi, I.a(I.X(ix - 3), iy, iz));
        t[7] = ld(tpsi, I.a(I.X(ix - 4), iy, iz));
        zc_t v = rmul(lapt[0], t[3] + t[4]) + rmul(lapt[1], t[2] + t[5]) +
                 rmul(lapt[2], t[1] + t[6]) + rmul(lapt[3], t[0] + t[7]);
        zc_t w = rmul(nabt[0], t[3] - t[4]) + rmul(nabt[1], t[2] - t[5]) +
                 rmul(nabt[2], t[1] - t[6]) + rmul(nabt[3], t[0] - t[7]);
        // y: t(1..4) = psi(y+1..y+4), t(5..8) = psi(y-1..y-4)
        for (int k = 0; k < 4; ++k) {
          t[k] = ld(tpsi, I.a(ix, I.Y(iy + k + 1), iz));
          t[k + 4] = ld(tpsi, I.a(ix, I.Y(iy - k - 1), iz));
        }
        v = (rmul(lapt[4], t[0] + t[4]) + rmul(lapt[5], t[1] + t[5]) +
             rmul(lapt[6], t[2] + t[6]) + rmul(lapt[7], t[3] + t[7])) + v;
        w = (rmul(nabt[4], t[0] - t[4]) + rmul(nabt[5], t[1] - t[5]) +
             rmul(nabt[6], t[2] - t[6]) + rmul(nabt[7], t[3] - t[7])) + w;
        for (int k = 0; k < 4; ++k) {
          t[k] = ld(tpsi, I.a(ix, iy, I.Z(iz + k + 1)));
          t[k + 4] = ld(tpsi, I.a(ix, iy, I.Z(iz - k - 1)));
        }
        v = (rmul(lapt[8], t[0] + t[4]) + rmul(lapt[9], t[1] + t[5]) +
             rmul(lapt[10], t[2] + t[6]) + rmul(lapt[11], t[3] + t[7])) + v;
        w = (rmul(nabt[8], t[0] - t[4]) + rmul(nabt[9], t[1] - t[5]) +
             rmul(nabt[10], t[2] - t[6]) + rmul(nabt[11], t[3] - t[7])) + w;
        const zc_t c = ld(tpsi, I.a(ix, iy, iz));
        const double vl = V[I.r(ix, iy, iz)];
        // V*psi + lap0*psi - 0.5*v - zI*w ;  zI*w = (-w_i, w_r)
        zc_t h = rmul(vl, c) + rmul(lap0, c) - rmul(0.5, v) - zc_t(-w.imag(), w.real());
        st(htpsi, I.a(ix, iy, iz), h);
      }
}

// One orbital of the non-orthogonal-lattice stencil, zstencil_nonorthogonal
// (stencil.f90:120-214): lattice-axis Laplacian sums v(d) and first
// derivatives w(d) (coef_nab, not k-weighted), htpsi = (V + lap0) psi
// - 1/2 sum F(d) v(d) - i sum Bk(d) w(d); then the mixed terms
// - 1/2 (F(4) d_z(w_y) + F(5) d_z(w_x) + F(6) d_y(w_x)) from the stored
// first derivatives (the reference's wrk array, read through the index maps).
void zstencil_nonorth_one(const sbo_system* s, const Idx& I, const double* tpsi, double* htpsi,
                          const double* V, double lap0, const double* Bk) {
  const double* lapt = s->coef_lap;
  const double* nab = s->coef_nab;
  const double* F = s->coef_F;
  std::vector<zc_t> wrk1(I.vol), wrk2(I.vol);
  auto T = [&](int x, int y, int z) { return ld(tpsi, I.a(x, y, z)); };
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
        zc_t v[3], w[3];
        for (int d = 0; d < 3; ++d) {
          zc_t vv(0.0, 0.0), ww(0.0, 0.0);
          for (int k = 1; k <= 4; ++k) {
            zc_t tp, tm;
            if (d == 0) {
              tp = T(I.X(ix + k), iy, iz);
              tm = T(I.X(ix - k), iy, iz);
            } else if (d == 1) {
              tp = T(ix, I.Y(iy + k), iz);
              tm = T(ix, I.Y(iy - k), iz);
            } else {
              tp = T(ix, iy, I.Z(iz + k));
              tm = T(ix, iy, I.Z(iz - k));
            }
            vv = vv + rmul(lapt[4 * d + k - 1], tp + tm);
            ww = ww + rmul(nab[4 * d + k - 1], tp - tm);
          }
          v[d] = vv;
          w[d] = ww;
        }
        const zc_t c = T(ix, iy, iz);
        const zc_t fv = rmul(F[0], v[0]) + rmul(F[1], v[1]) + rmul(F[2], v[2]);
        const zc_t bw = rmul(Bk[0], w[0]) + rmul(Bk[1], w[1]) + rmul(Bk[2], w[2]);
        // (V + lap0) psi - 0.5 (F.v) - zI (Bk.w)
        const zc_t h = rmul(V[I.r(ix, iy, iz)] + lap0, c) - rmul(0.5, fv) - zc_t(-bw.imag(), bw.real());
        st(htpsi, I.a(ix, iy, iz), h);
        wrk1[I.a(ix, iy, iz)] = w[0];
        wrk2[I.a(ix, iy, iz)] = w[1];
      }
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
        zc_t w1(0.0, 0.0), w2(0.0, 0.0), w3(0.0, 0.0);
        for (int k = 1; k <= 4; ++k) {
          w1 = w1 + rmul(nab[8 + k - 1], wrk2[I.a(ix, iy, I.Z(iz + k))] - wrk2[I.a(ix, iy, I.Z(iz - k))]);  // yz
          w2 = w2 + rmul(nab[8 + k - 1], wrk1[I.a(ix, iy, I.Z(iz + k))] - wrk1[I.a(ix, iy, I.Z(iz - k))]);  // zx
          w3 = w3 + rmul(nab[4 + k - 1], wrk1[I.a(ix, I.Y(iy + k), iz)] - wrk1[I.a(ix, I.Y(iy - k), iz)]);  // xy
        }
        const zc_t h = ld(htpsi, I.a(ix, iy, iz)) - rmul(0.5, rmul(F[3], w1) + rmul(F[4], w2) + rmul(F[5], w3));
        st(htpsi, I.a(ix, iy, iz), h);
      }
}

// One orbital of the single-scale (microscopic A) stencil,
// zstencil_microAc_typical_seq (zstencil_microac_core/typical/seq.f90): per
// point kAc = k + Ac(r), v the Laplacian sums, w(d) the first derivatives
// (coef_nab), htpsi = (V + lap0) psi - v/2 + |kAc|^2 psi / 2 - i kAc.w
// - i div(Ac) psi / 2.
void zstencil_microac_one(const sbo_system* s, const Idx& I, const double* tpsi, double* htpsi, const double* V,
                          const double* k) {
  const double* lapt = s->coef_lap;
  const double* nab = s->coef_nab;
  auto T = [&](int x, int y, int z) { return ld(tpsi, I.a(x, y, z)); };
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
        const long r = I.r(ix, iy, iz);
        const zc_t psi0 = T(ix, iy, iz);
        double kAc[3];
        for (int d = 0; d < 3; ++d) kAc[d] = k[d] + s->ac_micro[3 * r + d];
        const double div = s->div_ac[r];
        zc_t v(0.0, 0.0), w[3];
        for (int d = 0; d < 3; ++d) {
          zc_t vv(0.0, 0.0), ww(0.0, 0.0);
          for (int q = 1; q <= 4; ++q) {
            zc_t tp, tm;
            if (d == 0) {
              tp = T(I.X(ix + q), iy, iz);
              tm = T(I.X(ix - q), iy, iz);
            } else if (d == 1) {
              tp = T(ix, I.Y(iy + q), iz);
              tm = T(ix, I.Y(iy - q), iz);
            } else {
              tp = T(ix, iy, I.Z(iz + q));
              tm = T(ix, iy, I.Z(iz - q));
            }
            vv = vv + rmul(lapt[4 * d + q - 1], tp + tm);
            ww = ww + rmul(nab[4 * d + q - 1], tp - tm);
          }
          v = d == 0 ? vv : vv + v;
          w[d] = ww;
        }
        const zc_t kw = rmul(kAc[0], w[0]) + rmul(kAc[1], w[1]) + rmul(kAc[2], w[2]);
        const double k2 = kAc[0] * kAc[0] + kAc[1] * kAc[1] + kAc[2] * kAc[2];
        // - zI kw = (kw_i, -kw_r); - zI 0.5 div psi0 = (0.5 div psi0_i, -0.5 div psi0_r)
        const zc_t h = rmul(V[r] + s->coef_lap0, psi0) - rmul(0.5, v) + rmul(0.5 * k2, psi0) +
                       zc_t(kw.imag(), -kw.real()) + zc_t(0.5 * div * psi0.imag(), -0.5 * div * psi0.real());
        st(htpsi, I.a(ix, iy, iz), h);
      }
}

// One orbital of the symmetrized single-scale stencil, zstencil_microAc_symmetrized
// (stencil.f90:319-411): kAc = k + Ac(r), v the Laplacian sums, w(d) the first
// derivatives, x = sum_d sum_q nab(q,d) ((k_d + Ac_d(r + q e_d)) psi(r + q e_d)
// - (k_d + Ac_d(r - q e_d)) psi(r - q e_d)), htpsi = (V + lap0) psi - v/2
// + |kAc|^2 psi / 2 - (i/2) (kAc.w + x).  A neighbour outside an isolated grid
// has psi = 0, so its product is zero whatever Ac holds there.
void zstencil_microac_sym_one(const sbo_system* s, const Idx& I, const double* tpsi, double* htpsi,
                              const double* V, const double* k) {
  const double* lapt = s->coef_lap;
  const double* nab = s->coef_nab;
  auto T = [&](int x, int y, int z) { return ld(tpsi, I.a(x, y, z)); };
  auto inside = [&](int x, int y, int z) {
    return x >= s->is[0] && x <= s->ie[0] && y >= s->is[1] && y <= s->ie[1] && z >= s->is[2] && z <= s->ie[2];
  };
  auto A = [&](int d, int x, int y, int z) { return inside(x, y, z) ? s->ac_micro[3 * I.r(x, y, z) + d] : 0.0; };
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
        const long r = I.r(ix, iy, iz);
        const zc_t psi0 = T(ix, iy, iz);
        double kAc[3];
        for (int d = 0; d < 3; ++d) kAc[d] = k[d] + s->ac_micro[3 * r + d];
        zc_t v(0.0, 0.0), w[3], x(0.0, 0.0);
        for (int d = 0; d < 3; ++d) {
          zc_t vv(0.0, 0.0), ww(0.0, 0.0), xx(0.0, 0.0);
          for (int q = 1; q <= 4; ++q) {
            int px = ix, py = iy, pz = iz, mx = ix, my = iy, mz = iz;
            if (d == 0) {
              px = I.X(ix + q);
              mx = I.X(ix - q);
            } else if (d == 1) {
              py = I.Y(iy + q);
              my = I.Y(iy - q);
            } else {
              pz = I.Z(iz + q);
              mz = I.Z(iz - q);
            }
            const zc_t tp = T(px, py, pz), tm = T(mx, my, mz);
            vv = vv + rmul(lapt[4 * d + q - 1], tp + tm);
            ww = ww + rmul(nab[4 * d + q - 1], tp - tm);
            xx = xx + rmul(nab[4 * d + q - 1],
                           rmul(k[d] + A(d, px, py, pz), tp) - rmul(k[d] + A(d, mx, my, mz), tm));
          }
          v = d == 0 ? vv : vv + v;
          w[d] = ww;
          x = d == 0 ? xx : xx + x;
        }
        const zc_t kw = rmul(kAc[0], w[0]) + rmul(kAc[1], w[1]) + rmul(kAc[2], w[2]);
        const zc_t t = kw + x;
        const double k2 = kAc[0] * kAc[0] + kAc[1] * kAc[1] + kAc[2] * kAc[2];
        // - (i/2) t = (t_i / 2, -t_r / 2)
        const zc_t h = rmul(V[r] + s->coef_lap0, psi0) - rmul(0.5, v) + rmul(0.5 * k2, psi0) +
                       zc_t(0.5 * t.imag(), -0.5 * t.real());
        st(htpsi, I.a(ix, iy, iz), h);
      }
}

// One orbital of the real 25-point stencil.  stencil.f90:30-80.
void dstencil_one(const sbo_system* s, const Idx& I, const double* tpsi, double* htpsi,
                  const double* V, double lap0, const double* lapt, bool omp_grid) {
#pragma omp parallel for collapse(2) if (omp_grid)
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
        auto T = [&](int x, int y, int z) { return tpsi[I.a(x, y, z)]; };
        double v = lapt[0] * (T(I.X(ix + 1), iy, iz) + T(I.X(ix - 1), iy, iz)) +
                   lapt[1] * (T(I.X(ix + 2), iy, iz) + T(I.X(ix - 2), iy, iz)) +
                   lapt[2] * (T(I.X(ix + 3), iy, iz) + T(I.X(ix - 3), iy, iz)) +
                   lapt[3] * (T(I.X(ix + 4), iy, iz) + T(I.X(ix - 4), iy, iz));
        v = lapt[4] * (T(ix, I.Y(iy + 1), iz) + T(ix, I.Y(iy - 1), iz)) +
            lapt[5] * (T(ix, I.Y(iy + 2), iz) + T(ix, I.Y(iy - 2), iz)) +
            lapt[6] * (T(ix, I.Y(iy + 3), iz) + T(ix, I.Y(iy - 3), iz)) +
            lapt[7] * (T(ix, I.Y(iy + 4), iz) + T(ix, I.Y(iy - 4), iz)) + v;
        v = lapt[8] * (T(ix, iy, I.Z(iz + 1)) + T(ix, iy, I.Z(iz - 1))) +
            lapt[9] * (T(ix, iy, I.Z(iz + 2)) + T(ix, iy, I.Z(iz - 2))) +
            lapt[10] * (T(ix, iy, I.Z(iz + 3)) + T(ix, iy, I.Z(iz - 3))) +
            lapt[11] * (T(ix, iy, I.Z(iz + 4)) + T(ix, iy, I.Z(iz - 4))) + v;
        htpsi[I.a(ix, iy, iz)] = (V[I.r(ix, iy, iz)] + lap0) * T(ix, iy, iz) - 0.5 * v;
      }
}

inline long jx_off(const sbo_system* s, int c, int j, int ia) {
  return (c - 1) + 3L * ((j - 1) + (long)s->nps * (ia - 1));
}
inline long zekr_off(const sbo_system* s, int j, int ilma, int ik) {
  return (j - 1) + (long)s->nps * ((ilma - 1) + (long)s->nlma * (ik - 1));
}

// k+A dependent stencil coefficients. hamiltonian.f90:146-155.
void kac_coefs(const sbo_system* s, int ik, const double* vac, double* kAc, double& k_lap0,
               double* k_nabt) {
  if (s->periodic) {
    for (int d = 0; d < 3; ++d) kAc[d] = s->vec_k[3 * (ik - 1) + d] + vac[d];
    k_lap0 = s->coef_lap0 + 0.5 * (kAc[0] * kAc[0] + kAc[1] * kAc[1] + kAc[2] * kAc[2]);
    for (int d = 0; d < 3; ++d)
      for (int i = 0; i < 4; ++i) k_nabt[4 * d + i] = kAc[d] * s->coef_nab[4 * d + i];
  } else {
    kAc[0] = kAc[1] = kAc[2] = 0.0;
    k_lap0 = s->coef_lap0;
    for (int i = 0; i < 12; ++i) k_nabt[i] = 0.0;
  }
}

}  // namespace

extern "C" {

void sbo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int sbo_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void sbo_zstencil(const sbo_system* s, const double* tpsi, double* htpsi, const double* V_local,
                  double lap0, const double* lapt, const double* nabt) {
  Idx I(s);
  zstencil_one(s, I, tpsi, htpsi, V_local, lap0, lapt, nabt, s->stencil_rgrid_mode != 0);
}

void sbo_dstencil(const sbo_system* s, const double* tpsi, double* htpsi, const double* V_local,
                  double lap0, const double* lapt) {
  Idx I(s);
  dstencil_one(s, I, tpsi, htpsi, V_local, lap0, lapt, s->stencil_rgrid_mode != 0);
}

// update_kvector_nonlocalpt, hamiltonian.f90:847-903 (periodic);
// prep_pp.f90:618-619 (isolated: zekr_uV = uV, one k).
void sbo_update_kvector_nonlocalpt(sbo_system* s) {
  const int nk = s->periodic ? s->nk : 1;
#pragma omp parallel for collapse(2)
  for (int ik = 1; ik <= nk; ++ik)
    for (int ilma = 1; ilma <= s->nlma; ++ilma) {
      const int ia = s->ia_tbl[ilma - 1];
      double kAc[3];
      if (s->periodic) {
        for (int d = 0; d < 3; ++d) kAc[d] = s->vec_k[3 * (ik - 1) + d] + s->vec_Ac[d];
      }
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const double uv = s->uv[(j - 1) + (long)s->nps * (ilma - 1)];
        zc_t z;
        if (s->periodic) {
          const double x = s->rxyz[jx_off(s, 1, j, ia)];
          const double y = s->rxyz[jx_off(s, 2, j, ia)];
          const double zz = s->rxyz[jx_off(s, 3, j, ia)];
          const double th = kAc[0] * x + kAc[1] * y + kAc[2] * zz;
          // ekr = exp(zi*th); zekr = conjg(ekr)*uv
          z = zc_t(std::cos(th) * uv, -std::sin(th) * uv);
        } else {
          z = zc_t(uv, 0.0);
        }
        st(s->zekr, zekr_off(s, j, ilma, ik), z);
      }
    }
}

// Projections only: uvpsi(ilma, orb) = rinv_uvu * sum_j conj(zekr) psi(jxyz).
void sbo_zprojections(const sbo_system* s, const double* tpsi, double* uvpsi) {
  Idx I(s);
  const long norb = I.norb();
#pragma omp parallel for
  for (long o = 0; o < norb; ++o) {
    const int ik_eff = s->periodic ? (int)(o / ((long)s->nspin * s->no)) + 1 : 1;
    const double* psi = tpsi + 2 * I.vol * o;
    for (int ilma = 1; ilma <= s->nlma; ++ilma) {
      const int ia = s->ia_tbl[ilma - 1];
      zc_t u(0.0, 0.0);
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const int ix = s->jxyz[jx_off(s, 1, j, ia)];
        const int iy = s->jxyz[jx_off(s, 2, j, ia)];
        const int iz = s->jxyz[jx_off(s, 3, j, ia)];
        const zc_t zk = std::conj(ld(s->zekr, zekr_off(s, j, ilma, ik_eff)));
        u = u + cmul(zk, ld(psi, I.a(ix, iy, iz)));
      }
      u = rmul(s->rinv_uvu[ilma - 1], u);
      st(uvpsi, (ilma - 1) + (long)s->nlma * o, u);
    }
  }
}

// zpseudo CPU branch, nonlocal_potential.f90:351-382.
void sbo_zpseudo(const sbo_system* s, const double* tpsi, double* htpsi) {
  Idx I(s);
  const long norb = I.norb();
#pragma omp parallel for
  for (long o = 0; o < norb; ++o) {
    const int ik = (int)(o / ((long)s->nspin * s->no)) + 1;
    const int ik_eff = s->periodic ? ik : 1;
    const double* psi = tpsi + 2 * I.vol * o;
    double* hpsi = htpsi + 2 * I.vol * o;
    for (int ilma = 1; ilma <= s->nlma; ++ilma) {
      const int ia = s->ia_tbl[ilma - 1];
      zc_t u(0.0, 0.0);
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const int ix = s->jxyz[jx_off(s, 1, j, ia)];
        const int iy = s->jxyz[jx_off(s, 2, j, ia)];
        const int iz = s->jxyz[jx_off(s, 3, j, ia)];
        const zc_t zk = std::conj(ld(s->zekr, zekr_off(s, j, ilma, ik_eff)));
        u = u + cmul(zk, ld(psi, I.a(ix, iy, iz)));
      }
      u = rmul(s->rinv_uvu[ilma - 1], u);
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const int ix = s->jxyz[jx_off(s, 1, j, ia)];
        const int iy = s->jxyz[jx_off(s, 2, j, ia)];
        const int iz = s->jxyz[jx_off(s, 3, j, ia)];
        const zc_t wrk = cmul(u, ld(s->zekr, zekr_off(s, j, ilma, ik_eff)));
        const long off = I.a(ix, iy, iz);
        st(hpsi, off, ld(hpsi, off) + wrk);
      }
    }
  }
}

// dpseudo, nonlocal_potential.f90:26-171 (single r-space domain branch).
void sbo_dpseudo(const sbo_system* s, const double* tpsi, double* htpsi) {
  Idx I(s);
  const long norb = I.norb();
#pragma omp parallel for
  for (long o = 0; o < norb; ++o) {
    const double* psi = tpsi + I.vol * o;
    double* hpsi = htpsi + I.vol * o;
    for (int ilma = 1; ilma <= s->nlma; ++ilma) {
      const int ia = s->ia_tbl[ilma - 1];
      double u = 0.0;
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const int ix = s->jxyz[jx_off(s, 1, j, ia)];
        const int iy = s->jxyz[jx_off(s, 2, j, ia)];
        const int iz = s->jxyz[jx_off(s, 3, j, ia)];
        u = u + s->uv[(j - 1) + (long)s->nps * (ilma - 1)] * psi[I.a(ix, iy, iz)];
      }
      u = u * s->rinv_uvu[ilma - 1];
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const int ix = s->jxyz[jx_off(s, 1, j, ia)];
        const int iy = s->jxyz[jx_off(s, 2, j, ia)];
        const int iz = s->jxyz[jx_off(s, 3, j, ia)];
        hpsi[I.a(ix, iy, iz)] += u * s->uv[(j - 1) + (long)s->nps * (ilma - 1)];
      }
    }
  }
}

// add_imaginary_potential_for_absorbing_boundary_z (hamiltonian.f90:760-807):
// on each plane z = iz hgs(3), w = (0, -w0 (z1 - z) / dr) below z1 = dr,
// (0, -w0 (z - z2) / dr) above z2 = al(3) - dr, and htpsi += w tpsi.
static void cap_add(const sbo_system* s, const Idx& I, const double* tpsi, double* htpsi) {
  const double z1 = s->cap_dr, z2 = s->cap_al - s->cap_dr;
#pragma omp parallel for
  for (long o = 0; o < I.norb(); ++o)
    for (int iz = s->is[2]; iz <= s->ie[2]; ++iz) {
      const double z = iz * s->hgs[2];
      zc_t w;
      if (z <= z1) w = zc_t(0.0, -s->cap_w0 * (z1 - z) / s->cap_dr);
      else if (z >= z2) w = zc_t(0.0, -s->cap_w0 * (z - z2) / s->cap_dr);
      else continue;
      for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          const long i = I.vol * o + I.a(ix, iy, iz);
          st(htpsi, i, ld(htpsi, i) + w * ld(tpsi, i));
        }
    }
}

// hpsi, complex, orthogonal lattice: hamiltonian.f90:139-235 then zpseudo :424-435;
// non-orthogonal lattice: hamiltonian.f90:306-357 (kAc Cartesian, k_lap0 =
// coef_lap0 + |kAc|^2 / 2, Bk = rmatrix_B kAc) then zpseudo.
void sbo_hpsi(const sbo_system* s, const double* tpsi, double* htpsi) {
  Idx I(s);
  const bool grid_mode = s->stencil_rgrid_mode != 0;
  const long nxy = I.nx * I.ny * I.nz;
  if (s->ac_micro) {  // single-scale branch, hamiltonian.f90:236-298
#pragma omp parallel for collapse(3)
    for (int ik = 1; ik <= s->nk; ++ik)
      for (int io = 1; io <= s->no; ++io)
        for (int is = 1; is <= s->nspin; ++is) {
          const long o = I.orb(is, io, ik);
          if (s->symmetrized)  // hamiltonian.f90:239-256
            zstencil_microac_sym_one(s, I, tpsi + 2 * I.vol * o, htpsi + 2 * I.vol * o,
                                     s->V_local + nxy * (is - 1), s->vec_k + 3 * (ik - 1));
          else
            zstencil_microac_one(s, I, tpsi + 2 * I.vol * o, htpsi + 2 * I.vol * o, s->V_local + nxy * (is - 1),
                                 s->vec_k + 3 * (ik - 1));
        }
    if (s->cap_on) cap_add(s, I, tpsi, htpsi);  // hamiltonian.f90:300-303
    if (s->nlma > 0) sbo_zpseudo(s, tpsi, htpsi);
    return;
  }
  if (s->nonorth) {
#pragma omp parallel for collapse(3)
    for (int ik = 1; ik <= s->nk; ++ik)
      for (int io = 1; io <= s->no; ++io)
        for (int is = 1; is <= s->nspin; ++is) {
          double kAc[3], Bk[3];
          for (int d = 0; d < 3; ++d) kAc[d] = s->vec_k[3 * (ik - 1) + d] + s->vec_Ac[d];
          const double k_lap0 = s->coef_lap0 + 0.5 * (kAc[0] * kAc[0] + kAc[1] * kAc[1] + kAc[2] * kAc[2]);
          for (int d = 0; d < 3; ++d)
            Bk[d] = s->rmatrix_B[d] * kAc[0] + s->rmatrix_B[d + 3] * kAc[1] + s->rmatrix_B[d + 6] * kAc[2];
          const long o = I.orb(is, io, ik);
          zstencil_nonorth_one(s, I, tpsi + 2 * I.vol * o, htpsi + 2 * I.vol * o, s->V_local + nxy * (is - 1),
                               k_lap0, Bk);
        }
    if (s->nlma > 0) sbo_zpseudo(s, tpsi, htpsi);
    return;
  }
  if (grid_mode) {
    for (int ik = 1; ik <= s->nk; ++ik) {
      double kAc[3], k_lap0, k_nabt[12];
      kac_coefs(s, ik, s->vec_Ac, kAc, k_lap0, k_nabt);
      for (int io = 1; io <= s->no; ++io)
        for (int is = 1; is <= s->nspin; ++is) {
          const long o = I.orb(is, io, ik);
          zstencil_one(s, I, tpsi + 2 * I.vol * o, htpsi + 2 * I.vol * o,
                       s->V_local + nxy * (is - 1), k_lap0, s->coef_lap, k_nabt, true);
        }
    }
  } else {
#pragma omp parallel for collapse(3)
    for (int ik = 1; ik <= s->nk; ++ik)
      for (int io = 1; io <= s->no; ++io)
        for (int is = 1; is <= s->nspin; ++is) {
          double kAc[3], k_lap0, k_nabt[12];
          kac_coefs(s, ik, s->vec_Ac, kAc, k_lap0, k_nabt);
          const long o = I.orb(is, io, ik);
          zstencil_one(s, I, tpsi + 2 * I.vol * o, htpsi + 2 * I.vol * o,
                       s->V_local + nxy * (is - 1), k_lap0, s->coef_lap, k_nabt, false);
        }
  }
  if (s->cap_on) cap_add(s, I, tpsi, htpsi);  // hamiltonian.f90:231-234
  if (s->nlma > 0) sbo_zpseudo(s, tpsi, htpsi);
}

// hpsi with ttpsi (hamiltonian.f90:27 optional argument): after the stencil,
// ttpsi = htpsi - V_local * tpsi on the interior (:364-414), then the nonlocal
// term is added to htpsi only.
void sbo_hpsi_tt(const sbo_system* s, const double* tpsi, double* htpsi, double* ttpsi) {
  Idx I(s);
  const long nxy = I.nx * I.ny * I.nz;
  sbo_system s0 = *s;
  s0.nlma = 0;  // the stencil part of hpsi
  sbo_hpsi(&s0, tpsi, htpsi);
#pragma omp parallel for collapse(3)
  for (int ik = 1; ik <= s->nk; ++ik)
    for (int io = 1; io <= s->no; ++io)
      for (int is = 1; is <= s->nspin; ++is) {
        const long o = I.orb(is, io, ik);
        const double* V = s->V_local + nxy * (is - 1);
        const double* t = tpsi + 2 * I.vol * o;
        const double* h = htpsi + 2 * I.vol * o;
        double* tt = ttpsi + 2 * I.vol * o;
        for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
          for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
            for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
              const long i = I.a(ix, iy, iz);
              const double v = V[I.r(ix, iy, iz)];
              tt[2 * i] = h[2 * i] - v * t[2 * i];
              tt[2 * i + 1] = h[2 * i + 1] - v * t[2 * i + 1];
            }
      }
  if (s->nlma > 0) sbo_zpseudo(s, tpsi, htpsi);
}

// calc_eigen_energy, complex branch (total_energy.f90:505-775): per orbital
// esp = Re sum conj(psi) H psi * Hvol; E_kin = sum occ w Re sum conj(psi) T psi
// * Hvol; E_ion_nloc = sum occ w Hvol Re sum conj(psi) (H psi - (T psi + V psi)).
void sbo_calc_eigen_energy(const sbo_system* s, const double* tpsi, double* htpsi, double* ttpsi, double* esp,
                           double* e) {
  Idx I(s);
  const long nxy = I.nx * I.ny * I.nz;
  sbo_hpsi_tt(s, tpsi, htpsi, ttpsi);
  double ek = 0.0, en = 0.0;
  for (int is = 1; is <= s->nspin; ++is)
    for (int ik = 1; ik <= s->nk; ++ik)
      for (int io = 1; io <= s->no; ++io) {
        const long o = I.orb(is, io, ik);
        const double* V = s->V_local + nxy * (is - 1);
        const double* t = tpsi + 2 * I.vol * o;
        const double* h = htpsi + 2 * I.vol * o;
        const double* tt = ttpsi + 2 * I.vol * o;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
          for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
            for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
              const long i = I.a(ix, iy, iz);
              const double v = V[I.r(ix, iy, iz)];
              const double tr = t[2 * i], ti = t[2 * i + 1];
              s0 += tr * h[2 * i] + ti * h[2 * i + 1];
              s1 += tr * tt[2 * i] + ti * tt[2 * i + 1];
              const double nr = h[2 * i] - (tt[2 * i] + v * tr), ni = h[2 * i + 1] - (tt[2 * i + 1] + v * ti);
              s2 += tr * nr + ti * ni;
            }
        const double w = s->rocc[(io - 1) + (long)s->no * ((ik - 1) + (long)s->nk * (is - 1))] * s->wtk[ik - 1];
        esp[(io - 1) + (long)s->no * ((ik - 1) + (long)s->nk * (is - 1))] = s0 * s->hvol;
        ek += w * s1 * s->hvol;
        en += w * s->hvol * s2;
      }
  e[0] = ek;
  e[1] = en;
}

// hpsi, real orbitals: hamiltonian.f90:88-125 (dstencil + dpseudo).
void sbo_hpsi_real(const sbo_system* s, const double* tpsi, double* htpsi) {
  Idx I(s);
  const long nxy = I.nx * I.ny * I.nz;
  const long norb = I.norb();
  if (s->stencil_rgrid_mode) {
    for (long o = 0; o < norb; ++o) {
      const int is = (int)(o % s->nspin) + 1;
      dstencil_one(s, I, tpsi + I.vol * o, htpsi + I.vol * o, s->V_local + nxy * (is - 1),
                   s->coef_lap0, s->coef_lap, true);
    }
  } else {
#pragma omp parallel for
    for (long o = 0; o < norb; ++o) {
      const int is = (int)(o % s->nspin) + 1;
      dstencil_one(s, I, tpsi + I.vol * o, htpsi + I.vol * o, s->V_local + nxy * (is - 1),
                   s->coef_lap0, s->coef_lap, false);
    }
  }
  if (s->nlma > 0) sbo_dpseudo(s, tpsi, htpsi);
}

// taylor, taylor.f90:21-121 (tspsi_in is reused as scratch for even terms).
void sbo_taylor(const sbo_system* s, double* tspsi_in, double* tspsi_out, double* sshtpsi,
                const double* zc, int n_hamil) {
  Idx I(s);
  const long norb = I.norb();
  for (int nn = 1; nn <= n_hamil; ++nn) {
    const zc_t c(zc[2 * (nn - 1)], zc[2 * (nn - 1) + 1]);
    const bool odd = (nn % 2) == 1;
    if (odd) sbo_hpsi(s, tspsi_in, sshtpsi);
    else sbo_hpsi(s, sshtpsi, tspsi_in);
    const double* h = odd ? sshtpsi : tspsi_in;
#pragma omp parallel for collapse(3)
    for (long o = 0; o < norb; ++o)
      for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
        for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
          for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
            const long off = I.vol * o + I.a(ix, iy, iz);
            if (nn == 1)
              st(tspsi_out, off, ld(tspsi_in, off) + cmul(c, ld(h, off)));
            else
              st(tspsi_out, off, ld(tspsi_out, off) + cmul(c, ld(h, off)));
          }
  }
}

// calc_density, density_matrix.f90:150-232 (fixed summation order over k, o).
void sbo_calc_density(const sbo_system* s, const double* psi, double* rho) {
  Idx I(s);
  const long n = I.nx * I.ny * I.nz;
  for (int is = 1; is <= s->nspin; ++is) {
    double* r = rho + n * (is - 1);
#pragma omp parallel for collapse(2)
    for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
      for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          double acc = 0.0;
          for (int ik = 1; ik <= s->nk; ++ik)
            for (int io = 1; io <= s->no; ++io) {
              const long o = I.orb(is, io, ik);
              const double w2 = abs2(ld(psi, I.vol * o + I.a(ix, iy, iz)));
              acc = acc + w2 * s->rocc[(io - 1) + (long)s->no * ((ik - 1) + (long)s->nk * (is - 1))] *
                              s->wtk[ik - 1];
            }
          r[I.r(ix, iy, iz)] = acc;
        }
  }
}

// calc_microscopic_current (density_matrix.f90:726-845): per orbital
// (k, o, spin in the reference's loop order) micro_current's
// jw_d = Im(conj(psi) xtmp_d) + k_d |psi|^2, xtmp_d the coef_nab first
// derivative, then wrk2 += jw rocc wtk at every point.
void sbo_calc_microscopic_current(const sbo_system* s, const double* psi, double* curr) {
  Idx I(s);
  const double* nab = s->coef_nab;
#pragma omp parallel for collapse(2)
  for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
    for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
      for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int ik = 1; ik <= s->nk; ++ik)
          for (int io = 1; io <= s->no; ++io)
            for (int is = 1; is <= s->nspin; ++is) {
              const double* t = psi + 2 * I.vol * I.orb(is, io, ik);
              const zc_t p = std::conj(ld(t, I.a(ix, iy, iz)));
              const double ap = std::abs(p);
              const double* k = s->vec_k + 3 * (ik - 1);
              const double occ = s->rocc[(io - 1) + (long)s->no * ((ik - 1) + (long)s->nk * (is - 1))];
              for (int d = 0; d < 3; ++d) {
                zc_t tmp(0.0, 0.0);
                for (int q = 1; q <= 4; ++q) {
                  zc_t tp, tm;
                  if (d == 0) {
                    tp = ld(t, I.a(I.X(ix + q), iy, iz));
                    tm = ld(t, I.a(I.X(ix - q), iy, iz));
                  } else if (d == 1) {
                    tp = ld(t, I.a(ix, I.Y(iy + q), iz));
                    tm = ld(t, I.a(ix, I.Y(iy - q), iz));
                  } else {
                    tp = ld(t, I.a(ix, iy, I.Z(iz + q)));
                    tm = ld(t, I.a(ix, iy, I.Z(iz - q)));
                  }
                  tmp = tmp + rmul(nab[4 * d + q - 1], tp - tm);
                }
                const double jw = (p * tmp).imag() + k[d] * ap * ap;
                acc[d] = acc[d] + jw * occ * s->wtk[ik - 1];
              }
            }
        const long r = I.r(ix, iy, iz);
        for (int d = 0; d < 3; ++d) curr[3 * r + d] = acc[d];
      }
}

// Per-orbital current pieces: stencil_current (density_matrix.f90:465-530) and
// calc_current_nonlocal (:532-591).
void sbo_current_parts(const sbo_system* s, const double* psi_all, double* out) {
  Idx I(s);
  const long norb = I.norb();
#pragma omp parallel for
  for (long o = 0; o < norb; ++o) {
    const int is = (int)(o % s->nspin) + 1;
    const int io = (int)((o / s->nspin) % s->no) + 1;
    const int ik = (int)(o / ((long)s->nspin * s->no)) + 1;
    const double* psi = psi_all + 2 * I.vol * o;
    const double* nab = s->coef_nab;
    double rtmp = 0.0;
    zc_t xt(0, 0), yt(0, 0), zt(0, 0);
    for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
      for (int iy = s->is[1]; iy <= s->ie[1]; ++iy) {
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) rtmp = rtmp + abs2(ld(psi, I.a(ix, iy, iz)));
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          const zc_t cp = std::conj(ld(psi, I.a(ix, iy, iz)));
          xt = xt + cmul(rmul(nab[0], cp), ld(psi, I.a(I.X(ix + 1), iy, iz))) +
               cmul(rmul(nab[1], cp), ld(psi, I.a(I.X(ix + 2), iy, iz))) +
               cmul(rmul(nab[2], cp), ld(psi, I.a(I.X(ix + 3), iy, iz))) +
               cmul(rmul(nab[3], cp), ld(psi, I.a(I.X(ix + 4), iy, iz)));
        }
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          const zc_t cp = std::conj(ld(psi, I.a(ix, iy, iz)));
          yt = yt + cmul(rmul(nab[4], cp), ld(psi, I.a(ix, I.Y(iy + 1), iz))) +
               cmul(rmul(nab[5], cp), ld(psi, I.a(ix, I.Y(iy + 2), iz))) +
               cmul(rmul(nab[6], cp), ld(psi, I.a(ix, I.Y(iy + 3), iz))) +
               cmul(rmul(nab[7], cp), ld(psi, I.a(ix, I.Y(iy + 4), iz)));
        }
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          const zc_t cp = std::conj(ld(psi, I.a(ix, iy, iz)));
          zt = zt + cmul(rmul(nab[8], cp), ld(psi, I.a(ix, iy, I.Z(iz + 1)))) +
               cmul(rmul(nab[9], cp), ld(psi, I.a(ix, iy, I.Z(iz + 2)))) +
               cmul(rmul(nab[10], cp), ld(psi, I.a(ix, iy, I.Z(iz + 3)))) +
               cmul(rmul(nab[11], cp), ld(psi, I.a(ix, iy, I.Z(iz + 4))));
        }
      }
    double kAc[3];
    for (int d = 0; d < 3; ++d) kAc[d] = s->vec_k[3 * (ik - 1) + d] + s->vec_Ac[d];
    double j1[3], j2[3], j2b[3], jw[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) j1[d] = kAc[d] * rtmp;
    j2[0] = (xt * 2.0).imag();
    j2[1] = (yt * 2.0).imag();
    j2[2] = (zt * 2.0).imag();
    for (int d = 0; d < 3; ++d)
      j2b[d] = s->BT[d] * j2[0] + s->BT[d + 3] * j2[1] + s->BT[d + 6] * j2[2];
    // calc_current_nonlocal
    for (int ilma = 1; ilma <= s->nlma; ++ilma) {
      const int ia = s->ia_tbl[ilma - 1];
      zc_t u(0, 0), ur[3] = {zc_t(0, 0), zc_t(0, 0), zc_t(0, 0)};
      for (int j = 1; j <= s->mps[ia - 1]; ++j) {
        const double r[3] = {s->rxyz[jx_off(s, 1, j, ia)], s->rxyz[jx_off(s, 2, j, ia)],
                             s->rxyz[jx_off(s, 3, j, ia)]};
        const int ix = s->jxyz[jx_off(s, 1, j, ia)];
        const int iy = s->jxyz[jx_off(s, 2, j, ia)];
        const int iz = s->jxyz[jx_off(s, 3, j, ia)];
        const zc_t zk = std::conj(ld(s->zekr, zekr_off(s, j, ilma, ik)));
        const zc_t p = ld(psi, I.a(ix, iy, iz));
        u = u + cmul(zk, p);
        for (int d = 0; d < 3; ++d) ur[d] = ur[d] + cmul(rmul(r[d], zk), p);
      }
      u = rmul(s->rinv_uvu[ilma - 1], u);
      for (int d = 0; d < 3; ++d) jw[d] = jw[d] + cmul(std::conj(ur[d]), u).imag();
    }
    for (int d = 0; d < 3; ++d) jw[d] = jw[d] * 2.0;
    const double wgt = s->rocc[(io - 1) + (long)s->no * ((ik - 1) + (long)s->nk * (is - 1))] *
                       s->wtk[ik - 1];
    double* op = out + 10 * o;
    op[0] = rtmp;
    op[1] = j2[0];
    op[2] = j2[1];
    op[3] = j2[2];
    for (int d = 0; d < 3; ++d) op[4 + d] = jw[d];
    for (int d = 0; d < 3; ++d) op[7 + d] = (j1[d] + j2b[d] + jw[d]) * wgt;
  }
}

// calc_current, density_matrix.f90:240-463 (single domain, CPU branch).
void sbo_calc_current(const sbo_system* s, const double* psi, double* curr) {
  Idx I(s);
  const long norb = I.norb();
  std::vector<double> parts(10 * norb);
  sbo_current_parts(s, psi, parts.data());
  for (int is = 1; is <= s->nspin; ++is) {
    double w4[3] = {0, 0, 0};
    for (int ik = 1; ik <= s->nk; ++ik)
      for (int io = 1; io <= s->no; ++io) {
        const long o = I.orb(is, io, ik);
        for (int d = 0; d < 3; ++d) w4[d] = w4[d] + parts[10 * o + 7 + d];
      }
    for (int d = 0; d < 3; ++d) curr[3 * (is - 1) + d] = w4[d] / (double)s->ngrid;
  }
}

// calc_dip, dip.f90:114-225.
void sbo_calc_dip(const sbo_system* s, const double* rho, double* rbox) {
  Idx I(s);
  const long n = I.nx * I.ny * I.nz;
  for (int d = 0; d < 3; ++d) {
    const double shift = (s->lg_num[d] % 2 == 1) ? 0.0 : 0.5;
    double acc = 0.0;
    for (int is = 1; is <= s->nspin; ++is)
      for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
        for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
          for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
            const int c = d == 0 ? ix : (d == 1 ? iy : iz);
            acc = acc + ((double)c - shift) * rho[n * (is - 1) + I.r(ix, iy, iz)];
          }
    rbox[d] = acc;
  }
  double acc = 0.0;
  for (int is = 1; is <= s->nspin; ++is)
    for (long p = 0; p < n; ++p) acc = acc + rho[n * (is - 1) + p];
  rbox[3] = acc;
}

// Grid coordinate lg%coordinate(i, d) of set_gridcoordinate
// (initialization.f90:1125-1190): isolated grids i h (odd global size) or
// (i - 1/2) h (even), periodic grids (i - 1) h.
static double grid_coordinate(const sbo_system* s, int d, int i) {
  if (s->periodic) return (double)(i - 1) * s->hgs[d];
  return (s->lg_num[d] % 2 == 1) ? (double)i * s->hgs[d] : ((double)i - 0.5) * s->hgs[d];
}

// Impulse kick of the initial orbitals (initialization_rt.f90:382-423):
// R1 = epdir . r at every interior point, then zwf <- exp(i e_impulse R1) zwf
// for every (spin, orbital, k).
void sbo_impulse_kick(const sbo_system* s, double* psi, double e_impulse, const double epdir[3]) {
  Idx I(s);
  const long vol = I.vol;
  const int norb = s->nspin * s->no * s->nk;
  for (int o = 0; o < norb; ++o)
    for (int iz = s->is[2]; iz <= s->ie[2]; ++iz)
      for (int iy = s->is[1]; iy <= s->ie[1]; ++iy)
        for (int ix = s->is[0]; ix <= s->ie[0]; ++ix) {
          const double r1 = epdir[0] * grid_coordinate(s, 0, ix) + epdir[1] * grid_coordinate(s, 1, iy) +
                            epdir[2] * grid_coordinate(s, 2, iz);
          const std::complex<double> ph = std::exp(std::complex<double>(0.0, e_impulse * r1));
          double* z = psi + 2 * (vol * o + I.a(ix, iy, iz));
          const std::complex<double> v = ph * std::complex<double>(z[0], z[1]);
          z[0] = v.real();
          z[1] = v.imag();
        }
}

// calc_Ac_ext_t, em_field.f90:86-306 (impulse, Acos2, Asin2cos).
void sbo_calc_Ac_ext_t(int shape, double t0, double delta_t, int is, int ie, const double* epdir,
                       double f0, double omega, double tw, double phi_cep, double t1_start,
                       double e_impulse, double* Ac) {
  const double pi = 3.141592653589793238462643383279502884;
  for (int i = is; i <= ie; ++i) {
    double* a = Ac + 3L * (i - is);
    a[0] = a[1] = a[2] = 0.0;
    const double t = t0 + i * delta_t;
    if (shape == 0) {
      if (0.0 <= t)
        for (int d = 0; d < 3; ++d) a[d] = epdir[d] * e_impulse;
    } else if (shape == 1) {  // Asin2cos
      const double tt = t;
      if (tt < tw) {
        const double sn = std::sin(pi * tt / tw);
        for (int d = 0; d < 3; ++d)
          a[d] = -epdir[d] * f0 / omega * (sn * sn) * std::cos(omega * tt + phi_cep * 2.0 * pi);
      }
    } else if (shape == 2) {  // Acos2 with real polarisation
      const double tt = t - 0.5 * tw - t1_start;
      if (std::fabs(tt) < 0.5 * tw) {
        const double cs = std::cos(pi * tt / tw);
        // aimag(epdir * exp(i(omega tt + 2 pi phi)))
        const double ph = std::sin(omega * tt + phi_cep * 2.0 * pi);
        for (int d = 0; d < 3; ++d) a[d] = -f0 / omega * (cs * cs) * (epdir[d] * ph);
      }
    }
  }
}

// time loop body, time_evolution_step.f90:102-312, linear response
// (yn_fix_func='y' path: V_local fixed), middlepoint propagator.
// The self-consistent variant (sbo_rt_run_scf): after the density, the
// Hartree and exchange-correlation potentials of rho(t+dt) and update_vlocal,
// time_evolution_step.f90:184-207 with yn_fix_func = 'n' (nspin = 1 or 2; Hartree by
// poisson_ft on periodic grids, poisson_isolated_ft on isolated ones).
// method_poisson = 'cg' on isolated grids (time_evolution_step.f90:186-198):
// vh carries the potential from step to step (the CG start), with the two
// stored potentials of the extrapolation
struct ScfCg {
  int layout, lmax;
  const double* rion;
  int natom;
  int npole[3];
  double threshold;
  int maxiter;
  double* vh;     // in: Vh of the initial density; out: the last step's
  int* iters;     // [nt] iterations of each step's solve
};
struct ScfUpdate {
  const double* vpsl;
  const double* brl;
  double* vloc;  // the buffer s->V_local points to
  const ScfCg* cg = nullptr;
};

static int rt_run_impl(sbo_system* s, double* psi_a, double* psi_b, double* work, int nt, double dt,
                       const double* zc, int n_hamil, const double* Ac_ext, double* Ac_ind, double* Ac_tot,
                       int trans_longi, double* curr, double* rbox, double* rho_work, const ScfUpdate* scf) {
  const double pi = 3.141592653589793238462643383279502884;
  const long npts = (long)(s->ie[0] - s->is[0] + 1) * (s->ie[1] - s->is[1] + 1) * (s->ie[2] - s->is[2] + 1);
  std::vector<double> vh(scf ? npts : 0), vxc(scf ? npts * s->nspin : 0), stock1, stock2;
  std::vector<double> rho_tot(scf && s->nspin == 2 ? npts : 0);
  const ScfCg* cg = (scf && !s->periodic) ? scf->cg : nullptr;
  if (cg) {  // initialization_rt.f90:277-286
    vh.assign(cg->vh, cg->vh + npts);
    stock1 = vh;
    stock2 = vh;
  }
  double* in = psi_a;
  double* out = psi_b;
  int which = 1;
  // length gauge (calcVbox, em_field.f90:422-548; time_evolution_step.f90:95-116):
  // E_ext(itt) = -(Ac_ext(itt+1) - Ac_ext(itt)) / dt (initialization_rt.f90:180-183)
  const bool lgauge = !s->periodic && s->length_gauge;
  std::vector<double> veff(lgauge ? npts * s->nspin : 0);
  std::vector<double> cx[3];
  if (lgauge)
    for (int d = 0; d < 3; ++d)  // lg%coordinate, initialization.f90:1125-1190
      for (int i = s->is[d]; i <= s->ie[d]; ++i)
        cx[d].push_back(s->lg_num[d] % 2 == 1 ? i * s->hgs[d] : (i - 0.5) * s->hgs[d]);
  // AETRS: the stored potentials, vloc_old(:,1:2) = V_local (initialization_rt.f90:287-292)
  const long nv = npts * s->nspin;
  // predictor_corrector (time_evolution_step.f90:374-428): the loop's initial
  // potential (update_vlocal of a fixed potential), V_tmp, psi_tmp
  const bool pc = s->pred_corr && !s->aetrs;
  std::vector<double> pc_v0, pc_v, pc_psi, pc_vnew, pc_rho(pc && s->nspin == 2 ? npts : 0);
  if (pc) {
    Idx I(s);
    pc_v0.assign(s->V_local, s->V_local + nv);
    pc_v.resize(nv);
    pc_vnew.resize(nv);
    pc_psi.resize(2 * I.vol * I.norb());
  }
  std::vector<double> old1, old2, vuse;
  if (s->aetrs) {
    old1.assign(s->V_local, s->V_local + nv);
    old2 = old1;
    vuse.resize(nv);
  }
  for (int itt = 1; itt <= nt; ++itt) {
    const double* v_base = s->V_local;
    if (lgauge) {
      double E[3];
      for (int d = 0; d < 3; ++d) E[d] = -(Ac_ext[3 * (itt + 1) + d] - Ac_ext[3 * itt + d]) / dt;
      const long nx = (long)cx[0].size(), ny = (long)cx[1].size();
      for (int is = 0; is < s->nspin; ++is)
        for (long p = 0; p < npts; ++p) {
          const long x = p % nx, y = (p / nx) % ny, z = p / (nx * ny);
          const double vb = 0.0 + (E[0] * cx[0][x] + E[1] * cx[1][y] + E[2] * cx[2][z]);
          veff[is * npts + p] = v_base[is * npts + p] + vb;
        }
      s->V_local = veff.data();
    }
    if (s->periodic) {  // middlepoint: (A(itt) + A(itt-1)) / 2; aetrs: A(itt)
      for (int d = 0; d < 3; ++d)
        s->vec_Ac[d] = s->aetrs ? Ac_tot[3 * itt + d] : 0.5 * (Ac_tot[3 * itt + d] + Ac_tot[3 * (itt - 1) + d]);
      if (s->nlma > 0) sbo_update_kvector_nonlocalpt(s);
    }
    if (pc) {
      const double* Vt = s->V_local;  // V_tmp
      std::copy(in, in + pc_psi.size(), pc_psi.begin());
      sbo_taylor(s, in, out, work, zc, n_hamil);
      sbo_calc_density(s, out, rho_work);
      const double* Vn = pc_v0.data();
      if (scf) {
        const int num[3] = {s->ie[0] - s->is[0] + 1, s->ie[1] - s->is[1] + 1, s->ie[2] - s->is[2] + 1};
        const double* rho_h = rho_work;
        if (s->nspin == 2) {
          for (long i = 0; i < npts; ++i) pc_rho[i] = (0.0 + rho_work[i]) + rho_work[npts + i];
          rho_h = pc_rho.data();
        }
        double exc = 0.0;
        if (s->periodic) {
          sbo_poisson_ft(num, scf->brl, rho_h, vh.data());
        } else if (cg) {  // hartree from the current Vh (no extrapolation here)
          int it = 0;
          sbo_poisson_isolated_cg(s, rho_h, vh.data(), cg->layout, cg->lmax, cg->rion, cg->natom, cg->npole,
                                  cg->threshold, cg->maxiter, &it);
        } else {
          sbo_poisson_isolated_ft(num, scf->brl, rho_h, vh.data());
        }
        if (s->nspin == 2)
          sbo_exc_cor_pz_sp(npts, rho_work, s->hvol, vxc.data(), &exc);
        else
          sbo_exc_cor_pz(npts, rho_work, s->hvol, vxc.data(), &exc);
        sbo_update_vlocal(npts, s->nspin, scf->vpsl, vh.data(), vxc.data(), pc_vnew.data());
        Vn = pc_vnew.data();
      }
      for (long i = 0; i < nv; ++i) pc_v[i] = 0.5 * (Vt[i] + Vn[i]);
      std::copy(pc_psi.begin(), pc_psi.end(), in);
      s->V_local = pc_v.data();
    }
    sbo_taylor(s, in, out, work, zc, n_hamil);
    if (s->aetrs) {  // time_evolution_half_step_etrs, time_evolution_step.f90:430-470
      const double* V = s->V_local;
      double E[3] = {0.0, 0.0, 0.0};
      if (lgauge) {  // E_ext(itt + 1), with E_ext(nt + 1) = E_ext(nt)
        const int j = itt + 1 <= nt ? itt + 1 : nt;
        for (int d = 0; d < 3; ++d) E[d] = -(Ac_ext[3 * (j + 1) + d] - Ac_ext[3 * j + d]) / dt;
      }
      const long nx = s->ie[0] - s->is[0] + 1, ny = s->ie[1] - s->is[1] + 1;
      for (long i = 0; i < nv; ++i) {
        const double vn = 3.0 * V[i] - 3.0 * old1[i] + old2[i];
        old2[i] = old1[i];
        old1[i] = V[i];
        vuse[i] = vn;
        if (lgauge) {  // + Vbox(itt + 1)
          const long p = i % npts;
          const long x = p % nx, y = (p / nx) % ny, z = p / (nx * ny);
          vuse[i] = vuse[i] + (0.0 + (E[0] * cx[0][x] + E[1] * cx[1][y] + E[2] * cx[2][z]));
        }
      }
      s->V_local = vuse.data();
      if (s->periodic) {
        for (int d = 0; d < 3; ++d)
          s->vec_Ac[d] = Ac_ext[3 * (itt + 1) + d] + 2.0 * Ac_ind[3 * itt + d] - Ac_ind[3 * (itt - 1) + d];
        if (s->nlma > 0) sbo_update_kvector_nonlocalpt(s);
      }
      Idx I(s);
      std::copy(out, out + 2 * I.vol * I.norb(), in);  // spsi_in%zwf = spsi_out%zwf
      sbo_taylor(s, in, out, work, zc, n_hamil);
    }
    s->V_local = v_base;  // the step's update_vlocal: the field-free potential again
    if (s->gs_interval >= 1 && itt % s->gs_interval == 0)  // time_evolution_step.f90:149-152
      sbo_gram_schmidt_complex(s, out);
    sbo_calc_density(s, out, rho_work);
    if (scf) {
      const int num[3] = {s->ie[0] - s->is[0] + 1, s->ie[1] - s->is[1] + 1, s->ie[2] - s->is[2] + 1};
      double exc = 0.0;
      // rho = sum over spins of rho_s (time_evolution_step.f90:160-170)
      const double* rho_h = rho_work;
      if (s->nspin == 2) {
        for (long i = 0; i < npts; ++i) rho_tot[i] = (0.0 + rho_work[i]) + rho_work[npts + i];
        rho_h = rho_tot.data();
      }
      if (s->periodic) {
        sbo_poisson_ft(num, scf->brl, rho_h, vh.data());
      } else if (cg) {
        if (itt != 1)
          for (long i = 0; i < npts; ++i) {
            vh[i] = 2.0 * stock1[i] - stock2[i];
            stock2[i] = stock1[i];
          }
        int it = 0;
        sbo_poisson_isolated_cg(s, rho_h, vh.data(), cg->layout, cg->lmax, cg->rion, cg->natom, cg->npole,
                                cg->threshold, cg->maxiter, &it);
        if (cg->iters) cg->iters[itt - 1] = it;
        if (itt != 1) stock1 = vh;
      } else {
        sbo_poisson_isolated_ft(num, scf->brl, rho_h, vh.data());
      }
      if (s->nspin == 2)
        sbo_exc_cor_pz_sp(npts, rho_work, s->hvol, vxc.data(), &exc);
      else
        sbo_exc_cor_pz(npts, rho_work, s->hvol, vxc.data(), &exc);
      sbo_update_vlocal(npts, s->nspin, scf->vpsl, vh.data(), vxc.data(), scf->vloc);
    }
    if (s->periodic) {
      for (int d = 0; d < 3; ++d) s->vec_Ac[d] = Ac_tot[3 * itt + d];
      double c[6] = {0, 0, 0, 0, 0, 0};
      sbo_calc_current(s, out, c);
      double ctot[3];
      for (int d = 0; d < 3; ++d) ctot[d] = s->nspin == 2 ? c[d] + c[3 + d] : c[d];
      for (int d = 0; d < 3; ++d) curr[3 * (itt - 1) + d] = ctot[d];
      // calc_emfields, em_field.f90:24-70
      for (int d = 0; d < 3; ++d) {
        if (trans_longi == 1)
          Ac_ind[3 * (itt + 1) + d] = 2.0 * Ac_ind[3 * itt + d] - Ac_ind[3 * (itt - 1) + d] -
                                      4.0 * pi * ctot[d] * dt * dt;
        else
          Ac_ind[3 * (itt + 1) + d] = 0.0;
        Ac_tot[3 * (itt + 1) + d] = Ac_ext[3 * (itt + 1) + d] + Ac_ind[3 * (itt + 1) + d];
      }
    }
    sbo_calc_dip(s, rho_work, rbox + 4 * (itt - 1));
    double* t = in;
    in = out;
    out = t;
    which = 1 - which;
  }
  if (cg) std::copy(vh.begin(), vh.end(), cg->vh);
  // after the last swap "in" holds the newest orbitals
  return (in == psi_a) ? 0 : 1;
}

int sbo_rt_run(sbo_system* s, double* psi_a, double* psi_b, double* work, int nt, double dt,
               const double* zc, int n_hamil, const double* Ac_ext, double* Ac_ind,
               double* Ac_tot, int trans_longi, double* curr, double* rbox, double* rho_work) {
  return rt_run_impl(s, psi_a, psi_b, work, nt, dt, zc, n_hamil, Ac_ext, Ac_ind, Ac_tot, trans_longi, curr, rbox,
                     rho_work, nullptr);
}

int sbo_rt_run_scf(sbo_system* s, double* psi_a, double* psi_b, double* work, int nt, double dt,
                   const double* zc, int n_hamil, const double* Ac_ext, double* Ac_ind,
                   double* Ac_tot, int trans_longi, double* curr, double* rbox, double* rho_work,
                   const double* vpsl, const double brl[9], double* vloc) {
  const ScfUpdate u{vpsl, brl, vloc};
  const double* saved = s->V_local;
  s->V_local = vloc;
  const int r = rt_run_impl(s, psi_a, psi_b, work, nt, dt, zc, n_hamil, Ac_ext, Ac_ind, Ac_tot, trans_longi, curr,
                            rbox, rho_work, &u);
  s->V_local = saved;
  return r;
}

int sbo_rt_run_scf_cg(sbo_system* s, double* psi_a, double* psi_b, double* work, int nt, double dt,
                      const double* zc, int n_hamil, const double* Ac_ext, double* Ac_ind, double* Ac_tot,
                      int trans_longi, double* curr, double* rbox, double* rho_work, const double* vpsl,
                      double* vloc, double* vh, int layout, int lmax, const double* rion, int natom,
                      const int npole_xyz[3], double threshold, int maxiter, int* iters) {
  if (s->periodic) return -1;
  ScfCg cg{layout, lmax, rion, natom, {npole_xyz[0], npole_xyz[1], npole_xyz[2]}, threshold, maxiter, vh, iters};
  ScfUpdate u{vpsl, nullptr, vloc, &cg};
  const double* saved = s->V_local;
  s->V_local = vloc;
  const int r = rt_run_impl(s, psi_a, psi_b, work, nt, dt, zc, n_hamil, Ac_ext, Ac_ind, Ac_tot, trans_longi, curr,
                            rbox, rho_work, &u);
  s->V_local = saved;
  return r;
}

}  // extern "C"
