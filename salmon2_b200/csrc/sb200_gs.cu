// sb200_gs.cu -- ground state on real orbitals (one k-point): real hpsi
// (dstencil + dpseudo), the band-by-band preconditioned CG eigensolver of
// gscg_rwf, classical Gram-Schmidt and the subspace diagonalisation, all on
// the device.  Orbitals use the resident layout psi[o][z][y][x] (double),
// o = ispin + nspin*io, with the context's grid, V_local and projector tables.
//
// Every reduction is deterministic: per-CTA partial sums in a fixed order,
// then a fixed-order sum of the partials by the consumer.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "sb200_gs.cuh"
#include "sb200_internal.cuh"

namespace sb200 {
namespace {

constexpr int RT = 256;            // threads of the reduction kernels
constexpr int DOT_PTS = RT * 8;    // points per reduction CTA

// ---------------------------------------------------------------------------
// real hpsi: 25-point Laplacian + V_local (stencil.f90:30-80) and the KB term
// (nonlocal_potential.f90:26-171), one thread per point, x/y/z neighbours
// through L1 (tables from the complex path: pmap entries carry uV).
// ---------------------------------------------------------------------------
struct RArgs {
  int nx, ny, nz, periodic, nspin, nlma, natom, nps, totpts;
  long npts;
  double lap0, lapt[12];
  const double* vloc;
  const int *pmap, *ent_lma;
  const double* ent_uv;
  const double* proj;  // [norb][nlma]
  const int *atom_start, *mps, *lma_start, *nproj, *pt_lin;
  const double *uv, *rinv;
};

__device__ __forceinline__ int wrap(int q, int n, int periodic, bool& ok) {
  if (periodic) {
    q = q < 0 ? q + n : (q >= n ? q - n : q);
    ok = true;
  } else {
    ok = (q >= 0) && (q < n);
  }
  return q;
}

__global__ void __launch_bounds__(256) k_dhpsi(const double* __restrict__ in, double* __restrict__ out, RArgs a) {
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= a.npts) return;
  const int o = blockIdx.y;
  const int x = (int)(p % a.nx), y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
  const double* src = in + (long)o * a.npts;
  const long sy = a.nx, sz = (long)a.nx * a.ny;
  double v[3];
  const int c3[3] = {x, y, z}, n3[3] = {a.nx, a.ny, a.nz};
  const long st3[3] = {1, sy, sz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double acc = 0.0;
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      bool okp, okm;
      const int qp = wrap(c3[d] + s, n3[d], a.periodic, okp);
      const int qm = wrap(c3[d] - s, n3[d], a.periodic, okm);
      const double tp = okp ? __ldg(src + p + (qp - c3[d]) * st3[d]) : 0.0;
      const double tm = okm ? __ldg(src + p + (qm - c3[d]) * st3[d]) : 0.0;
      acc += a.lapt[4 * d + s - 1] * (tp + tm);
    }
    v[d] = acc;
  }
  const double vs = v[2] + (v[1] + v[0]);
  double h = (__ldg(a.vloc + (long)(o % a.nspin) * a.npts + p) + a.lap0) * __ldg(src + p) - 0.5 * vs;
  if (a.nlma > 0) {
    const int pm = __ldg(a.pmap + p);
    if (pm >= 0) {
      const double* pj = a.proj + (long)o * a.nlma;
      const int e1 = (pm >> 8) + (pm & 255);
      for (int e = pm >> 8; e < e1; ++e) h += pj[__ldg(a.ent_lma + e)] * __ldg(a.ent_uv + e);
    }
  }
  out[(long)o * a.npts + p] = h;
}

// real projections uVpsi = rinv * sum_j uV(j,ilma) psi(jxyz): warp per (orbital, atom)
__global__ void __launch_bounds__(128) k_dproject(const double* __restrict__ in, double* __restrict__ proj, RArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int atom = blockIdx.x * 4 + warp;
  if (atom >= a.natom) return;
  const int o = blockIdx.y;
  const double* psi = in + (long)o * a.npts;
  const int start = a.atom_start[atom], m = a.mps[atom];
  const int lma0 = a.lma_start[atom], np = a.nproj[atom];
  for (int q0 = 0; q0 < np; q0 += 4) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j = lane; j < m; j += 32) {
      const double v = __ldg(psi + a.pt_lin[start + j]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q0 + q < np) acc[q] += __ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j) * v;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (lane == 0)
      for (int q = 0; q < 4; ++q)
        if (q0 + q < np) proj[(long)o * a.nlma + lma0 + q0 + q] = acc[q] * a.rinv[lma0 + q0 + q];
  }
}

// ---------------------------------------------------------------------------
// per-orbital dot products: part[o][b][k] for up to 3 products at once
// ---------------------------------------------------------------------------
struct DotArgs {
  long npts;
  int nblk, ndot;
  const double *x0, *y0, *x1, *y1, *x2, *y2;
  double* part;  // [norb][nblk][3]
};

__global__ void __launch_bounds__(RT) k_dots(DotArgs a) {
  __shared__ double red[3][RT];
  const int o = blockIdx.y;
  const long base = (long)o * a.npts;
  double s[3] = {0.0, 0.0, 0.0};
  const long p0 = (long)blockIdx.x * DOT_PTS;
  for (int it = 0; it < DOT_PTS / RT; ++it) {
    const long p = p0 + it * RT + threadIdx.x;
    if (p >= a.npts) break;
    s[0] += a.x0[base + p] * a.y0[base + p];
    if (a.ndot > 1) s[1] += a.x1[base + p] * a.y1[base + p];
    if (a.ndot > 2) s[2] += a.x2[base + p] * a.y2[base + p];
  }
  for (int k = 0; k < 3; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int st = RT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 3) a.part[((long)o * a.nblk + blockIdx.x) * 3 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_dots_final(const double* __restrict__ part, int norb, int nblk, double hvol, double* __restrict__ out) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= norb) return;
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[((long)o * nblk + b) * 3 + k];
    out[3 * o + k] = s * hvol;
  }
}

// ---------------------------------------------------------------------------
// CG vector updates with per-orbital coefficients (conjugate_gradient.f90)
// ---------------------------------------------------------------------------
enum { U_GK = 0, U_PK, U_PKO, U_SCALE, U_XH, U_PSI };
struct UpdArgs {
  long npts, n;
  int op;
  const double* coef;  // per-orbital coefficient block (see k_cg_scalars)
  double *a, *b, *c, *d;
};

__global__ void k_cg_update(UpdArgs u) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < u.n; i += (long)gridDim.x * blockDim.x) {
    const int o = (int)(i / u.npts);
    const double* cf = u.coef + CG_NC * o;
    switch (u.op) {
      case U_GK:  // gk = hxk - xkHxk * xk           (a = gk, b = hxk, c = xk)
        u.a[i] = u.b[i] - cf[CG_XKHXK] * u.c[i];
        break;
      case U_PK:  // pk = g + uk * pk                   (a = pk, b = g or pre_g)
        u.a[i] = u.b[i] + cf[CG_UK] * u.a[i];
        break;
      case U_PKO:  // pko = pk - zs * xk                (a = pko, b = pk, c = xk)
        u.a[i] = u.b[i] - cf[CG_ZS] * u.c[i];
        break;
      case U_SCALE:  // pko = pko / sqrt(sum)
        u.a[i] = u.a[i] / sqrt(cf[CG_SUM]);
        break;
      case U_XH: {  // xk = cx xk + cp pko ; hxk = cx hxk + cp hwf  (a=xk, b=pko, c=hxk, d=hwf)
        u.a[i] = cf[CG_CX] * u.a[i] + cf[CG_CP] * u.b[i];
        u.c[i] = cf[CG_CX] * u.c[i] + cf[CG_CP] * u.d[i];
        break;
      }
      case U_PSI: {  // psi = xk / sqrt(xkxk) when 1e-16 < |xkxk| <= 1e30   (a = psi, b = xk)
        const double q = cf[CG_XKXK];
        if (1e-16 < fabs(q) && fabs(q) <= 1e30) u.a[i] = u.b[i] / sqrt(q);
        break;
      }
    }
  }
}

// per-orbital scalar algebra of gscg_rwf; `stage` selects which block of the
// iteration is being completed; dots = latest k_dots_final output [o][3]
__global__ void k_cg_scalars(double* __restrict__ coef, const double* __restrict__ dots, int norb, int stage,
                             int iter) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= norb) return;
  double* cf = coef + CG_NC * o;
  const double* d = dots + 3 * o;
  switch (stage) {
    case 0:  // initial <xk|H|xk>
      cf[CG_XKHXK] = d[0];
      break;
    case 1: {  // sum = <(pre)g|g>; uk; gkgk = sum
      const double sum = d[0];
      cf[CG_UK] = (iter == 1) ? 0.0 : ((fabs(cf[CG_GKGK]) > 1e-16) ? sum / cf[CG_GKGK] : 0.0);
      cf[CG_GKGK] = sum;
      break;
    }
    case 2:  // zs = <xk|pk>
      cf[CG_ZS] = d[0];
      break;
    case 3:  // sum = <pko|pko>
      cf[CG_SUM] = d[0];
      break;
    case 4: {  // xkHpk, pkHpk -> ev, cx, cp
      const double xkHxk = cf[CG_XKHXK], xkHpk = d[0], pkHpk = d[1];
      const double ev = 0.5 * ((xkHxk + pkHpk) - sqrt((xkHxk - pkHpk) * (xkHxk - pkHpk) +
                                                      4.0 * fabs(xkHpk) * fabs(xkHpk)));
      double cx, cp;
      if (fabs(ev - xkHxk) > 1e-16) {
        cx = xkHpk / (ev - xkHxk);
        cp = 1.0 / sqrt(1.0 + fabs(cx) * fabs(cx));
        cx = cx * cp;
      } else {
        cx = 1.0;
        cp = 0.0;
      }
      cf[CG_CX] = cx;
      cf[CG_CP] = cp;
      break;
    }
    case 5:  // xkHxk, xkxk after the update
      cf[CG_XKHXK] = d[0];
      cf[CG_XKXK] = d[1];
      break;
  }
}

// low-pass preconditioner (preconditioning.f90:25-77), 3-point Laplacian
__global__ void k_precond(const double* __restrict__ g, double* __restrict__ pre, RArgs a, double hx2, double hy2,
                          double hz2, double omega_d) {
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= a.npts) return;
  const int o = blockIdx.y;
  const int x = (int)(p % a.nx), y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
  const double* t = g + (long)o * a.npts;
  const double c = t[p];
  auto nb = [&](int q, int n, int cc, long st) -> double {
    bool ok;
    const int w = wrap(q, n, a.periodic, ok);
    return ok ? t[p + (w - cc) * st] : 0.0;
  };
  const double v = (nb(x + 1, a.nx, x, 1) - 2.0 * c + nb(x - 1, a.nx, x, 1)) / hx2 +
                   (nb(y + 1, a.ny, y, a.nx) - 2.0 * c + nb(y - 1, a.ny, y, a.nx)) / hy2 +
                   (nb(z + 1, a.nz, z, (long)a.nx * a.ny) - 2.0 * c + nb(z - 1, a.nz, z, (long)a.nx * a.ny)) / hz2;
  pre[(long)o * a.npts + p] = omega_d * (2.0 * c - omega_d * (-0.5 * v));
}

// ---------------------------------------------------------------------------
// Tall-skinny products for Gram-Schmidt and the subspace matrix:
//   part[b][i][j] = sum_{p in chunk b} A[i][p] * B[j][p], i < m, j < n
// One CTA = one 32 x 32 output tile over a point chunk; fixed summation order.
// ---------------------------------------------------------------------------
constexpr int GT = 32, GK = 64;
__global__ void __launch_bounds__(256) k_gram_part(const double* __restrict__ A, int m, const double* __restrict__ B,
                                                   int n, long npts, long chunk, double* __restrict__ part) {
  __shared__ double As[GT][GK + 1], Bs[GT][GK + 1];
  const int ti = blockIdx.x, tj = blockIdx.y, b = blockIdx.z;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // each thread: 2 x 2 outputs
  const long p0 = (long)b * chunk, p1 = min(npts, p0 + chunk);
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (long pp = p0; pp < p1; pp += GK) {
    for (int c = threadIdx.x; c < GT * GK; c += 256) {
      const int r = c / GK, k = c % GK;
      const int i = ti * GT + r, j = tj * GT + r;
      const long p = pp + k;
      As[r][k] = (i < m && p < p1) ? A[(long)i * npts + p] : 0.0;
      Bs[r][k] = (j < n && p < p1) ? B[(long)j * npts + p] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < GK; ++k) {
      const double a0 = As[2 * ty][k], a1 = As[2 * ty + 1][k];
      const double b0 = Bs[2 * tx][k], b1 = Bs[2 * tx + 1][k];
      acc[0][0] += a0 * b0;
      acc[0][1] += a0 * b1;
      acc[1][0] += a1 * b0;
      acc[1][1] += a1 * b1;
    }
    __syncthreads();
  }
  for (int u = 0; u < 2; ++u)
    for (int v = 0; v < 2; ++v) {
      const int i = ti * GT + 2 * ty + u, j = tj * GT + 2 * tx + v;
      if (i < m && j < n) part[((long)b * m + i) * n + j] = acc[u][v];
    }
}

__global__ void k_gram_final(const double* __restrict__ part, int nb, long mn, double scale, double* __restrict__ out) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < mn; q += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(long)b * mn + q];
    out[q] = s * scale;
  }
}

// Y[j][p] = beta * Y[j][p] + alpha * sum_i X[i][p] * M[i][j]; M column-major m x n
__global__ void __launch_bounds__(256) k_rotate(const double* __restrict__ X, int m, const double* __restrict__ M,
                                                int n, long npts, double alpha, double beta, double* __restrict__ Y) {
  __shared__ double Ms[GT][GT + 1];
  const long p = blockIdx.x * 256L + threadIdx.x;
  const int j0 = blockIdx.y * GT;
  double acc[GT];
#pragma unroll
  for (int u = 0; u < GT; ++u) acc[u] = 0.0;
  for (int i0 = 0; i0 < m; i0 += GT) {
    for (int c = threadIdx.x; c < GT * GT; c += 256) {
      const int ii = c / GT, jj = c % GT;
      Ms[ii][jj] = (i0 + ii < m && j0 + jj < n) ? M[(long)(j0 + jj) * m + (i0 + ii)] : 0.0;
    }
    __syncthreads();
    if (p < npts) {
      for (int ii = 0; ii < GT && i0 + ii < m; ++ii) {
        const double x = X[(long)(i0 + ii) * npts + p];
#pragma unroll
        for (int u = 0; u < GT; ++u) acc[u] += x * Ms[ii][u];
      }
    }
    __syncthreads();
  }
  if (p < npts)
    for (int u = 0; u < GT; ++u)
      if (j0 + u < n) {
        const long q = (long)(j0 + u) * npts + p;
        Y[q] = alpha * acc[u] + (beta != 0.0 ? beta * Y[q] : 0.0);
      }
}

// y[p] = y[p] - x[p] * coef  (one orbital) and norm handled by dots
__global__ void k_axpy(double* __restrict__ y, const double* __restrict__ x, double a, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + y[i];
}

// single vector: partial sums of squares, then scale by 1/sqrt(hvol * sum)
__global__ void __launch_bounds__(RT) k_sq_part(const double* __restrict__ y, long n, double* __restrict__ part) {
  __shared__ double red[RT];
  double s = 0.0;
  const long p0 = (long)blockIdx.x * DOT_PTS;
  for (int it = 0; it < DOT_PTS / RT; ++it) {
    const long p = p0 + it * RT + threadIdx.x;
    if (p >= n) break;
    s += y[p] * y[p];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = RT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_scale_norm(double* __restrict__ y, long n, const double* __restrict__ part, int nblk, double hvol) {
  __shared__ double f;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[b];
    f = 1.0 / sqrt(s * hvol);
  }
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = f * y[i];
}

__global__ void k_relayout_real(const double* __restrict__ src, double* __restrict__ dst, int nx, int ny, int nz,
                                int nxa, int nya, long vola, int ox, int oy, int oz, int norb, int to_ref) {
  const long npts = (long)nx * ny * nz;
  const long total = npts * norb;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long o = i / npts, p = i % npts;
    const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
    const long r = o * vola + (x + ox) + (long)nxa * ((y + oy) + (long)nya * (z + oz));
    if (to_ref) dst[r] = src[i];
    else dst[i] = src[r];
  }
}

int gridsz(long n) {
  long b = (n + 255) / 256;
  if (b > 148L * 32) b = 148L * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static RArgs rargs(sb200_ctx* c) {
  RArgs a;
  a.nx = c->g.nx;
  a.ny = c->g.ny;
  a.nz = c->g.nz;
  a.periodic = c->g.periodic;
  a.nspin = c->orb.nspin;
  a.nlma = c->pp.nlma;
  a.natom = c->pp.natom;
  a.nps = c->pp.nps;
  a.totpts = c->pp.totpts;
  a.npts = c->g.npts;
  a.lap0 = c->g.coef_lap0;
  for (int i = 0; i < 12; ++i) a.lapt[i] = c->g.coef_lap[i];
  a.vloc = c->d_vloc;
  a.pmap = c->pp.d_pmap;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_uv = c->pp.d_ent_uv;
  a.proj = c->gs.d_proj;
  a.atom_start = c->pp.d_atom_start;
  a.mps = c->pp.d_mps;
  a.lma_start = c->pp.d_lma_start;
  a.nproj = c->pp.d_nproj;
  a.pt_lin = c->pp.d_pt_lin;
  a.uv = c->pp.d_uv;
  a.rinv = c->pp.d_rinv;
  return a;
}

int gs_ensure(sb200_ctx* c, bool cg_work) {
  GSState& s = c->gs;
  const long n = c->g.npts * c->orb.norb;
  const int norb = c->orb.norb;
  const int nblk = (int)((c->g.npts + DOT_PTS - 1) / DOT_PTS);
  if (s.n != n || s.norb != norb) {
    dfree(s.d_proj);
    dfree(s.d_part);
    dfree(s.d_dots);
    dfree(s.d_coef);
    dfree(s.d_work);
    s.n = n;
    s.norb = norb;
    s.nblk = nblk;
    s.have_work = false;
    TRY_GS(dalloc(&s.d_proj, (size_t)norb * (c->pp.nlma > 0 ? c->pp.nlma : 1)));
    TRY_GS(dalloc(&s.d_part, (size_t)norb * nblk * 3));
    TRY_GS(dalloc(&s.d_dots, (size_t)norb * 3));
    TRY_GS(dalloc(&s.d_coef, (size_t)norb * CG_NC));
  }
  if (cg_work && !s.have_work) {
    TRY_GS(dalloc(&s.d_work, (size_t)n * 7));
    s.have_work = true;
  }
  return SB200_OK;
}

int gs_hpsi(sb200_ctx* c, const double* in, double* out) {
  RArgs a = rargs(c);
  if (a.nlma > 0) {
    dim3 g((a.natom + 3) / 4, c->orb.norb);
    k_dproject<<<g, 128, 0, c->stream>>>(in, c->gs.d_proj, a);
    SB_LAUNCH_CHECK("k_dproject");
  }
  dim3 g((unsigned)((a.npts + 255) / 256), c->orb.norb);
  k_dhpsi<<<g, 256, 0, c->stream>>>(in, out, a);
  SB_LAUNCH_CHECK("k_dhpsi");
  return SB200_OK;
}

// up to three per-orbital dot products into gs.d_dots[o][0..2] (times hvol)
int gs_dots(sb200_ctx* c, int ndot, const double* x0, const double* y0, const double* x1 = nullptr,
            const double* y1 = nullptr, const double* x2 = nullptr, const double* y2 = nullptr) {
  GSState& s = c->gs;
  DotArgs d;
  d.npts = c->g.npts;
  d.nblk = s.nblk;
  d.ndot = ndot;
  d.x0 = x0;
  d.y0 = y0;
  d.x1 = x1;
  d.y1 = y1;
  d.x2 = x2;
  d.y2 = y2;
  d.part = s.d_part;
  dim3 g(s.nblk, c->orb.norb);
  k_dots<<<g, RT, 0, c->stream>>>(d);
  SB_LAUNCH_CHECK("k_dots");
  k_dots_final<<<(c->orb.norb + 127) / 128, 128, 0, c->stream>>>(s.d_part, c->orb.norb, s.nblk, c->g.hvol,
                                                                  s.d_dots);
  SB_LAUNCH_CHECK("k_dots_final");
  return SB200_OK;
}

int gs_scalars(sb200_ctx* c, int stage, int iter) {
  k_cg_scalars<<<(c->orb.norb + 127) / 128, 128, 0, c->stream>>>(c->gs.d_coef, c->gs.d_dots, c->orb.norb, stage,
                                                                  iter);
  SB_LAUNCH_CHECK("k_cg_scalars");
  return SB200_OK;
}

int gs_update(sb200_ctx* c, int op, double* a, double* b = nullptr, double* cc = nullptr, double* d = nullptr) {
  UpdArgs u;
  u.npts = c->g.npts;
  u.n = c->gs.n;
  u.op = op;
  u.coef = c->gs.d_coef;
  u.a = a;
  u.b = b;
  u.c = cc;
  u.d = d;
  k_cg_update<<<gridsz(u.n), 256, 0, c->stream>>>(u);
  SB_LAUNCH_CHECK("k_cg_update");
  return SB200_OK;
}

int gs_precond(sb200_ctx* c, const double* g, double* pre, double alpha) {
  RArgs a = rargs(c);
  const double h0 = c->g.hgs[0], h1 = c->g.hgs[1], h2 = c->g.hgs[2];
  const double omega = 2.0 * (1.0 - alpha);
  const double d = -0.5 * ((-2.0) / (h0 * h0) + (-2.0) / (h1 * h1) + (-2.0) / (h2 * h2));
  dim3 gr((unsigned)((a.npts + 255) / 256), c->orb.norb);
  k_precond<<<gr, 256, 0, c->stream>>>(g, pre, a, h0 * h0, h1 * h1, h2 * h2, omega / d);
  SB_LAUNCH_CHECK("k_precond");
  return SB200_OK;
}

// C (m x n, row-major [i][j]) = scale * A(m orbitals) . B(n orbitals)
// ---- complex column Gram-Schmidt (gram_schmidt_col_complex8) -------------
// Orbitals io of one (k, spin) group sit `stride` complex values apart.
// part[io2][b] = sum over the points of block b of conj(psi_io2) psi_io1
__global__ void __launch_bounds__(RT) k_zgs_dots(const double2* __restrict__ psi, long stride, int io1, long npts,
                                                 double2* __restrict__ part, int nb) {
  __shared__ double rr[RT], ri[RT];
  const int io2 = blockIdx.y;
  const double2* a = psi + stride * io2;
  const double2* b = psi + stride * io1;
  double sr = 0.0, si = 0.0;
  const long p0 = (long)blockIdx.x * DOT_PTS;
  for (int it = 0; it < DOT_PTS / RT; ++it) {
    const long p = p0 + it * RT + threadIdx.x;
    if (p < npts) {
      const double2 x = a[p], y = b[p];
      sr += x.x * y.x + x.y * y.y;
      si += x.x * y.y - x.y * y.x;
    }
  }
  rr[threadIdx.x] = sr;
  ri[threadIdx.x] = si;
  __syncthreads();
  for (int st = RT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      rr[threadIdx.x] += rr[threadIdx.x + st];
      ri[threadIdx.x] += ri[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(long)io2 * nb + blockIdx.x] = make_double2(rr[0], ri[0]);
}

// coeff[io2] = hvol * sum_b part[io2][b] (blocks in order)
__global__ void k_zgs_coeff(const double2* __restrict__ part, int nb, int m, double hvol,
                            double2* __restrict__ coeff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double sr = 0.0, si = 0.0;
  for (int b = 0; b < nb; ++b) {
    sr += part[(long)i * nb + b].x;
    si += part[(long)i * nb + b].y;
  }
  coeff[i] = make_double2(sr * hvol, si * hvol);
}

// psi_io1 <- psi_io1 - sum_{io2 < io1} coeff[io2] psi_io2 (exclusion term
// accumulated in io2 order, then subtracted)
__global__ void k_zgs_sub(double2* __restrict__ psi, long stride, int io1, const double2* __restrict__ coeff,
                          long npts) {
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)gridDim.x * 256) {
    double2 exc = make_double2(0.0, 0.0);
    for (int io2 = 0; io2 < io1; ++io2) {
      const double2 cf = coeff[io2], x = psi[stride * io2 + p];
      exc = make_double2(cf.x * x.x - cf.y * x.y + exc.x, cf.x * x.y + cf.y * x.x + exc.y);
    }
    double2* w = psi + stride * io1 + p;
    *w = make_double2(-exc.x + w->x, -exc.y + w->y);
  }
}

// part[b] = sum over block b of |psi|^2
__global__ void __launch_bounds__(RT) k_zsq_part(const double2* __restrict__ y, long n, double* __restrict__ part) {
  __shared__ double r[RT];
  double s = 0.0;
  const long p0 = (long)blockIdx.x * DOT_PTS;
  for (int it = 0; it < DOT_PTS / RT; ++it) {
    const long p = p0 + it * RT + threadIdx.x;
    if (p < n) s += y[p].x * y[p].x + y[p].y * y[p].y;
  }
  r[threadIdx.x] = s;
  __syncthreads();
  for (int st = RT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) r[threadIdx.x] += r[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = r[0];
}

// y <- y / sqrt(hvol * sum_b part[b])
__global__ void k_zscale_norm(double2* __restrict__ y, long n, const double* __restrict__ part, int nb, double hvol) {
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[b];
  const double sc = 1.0 / sqrt(s * hvol);
  for (long p = blockIdx.x * 256L + threadIdx.x; p < n; p += (long)gridDim.x * 256)
    y[p] = make_double2(sc * y[p].x, sc * y[p].y);
}

int gs_gram(sb200_ctx* c, const double* A, int m, const double* B, int n, double scale, double* C_dev) {
  const long npts = c->g.npts;
  int nb = (int)((npts + 16383) / 16384);
  if (nb > 64) nb = 64;
  const long chunk = ((npts + nb - 1) / nb + GK - 1) / GK * GK;
  nb = (int)((npts + chunk - 1) / chunk);
  const size_t need = (size_t)nb * m * n;
  if (c->gs.gram_cap < need) {
    dfree(c->gs.d_gram);
    TRY_GS(dalloc(&c->gs.d_gram, need));
    c->gs.gram_cap = need;
  }
  dim3 g((m + GT - 1) / GT, (n + GT - 1) / GT, nb);
  k_gram_part<<<g, 256, 0, c->stream>>>(A, m, B, n, npts, chunk, c->gs.d_gram);
  SB_LAUNCH_CHECK("k_gram_part");
  k_gram_final<<<gridsz((long)m * n), 256, 0, c->stream>>>(c->gs.d_gram, nb, (long)m * n, scale, C_dev);
  SB_LAUNCH_CHECK("k_gram_final");
  return SB200_OK;
}

int gs_relayout(sb200_ctx* c, const double* src, double* dst, int norb, bool to_ref) {
  const GridInfo& g = c->g;
  const int nxa = g.ie_array[0] - g.is_array[0] + 1;
  const int nya = g.ie_array[1] - g.is_array[1] + 1;
  k_relayout_real<<<gridsz(g.npts * norb), 256, 0, c->stream>>>(src, dst, g.nx, g.ny, g.nz, nxa, nya,
                                                                 g.vol_array(), g.is[0] - g.is_array[0],
                                                                 g.is[1] - g.is_array[1], g.is[2] - g.is_array[2],
                                                                 norb, to_ref ? 1 : 0);
  SB_LAUNCH_CHECK("k_relayout_real");
  return SB200_OK;
}

int gs_axpy(sb200_ctx* c, double* y, const double* x, double a, long n) {
  k_axpy<<<gridsz(n), 256, 0, c->stream>>>(y, x, a, n);
  SB_LAUNCH_CHECK("k_axpy");
  return SB200_OK;
}

int gs_rotate(sb200_ctx* c, const double* X, int m, const double* M_dev, int n, double beta, double* Y) {
  dim3 g((unsigned)((c->g.npts + 255) / 256), (n + GT - 1) / GT);
  k_rotate<<<g, 256, 0, c->stream>>>(X, m, M_dev, n, c->g.npts, 1.0, beta, Y);
  SB_LAUNCH_CHECK("k_rotate");
  return SB200_OK;
}

// y <- y - sum_i coeff[i] * X_i  (exc accumulated in i order, then subtracted)
// Y -= X (X^T Y) hvol for Y of n orbitals: removes from every column of Y its
// components along the m orthonormal orbitals X (scratch: the small-matrix area)
int gs_project_out(sb200_ctx* c, const double* X, int m, double* Y, int n) {
  if (c->gs.mat_cap < (size_t)m * n) {
    dfree(c->gs.d_mat);
    TRY_GS(dalloc(&c->gs.d_mat, (size_t)m * n));
    c->gs.mat_cap = (size_t)m * n;
  }
  // gs_gram(Y, X) stores <Y_j, X_i> at j*m + i: the column-major M(i, j) k_rotate reads
  TRY_GS(gs_gram(c, Y, n, X, m, c->g.hvol, c->gs.d_mat));
  dim3 g((unsigned)((c->g.npts + 255) / 256), (n + GT - 1) / GT);
  k_rotate<<<g, 256, 0, c->stream>>>(X, m, c->gs.d_mat, n, c->g.npts, -1.0, 1.0, Y);
  SB_LAUNCH_CHECK("k_rotate");
  return SB200_OK;
}

int gs_rotate_sub(sb200_ctx* c, const double* X, int m, const double* coeff_dev, double* y) {
  dim3 g((unsigned)((c->g.npts + 255) / 256), 1);
  k_rotate<<<g, 256, 0, c->stream>>>(X, m, coeff_dev, 1, c->g.npts, -1.0, 1.0, y);
  SB_LAUNCH_CHECK("k_rotate");
  return SB200_OK;
}

// y <- y / sqrt(hvol * sum y^2), one orbital, deterministic
int gs_norm_scale(sb200_ctx* c, double* y) {
  const long n = c->g.npts;
  const int nblk = (int)((n + DOT_PTS - 1) / DOT_PTS);
  k_sq_part<<<nblk, RT, 0, c->stream>>>(y, n, c->gs.d_part);
  SB_LAUNCH_CHECK("k_sq_part");
  k_scale_norm<<<gridsz(n), 256, 0, c->stream>>>(y, n, c->gs.d_part, nblk, c->g.hvol);
  SB_LAUNCH_CHECK("k_scale_norm");
  return SB200_OK;
}

}  // namespace sb200

// ---------------------------------------------------------------------------
// C ABI of the ground-state path
// ---------------------------------------------------------------------------
using namespace sb200;

namespace {

int gs_ready(sb200_ctx* c) {
  if (!c) return set_error(SB200_ERR_INVALID_ARG, "null ctx");
  if (!c->g.set || !c->orb.set || !c->vloc_set)
    return set_error(SB200_ERR_STATE, "ground state needs sb200_set_grid / _set_orbitals / _set_vlocal first");
  if (c->orb.nk != 1) return set_error(SB200_ERR_UNSUPPORTED, "real-orbital ground state takes one k-point");
  return SB200_OK;
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int gs_mat(sb200_ctx* c, size_t n) {
  if (c->gs.mat_cap >= n) return SB200_OK;
  dfree(c->gs.d_mat);
  TRY_GS(dalloc(&c->gs.d_mat, n));
  c->gs.mat_cap = n;
  return SB200_OK;
}

int gs_relayout_all(sb200_ctx* c, const double* src_ref, double* dst_dev, double* dst_ref, const double* src_dev,
                    bool to_ref) {
  const size_t blk = (size_t)c->g.vol_array() * sizeof(double);
  const int norb = c->orb.norb;
  int chunk = (int)((size_t)(256u << 20) / blk);
  if (chunk < 1) chunk = 1;
  if (chunk > norb) chunk = norb;
  if (c->stage_bytes < blk * chunk) {
    if (c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    c->stage_bytes = 0;
    SB_CUDA(cudaMalloc(&c->d_stage, blk * chunk));
    c->stage_bytes = blk * chunk;
  }
  for (int o0 = 0; o0 < norb; o0 += chunk) {
    const int n = (o0 + chunk <= norb) ? chunk : norb - o0;
    if (!to_ref) {
      SB_CUDA(cudaMemcpyAsync(c->d_stage, (const char*)src_ref + blk * o0, blk * n, cudaMemcpyDefault, c->stream));
      TRY_GS(gs_relayout(c, (const double*)c->d_stage, dst_dev + c->g.npts * o0, n, false));
    } else {
      SB_CUDA(cudaMemsetAsync(c->d_stage, 0, blk * n, c->stream));
      TRY_GS(gs_relayout(c, src_dev + c->g.npts * o0, (double*)c->d_stage, n, true));
      SB_CUDA(cudaMemcpyAsync((char*)dst_ref + blk * o0, c->d_stage, blk * n, cudaMemcpyDefault, c->stream));
    }
    SB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return SB200_OK;
}

}  // namespace

extern "C" {

int sb200_gs_from_ref(sb200_ctx* c, const double* rwf_ref, double* psi_dev) {
  TRY_GS(gs_ready(c));
  if (!rwf_ref || !psi_dev) return set_error(SB200_ERR_INVALID_ARG, "null orbital pointer");
  DevGuard dg(c->device);
  return gs_relayout_all(c, rwf_ref, psi_dev, nullptr, nullptr, false);
}

int sb200_gs_to_ref(sb200_ctx* c, const double* psi_dev, double* rwf_ref) {
  TRY_GS(gs_ready(c));
  if (!rwf_ref || !psi_dev) return set_error(SB200_ERR_INVALID_ARG, "null orbital pointer");
  DevGuard dg(c->device);
  return gs_relayout_all(c, nullptr, nullptr, rwf_ref, psi_dev, true);
}

int sb200_hpsi_real(sb200_ctx* c, const double* tpsi, double* htpsi) {
  TRY_GS(gs_ready(c));
  if (!tpsi || !htpsi || tpsi == htpsi) return set_error(SB200_ERR_INVALID_ARG, "tpsi/htpsi null or aliased");
  DevGuard dg(c->device);
  TRY_GS(gs_ensure(c, false));
  return gs_hpsi(c, tpsi, htpsi);
}

int sb200_gscg(sb200_ctx* c, double* psi, int ncg, int precondition, double alpha_pre, double* esp) {
  TRY_GS(gs_ready(c));
  if (!psi || ncg < 1 || precondition < SB200_PRECOND_NONE || precondition > SB200_PRECOND_LEARNED)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_gscg: bad argument");
  if (precondition == SB200_PRECOND_LEARNED && !c->learned_set)
    return set_error(SB200_ERR_STATE, "learned preconditioner weights not set");
  DevGuard dg(c->device);
  TRY_GS(gs_ensure(c, true));
  const long n = c->gs.n;
  double* w = c->gs.d_work;
  double *xk = w, *hxk = w + n, *pk = w + 2 * n, *gk = w + 3 * n, *pre = w + 4 * n, *pko = w + 5 * n,
         *hwf = w + 6 * n;
  SB_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * 7 * n, c->stream));
  SB_CUDA(cudaMemcpyAsync(xk, psi, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  TRY_GS(gs_hpsi(c, xk, hxk));
  TRY_GS(gs_dots(c, 1, xk, hxk));
  TRY_GS(gs_scalars(c, 0, 0));
  for (int iter = 1; iter <= ncg; ++iter) {
    TRY_GS(gs_update(c, U_GK, gk, hxk, xk));
    const double* g_for_p = gk;
    if (precondition == SB200_PRECOND_LOWPASS) {
      TRY_GS(gs_precond(c, gk, pre, alpha_pre));
      TRY_GS(gs_dots(c, 1, pre, gk));
      g_for_p = pre;
    } else if (precondition == SB200_PRECOND_LEARNED) {
      TRY_GS(learned_precond_apply(c, gk, xk, pre));
      TRY_GS(gs_dots(c, 1, pre, gk));
      g_for_p = pre;
    } else {
      TRY_GS(gs_dots(c, 1, gk, gk));
    }
    // the network direction is not a fixed linear preconditioner: with it the
    // conjugation restarts every iteration (uk = 0, as in the first iteration)
    TRY_GS(gs_scalars(c, 1, precondition == SB200_PRECOND_LEARNED ? 1 : iter));
    TRY_GS(gs_update(c, U_PK, pk, (double*)g_for_p));
    TRY_GS(gs_dots(c, 1, xk, pk));
    TRY_GS(gs_scalars(c, 2, iter));
    TRY_GS(gs_update(c, U_PKO, pko, pk, xk));
    TRY_GS(gs_dots(c, 1, pko, pko));
    TRY_GS(gs_scalars(c, 3, iter));
    TRY_GS(gs_update(c, U_SCALE, pko));
    TRY_GS(gs_hpsi(c, pko, hwf));
    TRY_GS(gs_dots(c, 2, xk, hwf, pko, hwf));
    TRY_GS(gs_scalars(c, 4, iter));
    TRY_GS(gs_update(c, U_XH, xk, pko, hxk, hwf));
    TRY_GS(gs_dots(c, 2, xk, hxk, xk, xk));
    TRY_GS(gs_scalars(c, 5, iter));
    TRY_GS(gs_update(c, U_PSI, psi, xk));
  }
  if (esp) {
    std::vector<double> cf((size_t)c->orb.norb * CG_NC);
    SB_CUDA(cudaMemcpyAsync(cf.data(), c->gs.d_coef, cf.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
    for (int o = 0; o < c->orb.norb; ++o) esp[o] = cf[(size_t)o * CG_NC + CG_XKHXK] / cf[(size_t)o * CG_NC + CG_XKXK];
  }
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

// gram_schmidt_col_real8 (gram_schmidt_orth.f90:59-230): classical GS, the
// coefficients of orbital io1 taken against its original vector.
int sb200_gram_schmidt_real(sb200_ctx* c, double* psi) {
  TRY_GS(gs_ready(c));
  if (!psi) return set_error(SB200_ERR_INVALID_ARG, "null psi");
  DevGuard dg(c->device);
  TRY_GS(gs_ensure(c, false));
  const int nspin = c->orb.nspin, no = c->orb.no;
  const long npts = c->g.npts;
  TRY_GS(gs_mat(c, (size_t)no + 8));
  double* coeff = c->gs.d_mat;
  // orbitals of one spin are strided by nspin blocks: gather per spin
  double* buf = nullptr;
  if (nspin > 1) {
    TRY_GS(gs_ensure(c, true));
    buf = c->gs.d_work;  // [no][npts] of the current spin + 1 scratch block
  }
  for (int is = 0; is < nspin; ++is) {
    double* P = psi;
    if (nspin > 1) {
      for (int io = 0; io < no; ++io)
        SB_CUDA(cudaMemcpyAsync(buf + npts * io, psi + npts * ((long)io * nspin + is), sizeof(double) * npts,
                                cudaMemcpyDeviceToDevice, c->stream));
      P = buf;
    }
    for (int io1 = 0; io1 < no; ++io1) {
      double* w1 = P + npts * io1;
      if (io1 > 0) {
        // coeff(io2) = hvol <psi_io2 | psi_io1>, io2 < io1 ; w1 -= sum coeff * psi_io2
        TRY_GS(gs_gram(c, P, io1, w1, 1, c->g.hvol, coeff));
        TRY_GS(gs_rotate_sub(c, P, io1, coeff, w1));
      }
      TRY_GS(gs_norm_scale(c, w1));
    }
    if (nspin > 1)
      for (int io = 0; io < no; ++io)
        SB_CUDA(cudaMemcpyAsync(psi + npts * ((long)io * nspin + is), buf + npts * io, sizeof(double) * npts,
                                cudaMemcpyDeviceToDevice, c->stream));
  }
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

}  // extern "C"

namespace sb200 {
// scratch of gs_complex_issue: part [no][nb], coeff [no]
size_t gs_complex_part_len(const sb200_ctx* c) {
  const long nb = (c->g.npts + DOT_PTS - 1) / DOT_PTS;
  return (size_t)c->orb.no * (size_t)nb;
}

// gram_schmidt_col_complex8's launches for every (k, spin) group, on the
// context's stream, with caller-given scratch: no allocation, no host wait
// (also issued inside the time loop's CUDA graph)
int gs_complex_issue(sb200_ctx* c, double2* z, double2* part, double2* coeff) {
  const int nspin = c->orb.nspin, no = c->orb.no, nk = c->orb.nk;
  const long npts = c->g.npts;
  const int nb = (int)((npts + DOT_PTS - 1) / DOT_PTS);
  const long stride = (long)nspin * npts;
  for (int ik = 0; ik < nk; ++ik)
    for (int is = 0; is < nspin; ++is) {
      double2* base = z + npts * ((long)is + (long)nspin * no * ik);
      for (int io1 = 0; io1 < no; ++io1) {
        double2* w1 = base + stride * io1;
        if (io1 > 0) {
          k_zgs_dots<<<dim3(nb, io1), RT, 0, c->stream>>>(base, stride, io1, npts, part, nb);
          k_zgs_coeff<<<(io1 + 127) / 128, 128, 0, c->stream>>>(part, nb, io1, c->g.hvol, coeff);
          k_zgs_sub<<<gridsz(npts), 256, 0, c->stream>>>(base, stride, io1, coeff, npts);
        }
        k_zsq_part<<<nb, RT, 0, c->stream>>>(w1, npts, (double*)part);
        k_zscale_norm<<<gridsz(npts), 256, 0, c->stream>>>(w1, npts, (const double*)part, nb, c->g.hvol);
      }
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_error(e, "complex Gram-Schmidt");
    }
  return SB200_OK;
}
}  // namespace sb200

extern "C" {

// gram_schmidt_col_complex8 (gram_schmidt_orth.f90:1069-1242) for every
// (k, spin) group of the complex orbital block, orbitals in order.
int sb200_gram_schmidt_complex(sb200_ctx* c, double* psi) {
  if (!c) return set_error(SB200_ERR_INVALID_ARG, "null ctx");
  if (!c->g.set || !c->orb.set) return set_error(SB200_ERR_STATE, "sb200_set_grid / _set_orbitals first");
  if (!psi) return set_error(SB200_ERR_INVALID_ARG, "null psi");
  DevGuard dg(c->device);
  const int nspin = c->orb.nspin, no = c->orb.no, nk = c->orb.nk;
  const long npts = c->g.npts;
  const int nb = (int)((npts + DOT_PTS - 1) / DOT_PTS);
  double2* part = nullptr;
  double2* coeff = nullptr;
  TRY_GS(dalloc(&part, (size_t)no * nb));
  int r = dalloc(&coeff, (size_t)no);
  (void)nspin;
  (void)nk;
  if (r == SB200_OK) r = gs_complex_issue(c, (double2*)psi, part, coeff);
  if (r == SB200_OK) {
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) r = cuda_error(e, "complex Gram-Schmidt");
  }
  dfree(part);
  dfree(coeff);
  return r;
}

// ssdg_rwf (subspace_diagonalization.f90:62-238): H_sub = <psi_i|H|psi_j>,
// its eigenvectors on the GPU (sb200_eigh.cu), psi <- psi V, normalised.
// evals(no*nspin) host.
int sb200_subspace_diag_real(sb200_ctx* c, double* psi, double* evals) {
  TRY_GS(gs_ready(c));
  if (!psi) return set_error(SB200_ERR_INVALID_ARG, "null psi");
  DevGuard dg(c->device);
  TRY_GS(gs_ensure(c, true));
  const int nspin = c->orb.nspin, no = c->orb.no;
  const long npts = c->g.npts;
  if (nspin != 1) return set_error(SB200_ERR_UNSUPPORTED, "subspace diagonalisation implemented for nspin = 1");
  double* hpsi = c->gs.d_work;
  double* rot = c->gs.d_work + c->gs.n;
  TRY_GS(gs_hpsi(c, psi, hpsi));
  // work: M (no^2), V (no^2), eigensolver scratch (2 no^2), w (no), info
  const size_t nn = (size_t)no * no;
  TRY_GS(gs_mat(c, 4 * nn + no + 8));
  double* M = c->gs.d_mat;
  double* V = M + nn;
  double* ework = M + 2 * nn;
  double* w = M + 4 * nn;
  int* info = (int*)(w + no);
  TRY_GS(gs_gram(c, psi, no, hpsi, no, c->g.hvol, M));
  // M[i][j] row-major = <psi_i|H psi_j>; the eigensolver reads its upper
  // triangle (dsyev with uplo = 'U'), on the GPU
  TRY_GS(launch_eigh(c, M, no, ework, V, w, info));
  TRY_GS(gs_rotate(c, psi, no, V, no, 0.0, rot));
  for (int io = 0; io < no; ++io) TRY_GS(gs_norm_scale(c, rot + npts * io));
  SB_CUDA(cudaMemcpyAsync(psi, rot, sizeof(double) * npts * no, cudaMemcpyDeviceToDevice, c->stream));
  std::vector<double> hw(no + 1);
  SB_CUDA(cudaMemcpyAsync(hw.data(), w, sizeof(double) * (no + 1), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  int hinfo = 0;
  std::memcpy(&hinfo, &hw[no], sizeof(int));
  if (hinfo != 0) return set_error(SB200_ERR_UNSUPPORTED, "subspace eigensolver: QL iterations did not converge");
  if (evals)
    for (int i = 0; i < no; ++i) evals[i] = hw[i];
  return SB200_OK;
}

}  // extern "C"
