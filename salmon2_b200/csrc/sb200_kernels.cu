// sb200_kernels.cu -- device kernels of the FP64 hpsi / Taylor / observables
// path on the resident orbital layout psi[o][z][y][x] (complex double).
#include <cuda_runtime.h>

#include "sb200_bodies.cuh"
#include "sb200_internal.cuh"

namespace sb200 {
namespace {

using namespace body;

// ---------------------------------------------------------------------------
// k-point coefficients and projector phases (hamiltonian.f90:146-155,847-903)
// ---------------------------------------------------------------------------
struct PrepArgs {
  int nk, totpts, periodic, a_mode;
  int itt;                      // < 0: read *step
  double coef_lap0, coef_nab[12];
  const double* vec_k;          // [nk][3]
  const double* A;              // a_mode 0: A[3]; 1, 2: Ac_tot(3, 0:nt+1); 3: Ac_ext
  const double* A2;             // a_mode 3: Ac_ind(3, 0:nt+1)
  const int* step;
  const double* pt_r;           // [totpts][3]
  double* kcoef;                // [nk][KC]
  double2* phase;               // [nk][totpts] or null
  int nent;                     // scatter entries (0: none)
  const int* ent_pt;
  const double* ent_uv;
  double2* ent_zk;              // [nk][nent] zekr_uV per entry, or null
  int npair;                    // (point, atom) pairs (0: none)
  const int* pair_fp;
  double2* pair_ph;             // [nk][npair] exp(i kAc.r), or null
  double rB[9];                 // rmatrix_B (identity on orthogonal cells)
};

__global__ void k_prep(PrepArgs a) {
  const int per = a.totpts > 0 ? a.totpts : 1;
  const long items = (long)a.nk * per;
  int itt = a.itt;
  if (a.a_mode != 0 && itt < 0) itt = *a.step;
  double A[3];
  for (int d = 0; d < 3; ++d) {
    if (a.a_mode == 0) A[d] = a.A[d];
    else if (a.a_mode == 1) A[d] = 0.5 * (a.A[3 * itt + d] + a.A[3 * (itt - 1) + d]);
    else if (a.a_mode == 2) A[d] = a.A[3 * itt + d];
    else  // the AETRS prediction of A(itt+1), time_evolution_step.f90:466-470
      A[d] = a.A[3 * (itt + 1) + d] + 2.0 * a.A2[3 * itt + d] - a.A2[3 * (itt - 1) + d];
  }
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < items; i += (long)gridDim.x * blockDim.x) {
    const int k = (int)(i / per);
    const int j = (int)(i % per);
    double kAc[3];
    for (int d = 0; d < 3; ++d) kAc[d] = a.periodic ? a.vec_k[3 * k + d] + A[d] : 0.0;
    if (j == 0) {
      double* kc = a.kcoef + (long)KC * k;
      kc[0] = kAc[0];
      kc[1] = kAc[1];
      kc[2] = kAc[2];
      kc[3] = a.periodic ? a.coef_lap0 + 0.5 * (kAc[0] * kAc[0] + kAc[1] * kAc[1] + kAc[2] * kAc[2])
                         : a.coef_lap0;
      for (int q = 0; q < 12; ++q) kc[4 + q] = a.periodic ? kAc[q / 4] * a.coef_nab[q] : 0.0;
      // B (k+A): the lattice-axis components of the non-orthogonal hpsi (hamiltonian.f90:338-343)
      for (int d = 0; d < 3; ++d) kc[16 + d] = a.rB[d] * kAc[0] + a.rB[d + 3] * kAc[1] + a.rB[d + 6] * kAc[2];
      kc[19] = 0.0;
    }
    if (a.phase != nullptr && a.totpts > 0) {
      const double* r = a.pt_r + 3L * j;
      const double th = kAc[0] * r[0] + kAc[1] * r[1] + kAc[2] * r[2];
      double s, c;
      sincos(th, &s, &c);
      a.phase[(long)k * a.totpts + j] = make_double2(c, s);
    }
  }
  // zekr_uV = conj(exp(i kAc.r)) uV of every scatter entry (same sincos as the phase)
  if (a.ent_zk != nullptr && a.nent > 0) {
    const long ne = (long)a.nk * a.nent;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ne; i += (long)gridDim.x * blockDim.x) {
      const int k = (int)(i / a.nent);
      const int e = (int)(i % a.nent);
      const double* r = a.pt_r + 3L * a.ent_pt[e];
      double kAc[3];
      for (int d = 0; d < 3; ++d) kAc[d] = a.vec_k[3 * k + d] + A[d];
      const double th = kAc[0] * r[0] + kAc[1] * r[1] + kAc[2] * r[2];
      double s, c;
      sincos(th, &s, &c);
      const double uv = a.ent_uv[e];
      a.ent_zk[i] = make_double2(c * uv, -s * uv);
    }
  }
  // pair phases exp(i kAc.r) (the same sincos as the point phases)
  if (a.pair_ph != nullptr && a.npair > 0) {
    const long npr = (long)a.nk * a.npair;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npr; i += (long)gridDim.x * blockDim.x) {
      const int k = (int)(i / a.npair);
      const double* r = a.pt_r + 3L * a.pair_fp[(int)(i % a.npair)];
      double kAc[3];
      for (int d = 0; d < 3; ++d) kAc[d] = a.vec_k[3 * k + d] + A[d];
      const double th = kAc[0] * r[0] + kAc[1] * r[1] + kAc[2] * r[2];
      double sn, cs;
      sincos(th, &sn, &cs);
      a.pair_ph[i] = make_double2(cs, sn);
    }
  }
}

template <int NP, typename TIN>
__global__ void __launch_bounds__(128) k_project(const TIN* __restrict__ in, double2* __restrict__ proj,
                                                 ProjArgs a) {
  const int atom = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (atom >= a.natom) return;
  project_atom<NP, TIN>(in, proj, a, atom, blockIdx.y);
}

// Small systems (few orbitals x atoms): one (atom, orbital) pair per CTA of
// eight warps; warp w computes sub-sum w of project_sub, the sub-sums are
// added in warp order in shared memory (a fixed order) and scaled by rinv.
template <int NP, typename TIN>
__global__ void __launch_bounds__(256) k_project_split(const TIN* __restrict__ in, double2* __restrict__ proj,
                                                       ProjArgs a) {
  __shared__ double2 red[8][NP];
  const int atom = blockIdx.x, o = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ik = o / a.nspin_no;
  const TIN* psi = in + (long)o * a.npts;
  const int start = a.atom_start[atom], m = a.mps[atom];
  const int lma0 = a.lma_start[atom], np = a.nproj[atom];
  const double2* ph = a.phase + (a.phase_per_k ? (long)ik * a.totpts : 0L) + start;
  for (int q0 = 0; q0 < np; q0 += NP) {
    double2 acc[NP];
    project_sub<NP, TIN>(psi, ph, a, start, m, lma0, np, q0, warp, acc);
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < NP; ++q) red[warp][q] = acc[q];
    }
    __syncthreads();
    if (threadIdx.x < NP && q0 + (int)threadIdx.x < np) {
      const int q = threadIdx.x;
      double2 t = red[0][q];
      for (int w = 1; w < 8; ++w) t = cadd(t, red[w][q]);
      const int lma = lma0 + q0 + q;
      proj[(long)o * a.nlma + lma] = cscal(a.rinv[lma], t);
    }
    __syncthreads();
  }
}

// Nonlocal current pieces per (orbital, atom): sum over the atom's projectors
// of Im(conj(<r_d zekr|psi>) * rinv <zekr|psi>)  (density_matrix.f90:532-591).
// (at most 128 registers: four CTAs per SM)
template <int NP>
__global__ void __launch_bounds__(128, 4) k_project_moments(const double2* __restrict__ in, double* __restrict__ jw,
                                                         ProjArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int atom = blockIdx.x * 4 + warp;
  if (atom >= a.natom) return;
  const int o = blockIdx.y;
  const int ik = o / a.nspin_no;
  const double2* psi = in + (long)o * a.npts;
  const int start = a.atom_start[atom], m = a.mps[atom];
  const int lma0 = a.lma_start[atom], np = a.nproj[atom];
  const double2* ph = a.phase + (a.phase_per_k ? (long)ik * a.totpts : 0L) + start;
  double jx = 0.0, jy = 0.0, jz = 0.0;
  for (int q0 = 0; q0 < np; q0 += NP) {
    double2 u[NP], ur[NP][3];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      u[q] = make_double2(0.0, 0.0);
      ur[q][0] = ur[q][1] = ur[q][2] = make_double2(0.0, 0.0);
    }
#pragma unroll 2
    for (int j = lane; j < m; j += 32) {
      const double2 v = __ldg(psi + a.pt_lin[start + j]);
      const double2 ev = cmul(__ldg(ph + j), v);  // conj(zekr_uV) / uV times psi, once per point
      const double* r = a.pt_r + 3L * (start + j);
      const double r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2);
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        if (q0 + q < np) {
          const double2 t = cscal(__ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j), ev);
          u[q] = cadd(u[q], t);
          ur[q][0] = cadd(ur[q][0], cscal(r0, t));
          ur[q][1] = cadd(ur[q][1], cscal(r1, t));
          ur[q][2] = cadd(ur[q][2], cscal(r2, t));
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        u[q].x += __shfl_xor_sync(0xffffffffu, u[q].x, off);
        u[q].y += __shfl_xor_sync(0xffffffffu, u[q].y, off);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          ur[q][d].x += __shfl_xor_sync(0xffffffffu, ur[q][d].x, off);
          ur[q][d].y += __shfl_xor_sync(0xffffffffu, ur[q][d].y, off);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      if (q0 + q < np) {
        const double2 us = cscal(a.rinv[lma0 + q0 + q], u[q]);
        // Im(conj(ur) * us)
        jx += ur[q][0].x * us.y - ur[q][0].y * us.x;
        jy += ur[q][1].x * us.y - ur[q][1].y * us.x;
        jz += ur[q][2].x * us.y - ur[q][2].y * us.x;
      }
    }
  }
  if (lane == 0) {
    double* out = jw + 3L * ((long)o * a.natom + atom);
    out[0] = jx;
    out[1] = jy;
    out[2] = jz;
  }
}

// ---------------------------------------------------------------------------
// hpsi: 25-point Laplacian + Bloch gradient + V_local (zstencil_typical_seq,
// seq.f90:65-122) + KB scatter through the inverse map (one owner thread per
// point, ilma ascending as in nonlocal_potential.f90:368-375), with the Taylor
// accumulation of taylor.f90:47-117 fused as an epilogue.
// ---------------------------------------------------------------------------
struct HArgs {
  int nx, ny, nz, periodic, nspin, nspin_no, nlma, nent, phase_per_k;
  long npts;
  double lapt[12];
  const double* kcoef;
  const double* vloc;
  const int *pmap, *ent_lma;
  const double2* ent_zk;
  const double2* proj;
  double2 zc;
  const double* cap;  // absorbing boundary: w(z) per plane, or null
};

// the absorbing boundary's -i w(z) psi (add_imaginary_potential_for_absorbing_boundary_z,
// hamiltonian.f90:760-807), after the stencil and before the nonlocal term
__device__ __forceinline__ void add_cap(const HArgs& a, int z, double2 c, double2& h) {
  if (!a.cap) return;
  const double wv = __ldg(a.cap + z);
  if (wv != 0.0) {
    h.x += wv * c.y;
    h.y -= wv * c.x;
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_hpsi(const double2* __restrict__ in, double2* __restrict__ hout,
                                              double2* __restrict__ acc, HArgs a) {
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= a.npts) return;
  const int o = blockIdx.y;
  const int x = (int)(p % a.nx);
  const int y = (int)((p / a.nx) % a.ny);
  const int z = (int)(p / ((long)a.nx * a.ny));
  const double2* src = in + (long)o * a.npts;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const long sy = a.nx, sz = (long)a.nx * a.ny;

  double2 v = make_double2(0.0, 0.0), w = make_double2(0.0, 0.0);
  {  // x
    double2 vx = make_double2(0.0, 0.0), wx = make_double2(0.0, 0.0);
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      bool okp, okm;
      const int xp = nbr(x, s, a.nx, a.periodic, okp);
      const int xm = nbr(x, -s, a.nx, a.periodic, okm);
      const double2 tp = ldz(src, p - x + xp, okp);
      const double2 tm = ldz(src, p - x + xm, okm);
      vx = cadd(vx, cscal(a.lapt[s - 1], cadd(tp, tm)));
      wx = cadd(wx, cscal(kc[4 + s - 1], csub(tp, tm)));
    }
    v = vx;
    w = wx;
  }
  {  // y
    double2 vy = make_double2(0.0, 0.0), wy = make_double2(0.0, 0.0);
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      bool okp, okm;
      const int yp = nbr(y, s, a.ny, a.periodic, okp);
      const int ym = nbr(y, -s, a.ny, a.periodic, okm);
      const double2 tp = ldz(src, p + (long)(yp - y) * sy, okp);
      const double2 tm = ldz(src, p + (long)(ym - y) * sy, okm);
      vy = cadd(vy, cscal(a.lapt[4 + s - 1], cadd(tp, tm)));
      wy = cadd(wy, cscal(kc[8 + s - 1], csub(tp, tm)));
    }
    v = cadd(vy, v);
    w = cadd(wy, w);
  }
  {  // z
    double2 vz = make_double2(0.0, 0.0), wz = make_double2(0.0, 0.0);
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      bool okp, okm;
      const int zp = nbr(z, s, a.nz, a.periodic, okp);
      const int zm = nbr(z, -s, a.nz, a.periodic, okm);
      const double2 tp = ldz(src, p + (long)(zp - z) * sz, okp);
      const double2 tm = ldz(src, p + (long)(zm - z) * sz, okm);
      vz = cadd(vz, cscal(a.lapt[8 + s - 1], cadd(tp, tm)));
      wz = cadd(wz, cscal(kc[12 + s - 1], csub(tp, tm)));
    }
    v = cadd(vz, v);
    w = cadd(wz, w);
  }
  const double2 c = __ldg(src + p);
  const double vl = __ldg(a.vloc + (long)ispin * a.npts + p);
  const double lap0 = kc[3];
  double2 h;
  h.x = vl * c.x + lap0 * c.x - 0.5 * v.x + w.y;
  h.y = vl * c.y + lap0 * c.y - 0.5 * v.y - w.x;
  add_cap(a, z, c, h);
  if (MODE == 9) {  // ttpsi = htpsi - V_local tpsi before the nonlocal term (hamiltonian.f90:364-414)
    hout[(long)o * a.npts + p] = make_double2(h.x - vl * c.x, h.y - vl * c.y);
    return;
  }

  if (a.nlma > 0) {
    const int pm = __ldg(a.pmap + p);
    if (pm >= 0) {
      const double2* pj = a.proj + (long)o * a.nlma;
      const double2* zk = a.ent_zk + (a.phase_per_k ? (long)ik * a.nent : 0L);
      const int e1 = (pm >> 8) + (pm & 255);
      for (int e = pm >> 8; e < e1; ++e) h = cadd(h, cmul(pj[__ldg(a.ent_lma + e)], __ldg(zk + e)));
    }
  }
  const long gi = (long)o * a.npts + p;
  if (MODE <= 2) hout[gi] = h;
  if (MODE == 1 || MODE == 4) acc[gi] = cadd(c, cmul(a.zc, h));
  if (MODE == 2 || MODE == 3) acc[gi] = cadd(acc[gi], cmul(a.zc, h));
}

__global__ void __launch_bounds__(OBS_THREADS) k_observables(const double2* __restrict__ in, double* __restrict__ part,
                                                             ObsArgs a) {
  if (a.periodic) obs_block<true>(in, part, a, blockIdx.x, blockIdx.y);
  else obs_block<false>(in, part, a, blockIdx.x, blockIdx.y);
}

// Observables of a periodic grid as a z sweep (same quantities as
// obs_block): one CTA per 32 x 8 column tile x z chunk x orbital; the plane
// with its forward halo (+1..+4 in x and y, wrapped) in shared memory, the
// forward z neighbours in a register window, so psi is read about once.
// Writes partial block b = zchunk * ntiles + tile of the orbital; blocks
// ntiles * nzc .. nblk - 1 are written as zeros by the first CTA.
constexpr int OS_TX = 32, OS_TY = 8, OS_SX = OS_TX + ND, OS_SY = OS_TY + ND;
__global__ void __launch_bounds__(256) k_obs_sweep(const double2* __restrict__ in, double* __restrict__ part,
                                                   ObsArgs a, int zchunk) {
  __shared__ double2 pl[OS_SY * OS_SX];
  __shared__ double red[OBS_NQ][8];
  const int t = threadIdx.x, tx = t & 31, ty = t >> 5;
  const int ntx = (a.nx + OS_TX - 1) / OS_TX;
  const int ntiles = ntx * ((a.ny + OS_TY - 1) / OS_TY);
  const int x0 = ((int)blockIdx.x % ntx) * OS_TX, y0 = ((int)blockIdx.x / ntx) * OS_TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool active = x < a.nx && y < a.ny;
  const int z0 = blockIdx.y * zchunk, z1 = min(a.nz, z0 + zchunk);
  const int o = blockIdx.z;
  const double2* src = in + (long)o * a.npts;
  const long sz = (long)a.nx * a.ny;
  auto wz = [&](int z) { int q = z % a.nz; return q < 0 ? q + a.nz : q; };
  // halo cell of this thread (cells of the 12 x 36 area outside the tile)
  int hslot = -1;
  long hoff = 0;
  if (t < OS_SX * OS_SY - OS_TX * OS_TY) {
    int hx, hy;
    if (t < ND * OS_SX) {  // rows below the tile's forward edge
      hy = OS_TY + t / OS_SX;
      hx = t % OS_SX;
    } else {               // the forward x strip of the tile rows
      const int c = t - ND * OS_SX;
      hy = c / ND;
      hx = OS_TX + c % ND;
    }
    hslot = hy * OS_SX + hx;
    const int gx = (x0 + hx) % a.nx, gy = (y0 + hy) % a.ny;
    hoff = (long)gy * a.nx + gx;
  }
  const long pxy = (long)y * a.nx + x;
  double2 w[ND + 1];
#pragma unroll
  for (int k = 0; k <= ND; ++k) w[k] = active ? __ldg(src + wz(z0 + k) * sz + pxy) : make_double2(0.0, 0.0);
  double q[OBS_NQ];
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) q[i] = 0.0;
  double2 hq = hslot >= 0 ? __ldg(src + (long)z0 * sz + hoff) : make_double2(0.0, 0.0);
  for (int z = z0; z < z1; ++z) {
    if (active) pl[(ty)*OS_SX + tx] = w[0];
    if (hslot >= 0) pl[hslot] = hq;
    // the next plane's loads are issued before this plane's sums
    const double2 nxt = (active && z + 1 < z1) ? __ldg(src + wz(z + ND + 1) * sz + pxy) : make_double2(0.0, 0.0);
    if (hslot >= 0 && z + 1 < z1) hq = __ldg(src + (long)(z + 1) * sz + hoff);
    __syncthreads();
    if (active) {
      const double2 c = w[0];
      const double r2 = c.x * c.x + c.y * c.y;
      q[0] += r2;
      double ix = 0.0, iy = 0.0, iz = 0.0;
#pragma unroll
      for (int s = 1; s <= ND; ++s) {
        const double2 txv = pl[ty * OS_SX + tx + s];
        const double2 tyv = pl[(ty + s) * OS_SX + tx];
        const double2 tzv = w[s];
        ix += a.nab[s - 1] * (c.x * txv.y - c.y * txv.x);
        iy += a.nab[4 + s - 1] * (c.x * tyv.y - c.y * tyv.x);
        iz += a.nab[8 + s - 1] * (c.x * tzv.y - c.y * tzv.x);
      }
      q[1] += ix;
      q[2] += iy;
      q[3] += iz;
      q[4] += ((double)x + a.off[0]) * r2;
      q[5] += ((double)y + a.off[1]) * r2;
      q[6] += ((double)z + a.off[2]) * r2;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < ND; ++k) w[k] = w[k + 1];
    w[ND] = nxt;
  }
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) q[i] += __shfl_xor_sync(0xffffffffu, q[i], off);
  }
  if (tx == 0)
    for (int i = 0; i < OBS_NQ; ++i) red[i][ty] = q[i];
  __syncthreads();
  const int b = blockIdx.y * ntiles + blockIdx.x;
  if (t < OBS_NQ) {
    double sum = 0.0;
    for (int wv = 0; wv < 8; ++wv) sum += red[t][wv];
    part[((long)o * a.nblk + b) * OBS_NQ + t] = sum;
  }
  if (blockIdx.x == 0 && blockIdx.y == 0)
    for (int i = ntiles * gridDim.y * OBS_NQ + t; i < a.nblk * OBS_NQ; i += blockDim.x)
      part[(long)o * a.nblk * OBS_NQ + i] = 0.0;
}

__global__ void __launch_bounds__(256) k_finalize(FinArgs a) { finalize_body(a); }

__global__ void __launch_bounds__(256) k_collapse(const double* __restrict__ part, int nblk,
                                                  const double* __restrict__ jw, int natom, long nitems,
                                                  double* __restrict__ out) {
  const long item = (blockIdx.x * 256L + threadIdx.x) >> 5;  // one warp per item
  if (item < nitems) collapse_item(part, nblk, jw, natom, item, out);
}

// rho(p, ispin) = sum_{ik, io} w |psi|^2 (density_matrix.f90:150-232)
// rho of one chunk of (io, ik) orbitals per spin, rocc*wtk weighted.  A block
// is 32 points x 8 orbital slices: slice y sums the chunk's orbitals
// j = j0 + y, j0 + y + 8, ... and the eight slice sums are added in slice
// order.  With one chunk the result goes straight to rho; with several,
// part[chunk][is][p] holds the chunk sums and k_density_sum adds them in chunk
// order.  The chunk count depends only on the grid and orbital counts, so the
// summation order is fixed.
__global__ void __launch_bounds__(256) k_density(const double2* __restrict__ in, double* __restrict__ out, long npts,
                                                 int nspin, int nos, int nper, const double* __restrict__ weight) {
  __shared__ double red[8][32];
  const long p = blockIdx.x * 32L + threadIdx.x;
  const int j0 = blockIdx.y * nper;
  const int j1 = min(nos, j0 + nper);
  for (int is = 0; is < nspin; ++is) {
    double acc = 0.0;
    if (p < npts)
      for (int j = j0 + (int)threadIdx.y; j < j1; j += 8) {  // j = io + no * ik
        const long o = is + (long)nspin * j;
        const double2 c = __ldg(in + o * npts + p);
        acc += (c.x * c.x + c.y * c.y) * weight[o];
      }
    red[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && p < npts) {
      double t = red[0][threadIdx.x];
      for (int k = 1; k < 8; ++k) t += red[k][threadIdx.x];
      out[((long)blockIdx.y * nspin + is) * npts + p] = t;
    }
    __syncthreads();
  }
}

__global__ void k_density_sum(const double* __restrict__ part, double* __restrict__ rho, long n, int nchunk) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int c = 0; c < nchunk; ++c) acc += part[(long)c * n + i];
    rho[i] = acc;
  }
}

// calc_dip partial sums over a rho field (dip.f90:114-225).
__global__ void __launch_bounds__(256) k_dip_part(const double* __restrict__ rho, double* __restrict__ part,
                                                  long npts, int nspin, int nx, int ny, double o0, double o1,
                                                  double o2) {
  __shared__ double red[4][256];
  double q[4] = {0, 0, 0, 0};
  for (long i = blockIdx.x * 256L + threadIdx.x; i < npts * nspin; i += (long)gridDim.x * 256) {
    const long p = i % npts;
    const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
    const double r = rho[i];
    q[0] += ((double)x + o0) * r;
    q[1] += ((double)y + o1) * r;
    q[2] += ((double)z + o2) * r;
    q[3] += r;
  }
  for (int i = 0; i < 4; ++i) red[i][threadIdx.x] = q[i];
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int i = 0; i < 4; ++i) red[i][threadIdx.x] += red[i][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_dip_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  if (threadIdx.x < 4) {
    double acc = 0.0;
    for (int b = 0; b < nblk; ++b) acc += part[b * 4 + threadIdx.x];
    out[threadIdx.x] = acc;
  }
}

// reference layout <-> resident layout for a chunk of orbitals
__global__ void k_relayout(const double2* __restrict__ src, double2* __restrict__ dst, int nx, int ny, int nz,
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

int grid_for(long items, int threads) {
  long b = (items + threads - 1) / threads;
  if (b > 148L * 64) b = 148L * 64;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int launch_prep_k(sb200_ctx* c, const double* d_A, int a_mode, int itt, double* d_kcoef, bool phases) {
  PrepArgs a;
  a.nk = c->orb.nk;
  a.totpts = c->pp.totpts;
  a.periodic = c->g.periodic;
  a.a_mode = a_mode;
  a.itt = itt;
  a.coef_lap0 = c->g.coef_lap0;
  for (int i = 0; i < 12; ++i) a.coef_nab[i] = c->g.coef_nab[i];
  a.vec_k = c->d_vec_k;
  a.A = d_A;
  a.A2 = c->rt.d_Ac_ind;
  a.step = c->rt.d_step;
  a.pt_r = c->pp.d_pt_r;
  a.kcoef = d_kcoef;
  a.phase = (phases && c->g.periodic && c->pp.totpts > 0) ? c->pp.d_phase : nullptr;
  a.nent = c->pp.nent;
  a.ent_pt = c->pp.d_ent_pt;
  a.ent_uv = c->pp.d_ent_uv;
  a.ent_zk = (phases && c->g.periodic && c->pp.nent > 0) ? c->pp.d_ent_zk : nullptr;
  a.npair = c->pp.npair;
  a.pair_fp = c->pp.d_pair_fp;
  a.pair_ph = (phases && c->g.periodic && c->pp.npair > 0) ? c->pp.d_pair_ph : nullptr;
  for (int i = 0; i < 9; ++i) a.rB[i] = c->g.rB[i];
  long items = (long)a.nk * (a.totpts > 0 ? a.totpts : 1);
  if ((long)a.nk * a.nent > items) items = (long)a.nk * a.nent;
  if ((long)a.nk * a.npair > items) items = (long)a.nk * a.npair;
  k_prep<<<grid_for(items, 256), 256, 0, c->stream>>>(a);
  SB_LAUNCH_CHECK("k_prep");
  return SB200_OK;
}

ProjArgs make_proj_args(const sb200_ctx* c) {
  ProjArgs a;
  a.npts = c->g.npts;
  a.natom = c->pp.natom;
  // the eight-warp order while the pairs are fewer than 8 per SM (148 SMs),
  // or always with project_variant 3; the batched kernel follows the flag too
  a.split = (c->project_variant == 3 ||
             (c->project_variant == 1 && (long)c->pp.natom * c->orb.norb < 148L * 8)) ? 1 : 0;
  a.nlma = c->pp.nlma;
  a.nps = c->pp.nps;
  a.totpts = c->pp.totpts;
  a.nspin_no = c->orb.nspin * c->orb.no;
  a.phase_per_k = c->g.periodic;
  a.atom_start = c->pp.d_atom_start;
  a.mps = c->pp.d_mps;
  a.lma_start = c->pp.d_lma_start;
  a.nproj = c->pp.d_nproj;
  a.pt_lin = c->pp.d_pt_lin;
  a.uv = c->pp.d_uv;
  a.rinv = c->pp.d_rinv;
  a.pt_r = c->pp.d_pt_r;
  a.phase = c->pp.d_phase;
  return a;
}

int launch_project(sb200_ctx* c, const void* in, double2* proj, bool in32) {
  if (c->pp.nlma == 0) return SB200_OK;
  // the tensor-core form (sb200_project_mma.cu) when a k-point has at least
  // one full 16-orbital tile, else one CTA per (orbital, atom) while the pairs
  // are fewer than 8 per SM (148 SMs), else one warp per pair
  const int nspin_no = c->orb.nspin * c->orb.no;
  if (c->project_variant == 2 || (c->project_variant == 1 && nspin_no >= 16)) {
    const int r = launch_project_dmma(c, in, proj, in32);
    if (r != SB200_ERR_UNSUPPORTED) return r;
  }
  ProjArgs a = make_proj_args(c);
  if (a.split) {
    dim3 grid(a.natom, c->orb.norb);
    if (in32) k_project_split<4, float2><<<grid, 256, 0, c->stream>>>((const float2*)in, proj, a);
    else k_project_split<4, double2><<<grid, 256, 0, c->stream>>>((const double2*)in, proj, a);
    SB_LAUNCH_CHECK("k_project_split");
    return SB200_OK;
  }
  dim3 grid((a.natom + 3) / 4, c->orb.norb);
  if (in32) k_project<4, float2><<<grid, 128, 0, c->stream>>>((const float2*)in, proj, a);
  else k_project<4, double2><<<grid, 128, 0, c->stream>>>((const double2*)in, proj, a);
  SB_LAUNCH_CHECK("k_project");
  return SB200_OK;
}

// psi <- exp(i e_impulse epdir.r) psi on every orbital, r the grid coordinate
// of set_gridcoordinate (initialization.f90:1125-1190)
__global__ void k_impulse_kick(double2* __restrict__ psi, long npts, long norb, int nx, int ny, KickArgs k) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npts * norb; i += (long)gridDim.x * blockDim.x) {
    const long p = i % npts;
    const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
    const double r1 = k.ep[0] * (k.h[0] * (x + k.c0[0])) + k.ep[1] * (k.h[1] * (y + k.c0[1])) +
                      k.ep[2] * (k.h[2] * (z + k.c0[2]));
    double sn, cs;
    sincos(k.e * r1, &sn, &cs);
    const double2 v = psi[i];
    psi[i] = make_double2(cs * v.x - sn * v.y, cs * v.y + sn * v.x);
  }
}

int launch_impulse_kick(sb200_ctx* c, double2* psi, double e_impulse, const double epdir[3]) {
  KickArgs k;
  k.e = e_impulse;
  for (int d = 0; d < 3; ++d) {
    k.ep[d] = epdir[d];
    k.h[d] = c->g.hgs[d];
    // coordinate of resident index x: (is + x - 1) h periodic; (is + x) h or (is + x - 1/2) h isolated
    k.c0[d] = c->g.periodic ? (double)(c->g.is[d] - 1)
                            : (c->g.lg_num[d] % 2 == 1 ? (double)c->g.is[d] : (double)c->g.is[d] - 0.5);
  }
  const long n = c->g.npts * c->orb.norb;
  const unsigned blocks = (unsigned)((n + 255) / 256 < 148 * 32 ? (n + 255) / 256 : 148 * 32);
  k_impulse_kick<<<blocks, 256, 0, c->stream>>>(psi, c->g.npts, c->orb.norb, c->g.nx, c->g.ny, k);
  SB_LAUNCH_CHECK("k_impulse_kick");
  return SB200_OK;
}

int launch_project_moments(sb200_ctx* c, const double2* psi) {
  if (c->pp.nlma == 0) return SB200_OK;
  ProjArgs a = make_proj_args(c);
  dim3 grid((a.natom + 3) / 4, c->orb.norb);
  k_project_moments<4><<<grid, 128, 0, c->stream>>>(psi, c->d_jw, a);
  SB_LAUNCH_CHECK("k_project_moments");
  return SB200_OK;
}

namespace {
HArgs make_hargs(const sb200_ctx* c, double2 zc) {
  HArgs a;
  a.nx = c->g.nx;
  a.ny = c->g.ny;
  a.nz = c->g.nz;
  a.periodic = c->g.periodic;
  a.nspin = c->orb.nspin;
  a.nspin_no = c->orb.nspin * c->orb.no;
  a.nlma = c->pp.nlma;
  a.nent = c->pp.nent;
  a.phase_per_k = c->g.periodic;
  a.npts = c->g.npts;
  for (int i = 0; i < 12; ++i) a.lapt[i] = c->g.coef_lap[i];
  a.kcoef = c->d_kcoef;
  a.vloc = c->d_vloc;
  a.pmap = c->pp.d_pmap;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_zk = c->pp.d_ent_zk;
  a.proj = c->d_proj;
  a.zc = zc;
  a.cap = c->cap_on ? c->d_cap : nullptr;
  return a;
}

// per (orbital, block): Re sum conj(psi) h, Re sum conj(psi) tt and
// Re sum conj(psi) (h - (tt + V psi)), fixed-order tree in shared memory
__global__ void __launch_bounds__(256) k_energy_part(const double2* __restrict__ psi, const double2* __restrict__ h,
                                                     const double2* __restrict__ tt, const double* __restrict__ vloc,
                                                     long npts, int nspin, double* __restrict__ part, int nblk) {
  __shared__ double r[3][256];
  const long o = blockIdx.y;
  const double* V = vloc + (long)(o % nspin) * npts;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)nblk * 256) {
    const long i = o * npts + p;
    const double2 c = psi[i], hv = h[i], tv = tt[i];
    const double v = V[p];
    s0 += c.x * hv.x + c.y * hv.y;
    s1 += c.x * tv.x + c.y * tv.y;
    s2 += c.x * (hv.x - (tv.x + v * c.x)) + c.y * (hv.y - (tv.y + v * c.y));
  }
  r[0][threadIdx.x] = s0;
  r[1][threadIdx.x] = s1;
  r[2][threadIdx.x] = s2;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 3; ++q) r[q][threadIdx.x] += r[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[(o * nblk + blockIdx.x) * 3 + threadIdx.x] = r[threadIdx.x][0];
}
}  // namespace

// ttpsi of hpsi (the kinetic part) with the per-point kernel
int launch_hpsi_kinetic(sb200_ctx* c, const double2* in, double2* tt) {
  if (c->g.nonorth || c->microac)
    return set_error(SB200_ERR_UNSUPPORTED, "ttpsi on a non-orthogonal lattice or with a microscopic A is not supported");
  const HArgs a = make_hargs(c, make_double2(0.0, 0.0));
  dim3 grid((unsigned)((c->g.npts + 255) / 256), c->orb.norb);
  k_hpsi<9><<<grid, 256, 0, c->stream>>>(in, tt, nullptr, a);
  SB_LAUNCH_CHECK("k_hpsi(kinetic)");
  return SB200_OK;
}

// per-orbital partial energy sums: part[norb][nblk][3]
int launch_energy_parts(sb200_ctx* c, const double2* psi, const double2* h, const double2* tt, double* part,
                        int nblk) {
  dim3 grid(nblk, c->orb.norb);
  k_energy_part<<<grid, 256, 0, c->stream>>>(psi, h, tt, c->d_vloc, c->g.npts, c->orb.nspin, part, nblk);
  SB_LAUNCH_CHECK("k_energy_part");
  return SB200_OK;
}

// ---------------------------------------------------------------------------
// hpsi on a non-orthogonal lattice (zstencil_nonorthogonal, stencil.f90:120-214,
// called from hamiltonian.f90:306-357), one thread per point in two passes:
// (1) the lattice-axis sums v_d = sum_s lapt(s,d) (t+ + t-) and the first
// derivatives w_d = sum_s nab(s,d) (t+ - t-), h = (V + k_lap0) psi
// - 1/2 sum F_d v_d - i sum Bk_d w_d with Bk = B (k+A); w_x and w_y stored;
// (2) the mixed terms - 1/2 (F_4 d_z w_y + F_5 d_z w_x + F_6 d_y w_x) from the
// stored derivatives, then the KB term through the inverse map and the Taylor
// epilogue of MODE.  Periodic grids only (the neighbours wrap).
// ---------------------------------------------------------------------------
struct NoArgs {
  double F[6], nab[12];
};

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__global__ void __launch_bounds__(256) k_hpsi_no1(const double2* __restrict__ in, double2* __restrict__ h1,
                                                  double2* __restrict__ wx, double2* __restrict__ wy, HArgs a,
                                                  NoArgs n) {
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= a.npts) return;
  const int o = blockIdx.y;
  const int x = (int)(p % a.nx), y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
  const double2* src = in + (long)o * a.npts;
  const int ik = o / a.nspin_no, ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const long sy = a.nx, sz = (long)a.nx * a.ny;
  double2 v[3], w[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double2 vv = make_double2(0.0, 0.0), ww = make_double2(0.0, 0.0);
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      long qp, qm;
      if (d == 0) {
        qp = p - x + wrapi(x + s, a.nx);
        qm = p - x + wrapi(x - s, a.nx);
      } else if (d == 1) {
        qp = p + (long)(wrapi(y + s, a.ny) - y) * sy;
        qm = p + (long)(wrapi(y - s, a.ny) - y) * sy;
      } else {
        qp = p + (long)(wrapi(z + s, a.nz) - z) * sz;
        qm = p + (long)(wrapi(z - s, a.nz) - z) * sz;
      }
      const double2 tp = __ldg(src + qp), tm = __ldg(src + qm);
      vv = cadd(vv, cscal(a.lapt[4 * d + s - 1], cadd(tp, tm)));
      ww = cadd(ww, cscal(n.nab[4 * d + s - 1], csub(tp, tm)));
    }
    v[d] = vv;
    w[d] = ww;
  }
  const double2 c = __ldg(src + p);
  const double dg = __ldg(a.vloc + (long)ispin * a.npts + p) + kc[3];
  const double2 fv = cadd(cadd(cscal(n.F[0], v[0]), cscal(n.F[1], v[1])), cscal(n.F[2], v[2]));
  const double2 bw = cadd(cadd(cscal(kc[16], w[0]), cscal(kc[17], w[1])), cscal(kc[18], w[2]));
  // (V + lap0) psi - 0.5 (F.v) - i (Bk.w)
  const long gi = (long)o * a.npts + p;
  h1[gi] = make_double2(dg * c.x - 0.5 * fv.x + bw.y, dg * c.y - 0.5 * fv.y - bw.x);
  wx[gi] = w[0];
  wy[gi] = w[1];
}

template <int MODE>
__global__ void __launch_bounds__(256) k_hpsi_no2(const double2* __restrict__ in, const double2* __restrict__ h1,
                                                  const double2* __restrict__ wx, const double2* __restrict__ wy,
                                                  double2* __restrict__ hout, double2* __restrict__ acc, HArgs a,
                                                  NoArgs n) {
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= a.npts) return;
  const int o = blockIdx.y;
  const int y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
  const long sy = a.nx, sz = (long)a.nx * a.ny;
  const long base = (long)o * a.npts;
  double2 w1 = make_double2(0.0, 0.0), w2 = make_double2(0.0, 0.0), w3 = make_double2(0.0, 0.0);
#pragma unroll
  for (int s = 1; s <= ND; ++s) {
    const long zp = base + p + (long)(wrapi(z + s, a.nz) - z) * sz, zm = base + p + (long)(wrapi(z - s, a.nz) - z) * sz;
    const long yp = base + p + (long)(wrapi(y + s, a.ny) - y) * sy, ym = base + p + (long)(wrapi(y - s, a.ny) - y) * sy;
    w1 = cadd(w1, cscal(n.nab[8 + s - 1], csub(__ldg(wy + zp), __ldg(wy + zm))));  // yz
    w2 = cadd(w2, cscal(n.nab[8 + s - 1], csub(__ldg(wx + zp), __ldg(wx + zm))));  // zx
    w3 = cadd(w3, cscal(n.nab[4 + s - 1], csub(__ldg(wx + yp), __ldg(wx + ym))));  // xy
  }
  const long gi = base + p;
  const double2 mix = cadd(cadd(cscal(n.F[3], w1), cscal(n.F[4], w2)), cscal(n.F[5], w3));
  double2 h = csub(__ldg(h1 + gi), cscal(0.5, mix));
  if (a.nlma > 0) {
    const int pm = __ldg(a.pmap + p);
    if (pm >= 0) {
      const int ik = o / a.nspin_no;
      const double2* pj = a.proj + (long)o * a.nlma;
      const double2* zk = a.ent_zk + (long)ik * a.nent;
      const int e1 = (pm >> 8) + (pm & 255);
      for (int e = pm >> 8; e < e1; ++e) h = cadd(h, cmul(pj[__ldg(a.ent_lma + e)], __ldg(zk + e)));
    }
  }
  const double2 c = __ldg(in + gi);
  if (MODE <= 2) hout[gi] = h;
  if (MODE == 1 || MODE == 4) acc[gi] = cadd(c, cmul(a.zc, h));
  if (MODE == 2 || MODE == 3) acc[gi] = cadd(acc[gi], cmul(a.zc, h));
}

// the scratch of the non-orthogonal hpsi (called before a graph capture, and by every launch)
int nonorth_prepare(sb200_ctx* c) {
  if (!c->g.nonorth) return SB200_OK;
  const size_t need = 3 * (size_t)c->orb.norb * (size_t)c->g.npts;
  if (c->nonorth_cap < need) {
    dfree(c->d_nonorth);
    c->nonorth_cap = 0;
    if (dalloc(&c->d_nonorth, need) != SB200_OK) return SB200_ERR_OOM;
    c->nonorth_cap = need;
  }
  return SB200_OK;
}

int launch_hpsi_nonorth(sb200_ctx* c, const HpsiLaunch& L) {
  if (L.mode > 4) return set_error(SB200_ERR_UNSUPPORTED, "the non-orthogonal hpsi has no mixed-precision modes");
  if (nonorth_prepare(c) != SB200_OK) return SB200_ERR_OOM;
  const size_t blk = (size_t)c->orb.norb * (size_t)c->g.npts;
  double2* h1 = c->d_nonorth;
  double2* wx = h1 + blk;
  double2* wy = wx + blk;
  const HArgs a = make_hargs(c, L.zc);
  NoArgs n;
  for (int i = 0; i < 6; ++i) n.F[i] = c->g.coefF[i];
  for (int i = 0; i < 12; ++i) n.nab[i] = c->g.coef_nab[i];
  dim3 grid((unsigned)((c->g.npts + 255) / 256), c->orb.norb);
  const double2* IN = (const double2*)L.in;
  double2* HOUT = (double2*)L.hout;
  k_hpsi_no1<<<grid, 256, 0, c->stream>>>(IN, h1, wx, wy, a, n);
  switch (L.mode) {
    case 0: k_hpsi_no2<0><<<grid, 256, 0, c->stream>>>(IN, h1, wx, wy, HOUT, L.out, a, n); break;
    case 1: k_hpsi_no2<1><<<grid, 256, 0, c->stream>>>(IN, h1, wx, wy, HOUT, L.out, a, n); break;
    case 2: k_hpsi_no2<2><<<grid, 256, 0, c->stream>>>(IN, h1, wx, wy, HOUT, L.out, a, n); break;
    case 3: k_hpsi_no2<3><<<grid, 256, 0, c->stream>>>(IN, h1, wx, wy, HOUT, L.out, a, n); break;
    default: k_hpsi_no2<4><<<grid, 256, 0, c->stream>>>(IN, h1, wx, wy, HOUT, L.out, a, n); break;
  }
  SB_LAUNCH_CHECK("k_hpsi_no1 / k_hpsi_no2");
  return SB200_OK;
}

// ---------------------------------------------------------------------------
// hpsi with a microscopic vector potential (single-scale Maxwell-TDDFT,
// zstencil_microAc_typical_seq, zstencil_microac_core/typical/seq.f90; called
// from hamiltonian.f90:236-298): per point kAc = k + Ac(r), h = (V + lap0) psi
// - v/2 + |kAc|^2 psi / 2 - i kAc.w - i div(Ac) psi / 2 with v the Laplacian
// sums and w_d the first derivatives (coef_nab); then the KB term and the
// Taylor epilogue of MODE, one thread per point.
// SYM (yn_symmetrized_stencil = 'y', zstencil_microAc_symmetrized,
// stencil.f90:319-411): no div term; instead the divergence of (k + Ac) psi
// taken with Ac at the neighbour points, X = sum_d sum_s nab(s,d)
// ((k_d + Ac_d(r + s e_d)) psi(r + s e_d) - (k_d + Ac_d(r - s e_d)) psi(r - s e_d)),
// and h = (V + lap0) psi - v/2 + |kAc|^2 psi / 2 - (i/2) (kAc.w + X).
// ---------------------------------------------------------------------------
template <int MODE, int SYM>
__global__ void __launch_bounds__(256) k_hpsi_micro(const double2* __restrict__ in, double2* __restrict__ hout,
                                                    double2* __restrict__ acc, HArgs a, NoArgs n,
                                                    const double* __restrict__ acm, const double* __restrict__ divac,
                                                    const double* __restrict__ vec_k, double lap0) {
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= a.npts) return;
  const int o = blockIdx.y;
  const int x = (int)(p % a.nx), y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
  const double2* src = in + (long)o * a.npts;
  const int ik = o / a.nspin_no, ispin = o % a.nspin;
  const long sy = a.nx, sz = (long)a.nx * a.ny;
  double2 v = make_double2(0.0, 0.0), w[3], X = make_double2(0.0, 0.0);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double2 vv = make_double2(0.0, 0.0), ww = make_double2(0.0, 0.0), xx = make_double2(0.0, 0.0);
    const double kd = SYM ? __ldg(vec_k + 3 * ik + d) : 0.0;
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      bool okp, okm;
      long qp, qm;
      if (d == 0) {
        qp = p - x + nbr(x, s, a.nx, a.periodic, okp);
        qm = p - x + nbr(x, -s, a.nx, a.periodic, okm);
      } else if (d == 1) {
        qp = p + (long)(nbr(y, s, a.ny, a.periodic, okp) - y) * sy;
        qm = p + (long)(nbr(y, -s, a.ny, a.periodic, okm) - y) * sy;
      } else {
        qp = p + (long)(nbr(z, s, a.nz, a.periodic, okp) - z) * sz;
        qm = p + (long)(nbr(z, -s, a.nz, a.periodic, okm) - z) * sz;
      }
      const double2 tp = ldz(src, qp, okp), tm = ldz(src, qm, okm);
      vv = cadd(vv, cscal(a.lapt[4 * d + s - 1], cadd(tp, tm)));
      ww = cadd(ww, cscal(n.nab[4 * d + s - 1], csub(tp, tm)));
      if (SYM) {  // outside an isolated grid psi is zero, and so is the product
        const double ap = okp ? kd + __ldg(acm + 3 * qp + d) : 0.0;
        const double am = okm ? kd + __ldg(acm + 3 * qm + d) : 0.0;
        xx = cadd(xx, cscal(n.nab[4 * d + s - 1], csub(cscal(ap, tp), cscal(am, tm))));
      }
    }
    v = d == 0 ? vv : cadd(vv, v);
    w[d] = ww;
    if (SYM) X = d == 0 ? xx : cadd(xx, X);
  }
  double kAc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) kAc[d] = __ldg(vec_k + 3 * ik + d) + __ldg(acm + 3 * p + d);
  const double2 c = __ldg(src + p);
  const double dg = __ldg(a.vloc + (long)ispin * a.npts + p) + lap0;
  const double hk = 0.5 * (kAc[0] * kAc[0] + kAc[1] * kAc[1] + kAc[2] * kAc[2]);
  const double2 kw = cadd(cadd(cscal(kAc[0], w[0]), cscal(kAc[1], w[1])), cscal(kAc[2], w[2]));
  double2 h;
  if (SYM) {
    const double2 t = cadd(kw, X);
    h.x = dg * c.x - 0.5 * v.x + hk * c.x + 0.5 * t.y;
    h.y = dg * c.y - 0.5 * v.y + hk * c.y - 0.5 * t.x;
  } else {
    const double div = __ldg(divac + p);
    h.x = dg * c.x - 0.5 * v.x + hk * c.x + kw.y + 0.5 * div * c.y;
    h.y = dg * c.y - 0.5 * v.y + hk * c.y - kw.x - 0.5 * div * c.x;
  }
  add_cap(a, z, c, h);
  if (a.nlma > 0) {
    const int pm = __ldg(a.pmap + p);
    if (pm >= 0) {
      const double2* pj = a.proj + (long)o * a.nlma;
      const double2* zk = a.ent_zk + (a.phase_per_k ? (long)ik * a.nent : 0L);
      const int e1 = (pm >> 8) + (pm & 255);
      for (int e = pm >> 8; e < e1; ++e) h = cadd(h, cmul(pj[__ldg(a.ent_lma + e)], __ldg(zk + e)));
    }
  }
  const long gi = (long)o * a.npts + p;
  if (MODE <= 2) hout[gi] = h;
  if (MODE == 1 || MODE == 4) acc[gi] = cadd(c, cmul(a.zc, h));
  if (MODE == 2 || MODE == 3) acc[gi] = cadd(acc[gi], cmul(a.zc, h));
}

int launch_hpsi_micro(sb200_ctx* c, const HpsiLaunch& L) {
  if (L.mode > 4) return set_error(SB200_ERR_UNSUPPORTED, "the single-scale hpsi has no mixed-precision modes");
  const HArgs a = make_hargs(c, L.zc);
  NoArgs n;
  for (int i = 0; i < 6; ++i) n.F[i] = 0.0;
  for (int i = 0; i < 12; ++i) n.nab[i] = c->g.coef_nab[i];
  dim3 grid((unsigned)((c->g.npts + 255) / 256), c->orb.norb);
  const double2* IN = (const double2*)L.in;
  double2* HOUT = (double2*)L.hout;
  const double lap0 = c->g.coef_lap0;
#define SB_MICRO(M, S) \
  k_hpsi_micro<M, S><<<grid, 256, 0, c->stream>>>(IN, HOUT, L.out, a, n, c->d_acm, c->d_divac, c->d_vec_k, lap0)
#define SB_MICRO_MODES(S)        \
  switch (L.mode) {              \
    case 0: SB_MICRO(0, S); break; \
    case 1: SB_MICRO(1, S); break; \
    case 2: SB_MICRO(2, S); break; \
    case 3: SB_MICRO(3, S); break; \
    default: SB_MICRO(4, S); break; \
  }
  if (c->micro_sym) {
    SB_MICRO_MODES(1)
  } else {
    SB_MICRO_MODES(0)
  }
#undef SB_MICRO_MODES
#undef SB_MICRO
  SB_LAUNCH_CHECK("k_hpsi_micro");
  return SB200_OK;
}

// ---------------------------------------------------------------------------
// Isolated system driven by a pulse in the length gauge (ae_shape1 /= 'impulse'):
// calcVbox (em_field.f90:422-548) Vbox = E_ext(itt).r with lg%coordinate, and
// V_local = V_local + Vbox before the Taylor step (time_evolution_step.f90:102-116);
// the step's update_vlocal restores the field-free potential, kept here in base.
// ---------------------------------------------------------------------------
__global__ void k_vbox(const double* __restrict__ base, double* __restrict__ v, float* __restrict__ v32,
                       const double* __restrict__ eext, const int* __restrict__ step, long n, int nspin, int nx,
                       int ny, double o0, double o1, double o2, double h0, double h1, double h2) {
  const int itt = *step;
  const double e0 = eext[3 * itt], e1 = eext[3 * itt + 1], e2 = eext[3 * itt + 2];
  const long tot = n * nspin;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const long p = i % n;
    const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
    const double vb = 0.0 + (e0 * ((o0 + x) * h0) + e1 * ((o1 + y) * h1) + e2 * ((o2 + z) * h2));
    const double val = base[i] + vb;
    v[i] = val;
    v32[i] = (float)val;
  }
}

__global__ void k_vloc_restore(const double* __restrict__ base, double* __restrict__ v, float* __restrict__ v32,
                               long tot) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    v[i] = base[i];
    v32[i] = (float)base[i];
  }
}

int launch_vbox(sb200_ctx* c, int kind) {
  const long n = c->g.npts;
  const int nspin = c->orb.nspin;
  double o[3];
  for (int d = 0; d < 3; ++d) o[d] = (double)c->g.is[d] - ((c->g.lg_num[d] % 2 == 1) ? 0.0 : 0.5);
  long nb = (n * nspin + 255) / 256;
  if (nb > 148L * 8) nb = 148L * 8;
  if (kind >= 0 && kernel_timing_mark(c, kind, true)) return SB200_ERR_CUDA;
  k_vbox<<<(unsigned)nb, 256, 0, c->stream>>>(c->d_vloc_base, c->d_vloc, c->d_vloc32, c->d_eext, c->rt.d_step, n,
                                              nspin, c->g.nx, c->g.ny, o[0], o[1], o[2], c->g.hgs[0], c->g.hgs[1],
                                              c->g.hgs[2]);
  SB_LAUNCH_CHECK("k_vbox");
  if (kind >= 0 && kernel_timing_mark(c, kind, false)) return SB200_ERR_CUDA;
  return SB200_OK;
}

// AETRS between the half steps (time_evolution_half_step_etrs,
// time_evolution_step.f90:430-463): V_new = 3 V - 3 V_old1 + V_old2, V_old2 =
// V_old1, V_old1 = V, V = V_new, plus Vbox(itt+1) in the length gauge
__global__ void k_aetrs_vloc(double* __restrict__ v, float* __restrict__ v32, double* __restrict__ old1,
                             double* __restrict__ old2, const double* __restrict__ eext,
                             const int* __restrict__ step, long n, int nspin, int nx, int ny, double o0, double o1,
                             double o2, double h0, double h1, double h2) {
  double e0 = 0.0, e1 = 0.0, e2 = 0.0;
  if (eext) {
    const int itt = *step + 1;
    e0 = eext[3 * itt];
    e1 = eext[3 * itt + 1];
    e2 = eext[3 * itt + 2];
  }
  const long tot = n * nspin;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const double vc = v[i];
    double vn = 3.0 * vc - 3.0 * old1[i] + old2[i];
    old2[i] = old1[i];
    old1[i] = vc;
    if (eext) {
      const long p = i % n;
      const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
      vn = vn + (0.0 + (e0 * ((o0 + x) * h0) + e1 * ((o1 + y) * h1) + e2 * ((o2 + z) * h2)));
    }
    v[i] = vn;
    v32[i] = (float)vn;
  }
}

int launch_aetrs_vloc(sb200_ctx* c) {
  const long n = c->g.npts;
  const int nspin = c->orb.nspin;
  double o[3];
  for (int d = 0; d < 3; ++d) o[d] = (double)c->g.is[d] - ((c->g.lg_num[d] % 2 == 1) ? 0.0 : 0.5);
  long nb = (n * nspin + 255) / 256;
  if (nb > 148L * 8) nb = 148L * 8;
  double* old1 = c->d_vloc_old;
  double* old2 = c->d_vloc_old + (size_t)n * nspin;
  k_aetrs_vloc<<<(unsigned)nb, 256, 0, c->stream>>>(c->d_vloc, c->d_vloc32, old1, old2,
                                                    c->lg_active ? c->d_eext : nullptr, c->rt.d_step, n, nspin,
                                                    c->g.nx, c->g.ny, o[0], o[1], o[2], c->g.hgs[0], c->g.hgs[1],
                                                    c->g.hgs[2]);
  SB_LAUNCH_CHECK("k_aetrs_vloc");
  return SB200_OK;
}

int launch_vloc_restore(sb200_ctx* c) {
  const long tot = c->g.npts * c->orb.nspin;
  long nb = (tot + 255) / 256;
  if (nb > 148L * 8) nb = 148L * 8;
  k_vloc_restore<<<(unsigned)nb, 256, 0, c->stream>>>(c->d_vloc_base, c->d_vloc, c->d_vloc32, tot);
  SB_LAUNCH_CHECK("k_vloc_restore");
  return SB200_OK;
}

// ---------------------------------------------------------------------------
// Microscopic current density of the single-scale theory,
// calc_microscopic_current / micro_current (density_matrix.f90:726-845):
// j_d(r) = sum_{k,o,s} rocc wtk (Im(conj(psi) dpsi_d) + k_d |psi|^2) with dpsi_d
// the coef_nab first derivative and k = vec_k (no A: the electron number
// current without rho A / c; no nonlocal part).  A block is 32 points x 8
// orbital slices of one chunk; slice y sums orbitals o0 + y, o0 + y + 8, ...
// in orbital order (k, o, spin as the reference's loops); the slice sums are
// added in slice order, the chunk sums (part[chunk][p][3]) in chunk order by
// k_micro_current_sum.  The chunk count depends only on the grid and orbital
// counts, so the summation order is fixed.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_micro_current(const double2* __restrict__ in, double* __restrict__ part,
                                                       HArgs a, NoArgs n, const double* __restrict__ vec_k,
                                                       const double* __restrict__ weight, int norb, int nper) {
  __shared__ double red[3][8][32];
  const long p = blockIdx.x * 32L + threadIdx.x;
  const int o0 = blockIdx.y * nper, o1 = min(norb, o0 + nper);
  double j[3] = {0.0, 0.0, 0.0};
  if (p < a.npts) {
    const int x = (int)(p % a.nx), y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
    const long sy = a.nx, sz = (long)a.nx * a.ny;
    for (int o = o0 + (int)threadIdx.y; o < o1; o += 8) {
      const double2* src = in + (long)o * a.npts;
      const int ik = o / a.nspin_no;
      const double2 c = __ldg(src + p);
      const double cc = c.x * c.x + c.y * c.y;
      const double wo = __ldg(weight + o);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double2 t = make_double2(0.0, 0.0);
#pragma unroll
        for (int s = 1; s <= ND; ++s) {
          bool okp, okm;
          long qp, qm;
          if (d == 0) {
            qp = p - x + nbr(x, s, a.nx, a.periodic, okp);
            qm = p - x + nbr(x, -s, a.nx, a.periodic, okm);
          } else if (d == 1) {
            qp = p + (long)(nbr(y, s, a.ny, a.periodic, okp) - y) * sy;
            qm = p + (long)(nbr(y, -s, a.ny, a.periodic, okm) - y) * sy;
          } else {
            qp = p + (long)(nbr(z, s, a.nz, a.periodic, okp) - z) * sz;
            qm = p + (long)(nbr(z, -s, a.nz, a.periodic, okm) - z) * sz;
          }
          t = cadd(t, cscal(n.nab[4 * d + s - 1], csub(ldz(src, qp, okp), ldz(src, qm, okm))));
        }
        // Im(conj(c) t) + k_d |c|^2
        const double jw = (c.x * t.y - c.y * t.x) + __ldg(vec_k + 3 * ik + d) * cc;
        j[d] += jw * wo;
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) red[d][threadIdx.y][threadIdx.x] = j[d];
  __syncthreads();
  if (threadIdx.y < 3 && p < a.npts) {
    const int d = threadIdx.y;
    double t = red[d][0][threadIdx.x];
    for (int k = 1; k < 8; ++k) t += red[d][k][threadIdx.x];
    part[((long)blockIdx.y * a.npts + p) * 3 + d] = t;
  }
}

__global__ void k_micro_current_sum(const double* __restrict__ part, double* __restrict__ curr, long n, int nchunk) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int c = 0; c < nchunk; ++c) acc += part[(long)c * n + i];
    curr[i] = acc;
  }
}

// curr [npts][3] (device) of the orbitals psi; part: scratch of
// micro_current_part_len(c) doubles
void micro_current_chunks(const sb200_ctx* c, long* pblocks, int* nchunk, int* nper) {
  const long pb = (c->g.npts + 31) / 32;
  const int norb = c->orb.norb;
  long want = (2L * 148 + pb - 1) / pb;  // about two blocks per SM
  long cap = (norb + 7) / 8;             // at least eight orbitals per chunk
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  const int per = (int)((norb + want - 1) / want);
  *pblocks = pb;
  *nper = per;
  *nchunk = (norb + per - 1) / per;
}

size_t micro_current_part_len(const sb200_ctx* c) {
  long pb;
  int nchunk, nper;
  micro_current_chunks(c, &pb, &nchunk, &nper);
  return (size_t)nchunk * (size_t)c->g.npts * 3;
}

int launch_micro_current(sb200_ctx* c, const double2* psi, double* curr, double* part) {
  long pb;
  int nchunk, nper;
  micro_current_chunks(c, &pb, &nchunk, &nper);
  const HArgs a = make_hargs(c, make_double2(0.0, 0.0));
  NoArgs n;
  for (int i = 0; i < 6; ++i) n.F[i] = 0.0;
  for (int i = 0; i < 12; ++i) n.nab[i] = c->g.coef_nab[i];
  k_micro_current<<<dim3((unsigned)pb, (unsigned)nchunk), dim3(32, 8), 0, c->stream>>>(psi, part, a, n, c->d_vec_k,
                                                                                      c->d_weight, c->orb.norb, nper);
  const long n3 = 3L * c->g.npts;
  long sblocks = (n3 + 255) / 256;
  if (sblocks > 148L * 8) sblocks = 148L * 8;
  k_micro_current_sum<<<(unsigned)sblocks, 256, 0, c->stream>>>(part, curr, n3, nchunk);
  SB_LAUNCH_CHECK("k_micro_current");
  return SB200_OK;
}

int launch_hpsi(sb200_ctx* c, const HpsiLaunch& L) {
  if (c->microac) return launch_hpsi_micro(c, L);
  if (c->g.nonorth) return launch_hpsi_nonorth(c, L);
  if (c->cap_on && L.mode >= 5)
    return set_error(SB200_ERR_UNSUPPORTED, "the absorbing boundary has no mixed-precision form");
  if (!c->cap_on && (c->stencil_variant == 1 || L.mode >= 5)) return launch_hpsi_tiled(c, L);
  const double2* IN = (const double2*)L.in;
  double2* HOUT = (double2*)L.hout;
  HArgs a;
  a.nx = c->g.nx;
  a.ny = c->g.ny;
  a.nz = c->g.nz;
  a.periodic = c->g.periodic;
  a.nspin = c->orb.nspin;
  a.nspin_no = c->orb.nspin * c->orb.no;
  a.nlma = c->pp.nlma;
  a.nent = c->pp.nent;
  a.phase_per_k = c->g.periodic;
  a.npts = c->g.npts;
  for (int i = 0; i < 12; ++i) a.lapt[i] = c->g.coef_lap[i];
  a.kcoef = c->d_kcoef;
  a.vloc = c->d_vloc;
  a.pmap = c->pp.d_pmap;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_zk = c->pp.d_ent_zk;
  a.proj = c->d_proj;
  a.zc = L.zc;
  a.cap = c->cap_on ? c->d_cap : nullptr;
  dim3 grid((unsigned)((c->g.npts + 255) / 256), c->orb.norb);
  switch (L.mode) {
    case 0: k_hpsi<0><<<grid, 256, 0, c->stream>>>(IN, HOUT, L.out, a); break;
    case 1: k_hpsi<1><<<grid, 256, 0, c->stream>>>(IN, HOUT, L.out, a); break;
    case 2: k_hpsi<2><<<grid, 256, 0, c->stream>>>(IN, HOUT, L.out, a); break;
    case 3: k_hpsi<3><<<grid, 256, 0, c->stream>>>(IN, HOUT, L.out, a); break;
    case 4: k_hpsi<4><<<grid, 256, 0, c->stream>>>(IN, HOUT, L.out, a); break;
    default: return set_error(SB200_ERR_UNSUPPORTED, "per-point hpsi kernel has no mixed-precision modes");
  }
  SB_LAUNCH_CHECK("k_hpsi");
  return SB200_OK;
}

ObsArgs make_obs_args(const sb200_ctx* c) {
  ObsArgs a;
  a.nx = c->g.nx;
  a.ny = c->g.ny;
  a.nz = c->g.nz;
  a.periodic = c->g.periodic;
  a.npts = c->g.npts;
  a.nblk = c->obs_blocks;
  for (int i = 0; i < 12; ++i) a.nab[i] = c->g.coef_nab[i];
  for (int d = 0; d < 3; ++d) a.off[d] = (double)c->g.is[d] - ((c->g.lg_num[d] % 2 == 1) ? 0.0 : 0.5);
  return a;
}

int launch_observables(sb200_ctx* c, const double2* psi) {
  ObsArgs a = make_obs_args(c);
  // z sweep (psi read about once for the current sums): periodic grids whose
  // x / y extents are multiples of the 32 x 8 tile
  if (c->g.periodic && c->g.nx % OS_TX == 0 && c->g.ny % OS_TY == 0) {
    const int ntiles = ((c->g.nx + OS_TX - 1) / OS_TX) * ((c->g.ny + OS_TY - 1) / OS_TY);
    int nzc = c->obs_blocks / ntiles;
    if (nzc < 1) nzc = 1;
    if (nzc > c->g.nz) nzc = c->g.nz;
    const int zchunk = (c->g.nz + nzc - 1) / nzc;
    nzc = (c->g.nz + zchunk - 1) / zchunk;
    if ((long)ntiles * nzc <= c->obs_blocks) {
      dim3 grid(ntiles, nzc, c->orb.norb);
      k_obs_sweep<<<grid, 256, 0, c->stream>>>(psi, c->d_obs, a, zchunk);
      SB_LAUNCH_CHECK("k_obs_sweep");
      return SB200_OK;
    }
  }
  dim3 grid(c->obs_blocks, c->orb.norb);
  k_observables<<<grid, OBS_THREADS, 0, c->stream>>>(psi, c->d_obs, a);
  SB_LAUNCH_CHECK("k_observables");
  return SB200_OK;
}

// itt >= 0: history index given by the host (API calls), results to d_result;
// itt < 0: RT loop, index from the device step counter.
FinArgs make_fin_args(const sb200_ctx* c, int itt, int trans_longi, double dt, int spin_filter, bool fused_obs) {
  FinArgs a;
  a.stage = 0;  // one pass (launch_finalize splits it for k-point shards)
  a.sums = nullptr;
  a.norb = c->orb.norb;
  a.jw_natom = fused_obs ? 1 : c->pp.natom;
  a.obs_stride = OBS_NQ;
  a.jw_stride = 3;
  a.nspin = c->orb.nspin;
  a.spin_filter = spin_filter;
  a.nspin_no = c->orb.nspin * c->orb.no;
  a.nblk = fused_obs ? 1 : c->obs_blocks;
  a.natom = c->pp.natom;
  a.periodic = c->g.periodic;
  a.itt = itt;
  a.trans_longi = trans_longi;
  a.ngrid_inv = 1.0 / (double)((long)c->g.lg_num[0] * c->g.lg_num[1] * c->g.lg_num[2]);
  a.dt = dt;
  a.part = c->d_obs;
  a.jw = (c->pp.nlma > 0 && c->g.periodic) ? c->d_jw : nullptr;
  a.weight = c->d_weight;
  a.vec_k = c->d_vec_k;
  a.step = c->rt.d_step;
  a.nonorth = c->g.nonorth;
  for (int i = 0; i < 9; ++i) a.rB[i] = c->g.rB[i];
  if (itt < 0) {
    a.Ac_cur = c->rt.d_Ac_tot;
    a.A_direct = 0;
    a.Ac_ind = c->rt.d_Ac_ind;
    a.Ac_tot = c->rt.d_Ac_tot;
    a.Ac_ext = c->rt.d_Ac_ext;
    a.curr_hist = c->rt.d_curr;
    a.rbox_hist = c->rt.d_rbox;
    a.result = nullptr;
    a.advance = 1;
  } else {
    a.Ac_cur = c->d_result + 8;  // A for the current is staged in result[8..10]
    a.A_direct = 1;
    a.Ac_ind = nullptr;
    a.Ac_tot = nullptr;
    a.Ac_ext = nullptr;
    a.curr_hist = nullptr;
    a.rbox_hist = nullptr;
    a.result = c->d_result;
    a.advance = 0;
  }
  return a;
}

int launch_finalize(sb200_ctx* c, int itt, int nt, int trans_longi, double dt, int spin_filter, bool fused_obs) {
  (void)nt;
  FinArgs a = make_fin_args(c, itt, trans_longi, dt, spin_filter, fused_obs);
  if (a.nblk > 1 || (a.jw != nullptr && a.jw_natom > 1)) {
    // per-orbital sums first, a warp per (orbital, quantity), so the one-CTA
    // final reduction reads one record per orbital
    const long nitems = (long)c->orb.norb * (OBS_NQ + 3);
    k_collapse<<<(unsigned)((nitems * 32 + 255) / 256), 256, 0, c->stream>>>(a.part, a.nblk, a.jw, a.jw_natom,
                                                                             nitems, c->d_obs1);
    SB_LAUNCH_CHECK("k_collapse");
    a.part = c->d_obs1;
    a.nblk = 1;
    a.obs_stride = OBS_NQ + 3;
    if (a.jw != nullptr) {
      a.jw = c->d_obs1 + OBS_NQ;
      a.jw_natom = 1;
      a.jw_stride = OBS_NQ + 3;
    }
  }
  a.stage = 0;
  a.sums = c->d_result + 16;
  if (shard_comm_set(c)) {
    // k-point shards: the 7 sums of every shard added over the ranks before
    // J(t) enters calc_emfields (comm_summation over icomm_rko,
    // density_matrix.f90:448)
    a.stage = 1;
    k_finalize<<<1, 256, 0, c->stream>>>(a);
    SB_LAUNCH_CHECK("k_finalize");
    int r = shard_sum(c, a.sums, 7);
    if (r != SB200_OK) return r;
    a.stage = 2;
  }
  k_finalize<<<1, 256, 0, c->stream>>>(a);
  SB_LAUNCH_CHECK("k_finalize");
  return SB200_OK;
}

// Orbital chunking of calc_density: enough (32-point block, orbital chunk)
// pairs for about eight blocks per SM, with at least 32 orbitals per chunk
// (four per orbital slice).
void density_chunks(const sb200_ctx* c, long* pblocks, int* nchunk, int* nper) {
  const long n = c->g.npts;
  const int nos = c->orb.no * c->orb.nk;
  *pblocks = (n + 31) / 32;
  long nc = (148L * 8 + *pblocks - 1) / *pblocks;
  const long cap = (nos + 31) / 32;
  if (nc > cap) nc = cap;
  if (nc < 1) nc = 1;
  *nper = (int)((nos + nc - 1) / nc);
  *nchunk = (nos + *nper - 1) / *nper;
}

// Sizes the chunk partial-sum buffer (outside any stream capture).
int density_prepare(sb200_ctx* c) {
  long pblocks;
  int nchunk, nper;
  density_chunks(c, &pblocks, &nchunk, &nper);
  if (nchunk <= 1) return SB200_OK;
  const size_t need = (size_t)nchunk * c->orb.nspin * c->g.npts;
  if (c->rho_part_cap >= need) return SB200_OK;
  dfree(c->d_rho_part);
  c->rho_part_cap = 0;
  if (dalloc(&c->d_rho_part, need)) return SB200_ERR_OOM;
  c->rho_part_cap = need;
  return SB200_OK;
}

int launch_density(sb200_ctx* c, const double2* psi, double* rho, int kind) {
  const long n = c->g.npts;
  const int nspin = c->orb.nspin;
  const int nos = c->orb.no * c->orb.nk;
  long pblocks;
  int nchunk, nper;
  density_chunks(c, &pblocks, &nchunk, &nper);
  // kind >= 0: each launch bracketed for sb200_kernel_times
  auto mark = [&](bool start) { return kind >= 0 ? kernel_timing_mark(c, kind, start) : SB200_OK; };
  if (nchunk <= 1) {
    if (mark(true)) return SB200_ERR_CUDA;
    k_density<<<dim3((unsigned)pblocks, 1), dim3(32, 8), 0, c->stream>>>(psi, rho, n, nspin, nos, nos, c->d_weight);
    SB_LAUNCH_CHECK("k_density");
    return mark(false);
  }
  if (density_prepare(c) != SB200_OK) return SB200_ERR_OOM;
  if (mark(true)) return SB200_ERR_CUDA;
  k_density<<<dim3((unsigned)pblocks, (unsigned)nchunk), dim3(32, 8), 0, c->stream>>>(psi, c->d_rho_part, n, nspin,
                                                                                     nos, nper, c->d_weight);
  if (mark(false) || mark(true)) return SB200_ERR_CUDA;
  long sblocks = (n * nspin + 255) / 256;
  if (sblocks > 148L * 8) sblocks = 148L * 8;
  k_density_sum<<<(unsigned)sblocks, 256, 0, c->stream>>>(c->d_rho_part, rho, n * nspin, nchunk);
  SB_LAUNCH_CHECK("k_density");
  return mark(false);
}

int launch_dip(sb200_ctx* c, const double* rho, double* d_out4) {
  const long n = c->g.npts * c->orb.nspin;
  int nblk = (int)((n + 255) / 256);
  const int cap = (int)((size_t)c->orb.norb * c->obs_blocks * OBS_NQ / 4);
  if (nblk > cap) nblk = cap;
  if (nblk > 1024) nblk = 1024;
  if (nblk < 1) nblk = 1;
  double o[3];
  for (int d = 0; d < 3; ++d) o[d] = (double)c->g.is[d] - ((c->g.lg_num[d] % 2 == 1) ? 0.0 : 0.5);
  k_dip_part<<<nblk, 256, 0, c->stream>>>(rho, c->d_obs, c->g.npts, c->orb.nspin, c->g.nx, c->g.ny, o[0], o[1],
                                          o[2]);
  SB_LAUNCH_CHECK("k_dip_part");
  k_dip_final<<<1, 32, 0, c->stream>>>(c->d_obs, nblk, d_out4);
  SB_LAUNCH_CHECK("k_dip_final");
  return SB200_OK;
}

int launch_relayout(sb200_ctx* c, const void* src, void* dst, int norb_chunk, bool to_ref) {
  const GridInfo& g = c->g;
  const int nxa = g.ie_array[0] - g.is_array[0] + 1;
  const int nya = g.ie_array[1] - g.is_array[1] + 1;
  const long total = g.npts * norb_chunk;
  k_relayout<<<grid_for(total, 256), 256, 0, c->stream>>>(
      (const double2*)src, (double2*)dst, g.nx, g.ny, g.nz, nxa, nya, g.vol_array(), g.is[0] - g.is_array[0],
      g.is[1] - g.is_array[1], g.is[2] - g.is_array[2], norb_chunk, to_ref ? 1 : 0);
  SB_LAUNCH_CHECK("k_relayout");
  return SB200_OK;
}

}  // namespace sb200
