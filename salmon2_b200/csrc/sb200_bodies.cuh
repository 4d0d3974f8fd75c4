// sb200_bodies.cuh -- device-function bodies shared by the per-system kernels
// (sb200_kernels.cu) and the batched persistent kernels (sb200_batch.cu):
// KB projections of one (orbital, atom) and the observable partial sums of
// one (orbital, point block), and the per-step final reduction.
#pragma once
#include <cuda_runtime.h>

#include "sb200_internal.cuh"

namespace sb200 {
namespace body {

constexpr double PI = 3.141592653589793238462643383279502884;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscal(double r, double2 a) { return make_double2(r * a.x, r * a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// neighbour coordinate along an axis of length n; periodic wrap or Dirichlet.
__device__ __forceinline__ int nbr(int c, int s, int n, int periodic, bool& ok) {
  int q = c + s;
  if (periodic) {
    q = q < 0 ? q + n : (q >= n ? q - n : q);
    ok = true;
  } else {
    ok = (q >= 0) && (q < n);
  }
  return q;
}

__device__ __forceinline__ double2 ldz(const double2* __restrict__ p, long i, bool ok) {
  return ok ? __ldg(p + i) : make_double2(0.0, 0.0);
}

// KB projections P(o, ilma) = rinv_uvu * sum_j conj(zekr_uV(j,ilma,k)) psi(jxyz)
// (nonlocal_potential.f90:358-367) for one warp = one (orbital, atom); the
// projectors of the atom are processed NP at a time so psi is gathered once
// per pass; deterministic butterfly reduction over the warp.
struct ProjArgs {
  long npts;
  int natom, nlma, nps, totpts, nspin_no, phase_per_k;
  int split;  // 1: the eight-warp summation order of project_sub (few pairs), 0: project_atom's
  const int *atom_start, *mps, *lma_start, *nproj, *pt_lin;
  const double *uv, *rinv, *pt_r;
  const double2* phase;
};

template <int NP, typename TIN>
__device__ __forceinline__ void project_atom(const TIN* __restrict__ in, double2* __restrict__ proj,
                                             const ProjArgs& a, const int atom, const int o) {
  const int lane = threadIdx.x & 31;
  const int ik = o / a.nspin_no;
  const TIN* psi = in + (long)o * a.npts;
  const int start = a.atom_start[atom], m = a.mps[atom];
  const int lma0 = a.lma_start[atom], np = a.nproj[atom];
  const double2* ph = a.phase + (a.phase_per_k ? (long)ik * a.totpts : 0L) + start;
  for (int q0 = 0; q0 < np; q0 += NP) {
    double2 acc[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) acc[q] = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int j = lane; j < m; j += 32) {  // unrolled: the gathers of four iterations in flight
      const TIN vi = __ldg(psi + a.pt_lin[start + j]);
      const double2 v = make_double2((double)vi.x, (double)vi.y);
      const double2 ev = cmul(__ldg(ph + j), v);  // conj(zekr_uV) / uV times psi
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        if (q0 + q < np) acc[q] = cadd(acc[q], cscal(__ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j), ev));
      }
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, off);
        acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, off);
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < NP; ++q)
        if (q0 + q < np) {
          const int lma = lma0 + q0 + q;
          proj[(long)o * a.nlma + lma] = cscal(a.rinv[lma], acc[q]);
        }
    }
  }
}

// The eight-warp summation order for few (orbital, atom) pairs: sub-sum w
// (0..7) of projectors q0 .. q0 + NP - 1 takes sphere points w*32 + lane +
// 256 k in increasing k, butterfly-reduced over the warp.  A CTA of eight
// warps computes the sub-sums side by side (k_project_split), one warp of the
// batched kernel one after the other; both add them in w order, so the two
// give the same bits.
template <int NP, typename TIN>
__device__ __forceinline__ void project_sub(const TIN* __restrict__ psi, const double2* __restrict__ ph,
                                            const ProjArgs& a, const int start, const int m, const int lma0,
                                            const int np, const int q0, const int w, double2 (&acc)[NP]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < NP; ++q) acc[q] = make_double2(0.0, 0.0);
#pragma unroll 2
  for (int j = w * 32 + lane; j < m; j += 256) {
    const TIN vi = __ldg(psi + a.pt_lin[start + j]);
    const double2 v = make_double2((double)vi.x, (double)vi.y);
    const double2 ev = cmul(__ldg(ph + j), v);
#pragma unroll
    for (int q = 0; q < NP; ++q)
      if (q0 + q < np) acc[q] = cadd(acc[q], cscal(__ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j), ev));
  }
#pragma unroll
  for (int q = 0; q < NP; ++q) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, off);
      acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, off);
    }
  }
}

// One warp, the eight-warp order: the projections of one (orbital, atom).
template <int NP, typename TIN>
__device__ __forceinline__ void project_atom_split(const TIN* __restrict__ in, double2* __restrict__ proj,
                                                   const ProjArgs& a, const int atom, const int o) {
  const int lane = threadIdx.x & 31;
  const int ik = o / a.nspin_no;
  const TIN* psi = in + (long)o * a.npts;
  const int start = a.atom_start[atom], m = a.mps[atom];
  const int lma0 = a.lma_start[atom], np = a.nproj[atom];
  const double2* ph = a.phase + (a.phase_per_k ? (long)ik * a.totpts : 0L) + start;
  for (int q0 = 0; q0 < np; q0 += NP) {
    double2 tot[NP], acc[NP];
    project_sub<NP, TIN>(psi, ph, a, start, m, lma0, np, q0, 0, tot);
    for (int w = 1; w < 8; ++w) {
      project_sub<NP, TIN>(psi, ph, a, start, m, lma0, np, q0, w, acc);
#pragma unroll
      for (int q = 0; q < NP; ++q) tot[q] = cadd(tot[q], acc[q]);
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < NP; ++q)
        if (q0 + q < np) {
          const int lma = lma0 + q0 + q;
          proj[(long)o * a.nlma + lma] = cscal(a.rinv[lma], tot[q]);
        }
    }
  }
}

// Local observables per orbital (stencil_current, density_matrix.f90:465-530;
// calc_dip moments, dip.f90:114-225) of one block of points.
struct ObsArgs {
  int nx, ny, nz, periodic, nblk;
  long npts;
  double nab[12];
  double off[3];   // is_d - shift_d
};

// CUR = false (isolated grids: no current) skips the neighbour sums, which
// the final reduction does not use there.
template <bool CUR>
__device__ __forceinline__ void obs_block(const double2* __restrict__ in, double* __restrict__ part,
                                          const ObsArgs& a, const int blk, const int o) {
  __shared__ double red[OBS_NQ][OBS_THREADS];
  const double2* src = in + (long)o * a.npts;
  double q[OBS_NQ];
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) q[i] = 0.0;
  const long base = (long)blk * OBS_THREADS * OBS_PTS_PER_THREAD;
  for (int it = 0; it < OBS_PTS_PER_THREAD; ++it) {
    const long p = base + (long)it * OBS_THREADS + threadIdx.x;
    if (p >= a.npts) break;
    const int pi = (int)p;  // a point of one orbital's grid: 32-bit index arithmetic
    const int x = pi % a.nx;
    const int y = (pi / a.nx) % a.ny;
    const int z = pi / (a.nx * a.ny);
    const double2 c = __ldg(src + p);
    const double r2 = c.x * c.x + c.y * c.y;
    q[0] += r2;
    double ix = 0.0, iy = 0.0, iz = 0.0;
#pragma unroll
    for (int s = 1; s <= (CUR ? ND : 0); ++s) {
      bool ok;
      const int xp = nbr(x, s, a.nx, a.periodic, ok);
      const double2 tx = ldz(src, p - x + xp, ok);
      ix += a.nab[s - 1] * (c.x * tx.y - c.y * tx.x);
      const int yp = nbr(y, s, a.ny, a.periodic, ok);
      const double2 ty = ldz(src, p + (long)(yp - y) * a.nx, ok);
      iy += a.nab[4 + s - 1] * (c.x * ty.y - c.y * ty.x);
      const int zp = nbr(z, s, a.nz, a.periodic, ok);
      const double2 tz = ldz(src, p + (long)(zp - z) * a.nx * a.ny, ok);
      iz += a.nab[8 + s - 1] * (c.x * tz.y - c.y * tz.x);
    }
    q[1] += ix;
    q[2] += iy;
    q[3] += iz;
    q[4] += ((double)x + a.off[0]) * r2;
    q[5] += ((double)y + a.off[1]) * r2;
    q[6] += ((double)z + a.off[2]) * r2;
  }
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) red[i][threadIdx.x] = q[i];
  __syncthreads();
  for (int s = OBS_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
#pragma unroll
      for (int i = 0; i < OBS_NQ; ++i) red[i][threadIdx.x] += red[i][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x < OBS_NQ)
    part[((long)o * a.nblk + blk) * OBS_NQ + threadIdx.x] = red[threadIdx.x][0];
  __syncthreads();  // red is reused by the next call of a persistent caller
}

// ---------------------------------------------------------------------------
// Final per-step reduction in one block: current J (calc_current), calc_dip
// rbox, calc_emfields; advances the device step counter.
// ---------------------------------------------------------------------------
struct FinArgs {
  int norb, nspin, nspin_no, nblk, natom, periodic, itt, trans_longi, advance, spin_filter;
  int jw_natom;            // atoms per orbital in jw (1 when already summed)
  int obs_stride, jw_stride;  // doubles per (orbital, block) record in part / per (orbital, atom) in jw
  double ngrid_inv, dt;
  const double* part;
  const double* jw;        // [norb][natom][3] or null
  const double* weight;
  const double* vec_k;
  const double* Ac_cur;    // a_mode: itt-indexed Ac_tot (history) or direct A[3] when itt_direct
  int A_direct;
  double* Ac_ind;
  double* Ac_tot;
  const double* Ac_ext;
  double* curr_hist;       // (3, nt) or null
  double* rbox_hist;       // (4, nt) or null
  double* result;          // [8] direct results (J3, rbox4) or null
  int* step;
  // shard sums: 0 one pass; 1 write the 7 sums (J before 1/Ngrid, rbox) to
  // sums and stop; 2 take the 7 sums from sums (all-reduced over the k-point
  // shards in between) and finish
  int stage;
  double* sums;
  // non-orthogonal lattice: the lattice-axis current sums are taken to
  // Cartesian components by B^T (density_matrix.f90:313, 413: wrk2 = BT wrk2)
  int nonorth;
  double rB[9];  // rmatrix_B, column-major
};

// Called by one CTA of 256 threads.
__device__ __forceinline__ void finalize_body(const FinArgs& a) {
  __shared__ double red[7][256];
  int itt = a.itt;
  if (itt < 0) itt = *a.step;
  double A[3] = {0.0, 0.0, 0.0};
  if (a.periodic) {
    for (int d = 0; d < 3; ++d) A[d] = a.A_direct ? a.Ac_cur[d] : a.Ac_cur[3 * itt + d];
  }
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
  for (int o = threadIdx.x; o < a.norb && a.stage != 2; o += blockDim.x) {
    if (a.spin_filter >= 0 && (o % a.nspin) != a.spin_filter) continue;
    double q[OBS_NQ] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < a.nblk; ++b)
      for (int i = 0; i < OBS_NQ; ++i) q[i] += a.part[((long)o * a.nblk + b) * a.obs_stride + i];
    const double w = a.weight[o];
    if (a.periodic) {
      const int ik = o / a.nspin_no;
      double jw[3] = {0.0, 0.0, 0.0};
      if (a.jw != nullptr)
        for (int at = 0; at < a.jw_natom; ++at)
          for (int d = 0; d < 3; ++d) jw[d] += a.jw[(long)a.jw_stride * ((long)o * a.jw_natom + at) + d];
      for (int d = 0; d < 3; ++d) {
        const double kAc = a.vec_k[3 * ik + d] + A[d];
        const double ql = a.nonorth ? a.rB[3 * d] * q[1] + a.rB[3 * d + 1] * q[2] + a.rB[3 * d + 2] * q[3] : q[1 + d];
        s[d] += (kAc * q[0] + 2.0 * ql + 2.0 * jw[d]) * w;
      }
    }
    for (int d = 0; d < 3; ++d) s[3 + d] += q[4 + d] * w;
    s[6] += q[0] * w;
  }
  for (int i = 0; i < 7; ++i) red[i][threadIdx.x] = s[i];
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int i = 0; i < 7; ++i) red[i][threadIdx.x] += red[i][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (a.stage == 1) {
      for (int i = 0; i < 7; ++i) a.sums[i] = red[i][0];
      return;
    }
    double tot[7];
    for (int i = 0; i < 7; ++i) tot[i] = a.stage == 2 ? a.sums[i] : red[i][0];
    double J[3], rb[4];
    for (int d = 0; d < 3; ++d) J[d] = tot[d] * a.ngrid_inv;
    for (int d = 0; d < 3; ++d) rb[d] = tot[3 + d];
    rb[3] = tot[6];
    if (a.result) {
      for (int d = 0; d < 3; ++d) a.result[d] = J[d];
      for (int d = 0; d < 4; ++d) a.result[3 + d] = rb[d];
    }
    if (a.curr_hist)
      for (int d = 0; d < 3; ++d) a.curr_hist[3L * (itt - 1) + d] = J[d];
    if (a.rbox_hist)
      for (int d = 0; d < 4; ++d) a.rbox_hist[4L * (itt - 1) + d] = rb[d];
    if (a.periodic && a.Ac_tot) {  // calc_emfields, em_field.f90:47-67
      for (int d = 0; d < 3; ++d) {
        double ind;
        if (a.trans_longi == SB200_TRANS_LO)
          ind = 2.0 * a.Ac_ind[3 * itt + d] - a.Ac_ind[3 * (itt - 1) + d] - 4.0 * PI * J[d] * a.dt * a.dt;
        else
          ind = 0.0;
        a.Ac_ind[3 * (itt + 1) + d] = ind;
        a.Ac_tot[3 * (itt + 1) + d] = a.Ac_ext[3 * (itt + 1) + d] + ind;
      }
    }
    if (a.advance) *a.step = itt + 1;
  }
}

// Per-orbital sums of the observable partials [norb][nblk][OBS_NQ] and of the
// nonlocal-current pieces [norb][natom][3], blocks and atoms in ascending
// order (the order the final reduction adds them): out [norb][OBS_NQ + 3].
// Thread per (orbital, quantity).
// One item (orbital o, quantity i) per warp: lane l sums the partials
// l, l + 32, ... in order, then a butterfly over the warp (a fixed order; for
// one or two partials the plain sum).  Called by all 32 lanes of the warp.
__device__ __forceinline__ void collapse_item(const double* __restrict__ part, int nblk,
                                              const double* __restrict__ jw, int natom, long item,
                                              double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long o = item / (OBS_NQ + 3);
  const int i = (int)(item % (OBS_NQ + 3));
  double s = 0.0;
  if (i < OBS_NQ) {
    for (int b = lane; b < nblk; b += 32) s += part[(o * nblk + b) * OBS_NQ + i];
  } else if (jw != nullptr) {
    for (int at = lane; at < natom; at += 32) s += jw[3 * (o * natom + at) + (i - OBS_NQ)];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) out[item] = s;
}

}  // namespace body

// argument blocks of one context (sb200_kernels.cu)
body::ProjArgs make_proj_args(const sb200_ctx* c);
body::ObsArgs make_obs_args(const sb200_ctx* c);
// itt >= 0: host-given history index, results to d_result; itt < 0: RT loop
body::FinArgs make_fin_args(const sb200_ctx* c, int itt, int trans_longi, double dt, int spin_filter,
                            bool fused_obs);
}  // namespace sb200
