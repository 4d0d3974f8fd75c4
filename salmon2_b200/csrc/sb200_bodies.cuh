// sb200_bodies.cuh -- device-function bodies shared by the per-system kernels
// (sb200_kernels.cu) and the batched persistent kernels (sb200_batch.cu):
// KB projections of one (orbital, atom) and the observable partial sums of
// one (orbital, point block).
#pragma once
#include <cuda_runtime.h>

#include "sb200_internal.cuh"

namespace sb200 {
namespace body {

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
    for (int j = lane; j < m; j += 32) {
      const TIN vi = __ldg(psi + a.pt_lin[start + j]);
      const double2 v = make_double2((double)vi.x, (double)vi.y);
      const double2 e = __ldg(ph + j);
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        if (q0 + q < np) {
          const double uv = __ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j);
          const double2 zk = make_double2(e.x * uv, e.y * uv);  // conj(zekr_uV)
          acc[q] = cadd(acc[q], cmul(zk, v));
        }
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

// Local observables per orbital (stencil_current, density_matrix.f90:465-530;
// calc_dip moments, dip.f90:114-225) of one block of points.
struct ObsArgs {
  int nx, ny, nz, periodic, nblk;
  long npts;
  double nab[12];
  double off[3];   // is_d - shift_d
};

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
    const int x = (int)(p % a.nx);
    const int y = (int)((p / a.nx) % a.ny);
    const int z = (int)(p / ((long)a.nx * a.ny));
    const double2 c = __ldg(src + p);
    const double r2 = c.x * c.x + c.y * c.y;
    q[0] += r2;
    double ix = 0.0, iy = 0.0, iz = 0.0;
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
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

}  // namespace body
}  // namespace sb200
