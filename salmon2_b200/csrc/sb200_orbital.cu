// sb200_orbital.cu -- orbital-resident kernels for small periodic grids (one
// CTA owns one whole 16^3 orbital).  Three forms:
//   * k_step_orbital_st / k_step_orbital (default): the whole Taylor step of
//     the orbital in one launch, every term's h kept on the SM (described at
//     the kernels below);
//   * k_term_orbital: one launch per Taylor term (described here);
//   * k_term_orbital_tma: the per-term form with persistent CTAs and bulk copies.
//
// Per-term form: each CTA loads its orbital once from HBM (16 independent 16-byte loads per
// thread: a full z column), keeps the column in registers for the z
// neighbours and all 16 xy planes in shared memory for the x / y neighbours.
// Because the CTA owns the whole orbital it also computes, from shared memory:
//   * the KB projections <beta|h> of its own input before the stencil (no
//     separate projection pass, nonlocal_potential.f90:358-367);
//   * in the last Taylor term, the observables of the new orbital: sum |psi|^2,
//     the forward-difference current sums (density_matrix.f90:465-530), the
//     dipole moments (dip.f90:114-225) and the nonlocal current projections
//     (density_matrix.f90:532-591), with the projector phases of this step.
// The arithmetic per point is that of zstencil_typical_seq
// (zstencil_core/typical/seq.f90:65-122) plus the owner-computes KB scatter and
// the Taylor epilogue (taylor.f90:47-117); HBM traffic is the algorithmic
// 48/64/64/48 bytes per point of the four Taylor terms.
#include <cuda_runtime.h>

#include "sb200_internal.cuh"
#include "sb200_orbital.cuh"
#include "sb200_tma.cuh"

namespace sb200 {
namespace {

constexpr int N = 16, NP = N * N, NT = NP;  // 16^3 grid, one thread per (x, y) column

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscal(double r, double2 a) { return make_double2(r * a.x, r * a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Projections P(lma) = rinv * sum_j conj(zekr_uV) v(pt_j) of the orbital held
// in shared memory: one warp per atom (NWARP warps), projectors four at a time.
template <int NWARP = NT / 32>
__device__ void project_from_smem(const double2* __restrict__ sm, double2* __restrict__ Ps, const OrbArgs& a,
                                  int ik) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double2* ph = a.phase + (long)ik * a.totpts;
  for (int atom = warp; atom < a.natom; atom += NWARP) {
    const int start = a.atom_start[atom], m = a.mps[atom];
    const int lma0 = a.lma_start[atom], np = a.nproj[atom];
    for (int q0 = 0; q0 < np; q0 += 4) {
      double2 acc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = make_double2(0.0, 0.0);
      for (int j = lane; j < m; j += 32) {
        const double2 v = sm[__ldg(a.pt_lin + start + j)];
        const double2 ev = cmul(__ldg(ph + start + j), v);  // conj(zekr)/uV times psi
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (q0 + q < np) acc[q] = cadd(acc[q], cscal(__ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j), ev));
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, off);
          acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, off);
        }
      }
      if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q0 + q < np) Ps[lma0 + q0 + q] = cscal(__ldg(a.rinv + lma0 + q0 + q), acc[q]);
      }
    }
  }
}

// Nonlocal current pieces sum_lma Im(conj(<r_d zekr|v>) rinv <zekr|v>) of the
// orbital in shared memory, computed by NWARP warps (this one is number
// `warp`); per-warp sums in wsum[warp][0..2].
template <int NWARP>
__device__ void current_nonlocal_from_smem(const double2* __restrict__ sm, const OrbArgs& a, int ik,
                                           double* __restrict__ wsum /* [NWARP][3] */,
                                           int warp = (int)(threadIdx.x >> 5)) {
  // one pass over the atom's sphere per four projectors: e psi(pt) once per
  // point, then <zekr|psi> and <r_d zekr|psi> of each projector
  const int lane = threadIdx.x & 31;
  const double2* ph = a.phase + (long)ik * a.totpts;
  double jx = 0.0, jy = 0.0, jz = 0.0;
  for (int atom = warp; atom < a.natom; atom += NWARP) {
    const int start = a.atom_start[atom], m = a.mps[atom];
    const int lma0 = a.lma_start[atom], np = a.nproj[atom];
    for (int q0 = 0; q0 < np; q0 += 4) {
      double2 u[4], ur[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        u[q] = make_double2(0.0, 0.0);
        ur[q][0] = ur[q][1] = ur[q][2] = u[q];
      }
#pragma unroll 2
      for (int j = lane; j < m; j += 32) {
        const double2 v = sm[__ldg(a.pt_lin + start + j)];
        const double2 ev = cmul(__ldg(ph + start + j), v);
        const double* r = a.pt_r + 3L * (start + j);
        const double r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (q0 + q < np) {
            const double2 tq = cscal(__ldg(a.uv + (long)(lma0 + q0 + q) * a.nps + j), ev);
            u[q] = cadd(u[q], tq);
            ur[q][0] = cadd(ur[q][0], cscal(r0, tq));
            ur[q][1] = cadd(ur[q][1], cscal(r1, tq));
            ur[q][2] = cadd(ur[q][2], cscal(r2, tq));
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
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
      for (int q = 0; q < 4; ++q) {
        if (q0 + q < np) {
          const double2 us = cscal(__ldg(a.rinv + lma0 + q0 + q), u[q]);
          jx += ur[q][0].x * us.y - ur[q][0].y * us.x;
          jy += ur[q][1].x * us.y - ur[q][1].y * us.x;
          jz += ur[q][2].x * us.y - ur[q][2].y * us.x;
        }
      }
    }
  }
  if (lane == 0) {
    wsum[warp * 3 + 0] = jx;
    wsum[warp * 3 + 1] = jy;
    wsum[warp * 3 + 2] = jz;
  }
}

template <int MODE>
__global__ void __launch_bounds__(NT, 2) k_term_orbital(const double2* __restrict__ in, double2* __restrict__ hout,
                                                        double2* __restrict__ acc, OrbArgs a) {
  extern __shared__ double2 smem[];
  double2* sm = smem;            // N planes of N x N
  double2* Ps = smem + N * NP;   // nlma projections
  const int o = blockIdx.x;
  const int t = threadIdx.x;
  const int tx = t & (N - 1), ty = t >> 4;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const double2* src = in + (long)o * a.npts;

  double2 col[N];
#pragma unroll
  for (int z = 0; z < N; ++z) col[z] = __ldg(src + z * NP + t);
#pragma unroll
  for (int z = 0; z < N; ++z) sm[z * NP + t] = col[z];
  __syncthreads();
  if (a.nlma > 0) {
    project_from_smem(sm, Ps, a, ik);
    __syncthreads();
  }
  // k + A factored out of the gradient: w = sum_d kAc_d sum_s nab_s (t+ - t-)
  const double kx = kc[0], ky = kc[1], kz = kc[2], lap0 = kc[3];
  int oxp[ND], oxm[ND], oyp[ND], oym[ND];
#pragma unroll
  for (int s = 1; s <= ND; ++s) {
    oxp[s - 1] = ty * N + ((tx + s) & (N - 1));
    oxm[s - 1] = ty * N + ((tx - s) & (N - 1));
    oyp[s - 1] = (((ty + s) & (N - 1)) << 4) + tx;
    oym[s - 1] = (((ty - s) & (N - 1)) << 4) + tx;
  }
  const double* vloc = a.vloc + (long)ispin * a.npts;
  const double2* zkk = a.ent_zk + (long)ik * a.nent;
  double2* hdst = hout + (long)o * a.npts;
  double2* adst = acc + (long)o * a.npts;
  // per-point operands of plane z+1 are loaded while plane z is computed
  double vl_n = __ldg(vloc + t);
  int pm_n = a.nlma > 0 ? __ldg(a.pmap + t) : -1;
  double2 ac_n = make_double2(0.0, 0.0);
  if (MODE == 2 || MODE == 3) ac_n = adst[t];
#pragma unroll
  for (int z = 0; z < N; ++z) {
    const double vl = vl_n;
    const int pm = pm_n;
    const double2 ac = ac_n;
    if (z + 1 < N) {
      vl_n = __ldg(vloc + (z + 1) * NP + t);
      if (a.nlma > 0) pm_n = __ldg(a.pmap + (z + 1) * NP + t);
      if (MODE == 2 || MODE == 3) ac_n = adst[(z + 1) * NP + t];
    }
    const double2* P = sm + z * NP;
    double2 vx = make_double2(0.0, 0.0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
    for (int s = 0; s < ND; ++s) {
      const double2 tp = P[oxp[s]], tm = P[oxm[s]];
      vx = cadd(vx, cscal(a.lapt[s], cadd(tp, tm)));
      wx = cadd(wx, cscal(a.nab[s], csub(tp, tm)));
    }
#pragma unroll
    for (int s = 0; s < ND; ++s) {
      const double2 tp = P[oyp[s]], tm = P[oym[s]];
      vy = cadd(vy, cscal(a.lapt[4 + s], cadd(tp, tm)));
      wy = cadd(wy, cscal(a.nab[4 + s], csub(tp, tm)));
    }
#pragma unroll
    for (int s = 0; s < ND; ++s) {
      const double2 tp = col[(z + s + 1) & (N - 1)], tm = col[(z - s - 1) & (N - 1)];
      vz = cadd(vz, cscal(a.lapt[8 + s], cadd(tp, tm)));
      wz = cadd(wz, cscal(a.nab[8 + s], csub(tp, tm)));
    }
    const double2 v = cadd(vz, cadd(vy, vx));
    const double2 w = cadd(cscal(kz, wz), cadd(cscal(ky, wy), cscal(kx, wx)));
    const double2 c = col[z];
    const int p = z * NP + t;
    double2 h;
    h.x = vl * c.x + lap0 * c.x - 0.5 * v.x + w.y;
    h.y = vl * c.y + lap0 * c.y - 0.5 * v.y - w.x;
    if (a.nlma > 0) {
      if (pm >= 0) {
        const int e1 = (pm >> 8) + (pm & 255);
        for (int e = pm >> 8; e < e1; ++e) h = cadd(h, cmul(Ps[__ldg(a.ent_lma + e)], __ldg(zkk + e)));
      }
    }
    if (MODE == 1 || MODE == 2) hdst[p] = h;
    if (MODE == 1 || MODE == 4) adst[p] = cadd(c, cmul(a.zc, h));
    else adst[p] = cadd(ac, cmul(a.zc, h));
  }
  if (MODE != 3 && MODE != 4) return;
  if (a.obs == nullptr) return;
  // ---- observables of the new orbital (last Taylor term) ----
  __shared__ double red[OBS_NQ][NT / 32];
  __syncthreads();  // all reads of the input planes are done
  // the new orbital: this thread's own column, just written (program order)
#pragma unroll
  for (int z = 0; z < N; ++z) sm[z * NP + t] = adst[z * NP + t];
  __syncthreads();
  double q[OBS_NQ];
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) q[i] = 0.0;
#pragma unroll 4
  for (int z = 0; z < N; ++z) {
    const double2 c = sm[z * NP + t];
    const double r2 = c.x * c.x + c.y * c.y;
    q[0] += r2;
    double ix = 0.0, iy = 0.0, iz = 0.0;
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      const double2 txv = sm[z * NP + ty * N + ((tx + s) & (N - 1))];
      const double2 tyv = sm[z * NP + (((ty + s) & (N - 1)) << 4) + tx];
      const double2 tzv = sm[((z + s) & (N - 1)) * NP + t];
      ix += a.nab[s - 1] * (c.x * txv.y - c.y * txv.x);
      iy += a.nab[4 + s - 1] * (c.x * tyv.y - c.y * tyv.x);
      iz += a.nab[8 + s - 1] * (c.x * tzv.y - c.y * tzv.x);
    }
    q[1] += ix;
    q[2] += iy;
    q[3] += iz;
    q[4] += ((double)tx + a.off[0]) * r2;
    q[5] += ((double)ty + a.off[1]) * r2;
    q[6] += ((double)z + a.off[2]) * r2;
  }
  // warp tree (deterministic), then warps in order
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) q[i] += __shfl_xor_sync(0xffffffffu, q[i], off);
  }
  const int warp = t >> 5, lane = t & 31;
  if (lane == 0)
    for (int i = 0; i < OBS_NQ; ++i) red[i][warp] = q[i];
  __shared__ double jws[NT / 32][3];
  if (a.nlma > 0) current_nonlocal_from_smem<NT / 32>(sm, a, ik, &jws[0][0]);
  __syncthreads();
  if (t < OBS_NQ) {
    double s = 0.0;
    for (int w = 0; w < NT / 32; ++w) s += red[t][w];
    a.obs[(long)o * OBS_NQ + t] = s;
  } else if (t >= 32 && t < 35 && a.jw != nullptr) {  // no nonlocal current without projectors
    double s = 0.0;
    if (a.nlma > 0)
      for (int w = 0; w < NT / 32; ++w) s += jws[w][t - 32];
    a.jw[3L * o + (t - 32)] = s;
  }
}


// ---------------------------------------------------------------------------
// Fused Taylor step: one CTA of 512 threads applies all n_hamil terms of
// taylor.f90:47-117 to one 16^3 orbital without leaving the SM.  h_{n-1} sits
// in one of two whole-orbital shared-memory buffers while h_n is written into
// the other; psi_out sits in a third.  Thread t owns column (x, y) = t mod 256
// for the eight planes z0 = 8 (t / 256) .. z0 + 7 and keeps those eight values
// of h_{n-1} in registers for the z neighbours; the four-plane halo owned by the
// other half of the column is read from shared memory.  Each term starts with
// the KB projections of h_{n-1} from shared memory.  HBM traffic per step is
// read psi + write psi_out (32 B per point) instead of 224 B for four separate
// term launches.  The operations per point and term, and their order, are
// those of k_term_orbital.
// ---------------------------------------------------------------------------
constexpr int NTF = 2 * NP;  // threads of the fused-step CTA
constexpr int HZ = N / 2;    // planes per thread

// Observables of the new orbital held in shared memory, after the last
// Taylor term of the fused step: warps 0-7 the local sums over whole columns,
// warps 8-15 the nonlocal current, as in k_term_orbital.
__device__ __forceinline__ void step_observables(const double2* __restrict__ accb, const OrbArgs& a, int o, int ik) {
  const int t = threadIdx.x;
  const int tx = t & (N - 1), ty = (t >> 4) & (N - 1);
  __shared__ double red[OBS_NQ][NP / 32];
  __shared__ double jws[NP / 32][3];
  const int warp = t >> 5, lane = t & 31;
  if (t < NP) {
    const double2* sm = accb;
    double q[OBS_NQ];
#pragma unroll
    for (int i = 0; i < OBS_NQ; ++i) q[i] = 0.0;
#pragma unroll 4
    for (int z = 0; z < N; ++z) {
      const double2 c = sm[z * NP + t];
      const double r2 = c.x * c.x + c.y * c.y;
      q[0] += r2;
      double ix = 0.0, iy = 0.0, iz = 0.0;
#pragma unroll
      for (int s = 1; s <= ND; ++s) {
        const double2 txv = sm[z * NP + ty * N + ((tx + s) & (N - 1))];
        const double2 tyv = sm[z * NP + (((ty + s) & (N - 1)) << 4) + tx];
        const double2 tzv = sm[((z + s) & (N - 1)) * NP + t];
        ix += a.nab[s - 1] * (c.x * txv.y - c.y * txv.x);
        iy += a.nab[4 + s - 1] * (c.x * tyv.y - c.y * tyv.x);
        iz += a.nab[8 + s - 1] * (c.x * tzv.y - c.y * tzv.x);
      }
      q[1] += ix;
      q[2] += iy;
      q[3] += iz;
      q[4] += ((double)tx + a.off[0]) * r2;
      q[5] += ((double)ty + a.off[1]) * r2;
      q[6] += ((double)z + a.off[2]) * r2;
    }
#pragma unroll
    for (int i = 0; i < OBS_NQ; ++i) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) q[i] += __shfl_xor_sync(0xffffffffu, q[i], off);
    }
    if (lane == 0)
      for (int i = 0; i < OBS_NQ; ++i) red[i][warp] = q[i];
  } else if (a.nlma > 0) {
    current_nonlocal_from_smem<NP / 32>(accb, a, ik, &jws[0][0], warp - NP / 32);
  }
  __syncthreads();
  if (t < OBS_NQ) {
    double s = 0.0;
    for (int w = 0; w < NP / 32; ++w) s += red[t][w];
    a.obs[(long)o * OBS_NQ + t] = s;
  } else if (t >= 32 && t < 35 && a.jw != nullptr) {  // no nonlocal current without projectors
    double s = 0.0;
    if (a.nlma > 0)
      for (int w = 0; w < NP / 32; ++w) s += jws[w][t - 32];
    a.jw[3L * o + (t - 32)] = s;
  }
}

template <bool OBS>
__global__ void __launch_bounds__(NTF, 1) k_step_orbital(const double2* __restrict__ in, double2* __restrict__ out,
                                                         OrbArgs a, StepZC zc, int nterm) {
  extern __shared__ double2 smem[];
  double2* bufs = smem;               // two whole-orbital buffers: h_{n-1}, h_n
  double2* accb = smem + 2 * N * NP;  // psi_out
  double2* Ps = accb + N * NP;        // projections of h_{n-1}
  const int o = blockIdx.x;
  const int t = threadIdx.x;
  const int col = t & (NP - 1);
  const int z0 = (t >> 8) * HZ;
  const int tx = col & (N - 1), ty = col >> 4;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const double2* src = in + (long)o * a.npts;

  double2 cv[HZ];
#pragma unroll
  for (int j = 0; j < HZ; ++j) cv[j] = __ldg(src + (z0 + j) * NP + col);
#pragma unroll
  for (int j = 0; j < HZ; ++j) bufs[(z0 + j) * NP + col] = cv[j];
  __syncthreads();
  const double kx = kc[0], ky = kc[1], kz = kc[2], lap0 = kc[3];
  int oxp[ND], oxm[ND], oyp[ND], oym[ND];
#pragma unroll
  for (int s = 1; s <= ND; ++s) {
    oxp[s - 1] = ty * N + ((tx + s) & (N - 1));
    oxm[s - 1] = ty * N + ((tx - s) & (N - 1));
    oyp[s - 1] = (((ty + s) & (N - 1)) << 4) + tx;
    oym[s - 1] = (((ty - s) & (N - 1)) << 4) + tx;
  }
  const double* vloc = a.vloc + (long)ispin * a.npts;
  const double2* zkk = a.ent_zk + (long)ik * a.nent;
  double2* odst = out + (long)o * a.npts;
  int b = 0;
  for (int nn = 0; nn < nterm; ++nn) {
    const double2* cur = bufs + b * (N * NP);
    double2* nxt = bufs + (b ^ 1) * (N * NP);
    if (a.nlma > 0) {
      project_from_smem<NTF / 32>(cur, Ps, a, ik);
      __syncthreads();
    }
    const bool last = nn == nterm - 1;
    const double2 zn = zc.v[nn];
    const double2* oth = cur + (z0 ^ HZ) * NP + col;  // the other half of this column
    double vl_n = __ldg(vloc + z0 * NP + col);
    int pm_n = a.nlma > 0 ? __ldg(a.pmap + z0 * NP + col) : -1;
    double2 hv[HZ];
#pragma unroll
    for (int j = 0; j < HZ; ++j) {
      const int z = z0 + j;
      const double vl = vl_n;
      const int pm = pm_n;
      if (j + 1 < HZ) {
        vl_n = __ldg(vloc + (z + 1) * NP + col);
        if (a.nlma > 0) pm_n = __ldg(a.pmap + (z + 1) * NP + col);
      }
      const double2* P = cur + z * NP;
      double2 vx = make_double2(0.0, 0.0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = P[oxp[s]], tm = P[oxm[s]];
        vx = cadd(vx, cscal(a.lapt[s], cadd(tp, tm)));
        wx = cadd(wx, cscal(a.nab[s], csub(tp, tm)));
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = P[oyp[s]], tm = P[oym[s]];
        vy = cadd(vy, cscal(a.lapt[4 + s], cadd(tp, tm)));
        wy = cadd(wy, cscal(a.nab[4 + s], csub(tp, tm)));
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = (j + s + 1 < HZ) ? cv[(j + s + 1) & (HZ - 1)] : oth[(j + s + 1 - HZ) * NP];
        const double2 tm = (j - s - 1 >= 0) ? cv[(j - s - 1) & (HZ - 1)] : oth[(j - s - 1 + HZ) * NP];
        vz = cadd(vz, cscal(a.lapt[8 + s], cadd(tp, tm)));
        wz = cadd(wz, cscal(a.nab[8 + s], csub(tp, tm)));
      }
      const double2 v = cadd(vz, cadd(vy, vx));
      const double2 w = cadd(cscal(kz, wz), cadd(cscal(ky, wy), cscal(kx, wx)));
      const double2 c = cv[j];
      const int p = z * NP + col;
      double2 h;
      h.x = vl * c.x + lap0 * c.x - 0.5 * v.x + w.y;
      h.y = vl * c.y + lap0 * c.y - 0.5 * v.y - w.x;
      if (a.nlma > 0) {
        if (pm >= 0) {
          const int e1 = (pm >> 8) + (pm & 255);
          for (int e = pm >> 8; e < e1; ++e) h = cadd(h, cmul(Ps[__ldg(a.ent_lma + e)], __ldg(zkk + e)));
        }
      }
      // psi_out = psi + zc_1 h_1 (first term), psi_out + zc_n h_n (later terms)
      const double2 nv = cadd(nn == 0 ? c : accb[p], cmul(zn, h));
      if (last) {
        odst[p] = nv;
        if (OBS) accb[p] = nv;
      } else {
        accb[p] = nv;
        nxt[p] = h;
        hv[j] = h;
      }
    }
    __syncthreads();  // h_n complete in nxt; reads of cur and Ps done
    if (!last) {
#pragma unroll
      for (int j = 0; j < HZ; ++j) cv[j] = hv[j];
      b ^= 1;
    }
  }
  if (!OBS) return;
  step_observables(accb, a, o, ik);
}


// ---------------------------------------------------------------------------
// Fused Taylor step with the KB tables in shared memory.  The (point, atom)
// pair tables of the CTA's k-point -- phase exp(i(k+A).r), the uV of the
// atom's projectors at the point, lma0 | nproj, the grid point -- and the map
// (atom, sphere point) -> pair are copied into shared memory once per step, so
// the projections of every term and the scatter read no global tables.  To
// make room psi_out is kept in registers (eight values per thread) and h_n is
// re-read from shared memory for the next term's z neighbours.  The scatter
// sums each atom's projectors first, sum_q uV_q P_q, then multiplies by the
// conjugate phase (the pair form of the tiled kernels).
// ---------------------------------------------------------------------------
template <bool OBS>
__global__ void __launch_bounds__(NTF, 1) k_step_orbital_st(const double2* __restrict__ in,
                                                            double2* __restrict__ out, OrbArgs a, StageArgs st,
                                                            StepZC zc, int nterm) {
  extern __shared__ double2 smem[];
  double2* bufs = smem;                            // two whole-orbital buffers
  double2* Ps = smem + 2 * N * NP;                 // projections of h_{n-1}
  double2* sph = Ps + a.nlma;                      // [npair] phase
  double* suv = (double*)(sph + st.npair);         // [4][npair] uV (projector-major: no bank conflicts)
  int* slma = (int*)(suv + 4L * st.npair);         // [npair] lma0 | nproj << 24
  int* spt = slma + st.npair;                      // [npair] grid point
  int* sapj = spt + st.npair;                      // [totpts] pair of (atom, sphere point)
  const int o = blockIdx.x;
  const int t = threadIdx.x;
  const int col = t & (NP - 1);
  const int z0 = (t >> 8) * HZ;
  const int tx = col & (N - 1), ty = col >> 4;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const double2* src = in + (long)o * a.npts;

  double2 cv[HZ];
#pragma unroll
  for (int j = 0; j < HZ; ++j) cv[j] = __ldg(src + (z0 + j) * NP + col);
  {
    const double2* gph = st.pair_ph + (long)ik * st.npair;
    for (int i = t; i < st.npair; i += NTF) {
      sph[i] = __ldg(gph + i);
      const double2 u01 = __ldg((const double2*)(st.pair_uv + 4L * i));
      const double2 u23 = __ldg((const double2*)(st.pair_uv + 4L * i + 2));
      suv[i] = u01.x;
      suv[st.npair + i] = u01.y;
      suv[2 * st.npair + i] = u23.x;
      suv[3 * st.npair + i] = u23.y;
      slma[i] = __ldg(st.pair_lma + i);
      spt[i] = __ldg(st.pair_pt + i);
    }
    for (int i = t; i < a.totpts; i += NTF) sapj[i] = __ldg(st.apj + i);
  }
#pragma unroll
  for (int j = 0; j < HZ; ++j) bufs[(z0 + j) * NP + col] = cv[j];
  __syncthreads();
  const double kx = kc[0], ky = kc[1], kz = kc[2], lap0 = kc[3];
  int oxp[ND], oxm[ND], oyp[ND], oym[ND];
#pragma unroll
  for (int s = 1; s <= ND; ++s) {
    oxp[s - 1] = ty * N + ((tx + s) & (N - 1));
    oxm[s - 1] = ty * N + ((tx - s) & (N - 1));
    oyp[s - 1] = (((ty + s) & (N - 1)) << 4) + tx;
    oym[s - 1] = (((ty - s) & (N - 1)) << 4) + tx;
  }
  const double* vloc = a.vloc + (long)ispin * a.npts;
  double2* odst = out + (long)o * a.npts;
  const int warp = t >> 5, lane = t & 31;
  double2 acc[HZ];
  int b = 0;
  for (int nn = 0; nn < nterm; ++nn) {
    const double2* cur = bufs + b * (N * NP);
    double2* nxt = bufs + (b ^ 1) * (N * NP);
    if (a.nlma > 0) {  // P(lma) = rinv sum_j uV e^{i(k+A).r_j} h(pt_j): one warp per atom
      for (int atom = warp; atom < a.natom; atom += NTF / 32) {
        const int start = __ldg(a.atom_start + atom), m = __ldg(a.mps + atom);
        const int lma0 = __ldg(a.lma_start + atom), np = __ldg(a.nproj + atom);
        if (np == 0) continue;  // no projectors: its sphere points have no pairs
        double2 pq[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) pq[q] = make_double2(0.0, 0.0);
        for (int j = lane; j < m; j += 32) {
          const int pr = sapj[start + j];
          const double2 ev = cmul(sph[pr], cur[spt[pr]]);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < np) pq[q] = cadd(pq[q], cscal(suv[q * st.npair + pr], ev));
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            pq[q].x += __shfl_xor_sync(0xffffffffu, pq[q].x, off);
            pq[q].y += __shfl_xor_sync(0xffffffffu, pq[q].y, off);
          }
        }
        if (lane == 0) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < np) Ps[lma0 + q] = cscal(__ldg(a.rinv + lma0 + q), pq[q]);
        }
      }
      __syncthreads();
    }
    const bool last = nn == nterm - 1;
    const double2 zn = zc.v[nn];
    const double2* oth = cur + (z0 ^ HZ) * NP + col;  // the other half of this column
    double vl_n = __ldg(vloc + z0 * NP + col);
    int pm_n = a.nlma > 0 ? __ldg(st.pmap2 + z0 * NP + col) : -1;
#pragma unroll
    for (int j = 0; j < HZ; ++j) {
      const int z = z0 + j;
      const double vl = vl_n;
      const int pm = pm_n;
      if (j + 1 < HZ) {
        vl_n = __ldg(vloc + (z + 1) * NP + col);
        if (a.nlma > 0) pm_n = __ldg(st.pmap2 + (z + 1) * NP + col);
      }
      const double2* P = cur + z * NP;
      double2 vx = make_double2(0.0, 0.0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = P[oxp[s]], tm = P[oxm[s]];
        vx = cadd(vx, cscal(a.lapt[s], cadd(tp, tm)));
        wx = cadd(wx, cscal(a.nab[s], csub(tp, tm)));
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = P[oyp[s]], tm = P[oym[s]];
        vy = cadd(vy, cscal(a.lapt[4 + s], cadd(tp, tm)));
        wy = cadd(wy, cscal(a.nab[4 + s], csub(tp, tm)));
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = (j + s + 1 < HZ) ? cv[(j + s + 1) & (HZ - 1)] : oth[(j + s + 1 - HZ) * NP];
        const double2 tm = (j - s - 1 >= 0) ? cv[(j - s - 1) & (HZ - 1)] : oth[(j - s - 1 + HZ) * NP];
        vz = cadd(vz, cscal(a.lapt[8 + s], cadd(tp, tm)));
        wz = cadd(wz, cscal(a.nab[8 + s], csub(tp, tm)));
      }
      const double2 v = cadd(vz, cadd(vy, vx));
      const double2 w = cadd(cscal(kz, wz), cadd(cscal(ky, wy), cscal(kx, wx)));
      const double2 c = cv[j];
      const int p = z * NP + col;
      double2 h;
      h.x = vl * c.x + lap0 * c.x - 0.5 * v.x + w.y;
      h.y = vl * c.y + lap0 * c.y - 0.5 * v.y - w.x;
      if (pm >= 0) {  // (point, atom) pairs of this point, atoms in ilma order
        const int p1 = (pm >> 8) + (pm & 255);
        for (int pr = pm >> 8; pr < p1; ++pr) {
          const int lm = slma[pr];
          const int l0 = lm & 0xffffff, np = lm >> 24;
          double2 sp = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < np) {
              const double u = suv[q * st.npair + pr];
              const double2 pv = Ps[l0 + q];
              sp = make_double2(fma(u, pv.x, sp.x), fma(u, pv.y, sp.y));
            }
          const double2 e = sph[pr];
          h = cadd(h, cmul(make_double2(e.x, -e.y), sp));
        }
      }
      // psi_out = psi + zc_1 h_1 (first term), psi_out + zc_n h_n (later terms)
      const double2 nv = cadd(nn == 0 ? c : acc[j], cmul(zn, h));
      acc[j] = nv;
      if (last) {
        odst[p] = nv;
        if (OBS) nxt[p] = nv;  // the new orbital, for the observables
      } else {
        nxt[p] = h;
      }
    }
    __syncthreads();  // h_n complete in nxt; reads of cur and Ps done
    if (!last) {
#pragma unroll
      for (int j = 0; j < HZ; ++j) cv[j] = nxt[(z0 + j) * NP + col];
      b ^= 1;
    }
  }
  if (!OBS) return;
  step_observables(bufs + (b ^ 1) * (N * NP), a, o, ik);
}


// ---------------------------------------------------------------------------
// Persistent form: one CTA of 256 threads per SM walks orbitals
// o = blockIdx.x, blockIdx.x + gridDim.x, ...  Whole orbitals (64 KB) arrive
// by bulk copy (TMA, cp.async.bulk) into two shared-memory buffers, so the
// copy of orbital i+1 overlaps the stencil of orbital i; the Taylor
// accumulator psi_out of the orbital (modes 2, 3) is copied in the same way
// into a third buffer.  Thread t owns column (x, y) = t and keeps its whole z
// column in registers (up to 255 registers per thread at one CTA per SM).
// The Bloch gradient is applied as kAc_d * sum_s nab_s (psi(+s) - psi(-s)).
// ---------------------------------------------------------------------------
constexpr int NT2 = NP;
constexpr unsigned ORB_BYTES = N * NP * sizeof(double2);

// KB projections of the orbital in shared memory: one warp per projector.
__device__ void project_lma_from_smem(const double2* __restrict__ sm, double2* __restrict__ Ps, const OrbArgs& a,
                                      int ik) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double2* ph = a.phase + (long)ik * a.totpts;
  for (int lma = warp; lma < a.nlma; lma += NT2 / 32) {
    const int atom = __ldg(a.lma_atom + lma);
    const int start = __ldg(a.atom_start + atom), m = __ldg(a.mps + atom);
    const double* uvr = a.uv + (long)lma * a.nps;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int j = lane; j < m; j += 32) {
      const double2 v = sm[__ldg(a.pt_lin + start + j)];
      const double2 e = __ldg(ph + start + j);
      const double uv = __ldg(uvr + j);
      acc = cadd(acc, cmul(make_double2(e.x * uv, e.y * uv), v));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
    }
    if (lane == 0) Ps[lma] = cscal(__ldg(a.rinv + lma), acc);
  }
}

// Stencil + KB scatter + Taylor epilogue of the 16 planes of one column.
template <int MODE>
__device__ __forceinline__ void column_all(const double2* __restrict__ sm, const double2* __restrict__ Ps,
                                           double2* __restrict__ accb, const double2 (&colv)[N], const OrbArgs& a,
                                           int col, int tx, int ty, int ispin, int ik, double2* __restrict__ hdst,
                                           double2* __restrict__ adst) {
  constexpr bool READ_ACC = (MODE == 2 || MODE == 3);
  const double* kc = a.kcoef + (long)KC * ik;
  const double kx = kc[0], ky = kc[1], kz = kc[2], lap0 = kc[3];
  const double* vloc = a.vloc + (long)ispin * a.npts;
  const double2* zkk = a.ent_zk + (long)ik * a.nent;
  double vl_n = __ldg(vloc + col);
  int pm_n = a.nlma > 0 ? __ldg(a.pmap + col) : -1;
#pragma unroll
  for (int z = 0; z < N; ++z) {
    const double vl = vl_n;
    const int pm = pm_n;
    if (z + 1 < N) {
      vl_n = __ldg(vloc + (z + 1) * NP + col);
      if (a.nlma > 0) pm_n = __ldg(a.pmap + (z + 1) * NP + col);
    }
    const double2* P = sm + z * NP;
    double2 vx = make_double2(0.0, 0.0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      const double2 tp = P[ty * N + ((tx + s) & (N - 1))], tm = P[ty * N + ((tx - s) & (N - 1))];
      vx = cadd(vx, cscal(a.lapt[s - 1], cadd(tp, tm)));
      wx = cadd(wx, cscal(a.nab[s - 1], csub(tp, tm)));
    }
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      const double2 tp = P[(((ty + s) & (N - 1)) << 4) + tx], tm = P[(((ty - s) & (N - 1)) << 4) + tx];
      vy = cadd(vy, cscal(a.lapt[4 + s - 1], cadd(tp, tm)));
      wy = cadd(wy, cscal(a.nab[4 + s - 1], csub(tp, tm)));
    }
#pragma unroll
    for (int s = 0; s < ND; ++s) {
      const double2 tp = colv[(z + s + 1) & (N - 1)], tm = colv[(z - s - 1) & (N - 1)];
      vz = cadd(vz, cscal(a.lapt[8 + s], cadd(tp, tm)));
      wz = cadd(wz, cscal(a.nab[8 + s], csub(tp, tm)));
    }
    const double2 v = cadd(vz, cadd(vy, vx));
    const double2 w = cadd(cscal(kz, wz), cadd(cscal(ky, wy), cscal(kx, wx)));
    const double2 c = colv[z];
    const int p = z * NP + col;
    double2 h;
    h.x = vl * c.x + lap0 * c.x - 0.5 * v.x + w.y;
    h.y = vl * c.y + lap0 * c.y - 0.5 * v.y - w.x;
    if (a.nlma > 0 && pm >= 0) {
      const int e1 = (pm >> 8) + (pm & 255);
      for (int e = pm >> 8; e < e1; ++e) h = cadd(h, cmul(Ps[__ldg(a.ent_lma + e)], __ldg(zkk + e)));
    }
    if (MODE == 1 || MODE == 2) hdst[p] = h;
    double2 nv;
    if (READ_ACC) nv = cadd(accb[p], cmul(a.zc, h));
    else nv = cadd(c, cmul(a.zc, h));
    adst[p] = nv;
    if (MODE == 3 || MODE == 4) accb[p] = nv;  // the new orbital, for the observables
  }
}

// Observables of the new orbital held in shared memory (last Taylor term).
__device__ __forceinline__ void observables_smem(const double2* __restrict__ sm, const OrbArgs& a, int o, int ik,
                                                 double (*red)[NT2 / 32], double (*jws)[3]) {
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  double q[OBS_NQ];
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) q[i] = 0.0;
#pragma unroll 4
  for (int z = 0; z < N; ++z) {
    const double2 c = sm[z * NP + t];
    const double r2 = c.x * c.x + c.y * c.y;
    q[0] += r2;
    double ix = 0.0, iy = 0.0, iz = 0.0;
#pragma unroll
    for (int s = 1; s <= ND; ++s) {
      const double2 txv = sm[z * NP + ty * N + ((tx + s) & (N - 1))];
      const double2 tyv = sm[z * NP + (((ty + s) & (N - 1)) << 4) + tx];
      const double2 tzv = sm[((z + s) & (N - 1)) * NP + t];
      ix += a.nab[s - 1] * (c.x * txv.y - c.y * txv.x);
      iy += a.nab[4 + s - 1] * (c.x * tyv.y - c.y * tyv.x);
      iz += a.nab[8 + s - 1] * (c.x * tzv.y - c.y * tzv.x);
    }
    q[1] += ix;
    q[2] += iy;
    q[3] += iz;
    q[4] += ((double)tx + a.off[0]) * r2;
    q[5] += ((double)ty + a.off[1]) * r2;
    q[6] += ((double)z + a.off[2]) * r2;
  }
#pragma unroll
  for (int i = 0; i < OBS_NQ; ++i) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) q[i] += __shfl_xor_sync(0xffffffffu, q[i], off);
  }
  const int warp = t >> 5, lane = t & 31;
  if (lane == 0)
    for (int i = 0; i < OBS_NQ; ++i) red[i][warp] = q[i];
  if (a.nlma > 0) current_nonlocal_from_smem<NT2 / 32>(sm, a, ik, &jws[0][0]);
  __syncthreads();
  if (t < OBS_NQ) {
    double s = 0.0;
    for (int w = 0; w < NT2 / 32; ++w) s += red[t][w];
    a.obs[(long)o * OBS_NQ + t] = s;
  } else if (t >= 32 && t < 35 && a.jw != nullptr) {  // no nonlocal current without projectors
    double s = 0.0;
    if (a.nlma > 0)
      for (int w = 0; w < NT2 / 32; ++w) s += jws[w][t - 32];
    a.jw[3L * o + (t - 32)] = s;
  }
}

template <int MODE>
__global__ void __launch_bounds__(NT2, 1) k_term_orbital_tma(const double2* __restrict__ in,
                                                             double2* __restrict__ hout, double2* __restrict__ acc,
                                                             OrbArgs a, int norb, int* __restrict__ err) {
  constexpr bool READ_ACC = (MODE == 2 || MODE == 3);
  extern __shared__ __align__(128) unsigned char smraw[];
  double2* bufs = (double2*)smraw;         // two orbital buffers
  double2* accb = bufs + 2 * N * NP;        // psi_out of the orbital / the new orbital
  double2* Ps = accb + N * NP;              // projections
  __shared__ __align__(8) uint64_t bar[3];  // buffer 0, buffer 1, accumulator
  __shared__ double red[OBS_NQ][NT2 / 32];
  __shared__ double jws[NT2 / 32][3];
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  const int G = gridDim.x;
  const int nmine = ((int)blockIdx.x < norb) ? (norb - (int)blockIdx.x + G - 1) / G : 0;
  const bool obs = (MODE == 3 || MODE == 4) && a.obs != nullptr;
  if (t == 0) {
    tma::mbar_init(&bar[0], 1);
    tma::mbar_init(&bar[1], 1);
    tma::mbar_init(&bar[2], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  if (t == 0) {
    for (int i = 0; i < 2 && i < nmine; ++i) {
      const long o = blockIdx.x + (long)i * G;
      tma::mbar_arrive_expect_tx(&bar[i], ORB_BYTES);
      tma::bulk_load(bufs + i * N * NP, in + o * a.npts, ORB_BYTES, &bar[i]);
    }
    if (READ_ACC && nmine > 0) {
      tma::mbar_arrive_expect_tx(&bar[2], ORB_BYTES);
      tma::bulk_load(accb, acc + (long)blockIdx.x * a.npts, ORB_BYTES, &bar[2]);
    }
  }
  // orbital buffers issued so far (the same count in every thread)
  int psi_issued = nmine < 2 ? nmine : 2;
  for (int i = 0; i < nmine; ++i) {
    const int o = blockIdx.x + i * G;
    const int b = i & 1;
    const double2* sm = bufs + b * N * NP;
    bool ok = tma::mbar_wait(&bar[b], (unsigned)((i >> 1) & 1));
    if (READ_ACC) ok = tma::mbar_wait(&bar[2], (unsigned)(i & 1)) && ok;
    if (!__syncthreads_and(ok)) {
      // a copy did not arrive in time: flag it, wait (bounded) for the other
      // orbital copy this CTA has in flight, and leave
      if (t == 0) {
        atomicExch(err, 1);
        for (int k = i + 1; k < psi_issued; ++k) tma::mbar_wait(&bar[k & 1], (unsigned)((k >> 1) & 1));
      }
      __syncthreads();
      return;
    }
    const int ik = o / a.nspin_no;
    const int ispin = o % a.nspin;
    if (a.nlma > 0) {
      project_lma_from_smem(sm, Ps, a, ik);
      __syncthreads();
    }
    double2 colv[N];
#pragma unroll
    for (int z = 0; z < N; ++z) colv[z] = sm[z * NP + t];
    column_all<MODE>(sm, Ps, accb, colv, a, t, tx, ty, ispin, ik, hout + (long)o * a.npts, acc + (long)o * a.npts);
    __syncthreads();  // buffer b, accb and Ps are free (accb holds the new orbital in modes 3, 4)
    if (obs) {
      observables_smem(accb, a, o, ik, red, jws);
      __syncthreads();
    }
    if (t == 0) {  // refill: orbital i+2 into buffer b, psi_out of orbital i+1 into accb
      tma::fence_proxy_async_smem();
      if (i + 2 < nmine) {
        const long o2 = blockIdx.x + (long)(i + 2) * G;
        tma::mbar_arrive_expect_tx(&bar[b], ORB_BYTES);
        tma::bulk_load(bufs + b * N * NP, in + o2 * a.npts, ORB_BYTES, &bar[b]);
      }
      if (READ_ACC && i + 1 < nmine) {
        const long o1 = blockIdx.x + (long)(i + 1) * G;
        tma::mbar_arrive_expect_tx(&bar[2], ORB_BYTES);
        tma::bulk_load(accb, acc + o1 * a.npts, ORB_BYTES, &bar[2]);
      }
    }
    if (i + 2 < nmine) psi_issued = i + 3;
  }
}
}  // namespace

bool orbital_kernel_applies(const sb200_ctx* c) {
  const GridInfo& g = c->g;
  return g.periodic && !g.nonorth && !c->microac && !c->cap_on && g.nx == N && g.ny == N && g.nz == N && c->stencil_variant == 1 &&
         c->pp.nlma <= ORB_MAX_NLMA && c->precision == SB200_PREC_FP64;
}

namespace {
OrbArgs make_orb_args(const sb200_ctx* c, double2 zc, bool with_obs) {
  OrbArgs a;
  a.npts = c->g.npts;
  a.nspin = c->orb.nspin;
  a.nspin_no = c->orb.nspin * c->orb.no;
  a.nlma = c->pp.nlma;
  a.natom = c->pp.natom;
  a.nps = c->pp.nps;
  a.totpts = c->pp.totpts;
  for (int i = 0; i < 12; ++i) {
    a.lapt[i] = c->g.coef_lap[i];
    a.nab[i] = c->g.coef_nab[i];
  }
  for (int d = 0; d < 3; ++d) a.off[d] = (double)c->g.is[d] - ((c->g.lg_num[d] % 2 == 1) ? 0.0 : 0.5);
  a.kcoef = c->d_kcoef;
  a.vloc = c->d_vloc;
  a.pmap = c->pp.d_pmap;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_zk = c->pp.d_ent_zk;
  a.nent = c->pp.nent;
  a.phase = c->pp.d_phase;
  a.atom_start = c->pp.d_atom_start;
  a.mps = c->pp.d_mps;
  a.lma_start = c->pp.d_lma_start;
  a.nproj = c->pp.d_nproj;
  a.pt_lin = c->pp.d_pt_lin;
  a.lma_atom = c->pp.d_lma_atom;
  a.pt_r = c->pp.d_pt_r;
  a.uv = c->pp.d_uv;
  a.rinv = c->pp.d_rinv;
  a.zc = zc;
  a.obs = with_obs ? c->d_obs : nullptr;
  a.jw = (with_obs && c->pp.nlma > 0) ? c->d_jw : nullptr;  // allocated only with projectors
  return a;
}
}  // namespace

bool step_orbital_applies(const sb200_ctx* c, int n_hamil) {
  return orbital_kernel_applies(c) && (c->orbital_variant >= 2) && n_hamil >= 1 && n_hamil <= STEP_MAX_NTERM;
}

// One launch for the whole Taylor step: psi_out = sum_n zc_n H^n psi (+ psi).
int launch_step_orbital(sb200_ctx* c, const double2* in, double2* out, const double2* zc, int n_hamil,
                        bool with_obs) {
  // dynamic shared memory: three orbital buffers and the projections, or (KB
  // tables staged) two orbital buffers, the projections and the pair tables
  constexpr size_t SMEM_MAX = 227 * 1024 - 2048;  // less the static arrays
  const size_t smem = 3 * (size_t)N * NP * sizeof(double2) + (size_t)ORB_MAX_NLMA * sizeof(double2);
  const PPInfo& pp = c->pp;
  const size_t smem_st = 2 * (size_t)N * NP * sizeof(double2) + (size_t)pp.nlma * sizeof(double2) +
                         (size_t)pp.npair * (sizeof(double2) + 4 * sizeof(double) + 2 * sizeof(int)) +
                         (size_t)pp.totpts * sizeof(int);
  const bool staged = (c->orbital_variant == 2 || c->orbital_variant == 4) && pp.nlma > 0 && pp.npair > 0 && pp.d_apj != nullptr &&
                      smem_st <= SMEM_MAX;
  static bool attr_set = false;
  if (!attr_set) {
    SB_CUDA(cudaFuncSetAttribute(k_step_orbital<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SB_CUDA(cudaFuncSetAttribute(k_step_orbital<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SB_CUDA(cudaFuncSetAttribute(k_step_orbital_st<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_MAX));
    SB_CUDA(cudaFuncSetAttribute(k_step_orbital_st<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_MAX));
    attr_set = true;
  }
  if (n_hamil < 1 || n_hamil > STEP_MAX_NTERM) return set_error(SB200_ERR_INVALID_ARG, "fused step: bad n_hamil");
  StepZC z;
  for (int i = 0; i < STEP_MAX_NTERM; ++i) z.v[i] = i < n_hamil ? zc[i] : make_double2(0.0, 0.0);
  const OrbArgs a = make_orb_args(c, zc[0], with_obs);
  if (c->orbital_variant == 4) {  // register-blocked form, when its tables fit
    const int r = launch_step_blk(c, in, out, a, z, n_hamil, with_obs);
    if (r != SB200_ERR_UNSUPPORTED) return r;
  }
  dim3 grid(c->orb.norb);
  if (staged) {
    StageArgs st;
    st.npair = pp.npair;
    st.pair_ph = pp.d_pair_ph;
    st.pair_uv = pp.d_pair_uv;
    st.pair_lma = pp.d_pair_lma;
    st.pair_pt = pp.d_pair_pt;
    st.apj = pp.d_apj;
    st.pmap2 = pp.d_pmap2;
    if (with_obs) k_step_orbital_st<true><<<grid, NTF, smem_st, c->stream>>>(in, out, a, st, z, n_hamil);
    else k_step_orbital_st<false><<<grid, NTF, smem_st, c->stream>>>(in, out, a, st, z, n_hamil);
    SB_LAUNCH_CHECK("k_step_orbital_st");
    return SB200_OK;
  }
  if (with_obs) k_step_orbital<true><<<grid, NTF, smem, c->stream>>>(in, out, a, z, n_hamil);
  else k_step_orbital<false><<<grid, NTF, smem, c->stream>>>(in, out, a, z, n_hamil);
  SB_LAUNCH_CHECK("k_step_orbital");
  return SB200_OK;
}

int launch_term_orbital(sb200_ctx* c, const HpsiLaunch& L, bool with_obs) {
  static bool attr_set = false, attr_set2 = false;
  const size_t smem = (size_t)N * NP * sizeof(double2) + (size_t)ORB_MAX_NLMA * sizeof(double2);
  const size_t smem2 = 3 * (size_t)ORB_BYTES + (size_t)ORB_MAX_NLMA * sizeof(double2);
  const bool persistent = c->orbital_variant == 1;
  if (!persistent && !attr_set) {
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  if (persistent && !attr_set2) {
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital_tma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital_tma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital_tma<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    SB_CUDA(cudaFuncSetAttribute(k_term_orbital_tma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    attr_set2 = true;
  }
  const OrbArgs a = make_orb_args(c, L.zc, with_obs);
  const double2* IN = (const double2*)L.in;
  double2* HOUT = (double2*)L.hout;
  if (persistent) {
    int sms = 148;
    SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    const int norb = c->orb.norb;
    const int g2 = norb < sms ? norb : sms;
    switch (L.mode) {
      case 1: k_term_orbital_tma<1><<<g2, NT2, smem2, c->stream>>>(IN, HOUT, L.out, a, norb, c->d_err); break;
      case 2: k_term_orbital_tma<2><<<g2, NT2, smem2, c->stream>>>(IN, HOUT, L.out, a, norb, c->d_err); break;
      case 3: k_term_orbital_tma<3><<<g2, NT2, smem2, c->stream>>>(IN, HOUT, L.out, a, norb, c->d_err); break;
      case 4: k_term_orbital_tma<4><<<g2, NT2, smem2, c->stream>>>(IN, HOUT, L.out, a, norb, c->d_err); break;
      default: return set_error(SB200_ERR_INVALID_ARG, "orbital kernel: unsupported mode");
    }
    SB_LAUNCH_CHECK("k_term_orbital_tma");
    return SB200_OK;
  }
  dim3 grid(c->orb.norb);
  switch (L.mode) {
    case 1: k_term_orbital<1><<<grid, NT, smem, c->stream>>>(IN, HOUT, L.out, a); break;
    case 2: k_term_orbital<2><<<grid, NT, smem, c->stream>>>(IN, HOUT, L.out, a); break;
    case 3: k_term_orbital<3><<<grid, NT, smem, c->stream>>>(IN, HOUT, L.out, a); break;
    case 4: k_term_orbital<4><<<grid, NT, smem, c->stream>>>(IN, HOUT, L.out, a); break;
    default: return set_error(SB200_ERR_INVALID_ARG, "orbital kernel: unsupported mode");
  }
  SB_LAUNCH_CHECK("k_term_orbital");
  return SB200_OK;
}

}  // namespace sb200
