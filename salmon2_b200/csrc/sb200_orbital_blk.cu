// sb200_orbital_blk.cu -- the fused Taylor step for periodic 16^3 orbitals
// with register blocking (default form of the periodic-bulk path).
//
// One CTA applies all n_hamil terms of taylor.f90:47-117 to one 16^3 orbital.
// Thread t owns a block of 2 (x) x 2 (y) x BZ (z) grid points: x = 2 bx + i,
// y = 2 by + j, z = BZ bz + l with (bx, by, bz) = (t % 8, (t / 8) % 8, t / 64),
// slot s = i + 2 j + 4 l; the CTA has 1024 / BZ threads (BZ = 2: 512, BZ = 4:
// 256).  Per term the thread keeps the values of h_{n-1} at its own points in
// registers and accumulates those of h_n in registers; only the 4-point halo
// of its block comes from shared memory: 8 x-neighbours per (y, z) row, 8
// y-neighbours per (x, z) column and 8 z-neighbours per (x, y) column, i.e.
// 12 (BZ = 2) or 10 (BZ = 4) loads of 16 bytes per point and term, against
// 24 for a point-per-thread sweep.
//
// Shared-memory layout of an orbital: index (z, y, x) = 256 z + 16 y + 8 (x % 2)
// + x / 2, i.e. each 16-point x row is stored as its 8 even then its 8 odd
// points.  The 8 threads of a quarter warp share (by, bz) and differ in bx, so
// every x, y or z neighbour load of a quarter warp touches 8 consecutive
// 16-byte words of one 128-byte row half: no bank conflicts.
//
// Tensor memory (TMEM, 256 columns of the SM's 512) holds per thread the
// Taylor accumulator psi_out of its 16 points (FP64 complex), the diagonal
// V_local + k_lap0 of its points and their KB point-map words, so neither
// registers nor shared memory carry them through the step.  The orbital
// buffer is updated in place between terms (three CTA barriers per term).
//
// Kleinman-Bylander term (nonlocal_potential.f90:351-382, pair form): the
// CTA's k-point tables -- phase exp(i (k+A).r), uV of the atom's projectors,
// and the shared-memory index of every flat sphere point, plus the
// point-major list of (point, atom) pairs -- are staged in shared memory once
// per step.  After each h_{n-1} is complete, one warp per atom computes its
// projections P_q = rinv_q sum_j uV_qj e^{i(k+A).r_j} h(r_j) (butterfly, all
// lanes get the sums) and then, for each of its sphere points, the
// contribution c_j = conj(e_j) sum_q uV_qj P_q into a per-point buffer.  The
// owner of a grid point adds the contributions of its pairs in atom (ilma)
// order.  The stencil arithmetic per point and neighbour pair is that of
// zstencil_typical_seq (zstencil_core/typical/seq.f90:65-122) with the
// coefficients folded: h += (-lapt/2)(t+ + t-) - i k_nabt (t+ - t-).
//
// After the last term (OBS), the observables of psi(t+dt) (sum |psi|^2, the
// forward-difference current sums of density_matrix.f90:465-530, the dipole
// moments of dip.f90:114-225 and the nonlocal current of
// density_matrix.f90:532-591) are reduced per orbital in a fixed order.
#include <cuda_runtime.h>

#include <cstdint>

#include "sb200_internal.cuh"
#include "sb200_orbital.cuh"
#include "sb200_tma.cuh"
#include "sb200_tmem.cuh"

namespace sb200 {
namespace {

constexpr int N = 16, NP = N * N, NPTS = N * NP;
constexpr uint32_t TMEM_COLS = 512;
// TMEM words (columns) per thread: psi_out 4 per point, diagonal 2 per point,
// point-map word 1 per point, then (warps that project one atom) 12 words per
// 32-point chunk of its sphere: the lane's uV of the atom's 4 projectors and
// its phase.  The NW / 4 warps of one lane quarter each use 2048 / NW of the
// 512 columns.
template <int BZ>
struct Blk {
  static constexpr int BT = 1024 / BZ;  // threads
  static constexpr int NW = BT / 32;    // warps
  static constexpr int NS = 4 * BZ;     // own points per thread
  static constexpr uint32_t TW_ACC = 0, TW_D = 4 * NS, TW_PM = 6 * NS, TW_KB = 7 * NS;
  static constexpr uint32_t TW_WARP = TMEM_COLS / (NW / 4);
  static constexpr int KB_CHUNKS = (int)(TW_WARP - TW_KB) / 12;  // sphere chunks a warp can keep
  static_assert(KB_CHUNKS >= 1, "TMEM words per thread");
};

// uV of the 4 projectors and the phase of one sphere point, kept in TMEM
__device__ __forceinline__ void kb_store(uint32_t taddr, const double (&u)[4], double2 e) {
  uint32_t w8[8], w4[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    w8[2 * q] = tmem::lo_word(u[q]);
    w8[2 * q + 1] = tmem::hi_word(u[q]);
  }
  w4[0] = tmem::lo_word(e.x);
  w4[1] = tmem::hi_word(e.x);
  w4[2] = tmem::lo_word(e.y);
  w4[3] = tmem::hi_word(e.y);
  tmem::st8(taddr, w8);
  tmem::st4(taddr + 8, w4);
}
__device__ __forceinline__ void kb_load(uint32_t taddr, double (&u)[4], double2& e) {
  uint32_t w8[8], w4[4];
  tmem::ld8(taddr, w8);
  tmem::ld4(taddr + 8, w4);
#pragma unroll
  for (int q = 0; q < 4; ++q) u[q] = tmem::as_double(w8[2 * q], w8[2 * q + 1]);
  e = make_double2(tmem::as_double(w4[0], w4[1]), tmem::as_double(w4[2], w4[3]));
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// h += A (tp + tm) - i B (tp - tm)  (A = -lapt/2, B = k_nabt of one direction and distance)
__device__ __forceinline__ void pair_acc(double2& h, const double2 tp, const double2 tm, const double A,
                                         const double B) {
  const double sx = tp.x + tm.x, sy = tp.y + tm.y, dx = tp.x - tm.x, dy = tp.y - tm.y;
  h.x = fma(A, sx, h.x);
  h.y = fma(A, sy, h.y);
  h.x = fma(B, dy, h.x);
  h.y = fma(-B, dx, h.y);
}

// Im(conj(c) t) weighted: the current sums of density_matrix.f90:465-530
__device__ __forceinline__ double cur_term(const double nab, const double2 c, const double2 t) {
  return nab * (c.x * t.y - c.y * t.x);
}

// Sum of NV doubles (NV = 2^m <= 32) over the 32 lanes of a warp, by
// reduce-scatter: at each level a lane keeps half of its live values and adds
// its partner's copy of them, so NV - 1 + (5 - m) shuffles replace the 5 NV of
// a butterfly per value.  Afterwards lane L holds the total of value
// L >> (5 - m) (fixed operation order: the result does not depend on timing).
template <int NV>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[NV], int lane) {
  static_assert(NV >= 1 && NV <= 32 && (NV & (NV - 1)) == 0, "NV");
#pragma unroll
  for (int lev = 0; lev < 5; ++lev) {
    const int off = 16 >> lev, n = NV >> lev;
    if (n > 1) {
      const bool upper = (lane & off) != 0;
#pragma unroll
      for (int i = 0; i < n / 2; ++i) {
        const double keep = upper ? v[n / 2 + i] : v[i];
        const double send = upper ? v[i] : v[n / 2 + i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
      }
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], off);
    }
  }
  return v[0];
}
template <int NV>
__device__ __forceinline__ int rs_lane(int k) {  // a lane holding value k after warp_reduce_scatter<NV>
  return k << (5 - (NV == 1 ? 0 : NV == 2 ? 1 : NV == 4 ? 2 : NV == 8 ? 3 : NV == 16 ? 4 : 5));
}

__device__ __forceinline__ int gidx(int x, int y, int z) { return (z << 8) | (y << 4) | x; }
__device__ __forceinline__ int sidx(int x, int y, int z) { return (z << 8) | (y << 4) | ((x & 1) << 3) | (x >> 1); }

// Projections of the orbital in shared memory and the KB contributions
// pc[pr] = conj(e) sum_q uV_q P_q of every (point, atom) pair pr, stored in
// point-major pair order so that each grid point's owner reads its pairs as
// one contiguous run; one warp per atom.  sap[fp] packs, for flat sphere
// point fp, its pair index (bits 12..30) and its shared-memory grid index
// (bits 0..11).  With `cached` (at most one atom per warp) each lane's uV and
// phase come from its TMEM words at tkb + 12 k (chunk k of 32 sphere points)
// instead of shared memory, which the gathers of both loops otherwise load
// twice per term.
template <int NW>
__device__ __forceinline__ void project_contrib(const double2* __restrict__ buf, const double2* __restrict__ sph,
                                                const double* __restrict__ suv, const int* __restrict__ sap,
                                                double2* __restrict__ pc, int TP, const int4* __restrict__ satm,
                                                const double* __restrict__ srinv, const OrbArgs& a, int warp,
                                                int lane, bool cached, uint32_t tkb) {
  for (int atom = warp; atom < a.natom; atom += NW) {
    const int4 at = satm[atom];
    const int start = at.x, m = at.y, lma0 = at.z, np = at.w;
    if (np == 0) continue;  // no projectors: no pairs
    const int nk = (m + 31) >> 5;
    double2 pq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) pq[q] = make_double2(0.0, 0.0);
    if (cached) {
      for (int k = 0; k < nk; ++k) {  // uniform over the warp (TMEM loads)
        double u[4];
        double2 e;
        kb_load(tkb + 12 * k, u, e);
        const int j = lane + 32 * k;
        if (j < m) {
          const double2 ev = cmul(e, buf[sap[start + j] & 4095]);
#pragma unroll
          for (int q = 0; q < 4; ++q) pq[q] = make_double2(fma(u[q], ev.x, pq[q].x), fma(u[q], ev.y, pq[q].y));
        }
      }
    } else {
#pragma unroll 3
      for (int j = lane; j < m; j += 32) {
        const int fp = start + j;
        const double2 ev = cmul(sph[fp], buf[sap[fp] & 4095]);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q < np) {
            const double u = suv[q * TP + fp];
            pq[q] = make_double2(fma(u, ev.x, pq[q].x), fma(u, ev.y, pq[q].y));
          }
      }
    }
    {  // sums over the warp, then every lane gets the four totals
      double v[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        v[2 * q] = pq[q].x;
        v[2 * q + 1] = pq[q].y;
      }
      const double r = warp_reduce_scatter<8>(v, lane);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        pq[q] = make_double2(__shfl_sync(0xffffffffu, r, rs_lane<8>(2 * q)),
                             __shfl_sync(0xffffffffu, r, rs_lane<8>(2 * q + 1)));
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double r = q < np ? srinv[lma0 + q] : 0.0;
      pq[q] = make_double2(r * pq[q].x, r * pq[q].y);
    }
    if (cached) {
      for (int k = 0; k < nk; ++k) {
        double u[4];
        double2 e;
        kb_load(tkb + 12 * k, u, e);
        const int j = lane + 32 * k;
        if (j < m) {
          double2 sp = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < 4; ++q) sp = make_double2(fma(u[q], pq[q].x, sp.x), fma(u[q], pq[q].y, sp.y));
          pc[sap[start + j] >> 12] = cmul(make_double2(e.x, -e.y), sp);
        }
      }
    } else {
#pragma unroll 3
      for (int j = lane; j < m; j += 32) {
        const int fp = start + j;
        double2 sp = make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q < np) {
            const double u = suv[q * TP + fp];
            sp = make_double2(fma(u, pq[q].x, sp.x), fma(u, pq[q].y, sp.y));
          }
        const double2 e = sph[fp];
        pc[sap[fp] >> 12] = cmul(make_double2(e.x, -e.y), sp);
      }
    }
  }
}

// Split form of the projections: two warps per atom (warp w takes atoms
// w / 2, w / 2 + NW / 2, ...; half w % 2 its sphere chunks k = w % 2, w % 2 + 2,
// ...), each leaving its partial sums of the atom's 4 complex projections in
// ppart[(2 atom + half) * 8 + v] (v = 2 q + re/im).  With `cached` the chunks'
// uV and phases come from the warp's TMEM words at tkb + 12 i (chunk hf + 2 i).
template <int NW>
__device__ __forceinline__ void project_half(const double2* __restrict__ buf, const double2* __restrict__ sph,
                                             const double* __restrict__ suv, const int* __restrict__ sap, int TP,
                                             const int4* __restrict__ satm, double* __restrict__ ppart,
                                             const OrbArgs& a, int warp, int lane, bool cached, uint32_t tkb) {
  const int hf = warp & 1;
  for (int atom = warp >> 1; atom < a.natom; atom += NW / 2) {
    const int4 at = satm[atom];
    const int start = at.x, m = at.y, np = at.w;
    if (np == 0) continue;  // uniform over the warp
    const int nk = (m + 31) >> 5;
    double2 pq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) pq[q] = make_double2(0.0, 0.0);
    if (cached) {
      for (int k = hf, i = 0; k < nk; k += 2, ++i) {
        double u[4];
        double2 e;
        kb_load(tkb + 12 * i, u, e);
        const int j = lane + 32 * k;
        if (j < m) {
          const double2 ev = cmul(e, buf[sap[start + j] & 4095]);
#pragma unroll
          for (int q = 0; q < 4; ++q) pq[q] = make_double2(fma(u[q], ev.x, pq[q].x), fma(u[q], ev.y, pq[q].y));
        }
      }
    } else {
      for (int k = hf; k < nk; k += 2) {
        const int j = lane + 32 * k;
        if (j < m) {
          const int fp = start + j;
          const double2 ev = cmul(sph[fp], buf[sap[fp] & 4095]);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < np) {
              const double u = suv[q * TP + fp];
              pq[q] = make_double2(fma(u, ev.x, pq[q].x), fma(u, ev.y, pq[q].y));
            }
        }
      }
    }
    double v[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      v[2 * q] = pq[q].x;
      v[2 * q + 1] = pq[q].y;
    }
    const double r = warp_reduce_scatter<8>(v, lane);  // lane 4 v holds value v
    if ((lane & 3) == 0) ppart[(2 * atom + hf) * 8 + (lane >> 2)] = r;
  }
}

// Split form of the contributions: P_q = rinv_q (half 0 + half 1) of each
// atom, then pc[pair] = conj(e) sum_q uV_q P_q for the warp's chunks (the same
// warp / chunk assignment as project_half).
template <int NW>
__device__ __forceinline__ void contrib_half(const double2* __restrict__ sph, const double* __restrict__ suv,
                                             const int* __restrict__ sap, double2* __restrict__ pc, int TP,
                                             const int4* __restrict__ satm, const double* __restrict__ srinv,
                                             const double* __restrict__ ppart, const OrbArgs& a, int warp,
                                             int lane, bool cached, uint32_t tkb) {
  const int hf = warp & 1;
  for (int atom = warp >> 1; atom < a.natom; atom += NW / 2) {
    const int4 at = satm[atom];
    const int start = at.x, m = at.y, lma0 = at.z, np = at.w;
    if (np == 0) continue;
    const int nk = (m + 31) >> 5;
    const double* p0 = ppart + 16 * atom;
    double2 pq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double r = q < np ? srinv[lma0 + q] : 0.0;
      pq[q] = make_double2(r * (p0[2 * q] + p0[8 + 2 * q]), r * (p0[2 * q + 1] + p0[9 + 2 * q]));
    }
    if (cached) {
      for (int k = hf, i = 0; k < nk; k += 2, ++i) {
        double u[4];
        double2 e;
        kb_load(tkb + 12 * i, u, e);
        const int j = lane + 32 * k;
        if (j < m) {
          double2 sp = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < 4; ++q) sp = make_double2(fma(u[q], pq[q].x, sp.x), fma(u[q], pq[q].y, sp.y));
          pc[sap[start + j] >> 12] = cmul(make_double2(e.x, -e.y), sp);
        }
      }
    } else {
      for (int k = hf; k < nk; k += 2) {
        const int j = lane + 32 * k;
        if (j < m) {
          const int fp = start + j;
          double2 sp = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < np) {
              const double u = suv[q * TP + fp];
              sp = make_double2(fma(u, pq[q].x, sp.x), fma(u, pq[q].y, sp.y));
            }
          const double2 e = sph[fp];
          pc[sap[fp] >> 12] = cmul(make_double2(e.x, -e.y), sp);
        }
      }
    }
  }
}

template <int BZ, bool OBS, bool SPLIT>
__global__ void __launch_bounds__(Blk<BZ>::BT, 1) k_step_blk(const double2* __restrict__ in,
                                                             double2* __restrict__ out, OrbArgs a, BlkArgs bk,
                                                             StepZC zc, int nterm) {
  constexpr int NW = Blk<BZ>::NW, NS = Blk<BZ>::NS;
  constexpr uint32_t TW_ACC = Blk<BZ>::TW_ACC, TW_D = Blk<BZ>::TW_D, TW_PM = Blk<BZ>::TW_PM;
  constexpr uint32_t TW_WARP = Blk<BZ>::TW_WARP, TW_KB = Blk<BZ>::TW_KB;
  extern __shared__ __align__(16) double2 smem[];
  const int T = a.totpts;
  const bool kb = a.nlma > 0;
  const int TP = bk.tpad;                   // T rounded up to a multiple of 4
  double2* buf = smem;                      // [4096] the orbital h_{n-1}, split-x layout
  double2* sph = buf + NPTS;                // [TP] phase of the CTA's k-point
  double* suv = (double*)(sph + TP);        // [4][TP] uV of the atom's projectors
  double* sr = suv + 4 * TP;                // [3][TP] coordinates of the sphere points
  double2* pc = (double2*)(sr + 3 * TP);    // [npair] KB contribution of each (point, atom) pair
  int* sap = (int*)(pc + bk.npair);         // [TP] pair index << 12 | shared-memory index of each sphere point
  int4* satm = (int4*)(sap + TP);           // [natom] first flat point, sphere size, first ilma, projectors
  double* srinv = (double*)(satm + (kb ? a.natom : 0));  // [nlma] rinv_uvu
  double* ppart = srinv + (kb ? a.nlma : 0);              // [natom][2][8] half projections (split form)
  __shared__ uint32_t s_tmem;
  __shared__ double kn[12];
  __shared__ double red[OBS_NQ][NW];
  __shared__ double jws[NW][3];
  __shared__ double nlred[OBS ? NW : 1][32];  // reduced nonlocal-current sums of each warp
  __shared__ __align__(8) uint64_t s_bar;             // completion of the table copies

  const int o = blockIdx.x, t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int bx = t & 7, by = (t >> 3) & 7, bz = t >> 6;
  const int z0 = BZ * bz;
  const int ik = o / a.nspin_no, ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;

  if (warp == 0) tmem::alloc(&s_tmem, TMEM_COLS);
  // the orbital of the CTA one wave of resident CTAs later, into L2
  if (t == 64 && bk.prefetch_ahead > 0 && o + bk.prefetch_ahead < (int)gridDim.x)
    tma::bulk_prefetch_l2(in + (long)(o + bk.prefetch_ahead) * a.npts, (unsigned)(a.npts * sizeof(double2)));
  if (t < 12) kn[t] = __ldg(kc + 4 + t);  // k_nabt(s, d) = kAc_d nab(s, d)
  if (kb && t == 32) {
    // the k-point's KB tables: bulk copies (no multicast) into shared memory,
    // completion counted on s_bar; they overlap the orbital load below
    tma::mbar_init(&s_bar, 1);
    tma::fence_barrier_init();
    const unsigned b_ph = 16u * T, b_uv = 32u * TP, b_r = 24u * TP, b_ap = 4u * TP;
    tma::mbar_arrive_expect_tx(&s_bar, b_ph + b_uv + b_r + b_ap);
    tma::bulk_load(sph, a.phase + (long)ik * T, b_ph, &s_bar);
    tma::bulk_load(suv, bk.uv4, b_uv, &s_bar);
    tma::bulk_load(sr, bk.r3, b_r, &s_bar);
    tma::bulk_load(sap, bk.sap, b_ap, &s_bar);
  }

  if (kb) {
    for (int i = t; i < a.natom; i += Blk<BZ>::BT)
      satm[i] = make_int4(__ldg(a.atom_start + i), __ldg(a.mps + i), __ldg(a.lma_start + i), __ldg(a.nproj + i));
    for (int i = t; i < a.nlma; i += Blk<BZ>::BT) srinv[i] = __ldg(a.rinv + i);
  }

  // psi -> registers and the shared orbital buffer
  const double2* src = in + (long)o * a.npts;
  double2 cv[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
    cv[s] = __ldg(src + gidx(x, y, z));
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
    buf[sidx(x, y, z)] = cv[s];
  }
  tmem::fence_before_sync();
  __syncthreads();
  tmem::fence_after_sync();
  const uint32_t tb = tmem::warp_addr(s_tmem, warp, (uint32_t)(warp >> 2) * TW_WARP);
  {  // diagonal V_local + k_lap0 and point-map words of the own points -> TMEM
    const double lap0 = __ldg(kc + 3);
    const double* vloc = a.vloc + (long)ispin * a.npts;
    uint32_t w[8];
#pragma unroll
    for (int hh = 0; hh < NS / 4; ++hh) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int s = 4 * hh + u;
        const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
        const double d = __ldg(vloc + gidx(x, y, z)) + lap0;
        w[2 * u] = tmem::lo_word(d);
        w[2 * u + 1] = tmem::hi_word(d);
      }
      tmem::st8(tb + TW_D + 8 * hh, w);
    }
#pragma unroll
    for (int hh = 0; hh < NS / 8; ++hh) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int s = 8 * hh + u;
        const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
        w[u] = kb ? (uint32_t)__ldg(bk.pmap2 + gidx(x, y, z)) : 0xffffffffu;
      }
      tmem::st8(tb + TW_PM + 8 * hh, w);
    }
  }
  // the tables have arrived (bounded wait; on expiry: flag, wait once more for
  // the copies in flight, skip the step, release TMEM)
  bool ok = true;
  if (kb) ok = tma::mbar_wait(&s_bar, 0);
  ok = __syncthreads_and(ok);
  if (!ok) {
    if (t == 0) {
      atomicExch(bk.err, 1);
      tma::mbar_wait(&s_bar, 0);
    }
    __syncthreads();
  }
  if (ok) {
  // KB cache: warp w < natom keeps its atom's uV and phases in TMEM for the step
  const bool kbc = kb && bk.kbcache != 0;
  const uint32_t tkb = tb + TW_KB;
  // (split form: warp w keeps chunks w % 2, w % 2 + 2, ... of atom w / 2)
  const int cw = SPLIT ? (warp >> 1) : warp, c0 = SPLIT ? (warp & 1) : 0, cs = SPLIT ? 2 : 1;
  if (kbc && cw < a.natom) {
    const int4 at = satm[cw];
    const int nk = (at.y + 31) >> 5;
    for (int k = c0, i = 0; k < nk; k += cs, ++i) {
      const int j = lane + 32 * k;
      double u[4] = {0.0, 0.0, 0.0, 0.0};
      double2 e = make_double2(0.0, 0.0);
      if (j < at.y) {
#pragma unroll
        for (int q = 0; q < 4; ++q) u[q] = suv[q * TP + at.x + j];
        e = sph[at.x + j];
      }
      kb_store(tkb + 12 * i, u, e);
    }
  }
  if (!SPLIT && kb) {
    project_contrib<NW>(buf, sph, suv, sap, pc, TP, satm, srinv, a, warp, lane, kbc, tkb);
    __syncthreads();
  }
  const int hm2 = (bx - 2) & 7, hm1 = (bx - 1) & 7, hp1 = (bx + 1) & 7, hp2 = (bx + 2) & 7;
  double2* odst = out + (long)o * a.npts;
  for (int nn = 0; nn < nterm; ++nn) {
    // split form: this warp's partial projections of h_{n-1}, before its stencil
    if (SPLIT && kb) project_half<NW>(buf, sph, suv, sap, TP, satm, ppart, a, warp, lane, kbc, tkb);
    double2 h[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) h[s] = make_double2(0.0, 0.0);
    // ---- x neighbours: per (y, z) row, x = 2 bx - 4 .. 2 bx + 5 ----
    {
      const double B1 = kn[0], B2 = kn[1], B3 = kn[2], B4 = kn[3];
      const double A1 = bk.mhl[0], A2 = bk.mhl[1], A3 = bk.mhl[2], A4 = bk.mhl[3];
#pragma unroll
      for (int r = 0; r < 2 * BZ; ++r) {
        const int j = r & 1, l = r >> 1;
        const double2* row = buf + ((z0 + l) << 8) + ((2 * by + j) << 4);
        const double2 vm4 = row[hm2], vm3 = row[8 + hm2], vm2 = row[hm1], vm1 = row[8 + hm1];
        const double2 vp2 = row[hp1], vp3 = row[8 + hp1], vp4 = row[hp2], vp5 = row[8 + hp2];
        const int s0 = 2 * j + 4 * l, s1 = s0 + 1;
        pair_acc(h[s0], cv[s1], vm1, A1, B1);
        pair_acc(h[s0], vp2, vm2, A2, B2);
        pair_acc(h[s0], vp3, vm3, A3, B3);
        pair_acc(h[s0], vp4, vm4, A4, B4);
        pair_acc(h[s1], vp2, cv[s0], A1, B1);
        pair_acc(h[s1], vp3, vm1, A2, B2);
        pair_acc(h[s1], vp4, vm2, A3, B3);
        pair_acc(h[s1], vp5, vm3, A4, B4);
      }
    }
    // ---- y neighbours: per (x, z) column, y = 2 by - 4 .. 2 by + 5 ----
    {
      const double B1 = kn[4], B2 = kn[5], B3 = kn[6], B4 = kn[7];
      const double A1 = bk.mhl[4], A2 = bk.mhl[5], A3 = bk.mhl[6], A4 = bk.mhl[7];
#pragma unroll
      for (int r = 0; r < 2 * BZ; ++r) {
        const int i = r & 1, l = r >> 1;
        const double2* col = buf + ((z0 + l) << 8) + (i << 3) + bx;
        const int y0 = 2 * by;
        const double2 vm4 = col[((y0 - 4) & 15) << 4], vm3 = col[((y0 - 3) & 15) << 4];
        const double2 vm2 = col[((y0 - 2) & 15) << 4], vm1 = col[((y0 - 1) & 15) << 4];
        const double2 vp2 = col[((y0 + 2) & 15) << 4], vp3 = col[((y0 + 3) & 15) << 4];
        const double2 vp4 = col[((y0 + 4) & 15) << 4], vp5 = col[((y0 + 5) & 15) << 4];
        const int s0 = i + 4 * l, s1 = s0 + 2;
        pair_acc(h[s0], cv[s1], vm1, A1, B1);
        pair_acc(h[s0], vp2, vm2, A2, B2);
        pair_acc(h[s0], vp3, vm3, A3, B3);
        pair_acc(h[s0], vp4, vm4, A4, B4);
        pair_acc(h[s1], vp2, cv[s0], A1, B1);
        pair_acc(h[s1], vp3, vm1, A2, B2);
        pair_acc(h[s1], vp4, vm2, A3, B3);
        pair_acc(h[s1], vp5, vm3, A4, B4);
      }
    }
    // ---- z neighbours: per (x, y) column, z = 4 bz - 4 .. 4 bz + 7 ----
    {
      const double Bz[4] = {kn[8], kn[9], kn[10], kn[11]};
      const double Az[4] = {bk.mhl[8], bk.mhl[9], bk.mhl[10], bk.mhl[11]};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = r & 1, j = r >> 1;
        const double2* col = buf + ((2 * by + j) << 4) + (i << 3) + bx;
        double2 zm[4], zp[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          zm[e] = col[((z0 - 4 + e) & 15) << 8];   // z offset e - 4
          zp[e] = col[((z0 + BZ + e) & 15) << 8];  // z offset BZ + e
        }
#pragma unroll
        for (int l = 0; l < BZ; ++l) {
          const int s = i + 2 * j + 4 * l;
#pragma unroll
          for (int d = 1; d <= 4; ++d) {
            const int ep = l + d, em = l - d;  // z offsets of the pair, -4 .. BZ + 3
            const double2 tp = ep < BZ ? cv[i + 2 * j + 4 * (ep % BZ)] : zp[(ep - BZ) & 3];
            const double2 tm = em >= 0 ? cv[i + 2 * j + 4 * (em % BZ)] : zm[(em + 4) & 3];
            pair_acc(h[s], tp, tm, Az[d - 1], Bz[d - 1]);
          }
        }
      }
    }
    if (SPLIT) {
      // every read of h_{n-1} and every partial projection is done; the
      // contributions of the finished projections, then the buffer is free
      __syncthreads();
      if (kb) {
        contrib_half<NW>(sph, suv, sap, pc, TP, satm, srinv, ppart, a, warp, lane, kbc, tkb);
        __syncthreads();
      }
    }
    // ---- diagonal, KB contributions, Taylor update (taylor.f90:47-117) ----
    const bool last = nn == nterm - 1;
    // zc(nn + 1) by constant indices (no local-memory copy of the argument)
    double2 zn = zc.v[0];
#pragma unroll
    for (int q = 1; q < STEP_MAX_NTERM; ++q)
      if (nn == q) zn = zc.v[q];
    uint32_t pw[NS];
#pragma unroll
    for (int hh = 0; hh < NS / 8; ++hh) {
      uint32_t w8[8];
      tmem::ld8(tb + TW_PM + 8 * hh, w8);
#pragma unroll
      for (int u = 0; u < 8; ++u) pw[8 * hh + u] = w8[u];
    }
#pragma unroll
    for (int q4 = 0; q4 < NS / 4; ++q4) {
      uint32_t dw[8], aw[16];
      tmem::ld8(tb + TW_D + 8 * q4, dw);
      if (nn > 0) tmem::ld16(tb + TW_ACC + 16 * q4, aw);
      double2 c1[4];  // each point's first pair, loaded before any is used
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int pm = (int)pw[4 * q4 + u];
        c1[u] = pm >= 0 ? pc[pm >> 8] : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int s = 4 * q4 + u;
        const double dg = tmem::as_double(dw[2 * u], dw[2 * u + 1]);
        double2 hs = make_double2(fma(dg, cv[s].x, h[s].x), fma(dg, cv[s].y, h[s].y));
        const int pm = (int)pw[s];
        if (pm >= 0) {  // the point's pairs, atoms in ilma order
          hs = make_double2(hs.x + c1[u].x, hs.y + c1[u].y);
          const int p1 = (pm >> 8) + (pm & 255);
          for (int pr = (pm >> 8) + 1; pr < p1; ++pr) {
            const double2 cc = pc[pr];
            hs = make_double2(hs.x + cc.x, hs.y + cc.y);
          }
        }
        h[s] = hs;
        // psi_out = psi + zc_1 h_1 (first term), psi_out + zc_n h_n (later terms)
        const double2 ao = nn == 0 ? cv[s]
                                   : make_double2(tmem::as_double(aw[4 * u], aw[4 * u + 1]),
                                                  tmem::as_double(aw[4 * u + 2], aw[4 * u + 3]));
        const double2 an = make_double2(fma(zn.x, hs.x, fma(-zn.y, hs.y, ao.x)),
                                        fma(zn.x, hs.y, fma(zn.y, hs.x, ao.y)));
        if (last) {
          const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
          odst[gidx(x, y, z)] = an;
          if (OBS) {
            cv[s] = an;  // the new orbital, for the observables
            if (SPLIT) buf[sidx(x, y, z)] = an;
          }
        } else {
          if (SPLIT) {  // h_n into the (no longer read) buffer
            const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
            buf[sidx(x, y, z)] = hs;
            cv[s] = hs;
          }
          aw[4 * u] = tmem::lo_word(an.x);
          aw[4 * u + 1] = tmem::hi_word(an.x);
          aw[4 * u + 2] = tmem::lo_word(an.y);
          aw[4 * u + 3] = tmem::hi_word(an.y);
        }
      }
      if (!last) tmem::st16(tb + TW_ACC + 16 * q4, aw);
    }
    if (SPLIT) {
      if (last && !OBS) break;
      __syncthreads();  // h_n (or psi(t + dt)) complete in the buffer
      if (last) break;
      continue;
    }
    if (last) break;
    __syncthreads();  // every read of h_{n-1} and of the contributions is done
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
      buf[sidx(x, y, z)] = h[s];
      cv[s] = h[s];
    }
    __syncthreads();
    if (kb) {
      project_contrib<NW>(buf, sph, suv, sap, pc, TP, satm, srinv, a, warp, lane, kbc, tkb);
      __syncthreads();
    }
  }
  if (OBS) {
    if (!SPLIT) {
      __syncthreads();  // the last term's reads of h_{n-1} are done
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int x = 2 * bx + (s & 1), y = 2 * by + ((s >> 1) & 1), z = z0 + (s >> 2);
        buf[sidx(x, y, z)] = cv[s];
      }
      __syncthreads();
    }
    double q[OBS_NQ];
#pragma unroll
    for (int i = 0; i < OBS_NQ; ++i) q[i] = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double r2 = cv[s].x * cv[s].x + cv[s].y * cv[s].y;
      q[0] += r2;
      q[4] += ((double)(2 * bx + (s & 1)) + a.off[0]) * r2;
      q[5] += ((double)(2 * by + ((s >> 1) & 1)) + a.off[1]) * r2;
      q[6] += ((double)(z0 + (s >> 2)) + a.off[2]) * r2;
    }
#pragma unroll
    for (int r = 0; r < 2 * BZ; ++r) {  // x: t(+1 .. +4)
      const int j = r & 1, l = r >> 1;
      const double2* row = buf + ((z0 + l) << 8) + ((2 * by + j) << 4);
      const double2 vp2 = row[hp1], vp3 = row[8 + hp1], vp4 = row[hp2], vp5 = row[8 + hp2];
      const int s0 = 2 * j + 4 * l, s1 = s0 + 1;
      q[1] += cur_term(a.nab[0], cv[s0], cv[s1]) + cur_term(a.nab[1], cv[s0], vp2) +
              cur_term(a.nab[2], cv[s0], vp3) + cur_term(a.nab[3], cv[s0], vp4);
      q[1] += cur_term(a.nab[0], cv[s1], vp2) + cur_term(a.nab[1], cv[s1], vp3) +
              cur_term(a.nab[2], cv[s1], vp4) + cur_term(a.nab[3], cv[s1], vp5);
    }
#pragma unroll
    for (int r = 0; r < 2 * BZ; ++r) {  // y
      const int i = r & 1, l = r >> 1;
      const double2* col = buf + ((z0 + l) << 8) + (i << 3) + bx;
      const int y0 = 2 * by;
      const double2 vp2 = col[((y0 + 2) & 15) << 4], vp3 = col[((y0 + 3) & 15) << 4];
      const double2 vp4 = col[((y0 + 4) & 15) << 4], vp5 = col[((y0 + 5) & 15) << 4];
      const int s0 = i + 4 * l, s1 = s0 + 2;
      q[2] += cur_term(a.nab[4], cv[s0], cv[s1]) + cur_term(a.nab[5], cv[s0], vp2) +
              cur_term(a.nab[6], cv[s0], vp3) + cur_term(a.nab[7], cv[s0], vp4);
      q[2] += cur_term(a.nab[4], cv[s1], vp2) + cur_term(a.nab[5], cv[s1], vp3) +
              cur_term(a.nab[6], cv[s1], vp4) + cur_term(a.nab[7], cv[s1], vp5);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {  // z
      const int i = r & 1, j = r >> 1;
      const double2* col = buf + ((2 * by + j) << 4) + (i << 3) + bx;
      double2 zp[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) zp[e] = col[((z0 + BZ + e) & 15) << 8];
#pragma unroll
      for (int l = 0; l < BZ; ++l) {
        const int s = i + 2 * j + 4 * l;
#pragma unroll
        for (int d = 1; d <= 4; ++d) {
          const int ep = l + d;
          const double2 tp = ep < BZ ? cv[i + 2 * j + 4 * (ep % BZ)] : zp[(ep - BZ) & 3];
          q[3] += cur_term(a.nab[8 + d - 1], cv[s], tp);
        }
      }
    }
    {
      static_assert(OBS_NQ <= 8, "local sums");
      double v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = i < OBS_NQ ? q[i] : 0.0;
      const double r = warp_reduce_scatter<8>(v, lane);
      const int k = lane >> 2;  // rs_lane<8>(k) = 4 k
      if ((lane & 3) == 0 && k < OBS_NQ) red[k][warp] = r;
    }
    // nonlocal current (density_matrix.f90:532-591): one warp per atom, or two
    // per atom in the split form (their sums combined in warp order)
    double jx = 0.0, jy = 0.0, jz = 0.0;
    // chunk k of the atom's sphere (TMEM cache word i) into v: v[2c], v[2c + 1] =
    // <beta_q|psi> (c = q < 4) and <r_d beta_q|psi> (c = 4 + 3 q + d)
    auto nl_chunk = [&](double (&v)[32], int start, int m, int np, int k, int i) {
      const int j = lane + 32 * k;
      double uc[4];
      double2 e;
      if (kbc) kb_load(tkb + 12 * i, uc, e);
      if (j >= m) return;
      const int fp = start + j;
      if (!kbc) {
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) uc[qq] = suv[qq * TP + fp];
        e = sph[fp];
      }
      const double2 ev = cmul(e, buf[sap[fp] & 4095]);
      const double r0 = sr[fp], r1 = sr[TP + fp], r2 = sr[2 * TP + fp];
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        if (qq < np) {
          const double u = uc[qq];
          const double tx = u * ev.x, ty = u * ev.y;
          v[2 * qq] += tx;
          v[2 * qq + 1] += ty;
          v[8 + 6 * qq] = fma(r0, tx, v[8 + 6 * qq]);
          v[9 + 6 * qq] = fma(r0, ty, v[9 + 6 * qq]);
          v[10 + 6 * qq] = fma(r1, tx, v[10 + 6 * qq]);
          v[11 + 6 * qq] = fma(r1, ty, v[11 + 6 * qq]);
          v[12 + 6 * qq] = fma(r2, tx, v[12 + 6 * qq]);
          v[13 + 6 * qq] = fma(r2, ty, v[13 + 6 * qq]);
        }
      }
    };
    // J contribution of one atom from its reduced sums s0 (+ s1, the other half)
    auto nl_atom = [&](const double* s0, const double* s1, int lma0, int np) {
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        if (qq < np) {
          auto g = [&](int i) { return s1 ? s0[i] + s1[i] : s0[i]; };
          const double rv = srinv[lma0 + qq];
          const double usx = rv * g(2 * qq), usy = rv * g(2 * qq + 1);
          const int b = 8 + 6 * qq;
          jx += g(b) * usy - g(b + 1) * usx;
          jy += g(b + 2) * usy - g(b + 3) * usx;
          jz += g(b + 4) * usy - g(b + 5) * usx;
        }
      }
    };
    if (kb && SPLIT) {
      const int rounds = (a.natom + NW / 2 - 1) / (NW / 2);
      for (int rd = 0; rd < rounds; ++rd) {  // uniform over the CTA
        const int atom = (warp >> 1) + rd * (NW / 2);
        const int4 at = atom < a.natom ? satm[atom] : make_int4(0, 0, 0, 0);
        double v[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 0.0;
        if (at.w > 0) {
          const int nk = (at.y + 31) >> 5;
          for (int k = warp & 1, i = 0; k < nk; k += 2, ++i) nl_chunk(v, at.x, at.y, at.w, k, i);
        }
        const double r = warp_reduce_scatter<32>(v, lane);  // lane L holds value L
        nlred[warp][lane] = r;
        __syncthreads();
        if ((warp & 1) == 0 && lane == 0 && at.w > 0) nl_atom(nlred[warp], nlred[warp + 1], at.z, at.w);
        __syncthreads();
      }
    } else if (kb) {
      for (int atom = warp; atom < a.natom; atom += NW) {
        const int4 at = satm[atom];
        const int start = at.x, m = at.y, lma0 = at.z, np = at.w;
        if (np == 0) continue;
        double v[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 0.0;
        const int nk = (m + 31) >> 5;
        for (int k = 0; k < nk; ++k) nl_chunk(v, start, m, np, k, k);
        const double r = warp_reduce_scatter<32>(v, lane);  // lane L holds value L
        nlred[warp][lane] = r;
        __syncwarp();
        if (lane == 0) nl_atom(nlred[warp], nullptr, lma0, np);
        __syncwarp();
      }
    }
    if (lane == 0) {
      jws[warp][0] = jx;
      jws[warp][1] = jy;
      jws[warp][2] = jz;
    }
    __syncthreads();
    if (t < OBS_NQ) {
      double sum = 0.0;
      for (int w = 0; w < NW; ++w) sum += red[t][w];
      a.obs[(long)o * OBS_NQ + t] = sum;
    } else if (t >= 32 && t < 35 && a.jw != nullptr) {  // no nonlocal current without projectors
      double sum = 0.0;
      for (int w = 0; w < NW; ++w) sum += jws[w][t - 32];
      a.jw[3L * o + (t - 32)] = sum;
    }
  }
  }  // ok
  tmem::fence_before_sync();
  __syncthreads();
  tmem::fence_after_sync();
  if (warp == 0) tmem::dealloc(s_tmem, TMEM_COLS);
}

}  // namespace

// Host-built tables of the blocked fused step, in its shared-memory layout
// (k-independent; the phases come per k from the context's phase table):
// uV of each flat sphere point for the atom's projectors [4][tpad] (zero past
// the atom's count), coordinates [3][tpad], and (pair index << 12) | the
// split-x shared-memory index of its grid point [tpad].  Only for 16^3 grids
// with the (point, atom) pair form and fewer than 2^19 pairs.
int blk_build_tables(sb200_ctx* c, const std::vector<int>& pt_lin, const std::vector<int>& apj,
                     const std::vector<double>& uv_lma, const std::vector<double>& pt_r,
                     const std::vector<int>& atom_start, const std::vector<int>& mps,
                     const std::vector<int>& lma_start, const std::vector<int>& nproj) {
  PPInfo& p = c->pp;
  const GridInfo& g = c->g;
  if (!(g.nx == N && g.ny == N && g.nz == N) || p.npair <= 0 || p.npair >= (1 << 19) || p.nprojmax > 4)
    return SB200_OK;
  const int T = p.totpts, TP = (T + 3) & ~3;
  std::vector<double> uv4(4 * (size_t)TP, 0.0), r3(3 * (size_t)TP, 0.0);
  std::vector<int> sap(TP, 0);
  for (size_t at = 0; at < atom_start.size(); ++at)
    for (int j = 0; j < mps[at]; ++j) {
      const int fp = atom_start[at] + j;
      for (int q = 0; q < nproj[at] && q < 4; ++q) uv4[(size_t)q * TP + fp] = uv_lma[(size_t)(lma_start[at] + q) * p.nps + j];
      for (int d = 0; d < 3; ++d) r3[(size_t)d * TP + fp] = pt_r[3 * (size_t)fp + d];
      const int q = pt_lin[fp];
      const int x = q & 15, y = (q >> 4) & 15, z = q >> 8;
      sap[fp] = ((apj[fp] & 0x7ffff) << 12) | (z << 8) | (y << 4) | ((x & 1) << 3) | (x >> 1);
    }
  int r = dalloc(&p.d_blk_uv, uv4.size());
  if (r == SB200_OK) r = dalloc(&p.d_blk_r, r3.size());
  if (r == SB200_OK) r = dalloc(&p.d_blk_sap, sap.size());
  if (r != SB200_OK) return r;
  SB_CUDA(cudaMemcpy(p.d_blk_uv, uv4.data(), uv4.size() * sizeof(double), cudaMemcpyHostToDevice));
  SB_CUDA(cudaMemcpy(p.d_blk_r, r3.data(), r3.size() * sizeof(double), cudaMemcpyHostToDevice));
  SB_CUDA(cudaMemcpy(p.d_blk_sap, sap.data(), sap.size() * sizeof(int), cudaMemcpyHostToDevice));
  SB_CUDA(cudaDeviceSynchronize());  // landed before the context's (non-blocking) stream reads them
  p.blk_tpad = TP;
  return SB200_OK;
}

// Shared memory of the blocked fused step for the context's KB tables (bytes),
// or 0 when the form does not apply.
size_t step_blk_smem(const sb200_ctx* c) {
  const PPInfo& pp = c->pp;
  const size_t T = pp.nlma > 0 ? (size_t)pp.totpts : 0;
  const size_t npair = pp.nlma > 0 ? (size_t)pp.npair : 0;
  if (pp.nlma > 0 && (pp.npair <= 0 || pp.d_pmap2 == nullptr || pp.d_blk_sap == nullptr))
    return 0;  // no (point, atom) pair form, or no staged tables (blk_build_tables)
  const size_t TP = pp.nlma > 0 ? (size_t)pp.blk_tpad : 0;
  (void)T;
  const size_t natom = pp.nlma > 0 ? (size_t)pp.natom : 0, nlma = pp.nlma > 0 ? (size_t)pp.nlma : 0;
  return (size_t)NPTS * sizeof(double2) + TP * (sizeof(double2) + 7 * sizeof(double) + sizeof(int)) +
         npair * sizeof(double2) + natom * sizeof(int4) + nlma * sizeof(double) + natom * 16 * sizeof(double);
}

int launch_step_blk(sb200_ctx* c, const double2* in, double2* out, const OrbArgs& a, const StepZC& z, int n_hamil,
                    bool with_obs) {
  const size_t smem = step_blk_smem(c);
  if (smem == 0) return SB200_ERR_UNSUPPORTED;
  // per instantiation: the dynamic shared memory it may take next to its static arrays
  static size_t cap[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (cap[0] == 0) {
    const void* fns[8] = {(const void*)k_step_blk<2, false, false>, (const void*)k_step_blk<2, true, false>,
                          (const void*)k_step_blk<4, false, false>, (const void*)k_step_blk<4, true, false>,
                          (const void*)k_step_blk<2, false, true>,  (const void*)k_step_blk<2, true, true>,
                          (const void*)k_step_blk<4, false, true>,  (const void*)k_step_blk<4, true, true>};
    int optin = 0;
    SB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    for (int i = 0; i < 8; ++i) {
      cudaFuncAttributes fa;
      SB_CUDA(cudaFuncGetAttributes(&fa, fns[i]));
      const size_t ci = (size_t)optin - fa.sharedSizeBytes;
      SB_CUDA(cudaFuncSetAttribute(fns[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ci));
      cap[i] = ci;
    }
  }
  const bool split = c->blk_split != 0;
  const int which = (split ? 4 : 0) + (c->blk_depth == 4 ? 2 : 0) + (with_obs ? 1 : 0);
  if (smem > cap[which]) return SB200_ERR_UNSUPPORTED;
  BlkArgs bk;
  for (int i = 0; i < 12; ++i) bk.mhl[i] = -0.5 * c->g.coef_lap[i];
  bk.npair = c->pp.nlma > 0 ? c->pp.npair : 0;
  bk.pmap2 = c->pp.d_pmap2;
  bk.tpad = c->pp.blk_tpad;
  bk.uv4 = c->pp.d_blk_uv;
  bk.r3 = c->pp.d_blk_r;
  bk.sap = c->pp.d_blk_sap;
  bk.err = c->d_err;
  {  // TMEM KB cache: at most one atom per warp (per warp pair in the split form) and
     // every sphere chunk of the warp within its TMEM words
    const int nw = c->blk_depth == 4 ? Blk<4>::NW : Blk<2>::NW;
    const int chunks = c->blk_depth == 4 ? Blk<4>::KB_CHUNKS : Blk<2>::KB_CHUNKS;
    const int nk = (c->pp.nps + 31) / 32;
    bk.kbcache = (c->pp.nlma > 0 && (split ? (c->pp.natom <= nw / 2 && (nk + 1) / 2 <= chunks)
                                           : (c->pp.natom <= nw && nk <= chunks)))
                     ? 1
                     : 0;
  }
  {  // one wave of resident CTAs (one per SM) ahead, unless switched off
    int nsm = 0;
    SB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    bk.prefetch_ahead = c->blk_prefetch ? nsm : 0;
  }
  dim3 grid(c->orb.norb);
#define SB_BLK_LAUNCH(BZ, OBS, SPLIT) \
  k_step_blk<BZ, OBS, SPLIT><<<grid, Blk<BZ>::BT, smem, c->stream>>>(in, out, a, bk, z, n_hamil)
  switch (which) {
    case 0: SB_BLK_LAUNCH(2, false, false); break;
    case 1: SB_BLK_LAUNCH(2, true, false); break;
    case 2: SB_BLK_LAUNCH(4, false, false); break;
    case 3: SB_BLK_LAUNCH(4, true, false); break;
    case 4: SB_BLK_LAUNCH(2, false, true); break;
    case 5: SB_BLK_LAUNCH(2, true, true); break;
    case 6: SB_BLK_LAUNCH(4, false, true); break;
    default: SB_BLK_LAUNCH(4, true, true); break;
  }
#undef SB_BLK_LAUNCH
  SB_LAUNCH_CHECK("k_step_blk");
  return SB200_OK;
}

}  // namespace sb200
