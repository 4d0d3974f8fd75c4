// sb200_tiled_body.cuh -- the tiled 2.5-D hpsi sweep as a device function,
// shared by the per-system kernel (sb200_stencil.cu) and the batched
// persistent kernel (sb200_batch.cu).  See sb200_stencil.cu for the design.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "sb200_internal.cuh"
#include "sb200_stencil.cuh"

// resident CTAs per SM the tiled kernel is compiled for (register budget):
// FP64 stencils keep 2 (no spills), FP32 stencils fit 3
#ifndef SB200_TILED_MINB64
#define SB200_TILED_MINB64 2
#endif
#ifndef SB200_TILED_MINB32
#define SB200_TILED_MINB32 3
#endif

namespace sb200 {
namespace tiled {

template <typename R>
struct Cx;
template <>
struct Cx<double> {
  using T = double2;
  static __device__ __forceinline__ T make(double x, double y) { return make_double2(x, y); }
};
template <>
struct Cx<float> {
  using T = float2;
  static __device__ __forceinline__ T make(float x, float y) { return make_float2(x, y); }
};

template <typename T>
__device__ __forceinline__ T cadd(T a, T b) {
  T r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename T>
__device__ __forceinline__ T csub(T a, T b) {
  T r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
template <typename T, typename R>
__device__ __forceinline__ T cscal(R s, T a) {
  T r;
  r.x = s * a.x;
  r.y = s * a.y;
  return r;
}
template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// Packed FP32 forms (sm_100 f32x2 instructions): one instruction per complex
// add / scale / fused multiply-add instead of two; every rounding is the
// scalar one (round to nearest per component).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
__device__ __forceinline__ float2 cscal(float s, float2 a) { return __fmul2_rn(make_float2(s, s), a); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}

// acc + l x (fused per component)
__device__ __forceinline__ double2 cfma(double l, double2 x, double2 acc) {
  return make_double2(fma(l, x.x, acc.x), fma(l, x.y, acc.y));
}
__device__ __forceinline__ float2 cfma(float l, float2 x, float2 acc) {
  return __ffma2_rn(make_float2(l, l), x, acc);
}

// vl c + lap0 c - v / 2: the local-potential, k_lap0 and Laplacian part of
// the stencil value (zstencil_typical_seq, seq.f90:112-118)
__device__ __forceinline__ double2 hcore(double vl, double lap0, double2 c, double2 v) {
  return make_double2(fma(-0.5, v.x, fma(vl, c.x, lap0 * c.x)), fma(-0.5, v.y, fma(vl, c.y, lap0 * c.y)));
}
__device__ __forceinline__ float2 hcore(float vl, float lap0, float2 c, float2 v) {
  return __ffma2_rn(make_float2(-0.5f, -0.5f), v, __ffma2_rn(make_float2(vl, vl), c, cscal(lap0, c)));
}

// KB term of one point in the (point, atom) pair form: for each atom whose
// sphere holds the point, conj(exp(i (k+A).r)) sum_q uV_q P(lma0 + q)
// (the zekr_uV of nonlocal_potential.f90:368-375 factored into the point's
// phase and the projectors' uV); pairs two at a time with their loads issued
// together.  P: this orbital's projections (shared or global memory).
template <typename R, typename C2>
__device__ __forceinline__ C2 kb_pairs(C2 h, int pm, const double2* __restrict__ P, const TiledArgs& a, int ik) {
  const double2* ph = a.pair_ph + (a.phase_per_k ? (long)ik * a.npair : 0L);
  const int p0 = pm >> 8, p1 = p0 + (pm & 255);
  for (int pr = p0; pr < p1; pr += 2) {
    int lm[2];
    double2 u01[2], u23[2], e[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int pp = min(pr + i, p1 - 1);
      lm[i] = __ldg(a.pair_lma + pp);
      u01[i] = __ldg((const double2*)(a.pair_uv + 4L * pp));
      u23[i] = __ldg((const double2*)(a.pair_uv + 4L * pp + 2));
      e[i] = __ldg(ph + pp);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (pr + i < p1) {
        const int l0 = lm[i] & 0xffffff, np = lm[i] >> 24;
        const double uq[4] = {u01[i].x, u01[i].y, u23[i].x, u23[i].y};
        C2 sp = Cx<R>::make(0, 0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q < np) {
            const double2 pv = P[l0 + q];
            sp = cfma((R)uq[q], Cx<R>::make((R)pv.x, (R)pv.y), sp);
          }
        h = cadd(h, cmul(Cx<R>::make((R)e[i].x, -(R)e[i].y), sp));
      }
    }
  }
  return h;
}

// The first (point, atom) pair of a point, loaded one plane ahead by the
// tensor-copy sweep (nearly every point inside a sphere has exactly one pair,
// so the scatter's dependent loads leave the critical path).  The weights and
// the conjugate phase are kept in the stencil's type: the same values
// kb_pairs converts at use.
template <typename R>
struct Pair1 {
  int lm;  // pair_lma of the pair (0: no pair)
  R u[4];
  R ex, ey;
};

template <typename R>
__device__ __forceinline__ void load_pair1(Pair1<R>& f, int pm, const TiledArgs& a, const double2* __restrict__ ph) {
  f.lm = 0;
  if (pm < 0 || (pm & 255) == 0) return;
  const int p0 = pm >> 8;
  f.lm = __ldg(a.pair_lma + p0);
  const double2 u01 = __ldg((const double2*)(a.pair_uv + 4L * p0));
  const double2 u23 = __ldg((const double2*)(a.pair_uv + 4L * p0 + 2));
  const double2 e = __ldg(ph + p0);
  f.u[0] = (R)u01.x;
  f.u[1] = (R)u01.y;
  f.u[2] = (R)u23.x;
  f.u[3] = (R)u23.y;
  f.ex = (R)e.x;
  f.ey = -(R)e.y;
}

// kb_pairs with its first pair taken from f (loaded ahead); the others, in the
// same order, as kb_pairs loads them: the same sums, bit for bit
template <typename R, typename C2 = typename Cx<R>::T>
__device__ __forceinline__ C2 kb_pairs_ahead(C2 h, int pm, const double2* __restrict__ P, const TiledArgs& a,
                                             int ik, const Pair1<R>& f) {
  const int p0 = pm >> 8, p1 = p0 + (pm & 255);
  if (p1 <= p0) return h;
  {
    const int l0 = f.lm & 0xffffff, np = f.lm >> 24;
    C2 sp = Cx<R>::make(0, 0);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (q < np) {
        const double2 pv = P[l0 + q];
        sp = cfma(f.u[q], Cx<R>::make((R)pv.x, (R)pv.y), sp);
      }
    h = cadd(h, cmul(Cx<R>::make(f.ex, f.ey), sp));
  }
  if (p1 > p0 + 1) h = kb_pairs<R>(h, ((p0 + 1) << 8) | (p1 - p0 - 1), P, a, ik);
  return h;
}

// wrap (periodic) or test (Dirichlet) a coordinate that may be up to 4 outside
__device__ __forceinline__ int wrapc(int q, int n, int periodic, bool& ok) {
  if (periodic) {
    q = q < 0 ? q + n : (q >= n ? q - n : q);
    ok = true;
  } else {
    ok = (q >= 0) && (q < n);
  }
  return q;
}

template <int MODE>
struct ModeT {
  using R = typename std::conditional<(MODE >= 6), float, double>::type;
  static constexpr bool store_h = (MODE <= 2) || (MODE >= 5 && MODE <= 7);
  static constexpr bool h32 = (MODE >= 5);  // h stored as complex64
};

// GRAD = false drops the Bloch gradient terms, which vanish identically on
// isolated grids (k + A = 0).
template <int TX, int TY, bool FULL, int MODE, bool GRAD = true>
__device__ __forceinline__ void tiled_body(const typename Cx<typename ModeT<MODE>::R>::T* __restrict__ in,
                                           void* __restrict__ hout, double2* __restrict__ acc,
                                           float2* __restrict__ d32, const TiledArgs& a, const int bx,
                                           const int by, const int bz) {
  using R = typename ModeT<MODE>::R;
  using C2 = typename Cx<R>::T;
  constexpr int HX = FULL ? 0 : ND;                 // halo width in shared memory
  constexpr int SX = TX + 2 * HX, SY = TY + 2 * HX;  // staged plane extents
  constexpr int NT = TX * TY;
  constexpr int NH0 = (SX * SY - NT + NT - 1) / NT;  // halo cells per thread
  constexpr int NH = NH0 > 0 ? NH0 : 1;
  constexpr int HXD = HX > 0 ? HX : 1;              // divisor guard for the full-plane case
  __shared__ C2 plane[2][SY * SX];

  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int ntx = (a.nx + TX - 1) / TX;
  const int x0 = (bx % ntx) * TX, y0 = (bx / ntx) * TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool active = (x < a.nx) && (y < a.ny);
  const int zc0 = by * a.zchunk;
  const int zc1 = min(a.nz, zc0 + a.zchunk);
  const int o = bz;
  const long sz = (long)a.nx * a.ny;
  const C2* src = in + (long)o * a.npts;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  // k+A factored out of the gradient: w_d = kAc_d * sum_s nab_s (t+ - t-)
  const R kx = (R)kc[0], ky = (R)kc[1], kz = (R)kc[2], lap0 = (R)kc[3];
  const int ctr = (ty + HX) * SX + (tx + HX);
  const long pxy = (long)y * a.nx + x;
  // column value at any plane index (prefetches run up to 7 planes past the
  // chunk): periodic wrap by repeated add / subtract, no integer division
  auto colval = [&](int z) -> C2 {
    int zz = z;
    bool ok = true;
    if (a.periodic) {
      while (zz < 0) zz += a.nz;
      while (zz >= a.nz) zz -= a.nz;
    } else {
      ok = (z >= 0) && (z < a.nz);
    }
    return (ok && active) ? __ldg(src + (long)zz * sz + pxy) : Cx<R>::make(0, 0);
  };
  // halo cells owned by this thread (fixed over the sweep): shared-memory slot
  // and in-plane offset, or -1 when the cell lies outside a Dirichlet grid
  int hslot[NH];
  long hoff[NH];
#pragma unroll
  for (int k = 0; k < NH; ++k) {
    hslot[k] = -1;
    hoff[k] = -1;
    if (FULL) continue;
    // enumerate the halo ring in a fixed order and take every NT-th cell
    const int idx = threadIdx.x + k * NT;
    if (idx >= SX * SY - NT) continue;
    int c = idx;  // c-th cell of the ring: rows above/below first, then sides
    int hx, hy;
    if (c < HX * SX) {
      hy = c / SX;
      hx = c % SX;
    } else if (c < 2 * HX * SX) {
      c -= HX * SX;
      hy = HX + TY + c / SX;
      hx = c % SX;
    } else {
      c -= 2 * HX * SX;
      hy = HX + c / (2 * HXD);
      const int side = c % (2 * HXD);
      hx = side < HX ? side : TX + side;
    }
    bool okx, oky;
    const int gx = wrapc(x0 + hx - HX, a.nx, a.periodic, okx);
    const int gy = wrapc(y0 + hy - HX, a.ny, a.periodic, oky);
    hslot[k] = hy * SX + hx;
    hoff[k] = (okx && oky) ? (long)gy * a.nx + gx : -1;
  }
  // in-tile cells past the grid edge hold the wrapped (or zero) neighbours
  long eoff = -1;
  if (!active && x < a.nx + ND && y < a.ny + ND) {
    bool okx, oky;
    const int gx = wrapc(x, a.nx, a.periodic, okx);
    const int gy = wrapc(y, a.ny, a.periodic, oky);
    if (okx && oky) eoff = (long)gy * a.nx + gx;
  }
  auto planeval = [&](long off, int z) -> C2 {
    return (off >= 0) ? __ldg(src + (long)z * sz + off) : Cx<R>::make(0, 0);
  };
  // sliding window w[k] = psi(x, y, z - 4 + k); prefetch queue of two planes
  C2 w[2 * ND + 1];
#pragma unroll
  for (int k = 0; k < 2 * ND + 1; ++k) w[k] = colval(zc0 - ND + k);
  C2 q1 = colval(zc0 + ND + 1);
  C2 q2 = colval(zc0 + ND + 2);
  const C2 czc = Cx<R>::make((R)a.zc.x, (R)a.zc.y);
  // operands of plane z prefetched one plane ahead
  C2 hq[NH];
  C2 eq = Cx<R>::make(0, 0);
#pragma unroll
  for (int k = 0; k < NH; ++k) hq[k] = planeval(hoff[k], zc0);
  if (!active) eq = planeval(eoff, zc0);
  const R* vsrc;
  if (sizeof(R) == 8) vsrc = (const R*)(a.vloc + (long)ispin * a.npts);
  else vsrc = (const R*)(a.vloc32 + (long)ispin * a.npts);
  R vl_n = active ? __ldg(vsrc + (long)zc0 * sz + pxy) : (R)0;
  int pm_n = (active && a.nlma > 0) ? __ldg(a.pmap + (long)zc0 * sz + pxy) : -1;

  int buf = 0;
  for (int z = zc0; z < zc1; ++z) {
    C2* P = plane[buf];
    if (active) P[ctr] = w[ND];
    else P[ctr] = eq;
#pragma unroll
    for (int k = 0; k < NH; ++k)
      if (hslot[k] >= 0) P[hslot[k]] = hq[k];
    const R vl = vl_n;
    const int pm = pm_n;
    if (z + 1 < zc1) {  // next plane's halo and per-point operands
#pragma unroll
      for (int k = 0; k < NH; ++k) hq[k] = planeval(hoff[k], z + 1);
      if (!active) eq = planeval(eoff, z + 1);
      if (active) {
        vl_n = __ldg(vsrc + (long)(z + 1) * sz + pxy);
        if (a.nlma > 0) pm_n = __ldg(a.pmap + (long)(z + 1) * sz + pxy);
      }
    }
    __syncthreads();
    if (active) {
      C2 vx = Cx<R>::make(0, 0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
      for (int s = 1; s <= ND; ++s) {
        int ip, im;
        if (FULL) {
          ip = ty * SX + (tx + s) % TX;
          im = ty * SX + (tx - s + TX) % TX;
        } else {
          ip = ctr + s;
          im = ctr - s;
        }
        const C2 tp = P[ip], tm = P[im];
        vx = cfma((R)a.lapt[s - 1], cadd(tp, tm), vx);
        if (GRAD) wx = cfma((R)a.nab[s - 1], csub(tp, tm), wx);
      }
#pragma unroll
      for (int s = 1; s <= ND; ++s) {
        int ip, im;
        if (FULL) {
          ip = ((ty + s) % TY) * SX + tx;
          im = ((ty - s + TY) % TY) * SX + tx;
        } else {
          ip = ctr + s * SX;
          im = ctr - s * SX;
        }
        const C2 tp = P[ip], tm = P[im];
        vy = cfma((R)a.lapt[4 + s - 1], cadd(tp, tm), vy);
        if (GRAD) wy = cfma((R)a.nab[4 + s - 1], csub(tp, tm), wy);
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const C2 tp = w[ND + 1 + s], tm = w[ND - 1 - s];
        vz = cfma((R)a.lapt[8 + s], cadd(tp, tm), vz);
        if (GRAD) wz = cfma((R)a.nab[8 + s], csub(tp, tm), wz);
      }
      const C2 v = cadd(vz, cadd(vy, vx));
      const C2 ww = cfma(kz, wz, cfma(ky, wy, cscal(kx, wx)));
      const C2 c = w[ND];
      const long p = (long)z * sz + pxy;
      C2 h;  // stencil value, then + KB term
      h = hcore(vl, lap0, c, v);
      if (GRAD) {
        h.x += ww.y;
        h.y -= ww.x;
      }
      if (a.nlma > 0 && pm >= 0 && a.use_pairs) {
        h = kb_pairs<R>(h, pm, a.proj + (long)o * a.nlma, a, ik);
      } else if (a.nlma > 0 && pm >= 0) {
        const double2* pj = a.proj + (long)o * a.nlma;
        const double2* zk = a.ent_zk + (a.phase_per_k ? (long)ik * a.nent : 0L);
        const int e0 = pm >> 8, e1 = e0 + (pm & 255);
        for (int e = e0; e < e1; e += 4) {  // entries four at a time, summed in entry order
          double2 pv[4], zv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int ee = min(e + i, e1 - 1);
            pv[i] = pj[__ldg(a.ent_lma + ee)];
            zv[i] = __ldg(zk + ee);
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if (e + i < e1)
              h = cadd(h, cmul(Cx<R>::make((R)pv[i].x, (R)pv[i].y), Cx<R>::make((R)zv[i].x, (R)zv[i].y)));
        }
      }
      const long gi = (long)o * a.npts + p;
      if (ModeT<MODE>::store_h) {
        if (ModeT<MODE>::h32) ((float2*)hout)[gi] = make_float2((float)h.x, (float)h.y);
        else ((double2*)hout)[gi] = make_double2((double)h.x, (double)h.y);
      }
      if (MODE == 1 || MODE == 4 || MODE == 5) {
        const double2 cd = make_double2((double)c.x, (double)c.y);
        const double2 hd = make_double2((double)h.x, (double)h.y);
        acc[gi] = cadd(cd, cmul(a.zc, hd));
      } else if (MODE == 2 || MODE == 3) {
        const double2 hd = make_double2((double)h.x, (double)h.y);
        acc[gi] = cadd(acc[gi], cmul(a.zc, hd));
      } else if (MODE == 6) {
        const C2 t = cmul(czc, h);
        d32[gi] = make_float2((float)t.x, (float)t.y);
      } else if (MODE == 7) {
        const float2 dd = d32[gi];
        const C2 t = cadd(Cx<R>::make((R)dd.x, (R)dd.y), cmul(czc, h));
        d32[gi] = make_float2((float)t.x, (float)t.y);
      } else if (MODE == 8) {
        const float2 dd = d32[gi];
        const C2 t = cadd(Cx<R>::make((R)dd.x, (R)dd.y), cmul(czc, h));
        acc[gi] = cadd(acc[gi], make_double2((double)t.x, (double)t.y));
      }
    }
    // advance the window; the next plane's loads were issued two planes ago
#pragma unroll
    for (int k = 0; k < 2 * ND; ++k) w[k] = w[k + 1];
    w[2 * ND] = q1;
    q1 = q2;
    q2 = colval(z + ND + 3);
    buf ^= 1;
  }
}

template <int TX, int TY, bool FULL, int MODE, bool GRAD>
__global__ void __launch_bounds__(TX * TY, (MODE >= 6) ? SB200_TILED_MINB32 : SB200_TILED_MINB64)
    k_hpsi_tiled(const typename Cx<typename ModeT<MODE>::R>::T* __restrict__ in, void* __restrict__ hout,
                 double2* __restrict__ acc, float2* __restrict__ d32, TiledArgs a) {
  tiled_body<TX, TY, FULL, MODE, GRAD>(in, hout, acc, d32, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

}  // namespace tiled
}  // namespace sb200
