// sb200_stencil.cu -- tiled hpsi kernel: 2.5-D sweep along z, FP64 or FP32.
//
// One CTA owns a TX x TY column tile of one orbital and sweeps a chunk of z
// planes.  Each thread keeps the nine z-neighbours of its column in registers
// (a sliding window fed two planes ahead from HBM), the current xy plane of the
// tile (plus a 4-deep halo, unless the tile is the whole periodic plane) is
// staged in shared memory for the x / y neighbours, and every point is read
// from HBM once per sweep (halo cells come from L1/L2).  The arithmetic is the
// 25-point Laplacian + Bloch gradient + V_local of zstencil_typical_seq
// (src/common/zstencil_core/typical/seq.f90:65-122), the KB scatter through the
// owner-computes inverse map (ilma ascending, nonlocal_potential.f90:368-375)
// and the Taylor accumulation of taylor.f90:47-117 as an epilogue.
//
// Epilogue modes (taylor.f90:43-119 with psi_out accumulated in FP64):
//   FP64 form: 0 h only | 1 h, out = in + zc h | 2 h, out += zc h |
//              3 out += zc h | 4 out = in + zc h
//   mixed form (terms n >= 2 in FP32, FP64 first term and accumulation):
//              5 FP64 stencil, h stored as complex64, out = in + zc h
//              6 FP32 stencil, h complex64, d = zc h (FP32 correction)
//              7 FP32 stencil, h complex64, d += zc h
//              8 FP32 stencil, out += (double)(d + zc h)
#include <cuda_runtime.h>

#include <type_traits>

#include "sb200_internal.cuh"
#include "sb200_stencil.cuh"

namespace sb200 {
namespace {

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

template <int TX, int TY, bool FULL, int MODE>
__global__ void __launch_bounds__(TX * TY, 2)
    k_hpsi_tiled(const typename Cx<typename ModeT<MODE>::R>::T* __restrict__ in, void* __restrict__ hout,
                 double2* __restrict__ acc, float2* __restrict__ d32, TiledArgs a) {
  using R = typename ModeT<MODE>::R;
  using C2 = typename Cx<R>::T;
  constexpr int HX = FULL ? 0 : ND;                 // halo width in shared memory
  constexpr int SX = TX + 2 * HX, SY = TY + 2 * HX;  // staged plane extents
  constexpr int NT = TX * TY;
  __shared__ C2 plane[2][SY * SX];

  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int ntx = (a.nx + TX - 1) / TX;
  const int x0 = (blockIdx.x % ntx) * TX, y0 = (blockIdx.x / ntx) * TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool active = (x < a.nx) && (y < a.ny);
  const int zc0 = blockIdx.y * a.zchunk;
  const int zc1 = min(a.nz, zc0 + a.zchunk);
  const int o = blockIdx.z;
  const long sz = (long)a.nx * a.ny;
  const C2* src = in + (long)o * a.npts;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const R lap0 = (R)kc[3];
  R nabx[ND], naby[ND], nabz[ND], lx[ND], ly[ND], lz[ND];
#pragma unroll
  for (int s = 0; s < ND; ++s) {
    nabx[s] = (R)kc[4 + s];
    naby[s] = (R)kc[8 + s];
    nabz[s] = (R)kc[12 + s];
    lx[s] = (R)a.lapt[s];
    ly[s] = (R)a.lapt[4 + s];
    lz[s] = (R)a.lapt[8 + s];
  }
  // shared-memory offsets of the x / y neighbours (constant over the sweep)
  int offxp[ND], offxm[ND], offyp[ND], offym[ND];
  const int ctr = (ty + HX) * SX + (tx + HX);
#pragma unroll
  for (int s = 1; s <= ND; ++s) {
    if (FULL) {
      offxp[s - 1] = ty * SX + (tx + s) % TX;
      offxm[s - 1] = ty * SX + (tx - s + TX) % TX;
      offyp[s - 1] = ((ty + s) % TY) * SX + tx;
      offym[s - 1] = ((ty - s + TY) % TY) * SX + tx;
    } else {
      offxp[s - 1] = ctr + s;
      offxm[s - 1] = ctr - s;
      offyp[s - 1] = ctr + s * SX;
      offym[s - 1] = ctr - s * SX;
    }
  }
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
  // sliding window w[k] = psi(x, y, z - 4 + k); prefetch queue of two planes
  C2 w[2 * ND + 1];
#pragma unroll
  for (int k = 0; k < 2 * ND + 1; ++k) w[k] = colval(zc0 - ND + k);
  C2 q1 = colval(zc0 + ND + 1);
  C2 q2 = colval(zc0 + ND + 2);
  const C2 czc = Cx<R>::make((R)a.zc.x, (R)a.zc.y);

  int buf = 0;
  for (int z = zc0; z < zc1; ++z) {
    C2* P = plane[buf];
    // stage plane z: interior from the window, halo from L1/L2; cells of
    // threads past the grid edge hold the wrapped (or zero) neighbours
    if (active) {
      P[ctr] = w[ND];
    } else {
      bool okx, oky;
      const int gx = wrapc(x, a.nx, a.periodic, okx);
      const int gy = wrapc(y, a.ny, a.periodic, oky);
      const bool near = (x < a.nx + ND) && (y < a.ny + ND);
      P[ctr] = (okx && oky && near) ? __ldg(src + (long)z * sz + (long)gy * a.nx + gx) : Cx<R>::make(0, 0);
    }
    if (!FULL) {
      for (int c = threadIdx.x; c < SX * SY; c += NT) {
        const int hx = c % SX, hy = c / SX;
        if (hx >= HX && hx < HX + TX && hy >= HX && hy < HX + TY) continue;
        bool okx, oky;
        const int gx = wrapc(x0 + hx - HX, a.nx, a.periodic, okx);
        const int gy = wrapc(y0 + hy - HX, a.ny, a.periodic, oky);
        P[c] = (okx && oky) ? __ldg(src + (long)z * sz + (long)gy * a.nx + gx) : Cx<R>::make(0, 0);
      }
    }
    __syncthreads();
    if (active) {
      C2 vx = Cx<R>::make(0, 0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const C2 tp = P[offxp[s]], tm = P[offxm[s]];
        vx = cadd(vx, cscal(lx[s], cadd(tp, tm)));
        wx = cadd(wx, cscal(nabx[s], csub(tp, tm)));
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const C2 tp = P[offyp[s]], tm = P[offym[s]];
        vy = cadd(vy, cscal(ly[s], cadd(tp, tm)));
        wy = cadd(wy, cscal(naby[s], csub(tp, tm)));
      }
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const C2 tp = w[ND + 1 + s], tm = w[ND - 1 - s];
        vz = cadd(vz, cscal(lz[s], cadd(tp, tm)));
        wz = cadd(wz, cscal(nabz[s], csub(tp, tm)));
      }
      const C2 v = cadd(vz, cadd(vy, vx));
      const C2 ww = cadd(wz, cadd(wy, wx));
      const C2 c = w[ND];
      const long p = (long)z * sz + pxy;
      R vl;
      if (sizeof(R) == 8) vl = (R)__ldg(a.vloc + (long)ispin * a.npts + p);
      else vl = (R)__ldg(a.vloc32 + (long)ispin * a.npts + p);
      C2 h;
      h.x = vl * c.x + lap0 * c.x - (R)0.5 * v.x + ww.y;
      h.y = vl * c.y + lap0 * c.y - (R)0.5 * v.y - ww.x;
      if (a.nlma > 0) {
        const int pm = __ldg(a.pmap + p);
        if (pm >= 0) {
          const double2* pj = a.proj + (long)o * a.nlma;
          const double2* zk = a.ent_zk + (a.phase_per_k ? (long)ik * a.nent : 0L);
          const int e1 = (pm >> 8) + (pm & 255);
          for (int e = pm >> 8; e < e1; ++e) {
            const double2 pv = pj[__ldg(a.ent_lma + e)];
            const double2 zv = __ldg(zk + e);
            h = cadd(h, cmul(Cx<R>::make((R)pv.x, (R)pv.y), Cx<R>::make((R)zv.x, (R)zv.y)));
          }
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

template <int TX, int TY, bool FULL, int MODE>
void launch_mode(const HpsiLaunch& L, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  using C2 = typename Cx<typename ModeT<MODE>::R>::T;
  k_hpsi_tiled<TX, TY, FULL, MODE><<<grid, TX * TY, 0, st>>>((const C2*)L.in, (void*)L.hout, L.out, L.d32, a);
}

template <int TX, int TY, bool FULL>
int launch_tiled_t(const HpsiLaunch& L, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  switch (L.mode) {
    case 0: launch_mode<TX, TY, FULL, 0>(L, a, grid, st); break;
    case 1: launch_mode<TX, TY, FULL, 1>(L, a, grid, st); break;
    case 2: launch_mode<TX, TY, FULL, 2>(L, a, grid, st); break;
    case 3: launch_mode<TX, TY, FULL, 3>(L, a, grid, st); break;
    case 4: launch_mode<TX, TY, FULL, 4>(L, a, grid, st); break;
    case 5: launch_mode<TX, TY, FULL, 5>(L, a, grid, st); break;
    case 6: launch_mode<TX, TY, FULL, 6>(L, a, grid, st); break;
    case 7: launch_mode<TX, TY, FULL, 7>(L, a, grid, st); break;
    case 8: launch_mode<TX, TY, FULL, 8>(L, a, grid, st); break;
    default: return set_error(SB200_ERR_INVALID_ARG, "tiled hpsi: unknown mode");
  }
  return SB200_OK;
}

}  // namespace

int launch_hpsi_tiled(sb200_ctx* c, const HpsiLaunch& L) {
  TiledArgs a;
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
  a.vloc32 = c->d_vloc32;
  a.pmap = c->pp.d_pmap;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_zk = c->pp.d_ent_zk;
  a.proj = c->d_proj;
  a.zc = L.zc;
  // tile choice: the whole plane for 16x16 periodic grids, else 32x8 (16x16
  // when the x extent is at most 16)
  const GridInfo& g = c->g;
  const bool full16 = g.periodic && g.nx == 16 && g.ny == 16;
  const int TXv = g.nx <= 16 ? 16 : 32;
  const int TYv = TXv == 16 ? 16 : 8;
  const int ntiles = ((g.nx + TXv - 1) / TXv) * ((g.ny + TYv - 1) / TYv);
  // z chunks: enough CTAs to fill the GPU (>= 8 per SM), chunks of >= 8 planes
  const long ctas = (long)ntiles * c->orb.norb;
  int nchunk = 1;
  while (ctas * nchunk < 148L * 8 && g.nz / (nchunk * 2) >= 8) nchunk *= 2;
  a.zchunk = (g.nz + nchunk - 1) / nchunk;
  const int nzc = (g.nz + a.zchunk - 1) / a.zchunk;
  dim3 grid(ntiles, nzc, c->orb.norb);
  int r;
  if (full16) r = launch_tiled_t<16, 16, true>(L, a, grid, c->stream);
  else if (TXv == 16) r = launch_tiled_t<16, 16, false>(L, a, grid, c->stream);
  else r = launch_tiled_t<32, 8, false>(L, a, grid, c->stream);
  if (r != SB200_OK) return r;
  SB_LAUNCH_CHECK("k_hpsi_tiled");
  return SB200_OK;
}

}  // namespace sb200
