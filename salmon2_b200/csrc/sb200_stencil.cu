// sb200_stencil.cu -- tiled FP64 hpsi kernel: 2.5-D sweep along z.
//
// One CTA owns a TX x TY column tile of one orbital and sweeps a chunk of z
// planes.  Each thread keeps the nine z-neighbours of its column in registers
// (a sliding window fed one plane ahead from HBM), the current xy plane of the
// tile (plus a 4-deep halo, unless the tile is the whole periodic plane) is
// staged in shared memory for the x / y neighbours, and every point is read
// from HBM once per sweep (halo cells come from L1/L2).  The arithmetic is the
// 25-point Laplacian + Bloch gradient + V_local of zstencil_typical_seq
// (src/common/zstencil_core/typical/seq.f90:65-122), the KB scatter through the
// owner-computes inverse map (ilma ascending, nonlocal_potential.f90:368-375)
// and the Taylor accumulation of taylor.f90:47-117 as an epilogue.
#include <cuda_runtime.h>

#include "sb200_internal.cuh"
#include "sb200_stencil.cuh"

namespace sb200 {
namespace {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscal(double r, double2 a) { return make_double2(r * a.x, r * a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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

template <int TX, int TY, bool FULL, int MODE>
__global__ void __launch_bounds__(TX * TY, 2) k_hpsi_tiled(const double2* __restrict__ in, double2* __restrict__ hout,
                                                        double2* __restrict__ acc, TiledArgs a) {
  constexpr int HX = FULL ? 0 : ND;                 // halo width in shared memory
  constexpr int SX = TX + 2 * HX, SY = TY + 2 * HX;  // staged plane extents
  constexpr int NT = TX * TY;
  __shared__ double2 plane[2][SY * SX];

  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int ntx = (a.nx + TX - 1) / TX;
  const int x0 = (blockIdx.x % ntx) * TX, y0 = (blockIdx.x / ntx) * TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool active = (x < a.nx) && (y < a.ny);
  const int zc0 = blockIdx.y * a.zchunk;
  const int zc1 = min(a.nz, zc0 + a.zchunk);
  const int o = blockIdx.z;
  const long sz = (long)a.nx * a.ny;
  const double2* src = in + (long)o * a.npts;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const double lap0 = kc[3];
  double nabx[ND], naby[ND], nabz[ND];
#pragma unroll
  for (int s = 0; s < ND; ++s) {
    nabx[s] = kc[4 + s];
    naby[s] = kc[8 + s];
    nabz[s] = kc[12 + s];
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
  // chunk, so the periodic wrap is a full modulo)
  auto colval = [&](int z) -> double2 {
    int zz = z;
    bool ok = true;
    if (a.periodic) zz = ((z % a.nz) + a.nz) % a.nz;
    else ok = (z >= 0) && (z < a.nz);
    return (ok && active) ? __ldg(src + (long)zz * sz + pxy) : make_double2(0.0, 0.0);
  };
  // sliding window w[k] = psi(x, y, z - 4 + k); prefetch queue of two planes
  double2 w[2 * ND + 1];
#pragma unroll
  for (int k = 0; k < 2 * ND + 1; ++k) w[k] = colval(zc0 - ND + k);
  double2 q1 = colval(zc0 + ND + 1);
  double2 q2 = colval(zc0 + ND + 2);

  int buf = 0;
  for (int z = zc0; z < zc1; ++z) {
    double2* P = plane[buf];
    // stage plane z: interior from the window, halo from L1/L2; cells of
    // threads past the grid edge hold the wrapped (or zero) neighbours
    if (active) {
      P[ctr] = w[ND];
    } else {
      bool okx, oky;
      const int gx = wrapc(x, a.nx, a.periodic, okx);
      const int gy = wrapc(y, a.ny, a.periodic, oky);
      const bool near = (x < a.nx + ND) && (y < a.ny + ND);
      P[ctr] = (okx && oky && near) ? __ldg(src + (long)z * sz + (long)gy * a.nx + gx) : make_double2(0.0, 0.0);
    }
    if (!FULL) {
      for (int c = threadIdx.x; c < SX * SY; c += NT) {
        const int hx = c % SX, hy = c / SX;
        if (hx >= HX && hx < HX + TX && hy >= HX && hy < HX + TY) continue;
        bool okx, oky;
        const int gx = wrapc(x0 + hx - HX, a.nx, a.periodic, okx);
        const int gy = wrapc(y0 + hy - HX, a.ny, a.periodic, oky);
        P[c] = (okx && oky) ? __ldg(src + (long)z * sz + (long)gy * a.nx + gx) : make_double2(0.0, 0.0);
      }
    }
    __syncthreads();
    if (active) {
      double2 vx = make_double2(0.0, 0.0), wx = make_double2(0.0, 0.0);
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = P[offxp[s]], tm = P[offxm[s]];
        vx = cadd(vx, cscal(a.lapt[s], cadd(tp, tm)));
        wx = cadd(wx, cscal(nabx[s], csub(tp, tm)));
      }
      double2 vy = make_double2(0.0, 0.0), wy = make_double2(0.0, 0.0);
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = P[offyp[s]], tm = P[offym[s]];
        vy = cadd(vy, cscal(a.lapt[4 + s], cadd(tp, tm)));
        wy = cadd(wy, cscal(naby[s], csub(tp, tm)));
      }
      double2 vz = make_double2(0.0, 0.0), wz = make_double2(0.0, 0.0);
#pragma unroll
      for (int s = 0; s < ND; ++s) {
        const double2 tp = w[ND + 1 + s], tm = w[ND - 1 - s];
        vz = cadd(vz, cscal(a.lapt[8 + s], cadd(tp, tm)));
        wz = cadd(wz, cscal(nabz[s], csub(tp, tm)));
      }
      const double2 v = cadd(vz, cadd(vy, vx));
      const double2 ww = cadd(wz, cadd(wy, wx));
      const double2 c = w[ND];
      const long p = (long)z * sz + pxy;
      const double vl = __ldg(a.vloc + (long)ispin * a.npts + p);
      double2 h;
      h.x = vl * c.x + lap0 * c.x - 0.5 * v.x + ww.y;
      h.y = vl * c.y + lap0 * c.y - 0.5 * v.y - ww.x;
      if (a.nlma > 0) {
        const int vi = __ldg(a.map + p);
        if (vi >= 0) {
          const int e1 = __ldg(a.vi_start + vi + 1);
          const double2* pj = a.proj + (long)o * a.nlma;
          const double2* ph = a.phase + (a.phase_per_k ? (long)ik * a.totpts : 0L);
          for (int e = __ldg(a.vi_start + vi); e < e1; ++e) {
            const double uv = __ldg(a.ent_uv + e);
            const double2 phs = __ldg(ph + __ldg(a.ent_pt + e));
            const double2 zk = make_double2(phs.x * uv, -phs.y * uv);
            h = cadd(h, cmul(pj[__ldg(a.ent_lma + e)], zk));
          }
        }
      }
      const long gi = (long)o * a.npts + p;
      if (MODE <= 2) hout[gi] = h;
      if (MODE == 1 || MODE == 4) acc[gi] = cadd(c, cmul(a.zc, h));
      if (MODE == 2 || MODE == 3) acc[gi] = cadd(acc[gi], cmul(a.zc, h));
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

template <int TX, int TY, bool FULL>
int launch_tiled_t(const HpsiLaunch& L, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  switch (L.mode) {
    case 0: k_hpsi_tiled<TX, TY, FULL, 0><<<grid, TX * TY, 0, st>>>(L.in, L.hout, L.out, a); break;
    case 1: k_hpsi_tiled<TX, TY, FULL, 1><<<grid, TX * TY, 0, st>>>(L.in, L.hout, L.out, a); break;
    case 2: k_hpsi_tiled<TX, TY, FULL, 2><<<grid, TX * TY, 0, st>>>(L.in, L.hout, L.out, a); break;
    case 3: k_hpsi_tiled<TX, TY, FULL, 3><<<grid, TX * TY, 0, st>>>(L.in, L.hout, L.out, a); break;
    default: k_hpsi_tiled<TX, TY, FULL, 4><<<grid, TX * TY, 0, st>>>(L.in, L.hout, L.out, a); break;
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
  a.totpts = c->pp.totpts;
  a.phase_per_k = c->g.periodic;
  a.npts = c->g.npts;
  for (int i = 0; i < 12; ++i) a.lapt[i] = c->g.coef_lap[i];
  a.kcoef = c->d_kcoef;
  a.vloc = c->d_vloc;
  a.map = c->pp.d_map;
  a.vi_start = c->pp.d_vi_start;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_pt = c->pp.d_ent_pt;
  a.ent_uv = c->pp.d_ent_uv;
  a.phase = c->pp.d_phase;
  a.proj = c->d_proj;
  a.zc = L.zc;
  // tile choice: the whole plane for small periodic grids, else 32x8 (16x16
  // when the x extent is at most 16)
  const GridInfo& g = c->g;
  const bool full16 = g.periodic && g.nx == 16 && g.ny == 16;
  int TXv = g.nx <= 16 ? 16 : 32;
  int TYv = TXv == 16 ? 16 : 8;
  const int ntiles = ((g.nx + TXv - 1) / TXv) * ((g.ny + TYv - 1) / TYv);
  // z chunks: enough CTAs to fill the GPU (>= 4 per SM), chunks of >= 8 planes
  long ctas = (long)ntiles * c->orb.norb;
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
