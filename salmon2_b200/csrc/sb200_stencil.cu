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

#include "sb200_internal.cuh"
#include "sb200_stencil.cuh"
#include "sb200_tiled_body.cuh"

namespace sb200 {
namespace {

using namespace tiled;

template <int TX, int TY, bool FULL, int MODE, bool GRAD>
void launch_mode(const HpsiLaunch& L, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  using C2 = typename Cx<typename ModeT<MODE>::R>::T;
  k_hpsi_tiled<TX, TY, FULL, MODE, GRAD><<<grid, TX * TY, 0, st>>>((const C2*)L.in, (void*)L.hout, L.out, L.d32, a);
}

template <int TX, int TY, bool FULL, bool GRAD>
int launch_tiled_t(const HpsiLaunch& L, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  switch (L.mode) {
    case 0: launch_mode<TX, TY, FULL, 0, GRAD>(L, a, grid, st); break;
    case 1: launch_mode<TX, TY, FULL, 1, GRAD>(L, a, grid, st); break;
    case 2: launch_mode<TX, TY, FULL, 2, GRAD>(L, a, grid, st); break;
    case 3: launch_mode<TX, TY, FULL, 3, GRAD>(L, a, grid, st); break;
    case 4: launch_mode<TX, TY, FULL, 4, GRAD>(L, a, grid, st); break;
    case 5: launch_mode<TX, TY, FULL, 5, GRAD>(L, a, grid, st); break;
    case 6: launch_mode<TX, TY, FULL, 6, GRAD>(L, a, grid, st); break;
    case 7: launch_mode<TX, TY, FULL, 7, GRAD>(L, a, grid, st); break;
    case 8: launch_mode<TX, TY, FULL, 8, GRAD>(L, a, grid, st); break;
    default: return set_error(SB200_ERR_INVALID_ARG, "tiled hpsi: unknown mode");
  }
  return SB200_OK;
}

}  // namespace

TiledArgs make_tiled_args(const sb200_ctx* c, double2 zc) {
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
  for (int i = 0; i < 12; ++i) {
    a.lapt[i] = c->g.coef_lap[i];
    a.nab[i] = c->g.periodic ? c->g.coef_nab[i] : 0.0;
  }
  a.kcoef = c->d_kcoef;
  a.vloc = c->d_vloc;
  a.vloc32 = c->d_vloc32;
  a.pmap = c->pp.d_pmap;
  a.ent_lma = c->pp.d_ent_lma;
  a.ent_zk = c->pp.d_ent_zk;
  a.proj = c->d_proj;
  a.use_pairs = (c->pp.nlma > 0 && c->pp.d_pmap2 != nullptr) ? 1 : 0;
  a.npair = c->pp.npair;
  a.pair_lma = c->pp.d_pair_lma;
  a.pair_uv = c->pp.d_pair_uv;
  a.pair_ph = c->pp.d_pair_ph;
  if (a.use_pairs) a.pmap = c->pp.d_pmap2;
  a.zc = zc;
  a.zchunk = c->g.nz;
  return a;
}

int launch_hpsi_tiled(sb200_ctx* c, const HpsiLaunch& L) {
  const int rt = launch_hpsi_tma(c, L);
  if (rt != SB200_ERR_UNSUPPORTED) return rt;
  TiledArgs a = make_tiled_args(c, L.zc);
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
  // isolated grids (k + A = 0) skip the gradient terms
  if (full16) r = launch_tiled_t<16, 16, true, true>(L, a, grid, c->stream);
  else if (TXv == 16) r = g.periodic ? launch_tiled_t<16, 16, false, true>(L, a, grid, c->stream)
                                     : launch_tiled_t<16, 16, false, false>(L, a, grid, c->stream);
  else r = g.periodic ? launch_tiled_t<32, 8, false, true>(L, a, grid, c->stream)
                      : launch_tiled_t<32, 8, false, false>(L, a, grid, c->stream);
  if (r != SB200_OK) return r;
  SB_LAUNCH_CHECK("k_hpsi_tiled");
  return SB200_OK;
}

}  // namespace sb200
