// sb200_tma_stencil.cu -- hpsi Taylor-term kernel fed by TMA tensor copies.
//
// One CTA (256 threads) owns a 32 x 8 column tile of one orbital and sweeps a
// chunk of z planes.  The input planes, each with its 4-deep x / y halo
// (40 x 16 complex values; 32 x 16 when the tile spans a periodic x extent of
// 32), are brought into an 8-slot shared-memory ring by
// cp.async.bulk.tensor (one elected thread, one mbarrier per slot), four
// planes ahead of use; the Taylor accumulator tiles (and the FP32 correction
// of the mixed form) arrive the same way into a 4-slot ring.  Threads keep the
// nine z neighbours of their column in registers, fed from the ring, and read
// the x / y neighbours from the current plane.  Copies that fall outside an
// isolated grid are zero-filled by the copy engine, which is exactly the zero
// Dirichlet halo; periodic grids wrap z and y by coordinates.
//
// The arithmetic per point is that of the tiled kernel (sb200_tiled_body.cuh):
// zstencil_typical_seq (zstencil_core/typical/seq.f90:65-122), the KB scatter
// through the owner-computes map (nonlocal_potential.f90:368-375) and the
// Taylor epilogue of taylor.f90:47-117 in the modes of sb200_stencil.cu.
//
// Every wait on a copy is bounded (sb200_tma.cuh); when one expires the CTA
// flags ctx->d_err, waits (bounded) for its other copies in flight and leaves.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "sb200_internal.cuh"
#include "sb200_stencil.cuh"
#include "sb200_tiled_body.cuh"
#include "sb200_tma.cuh"

namespace sb200 {
namespace {

using namespace tiled;

constexpr int TX = 32, TY = 8, NT = TX * TY, HALO = ND;
constexpr int RING = 8;   // input planes resident / in flight
constexpr int ARING = 4;  // accumulator planes in flight

struct TmaMaps {
  CUtensorMap in;    // input planes: (2 SX) x SY box, or (2 TX) x TY for the periodic centre rows
  CUtensorMap inh;   // periodic: (2 TX) x 4 halo rows
  CUtensorMap acc;   // FP64 accumulator tile (2 TX) x TY
  CUtensorMap d32;   // FP32 correction tile (2 TX) x TY
};

template <int MODE, bool PER>
struct Geo {
  using R = typename ModeT<MODE>::R;
  using C2 = typename Cx<R>::T;
  static constexpr int SX = PER ? TX : TX + 2 * HALO;
  static constexpr int SY = TY + 2 * HALO;
  static constexpr int PLANE = SX * SY;  // complex values per ring slot
  static constexpr unsigned PLANE_BYTES = PLANE * sizeof(C2);
  static constexpr bool ACC64 = (MODE == 2 || MODE == 3 || MODE == 8);  // reads psi_out
  static constexpr bool D32 = (MODE == 7 || MODE == 8);                 // reads the FP32 correction
  static constexpr unsigned ACC_BYTES = ACC64 ? NT * 16u : 0u;
  static constexpr unsigned D32_BYTES = D32 ? NT * 8u : 0u;
  static constexpr size_t RING_OFF = 0;
  static constexpr size_t ACC_OFF = RING_OFF + (size_t)RING * PLANE_BYTES;
  static constexpr size_t D32_OFF = ACC_OFF + (size_t)ARING * ACC_BYTES;
  static constexpr size_t BAR_OFF = D32_OFF + (size_t)ARING * D32_BYTES;
  static constexpr size_t SMEM = BAR_OFF + (RING + ARING) * sizeof(uint64_t) + 128;  // + alignment slack
};

template <int MODE, bool PER>
__device__ __forceinline__ void issue_plane(const TmaMaps& m, unsigned char* base, uint64_t* pbar, int r, int q,
                                            int x0, int y0, int o, int nz, int ny) {
  using G = Geo<MODE, PER>;
  const int slot = r & (RING - 1);
  unsigned char* dst = base + G::RING_OFF + (size_t)slot * G::PLANE_BYTES;
  tma::mbar_arrive_expect_tx(&pbar[slot], G::PLANE_BYTES);
  if (!PER) {
    tma::tensor_load_4d(dst, &m.in, 2 * (x0 - HALO), y0 - HALO, q, o, &pbar[slot]);
  } else {
    int qz = q % nz;
    if (qz < 0) qz += nz;
    const int ya = y0 - HALO < 0 ? y0 - HALO + ny : y0 - HALO;
    const int yb = y0 + TY >= ny ? y0 + TY - ny : y0 + TY;
    constexpr size_t ROW = (size_t)TX * sizeof(typename G::C2);
    tma::tensor_load_4d(dst, &m.inh, 0, ya, qz, o, &pbar[slot]);
    tma::tensor_load_4d(dst + HALO * ROW, &m.in, 0, y0, qz, o, &pbar[slot]);
    tma::tensor_load_4d(dst + (HALO + TY) * ROW, &m.inh, 0, yb, qz, o, &pbar[slot]);
  }
}

template <int MODE, bool PER>
__device__ __forceinline__ void issue_acc(const TmaMaps& m, unsigned char* base, uint64_t* abar, int k, int z,
                                          int x0, int y0, int o) {
  using G = Geo<MODE, PER>;
  const int slot = k & (ARING - 1);
  tma::mbar_arrive_expect_tx(&abar[slot], G::ACC_BYTES + G::D32_BYTES);
  if (G::ACC64) tma::tensor_load_4d(base + G::ACC_OFF + (size_t)slot * G::ACC_BYTES, &m.acc, 2 * x0, y0, z, o, &abar[slot]);
  if (G::D32) tma::tensor_load_4d(base + G::D32_OFF + (size_t)slot * G::D32_BYTES, &m.d32, 2 * x0, y0, z, o, &abar[slot]);
}

template <int MODE, bool PER>
__global__ void __launch_bounds__(NT, (MODE >= 6) ? 3 : 2)
    k_hpsi_tma(const __grid_constant__ TmaMaps maps, void* __restrict__ hout, double2* __restrict__ acc,
               float2* __restrict__ d32, TiledArgs a, int* __restrict__ err) {
  using G = Geo<MODE, PER>;
  using R = typename G::R;
  using C2 = typename G::C2;
  constexpr int SX = G::SX;
  extern __shared__ unsigned char smraw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
  const C2* ring = (const C2*)(base + G::RING_OFF);
  const double2* accr = (const double2*)(base + G::ACC_OFF);
  const float2* d32r = (const float2*)(base + G::D32_OFF);
  uint64_t* pbar = (uint64_t*)(base + G::BAR_OFF);
  uint64_t* abar = pbar + RING;

  const int t = threadIdx.x;
  const int tx = t & (TX - 1), ty = t / TX;
  const int ntx = (a.nx + TX - 1) / TX;
  const int x0 = ((int)blockIdx.x % ntx) * TX, y0 = ((int)blockIdx.x / ntx) * TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool active = (x < a.nx) && (y < a.ny);
  const int zc0 = blockIdx.y * a.zchunk;
  const int zc1 = min(a.nz, zc0 + a.zchunk);
  const int nsteps = zc1 - zc0;
  const int ntot = nsteps + 2 * HALO;  // input planes zc0-4 .. zc1+3
  const int o = blockIdx.z;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const R kx = (R)kc[0], ky = (R)kc[1], kz = (R)kc[2], lap0 = (R)kc[3];
  const int ctr = (ty + HALO) * SX + (PER ? tx : tx + HALO);
  const long sz = (long)a.nx * a.ny;
  const long pxy = (long)y * a.nx + x;
  constexpr bool GRAD = PER;

  if (t == 0) {
    for (int i = 0; i < RING + ARING; ++i) tma::mbar_init(&pbar[i], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  // copies issued / waited, tracked identically by every thread
  int p_issued = 0, p_waited = 0, a_issued = 0, a_waited = 0;
  const int pro = ntot < RING ? ntot : RING;
  if (t == 0) {
    for (int r = 0; r < pro; ++r)
      issue_plane<MODE, PER>(maps, base, pbar, r, zc0 - HALO + r, x0, y0, o, a.nz, a.ny);
    if (G::ACC64 || G::D32)
      for (int k = 0; k < ARING && k < nsteps; ++k) issue_acc<MODE, PER>(maps, base, abar, k, zc0 + k, x0, y0, o);
  }
  p_issued = pro;
  if (G::ACC64 || G::D32) a_issued = nsteps < ARING ? nsteps : ARING;

  bool ok = true;
  C2 w[2 * HALO + 1];
  // window planes zc0-4 .. zc0+3
#pragma unroll
  for (int r = 0; r < 2 * HALO; ++r) {
    ok = tma::mbar_wait(&pbar[r], 0u) && ok;
    w[r] = ring[(size_t)r * G::PLANE + ctr];
  }
  p_waited = 2 * HALO;
  bool all_ok = __syncthreads_and(ok);  // the same in every thread
  if (all_ok) {
    if (t == 0) {  // the four pre-window slots take planes zc0+4 .. zc0+7
      tma::fence_proxy_async_smem();
      for (int r = RING; r < RING + HALO && r < ntot; ++r)
        issue_plane<MODE, PER>(maps, base, pbar, r, zc0 - HALO + r, x0, y0, o, a.nz, a.ny);
    }
    p_issued = ntot < RING + HALO ? ntot : RING + HALO;

    const C2 czc = Cx<R>::make((R)a.zc.x, (R)a.zc.y);
    const R* vsrc;
    if (sizeof(R) == 8) vsrc = (const R*)(a.vloc + (long)ispin * a.npts);
    else vsrc = (const R*)(a.vloc32 + (long)ispin * a.npts);
    R vl_n = active ? __ldg(vsrc + (long)zc0 * sz + pxy) : (R)0;
    int pm_n = (active && a.nlma > 0) ? __ldg(a.pmap + (long)zc0 * sz + pxy) : -1;
    for (int k = 0; k < nsteps; ++k) {
      const int z = zc0 + k;
      const int rf = k + 2 * HALO;  // plane z+4 feeds the window
      ok = tma::mbar_wait(&pbar[rf & (RING - 1)], (unsigned)((rf / RING) & 1)) && ok;
      w[2 * HALO] = ring[(size_t)(rf & (RING - 1)) * G::PLANE + ctr];
      p_waited = rf + 1;
      if (G::ACC64 || G::D32) {
        ok = tma::mbar_wait(&abar[k & (ARING - 1)], (unsigned)((k / ARING) & 1)) && ok;
        a_waited = k + 1;
      }
      const R vl = vl_n;
      const int pm = pm_n;
      if (k + 1 < nsteps && active) {
        vl_n = __ldg(vsrc + (long)(z + 1) * sz + pxy);
        if (a.nlma > 0) pm_n = __ldg(a.pmap + (long)(z + 1) * sz + pxy);
      }
      if (active) {
        const C2* P = ring + (size_t)((k + HALO) & (RING - 1)) * G::PLANE;
        C2 vx = Cx<R>::make(0, 0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
        for (int s = 1; s <= HALO; ++s) {
          C2 tp, tm;
          if (PER) {
            tp = P[(ty + HALO) * SX + ((tx + s) & (TX - 1))];
            tm = P[(ty + HALO) * SX + ((tx - s) & (TX - 1))];
          } else {
            tp = P[ctr + s];
            tm = P[ctr - s];
          }
          vx = cadd(vx, cscal((R)a.lapt[s - 1], cadd(tp, tm)));
          if (GRAD) wx = cadd(wx, cscal((R)a.nab[s - 1], csub(tp, tm)));
        }
#pragma unroll
        for (int s = 1; s <= HALO; ++s) {
          const C2 tp = P[ctr + s * SX], tm = P[ctr - s * SX];
          vy = cadd(vy, cscal((R)a.lapt[4 + s - 1], cadd(tp, tm)));
          if (GRAD) wy = cadd(wy, cscal((R)a.nab[4 + s - 1], csub(tp, tm)));
        }
#pragma unroll
        for (int s = 0; s < HALO; ++s) {
          const C2 tp = w[HALO + 1 + s], tm = w[HALO - 1 - s];
          vz = cadd(vz, cscal((R)a.lapt[8 + s], cadd(tp, tm)));
          if (GRAD) wz = cadd(wz, cscal((R)a.nab[8 + s], csub(tp, tm)));
        }
        const C2 v = cadd(vz, cadd(vy, vx));
        const C2 c = w[HALO];
        C2 h;
        h.x = vl * c.x + lap0 * c.x - (R)0.5 * v.x;
        h.y = vl * c.y + lap0 * c.y - (R)0.5 * v.y;
        if (GRAD) {
          const C2 ww = cadd(cscal(kz, wz), cadd(cscal(ky, wy), cscal(kx, wx)));
          h.x += ww.y;
          h.y -= ww.x;
        }
        if (a.nlma > 0 && pm >= 0) {
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
        const long gi = (long)o * a.npts + (long)z * sz + pxy;
        const int ti = (k & (ARING - 1)) * NT + t;
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
          acc[gi] = cadd(accr[ti], cmul(a.zc, hd));
        } else if (MODE == 6) {
          const C2 tt = cmul(czc, h);
          d32[gi] = make_float2((float)tt.x, (float)tt.y);
        } else if (MODE == 7) {
          const float2 dd = d32r[ti];
          const C2 tt = cadd(Cx<R>::make((R)dd.x, (R)dd.y), cmul(czc, h));
          d32[gi] = make_float2((float)tt.x, (float)tt.y);
        } else if (MODE == 8) {
          const float2 dd = d32r[ti];
          const C2 tt = cadd(Cx<R>::make((R)dd.x, (R)dd.y), cmul(czc, h));
          acc[gi] = cadd(accr[ti], make_double2((double)tt.x, (double)tt.y));
        }
      }
#pragma unroll
      for (int i = 0; i < 2 * HALO; ++i) w[i] = w[i + 1];
      all_ok = __syncthreads_and(ok);
      if (!all_ok) break;
      if (t == 0) {  // refill the slots of plane z and of accumulator step k
        tma::fence_proxy_async_smem();
        const int rn = k + RING + HALO;  // plane z+8
        if (rn < ntot) issue_plane<MODE, PER>(maps, base, pbar, rn, zc0 - HALO + rn, x0, y0, o, a.nz, a.ny);
        if ((G::ACC64 || G::D32) && k + ARING < nsteps)
          issue_acc<MODE, PER>(maps, base, abar, k + ARING, z + ARING, x0, y0, o);
      }
      if (k + RING + HALO < ntot) p_issued = k + RING + HALO + 1;
      if ((G::ACC64 || G::D32) && k + ARING < nsteps) a_issued = k + ARING + 1;
    }
  }
  if (!all_ok) {
    // a copy did not arrive in time: flag it, wait (bounded) for the copies
    // still in flight into this CTA's shared memory, and leave
    if (t == 0) {
      atomicExch(err, 1);
      for (int r = p_waited; r < p_issued; ++r) tma::mbar_wait(&pbar[r & (RING - 1)], (unsigned)((r / RING) & 1));
      for (int k = a_waited; k < a_issued; ++k) tma::mbar_wait(&abar[k & (ARING - 1)], (unsigned)((k / ARING) & 1));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      cudaGetLastError();
  }
  return fn;
}

// 4-D map over an orbital block [norb][nz][ny][2 nx] of FP64 or FP32 reals
bool make_map(CUtensorMap* m, const void* base, bool f32, const GridInfo& g, int norb, int box0, int box1) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn || ((uintptr_t)base & 15) != 0) return false;
  const cuuint64_t es = f32 ? 4 : 8;
  const cuuint64_t dims[4] = {(cuuint64_t)2 * g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)norb};
  const cuuint64_t strides[3] = {dims[0] * es, dims[0] * es * g.ny, dims[0] * es * g.ny * g.nz};
  if (strides[0] % 16 != 0) return false;
  const cuuint32_t box[4] = {(cuuint32_t)box0, (cuuint32_t)box1, 1, 1};
  const cuuint32_t est[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                        const_cast<void*>(base), dims, strides, box, est, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int MODE, bool PER>
int launch_t(sb200_ctx* c, const TmaMaps& maps, const HpsiLaunch& L, const TiledArgs& a, dim3 grid) {
  using G = Geo<MODE, PER>;
  static bool attr = false;
  if (!attr) {
    SB_CUDA(cudaFuncSetAttribute(k_hpsi_tma<MODE, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    attr = true;
  }
  k_hpsi_tma<MODE, PER><<<grid, NT, G::SMEM, c->stream>>>(maps, L.hout, L.out, L.d32, a, c->d_err);
  SB_LAUNCH_CHECK("k_hpsi_tma");
  return SB200_OK;
}

template <bool PER>
int launch_mode(sb200_ctx* c, const TmaMaps& maps, const HpsiLaunch& L, const TiledArgs& a, dim3 grid) {
  switch (L.mode) {
    case 0: return launch_t<0, PER>(c, maps, L, a, grid);
    case 1: return launch_t<1, PER>(c, maps, L, a, grid);
    case 2: return launch_t<2, PER>(c, maps, L, a, grid);
    case 3: return launch_t<3, PER>(c, maps, L, a, grid);
    case 4: return launch_t<4, PER>(c, maps, L, a, grid);
    case 5: return launch_t<5, PER>(c, maps, L, a, grid);
    case 6: return launch_t<6, PER>(c, maps, L, a, grid);
    case 7: return launch_t<7, PER>(c, maps, L, a, grid);
    case 8: return launch_t<8, PER>(c, maps, L, a, grid);
    default: return set_error(SB200_ERR_INVALID_ARG, "tma hpsi: unknown mode");
  }
}

}  // namespace

// Applies to isolated grids of any shape and to periodic grids with nx = 32
// and ny a multiple of 8; FP32-input modes need an even nx.  Returns
// SB200_ERR_UNSUPPORTED (without launching) when the path does not apply.
int launch_hpsi_tma(sb200_ctx* c, const HpsiLaunch& L) {
  const GridInfo& g = c->g;
  if (c->tma_variant == 0) return SB200_ERR_UNSUPPORTED;
  const bool per = g.periodic != 0;
  if (per && !(g.nx == TX && g.ny % TY == 0 && g.nz >= 1)) return SB200_ERR_UNSUPPORTED;
  const bool in32 = L.mode >= 6;
  const int SXv = per ? TX : TX + 2 * HALO;
  const int norb = c->orb.norb;
  TmaMaps maps;
  memset(&maps, 0, sizeof(maps));
  if (!make_map(&maps.in, L.in, in32, g, norb, 2 * SXv, per ? TY : TY + 2 * HALO)) return SB200_ERR_UNSUPPORTED;
  if (per && !make_map(&maps.inh, L.in, in32, g, norb, 2 * TX, HALO)) return SB200_ERR_UNSUPPORTED;
  const bool acc64 = (L.mode == 2 || L.mode == 3 || L.mode == 8);
  const bool rd32 = (L.mode == 7 || L.mode == 8);
  if (acc64 && !make_map(&maps.acc, L.out, false, g, norb, 2 * TX, TY)) return SB200_ERR_UNSUPPORTED;
  if (rd32 && !make_map(&maps.d32, L.d32, true, g, norb, 2 * TX, TY)) return SB200_ERR_UNSUPPORTED;
  TiledArgs a = make_tiled_args(c, L.zc);
  const int ntiles = ((g.nx + TX - 1) / TX) * ((g.ny + TY - 1) / TY);
  // z chunks: long sweeps (each chunk re-reads 8 halo planes), split only
  // until there are about four CTAs per SM
  const long ctas = (long)ntiles * norb;
  int nchunk = 1;
  while (ctas * nchunk < 148L * 4 && g.nz / (nchunk * 2) >= 16) nchunk *= 2;
  a.zchunk = (g.nz + nchunk - 1) / nchunk;
  const int nzc = (g.nz + a.zchunk - 1) / a.zchunk;
  dim3 grid(ntiles, nzc, norb);
  return per ? launch_mode<true>(c, maps, L, a, grid) : launch_mode<false>(c, maps, L, a, grid);
}

}  // namespace sb200
