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
#include "sb200_tma_body.cuh"

namespace sb200 {
namespace {

using namespace tmak;

template <int MODE, bool PER>
__global__ void __launch_bounds__(NT, (MODE >= 6) ? 3 : 2)
    k_hpsi_tma(const __grid_constant__ TmaMaps maps, void* __restrict__ hout, double2* __restrict__ acc,
               float2* __restrict__ d32, TiledArgs a, int* __restrict__ err) {
  extern __shared__ unsigned char smraw[];
  unsigned char* base = tma_area(smraw);
  tma_init_barriers<MODE, PER>(base);
  uint32_t pmask = 0, amask = 0;
  tma_body<MODE, PER>(maps, hout, acc, d32, a, err, blockIdx.x, blockIdx.y, blockIdx.z, base, pmask, amask);
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

bool make_tma_map(CUtensorMap* m, const void* base, bool f32, const GridInfo& g, int norb, int box0, int box1) {
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
  if (!make_tma_map(&maps.in, L.in, in32, g, norb, 2 * SXv, per ? TY : TY + 2 * HALO)) return SB200_ERR_UNSUPPORTED;
  if (per && !make_tma_map(&maps.inh, L.in, in32, g, norb, 2 * TX, HALO)) return SB200_ERR_UNSUPPORTED;
  const bool acc64 = (L.mode == 2 || L.mode == 3 || L.mode == 8);
  const bool rd32 = (L.mode == 7 || L.mode == 8);
  if (acc64 && !make_tma_map(&maps.acc, L.out, false, g, norb, 2 * TX, TY)) return SB200_ERR_UNSUPPORTED;
  if (rd32 && !make_tma_map(&maps.d32, L.d32, true, g, norb, 2 * TX, TY)) return SB200_ERR_UNSUPPORTED;
  TiledArgs a = make_tiled_args(c, L.zc);
  const int ntiles = ((g.nx + TX - 1) / TX) * ((g.ny + TY - 1) / TY);
  // z chunks: the count that minimises waves x planes per CTA (each chunk
  // re-reads 8 halo planes), with the CTAs that fit on the GPU at once
  const long ctas = (long)ntiles * norb;
  int sms = 148;
  SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const long slots = (long)sms * ((L.mode >= 6) ? 3 : 2);
  int nchunk = 1;
  double best = 0.0;
  for (int n = 1; n <= 16 && (n == 1 || g.nz / n >= 8); ++n) {
    const int zc = (g.nz + n - 1) / n;
    const int nzc_n = (g.nz + zc - 1) / zc;
    const double cost = (double)((ctas * nzc_n + slots - 1) / slots) * (zc + 2 * HALO);
    if (n == 1 || cost < best) {
      best = cost;
      nchunk = n;
    }
  }
  a.zchunk = (g.nz + nchunk - 1) / nchunk;
  const int nzc = (g.nz + a.zchunk - 1) / a.zchunk;
  dim3 grid(ntiles, nzc, norb);
  return per ? launch_mode<true>(c, maps, L, a, grid) : launch_mode<false>(c, maps, L, a, grid);
}

}  // namespace sb200
