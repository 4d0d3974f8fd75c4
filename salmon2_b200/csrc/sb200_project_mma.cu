// sb200_project_mma.cu -- Kleinman-Bylander projections on the FP64 tensor
// cores (DMMA, mma.sync m8n8k4 f64) for grids whose orbitals of one k-point
// give the contraction a real orbital dimension (the supercell: 256 per k).
//
// P(o, lma) = rinv(lma) sum_j conj(zekr_uV(j, lma)) psi_o(r_j)
// (nonlocal_potential.f90:358-367), per atom and k-point, as one real GEMM
// over a tile of 16 orbitals:
//   C (16 x 8) = A (16 x 2K) B (2K x 8),
//   A[o][2j + c] = (Re, Im)_c psi_o(r_j)            (the gathered sphere values)
//   B[2j][q] = Re w_qj, B[2j + 1][q] = -Im w_qj      (columns 0..3: Re P_q)
//   B[2j][4 + q] = Im w_qj, B[2j + 1][4 + q] = Re w_qj  (columns 4..7: Im P_q)
// with w_qj = exp(i (k+A).r_j) uV(j, q) = conj(zekr_uV(j, q)), K = sphere
// points (padded to a multiple of 2), q the atom's (at most 4) projectors.
// One CTA of 64 threads per (atom, 16-orbital tile, k-point): the sphere
// values of its 16 orbitals are gathered from HBM by cp.async straight into
// the A tile (16-byte copies, the complex value's two doubles side by side;
// FP32 input: 8-byte copies, widened in place after the wait),
// the B tile is built from the k-point's phases and uV, and each warp runs
// the K/4 DMMA steps of one 8-orbital half.  Row strides of both tiles are
// 12 modulo 16 doubles, so the fragment loads of a half-warp hit 16
// different 8-byte bank pairs.  The products are summed by the tensor core
// in the fixed order of the k steps: deterministic.
#include <cuda_runtime.h>

#include <cstdint>

#include "sb200_bodies.cuh"
#include "sb200_internal.cuh"

namespace sb200 {
namespace {

constexpr int MT = 16;   // orbitals per CTA
constexpr int PT = 64;   // threads per CTA

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// D = A B + C for one 8x8x4 FP64 tile (A row-major fragment: element
// (lane / 4, lane % 4); B column-major fragment: element (lane % 4, lane / 4);
// C / D: elements (lane / 4, 2 (lane % 4)) and (lane / 4, 2 (lane % 4) + 1))
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <typename TIN>
__global__ void __launch_bounds__(PT) k_project_dmma(const TIN* __restrict__ in, double2* __restrict__ proj,
                                                     body::ProjArgs a, int stride) {
  extern __shared__ __align__(16) double sm[];
  double* As = sm;                  // [MT][stride]
  double* Bs = sm + MT * stride;    // [8][stride]
  const int atom = blockIdx.x;
  const int ik = blockIdx.z;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int start = __ldg(a.atom_start + atom), m = __ldg(a.mps + atom);
  const int lma0 = __ldg(a.lma_start + atom), np = __ldg(a.nproj + atom);
  const int kp = (2 * m + 3) & ~3;  // K of the GEMM, padded to the k step
  const int o0 = ik * a.nspin_no + blockIdx.y * MT;
  const int nrow = min(MT, a.nspin_no - blockIdx.y * MT);
  // A: the sphere values of the tile's orbitals (zero rows past the k-point's
  // orbitals, zero columns past the sphere)
  // each thread owns sphere points j = t, t + 64, ...: one load of the point
  // index, then the copies of that point for all 16 orbitals back to back
  for (int j = t; j < m; j += PT) {
    const TIN* src = in + (long)o0 * a.npts + __ldg(a.pt_lin + start + j);
#pragma unroll
    for (int r = 0; r < MT; ++r) {
      double* dst = As + r * stride + 2 * j;
      if (r < nrow) {
        // FP64: the value itself; FP32: its 8 bytes into the first slot,
        // widened in place by the same thread after the wait below
        if (sizeof(TIN) == 16) cp_async16(dst, src + (long)r * a.npts);
        else cp_async8(dst, src + (long)r * a.npts);
      } else {
        dst[0] = 0.0;
        dst[1] = 0.0;
      }
    }
  }
  for (int i = t; i < MT * (kp - 2 * m); i += PT) {
    const int r = i / (kp - 2 * m), c = 2 * m + i % (kp - 2 * m);
    As[r * stride + c] = 0.0;
  }
  // B: the k-point's weights w_qj = exp(i (k+A).r_j) uV(j, q)
  const double2* ph = a.phase + (a.phase_per_k ? (long)ik * a.totpts : 0L) + start;
  for (int j = t; j < kp / 2; j += PT) {
    const double2 e = j < m ? __ldg(ph + j) : make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double u = (j < m && q < np) ? __ldg(a.uv + (long)(lma0 + q) * a.nps + j) : 0.0;
      const double wr = u * e.x, wi = u * e.y;
      Bs[q * stride + 2 * j] = wr;
      Bs[q * stride + 2 * j + 1] = -wi;
      Bs[(4 + q) * stride + 2 * j] = wi;
      Bs[(4 + q) * stride + 2 * j + 1] = wr;
    }
  }
  cp_async_wait_all();
  if (sizeof(TIN) == 8) {  // each thread widens the FP32 values it copied
    for (int j = t; j < m; j += PT)
      for (int r = 0; r < nrow; ++r) {
        double* dst = As + r * stride + 2 * j;
        const float2 v = *reinterpret_cast<const float2*>(dst);
        dst[0] = (double)v.x;
        dst[1] = (double)v.y;
      }
  }
  __syncthreads();
  // each warp: rows 8 warp .. 8 warp + 7 of C over all k steps
  double d0 = 0.0, d1 = 0.0;
  const double* ap = As + (8 * warp + (lane >> 2)) * stride + (lane & 3);
  const double* bp = Bs + (lane >> 2) * stride + (lane & 3);
#pragma unroll 4
  for (int k = 0; k < kp; k += 4) dmma_8x8x4(d0, d1, ap[k], bp[k]);
  // lanes with lane % 4 in {0, 1} hold Re P of projectors 2 (lane % 4) + {0, 1};
  // the matching Im P sits two lanes up
  const double i0 = __shfl_down_sync(0xffffffffu, d0, 2);
  const double i1 = __shfl_down_sync(0xffffffffu, d1, 2);
  const int r = 8 * warp + (lane >> 2);
  if ((lane & 3) < 2 && r < nrow) {
    const int q0 = 2 * (lane & 3);
    double2* dst = proj + (long)(o0 + r) * a.nlma + lma0;
    if (q0 < np) dst[q0] = make_double2(__ldg(a.rinv + lma0 + q0) * d0, __ldg(a.rinv + lma0 + q0) * i0);
    if (q0 + 1 < np)
      dst[q0 + 1] = make_double2(__ldg(a.rinv + lma0 + q0 + 1) * d1, __ldg(a.rinv + lma0 + q0 + 1) * i1);
  }
}

}  // namespace

// Row stride (doubles) of the tiles for spheres of at most nps points, or 0
// when the tensor-core form does not apply (more than 4 projectors on an
// atom, or tiles larger than the shared memory).
int project_dmma_stride(const sb200_ctx* c) {
  const PPInfo& p = c->pp;
  if (p.nlma <= 0 || p.nprojmax > 4 || p.nps <= 0) return 0;
  const int kp = (2 * p.nps + 3) & ~3;
  const int stride = kp + ((12 - kp % 16) + 16) % 16;
  if ((size_t)(MT + 8) * stride * sizeof(double) > 160 * 1024) return 0;
  return stride;
}

int launch_project_dmma(sb200_ctx* c, const void* in, double2* proj, bool in32) {
  const int stride = project_dmma_stride(c);
  if (stride == 0) return SB200_ERR_UNSUPPORTED;
  const size_t smem = (size_t)(MT + 8) * stride * sizeof(double);
  static bool attr = false;
  if (!attr) {
    SB_CUDA(cudaFuncSetAttribute(k_project_dmma<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SB_CUDA(cudaFuncSetAttribute(k_project_dmma<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    attr = true;
  }
  const body::ProjArgs a = make_proj_args(c);
  const int nk = c->orb.norb / a.nspin_no;
  dim3 grid(a.natom, (a.nspin_no + MT - 1) / MT, nk);
  if (in32) k_project_dmma<float2><<<grid, PT, smem, c->stream>>>((const float2*)in, proj, a, stride);
  else k_project_dmma<double2><<<grid, PT, smem, c->stream>>>((const double2*)in, proj, a, stride);
  SB_LAUNCH_CHECK("k_project_dmma");
  return SB200_OK;
}

}  // namespace sb200
