// sb200_eigh.cu -- symmetric eigen-decomposition on the GPU in FP64 for the
// subspace diagonalisation of the ground state (the dsyev call of
// eigen_subdiag_lapack.f90:23-38, used by ssdg, subspace_diagonalization.f90).
//
// One CTA, in three stages, restating the published Householder-QL method
// (Householder reduction to tridiagonal form, accumulation of the
// reflections, implicit-shift QL iterations on the tridiagonal matrix with
// the rotations applied to the eigenvector matrix; Wilkinson and Reinsch,
// the tred2 / tql2 procedures), which is the scheme of LAPACK's dsyev:
//   1. A = Q T Q^T: for k = 0 .. n-3 the reflection H_k = I - tau v v^T that
//      zeroes column k below the subdiagonal; the trailing block is updated
//      by the symmetric rank-2 form B <- B - v w^T - w v^T with
//      p = tau B v, w = p - (tau / 2)(v.p) v.  All threads share each step:
//      reductions in shared memory, the matrix in global memory (L2).
//   2. Z = H_0 H_1 ... H_{n-3}, by applying the reflections to the identity
//      in reverse order.
//   3. QL sweeps: one thread computes each sweep's rotation sequence (a
//      chain of scalar recurrences), every thread then applies the whole
//      sequence to its own rows of Z.
// Eigenvalues ascending, eigenvectors as columns with their largest-magnitude
// component positive (the first one on a tie).  Loops are bounded: a
// tridiagonal eigenvalue that has not converged after 60 sweeps sets *info.
#include <cuda_runtime.h>

#include "sb200_internal.cuh"

namespace sb200 {
namespace {

constexpr int ET = 512;  // threads of the eigensolver CTA

__device__ __forceinline__ double block_sum(double v, double* red) {
  // fixed-order tree over the CTA (warp butterfly, then warps in order)
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();  // red may still be read by the previous call
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < ET / 32; ++w) s += red[w];
  return s;
}

// M: n x n, row-major <psi_i|H psi_j> (its upper triangle is used, as dsyev
// with uplo = 'U').  A: n x n work (column-major).  V: eigenvectors, V[i n + k]
// = component k of eigenvector i.  w: eigenvalues.  sm: 5 n doubles.
__global__ void __launch_bounds__(ET, 1) k_eigh(const double* __restrict__ M, int n, double* __restrict__ A,
                                                double* __restrict__ Z, double* __restrict__ V,
                                                double* __restrict__ w, int* __restrict__ info) {
  extern __shared__ double sm[];
  double* d = sm;          // [n] diagonal
  double* e = d + n;       // [n] subdiagonal e[i] = T(i+1, i), e[n-1] = 0
  double* tau = e + n;     // [n] reflection factors
  double* rc = tau + n;    // [n] rotation cosines of one QL sweep
  double* rs = rc + n;     // [n] rotation sines
  __shared__ double red[ET / 32];
  __shared__ double sc[4];
  __shared__ int lm[2];
  const int t = threadIdx.x;
  auto a = [&](int i, int j) -> double& { return A[i + (long)n * j]; };
  auto z = [&](int i, int j) -> double& { return Z[i + (long)n * j]; };
  for (long q = t; q < (long)n * n; q += ET) {
    const int i = (int)(q % n), j = (int)(q / n);
    A[q] = (i <= j) ? M[(long)i * n + j] : M[(long)j * n + i];
  }
  if (t == 0) *info = 0;
  __syncthreads();
  // ---- 1. tridiagonal form ----
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // length of the column below the diagonal
    double s2 = 0.0;
    for (int i = 1 + t; i < m; i += ET) s2 += a(k + 1 + i, k) * a(k + 1 + i, k);
    const double tail = block_sum(s2, red);
    const double x0 = a(k + 1, k);
    if (tail == 0.0) {  // already tridiagonal in this column
      if (t == 0) {
        tau[k] = 0.0;
        e[k] = x0;
      }
      __syncthreads();
      continue;
    }
    const double alpha = -copysign(sqrt(x0 * x0 + tail), x0);
    const double v0 = x0 - alpha;
    const double tk = 2.0 / (v0 * v0 + tail);
    __syncthreads();
    if (t == 0) {
      a(k + 1, k) = v0;  // v stored in column k below the diagonal: v = (v0, x1, x2, ...)
      tau[k] = tk;
      e[k] = alpha;
    }
    __syncthreads();
    // p = tau B v over the trailing block B = A(k+1.., k+1..); kept in column k
    // of the upper triangle, A(k, k+1+i) (unused from here on)
    for (int i = t; i < m; i += ET) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += a(k + 1 + i, k + 1 + j) * a(k + 1 + j, k);
      a(k, k + 1 + i) = tk * s;
    }
    __syncthreads();
    double vp = 0.0;
    for (int i = t; i < m; i += ET) vp += a(k + 1 + i, k) * a(k, k + 1 + i);
    const double K = 0.5 * tk * block_sum(vp, red);
    for (int i = t; i < m; i += ET) a(k, k + 1 + i) -= K * a(k + 1 + i, k);  // w
    __syncthreads();
    for (long q = t; q < (long)m * m; q += ET) {
      const int i = (int)(q % m), j = (int)(q / m);
      a(k + 1 + i, k + 1 + j) -= a(k + 1 + i, k) * a(k, k + 1 + j) + a(k, k + 1 + i) * a(k + 1 + j, k);
    }
    __syncthreads();
  }
  for (int i = t; i < n; i += ET) {
    d[i] = a(i, i);
    if (i == n - 2) e[i] = a(n - 1, n - 2);
    if (i == n - 1) e[i] = 0.0;
  }
  if (t == 0 && n >= 2) tau[n - 2] = 0.0;
  // ---- 2. Z = H_0 ... H_{n-3} ----
  for (long q = t; q < (long)n * n; q += ET) Z[q] = (q % n == q / n) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = n - 3; k >= 0; --k) {
    if (tau[k] == 0.0) continue;
    const int m = n - k - 1;
    // u_j = v . Z(k+1.., k+1+j), kept in row k of Z (its entries right of the
    // diagonal are still those of the identity: zero)
    for (int j = t; j < m; j += ET) {
      double s = 0.0;
      for (int i = 0; i < m; ++i) s += a(k + 1 + i, k) * z(k + 1 + i, k + 1 + j);
      z(k, k + 1 + j) = s;
    }
    __syncthreads();
    const double tk = tau[k];
    for (long q = t; q < (long)m * m; q += ET) {
      const int i = (int)(q % m), j = (int)(q / m);
      z(k + 1 + i, k + 1 + j) -= tk * a(k + 1 + i, k) * z(k, k + 1 + j);
    }
    __syncthreads();
    for (int j = t; j < m; j += ET) z(k, k + 1 + j) = 0.0;
    __syncthreads();
  }
  // ---- 3. implicit QL on (d, e), rotations applied to Z ----
  double f = 0.0, tst1 = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    while (true) {
      if (t == 0) {
        tst1 = fmax(tst1, fabs(d[l]) + fabs(e[l]));
        int mm = l;
        while (mm < n - 1 && tst1 + fabs(e[mm]) != tst1) ++mm;
        lm[0] = mm;
        lm[1] = 0;
        if (mm > l) {
          if (++iter > 60) {
            *info = 1;
            lm[0] = l;  // give up on this eigenvalue
          } else {
            // one QL sweep with the Wilkinson-type shift from the leading 2x2
            double g = d[l];
            double p = (d[l + 1] - g) / (2.0 * e[l]);
            double r = hypot(p, 1.0);
            d[l] = e[l] / (p + copysign(r, p));
            d[l + 1] = e[l] * (p + copysign(r, p));
            const double dl1 = d[l + 1];
            double h = g - d[l];
            for (int i = l + 2; i < n; ++i) d[i] -= h;
            f += h;
            p = d[mm];
            double c = 1.0, c2 = 1.0, c3 = 1.0, s = 0.0, s2 = 0.0;
            const double el1 = e[l + 1];
            for (int i = mm - 1; i >= l; --i) {
              c3 = c2;
              c2 = c;
              s2 = s;
              g = c * e[i];
              h = c * p;
              r = hypot(p, e[i]);
              e[i + 1] = s * r;
              s = e[i] / r;
              c = p / r;
              p = c * d[i] - s * g;
              d[i + 1] = h + s * (c * g + s * d[i]);
              rc[i] = c;
              rs[i] = s;
            }
            p = -s * s2 * c3 * el1 * e[l] / dl1;
            e[l] = s * p;
            d[l] = c * p;
            lm[1] = 1;
          }
        }
        sc[0] = f;
        sc[1] = tst1;
      }
      __syncthreads();
      const int mm = lm[0], swept = lm[1];
      f = sc[0];
      tst1 = sc[1];
      if (swept) {  // the sweep's rotations on every row of Z, in the sweep's order
        for (int row = t; row < n; row += ET) {
          for (int i = mm - 1; i >= l; --i) {
            const double c = rc[i], s = rs[i];
            const double zi = z(row, i), zi1 = z(row, i + 1);
            z(row, i + 1) = s * zi + c * zi1;
            z(row, i) = c * zi - s * zi1;
          }
        }
      }
      __syncthreads();
      if (!swept) break;
    }
    if (t == 0) {
      d[l] += f;
      e[l] = 0.0;
    }
    __syncthreads();
  }
  // ---- ascending order, sign convention, output ----
  for (int col = t; col < n; col += ET) {
    // rank of eigenvalue col (ties by index)
    int rank = 0;
    for (int j = 0; j < n; ++j) rank += (d[j] < d[col] || (d[j] == d[col] && j < col)) ? 1 : 0;
    int im = 0;
    for (int k = 1; k < n; ++k)
      if (fabs(z(k, col)) > fabs(z(im, col))) im = k;
    const double sg = z(im, col) < 0.0 ? -1.0 : 1.0;
    for (int k = 0; k < n; ++k) V[(long)rank * n + k] = sg * z(k, col);
    w[rank] = d[col];
  }
}

}  // namespace

// Eigenvalues (ascending) and eigenvectors of the symmetric n x n matrix whose
// upper triangle M holds (row-major), on c's stream.  work: 2 n^2 doubles.
// V[i n + k] = component k of eigenvector i.  info: device int (0, or 1 when
// the QL iterations did not converge).
int launch_eigh(sb200_ctx* c, const double* M, int n, double* work, double* V, double* w, int* info) {
  if (n < 1) return set_error(SB200_ERR_INVALID_ARG, "eigensolver: n < 1");
  const size_t smem = 5 * (size_t)n * sizeof(double);
  if (smem > 200 * 1024) return set_error(SB200_ERR_UNSUPPORTED, "eigensolver: matrix larger than 5120 x 5120");
  static bool attr = false;
  if (!attr) {
    SB_CUDA(cudaFuncSetAttribute(k_eigh, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  k_eigh<<<1, ET, smem, c->stream>>>(M, n, work, work + (size_t)n * n, V, w, info);
  SB_LAUNCH_CHECK("k_eigh");
  return SB200_OK;
}

}  // namespace sb200
