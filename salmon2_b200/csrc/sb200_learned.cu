// sb200_learned.cu -- learned 3-D convolutional preconditioner for the
// ground-state CG: forward / backward kernels, Adam, and the CG hook.
//
// Network (per orbital, on the real-space grid, zero padding = the isolated
// grid's Dirichlet boundary):
//   x0 = [g / rms(g), V_local]                  2 channels
//   x1 = relu(conv3(x0; W1, b1))                C channels
//   x2 = relu(conv3(x1; W2, b2))                C channels
//   y  = conv3(x2; W3, b3)                      1 channel
//   corr  = rms(g) * y, minus its components along the current orbitals
//   p     = lowpass(g) + corr                   (lowpass = preconditioning.f90:25-77)
//   pre_g = +p or -p, whichever keeps <pre_g, g> >= <lowpass(g), g> / 5,
//           else lowpass(g) (k_apply_direction)
// conv3 is a 3x3x3 convolution.  Weights are kept as FP32 masters and used as
// BF16 in the forward pass, with FP32 accumulation; gradients and Adam are FP32.
// The last layer starts at zero, so the untrained network is the reference's
// low-pass preconditioner.
//
// Loss for training samples (input g, V; offset lowpass(g)/rms(g); target
// direction t): the misalignment 1 - <p,t>^2 / (<p,p><t,t>) of the
// preconditioned direction p = offset + y with t, summed over the batch; t is
// minus the part of the CG iterate outside the converged occupied subspace
// (the training driver, salmon2_b200/learned.py, forms it).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "sb200_internal.cuh"

#define TRY_L(x)                    \
  do {                              \
    int _r = (x);                   \
    if (_r != SB200_OK) return _r;  \
  } while (0)

namespace sb200 {
namespace {

constexpr int C = SB200_LEARNED_CHANNELS;  // hidden channels
constexpr int K3 = 27;
constexpr int NW1 = C * 2 * K3, NB1 = C;
constexpr int NW2 = C * C * K3, NB2 = C;
constexpr int NW3 = 1 * C * K3, NB3 = 1;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NW1, OFF_W2 = OFF_B1 + NB1, OFF_B2 = OFF_W2 + NW2;
constexpr int OFF_W3 = OFF_B2 + NB2, OFF_B3 = OFF_W3 + NW3, NPARAM = OFF_B3 + NB3;
static_assert(NPARAM == SB200_LEARNED_NPARAM, "parameter count mismatch");

struct Net {
  int nx = 0, ny = 0, nz = 0;
  long npts = 0;
  int cap_batch = 0;
  float* d_w = nullptr;       // FP32 master parameters [NPARAM]
  __nv_bfloat16* d_wb = nullptr;  // BF16 copy used by the forward pass
  float* d_g = nullptr;       // gradients [NPARAM]
  float *d_m = nullptr, *d_v = nullptr;  // Adam moments
  long adam_t = 0;
  // activations for a batch: x0 [B][2][n], a1/x1 [B][C][n], a2/x2 [B][C][n], y [B][n]
  float *x0 = nullptr, *a1 = nullptr, *a2 = nullptr, *y = nullptr;
  float *gx1 = nullptr, *gx2 = nullptr, *gy = nullptr;  // gradient buffers
  float* tgt = nullptr;       // device copy of the training targets [B][n]
  float* off = nullptr;       // device copy of the prediction offsets [B][n]
  double* d_red = nullptr;    // reductions
  float* d_wpart = nullptr;   // weight-gradient partials
  long wpart_cap = 0;
  float* d_scale = nullptr;   // per-orbital rms(g)
  double* d_dots = nullptr;   // CG hook: per-orbital <pre, g> partials [norb][32][2]
  double* d_corr = nullptr;   // CG hook: network corrections of all orbitals [norb][npts]
  size_t corr_cap = 0;
};

// ---- conv forward: out[co][p] = b[co] + sum_ci sum_k W[co][ci][k] in[ci][p+k] ----
template <int CIN, int COUT, bool RELU>
__global__ void __launch_bounds__(256) k_conv_fwd(const float* __restrict__ in, float* __restrict__ pre,
                                                  float* __restrict__ out, const __nv_bfloat16* __restrict__ W,
                                                  const float* __restrict__ bias, int nx, int ny, int nz, long npts) {
  __shared__ float Ws[COUT * CIN * K3];
  for (int i = threadIdx.x; i < COUT * CIN * K3; i += blockDim.x) Ws[i] = __bfloat162float(W[i]);
  __syncthreads();
  const int b = blockIdx.y;
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= npts) return;
  const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = bias[co];
  const float* src = in + (long)b * CIN * npts;
  for (int k = 0; k < K3; ++k) {
    const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    const int xx = x + dx, yy = y + dy, zz = z + dz;
    if (xx < 0 || xx >= nx || yy < 0 || yy >= ny || zz < 0 || zz >= nz) continue;
    const long q = p + dx + (long)dy * nx + (long)dz * nx * ny;
#pragma unroll 4
    for (int ci = 0; ci < CIN; ++ci) {
      const float v = src[(long)ci * npts + q];
#pragma unroll
      for (int co = 0; co < COUT; ++co) acc[co] += Ws[(co * CIN + ci) * K3 + k] * v;
    }
  }
#pragma unroll
  for (int co = 0; co < COUT; ++co) {
    const long i = ((long)b * COUT + co) * npts + p;
    if (pre) pre[i] = acc[co];
    out[i] = RELU ? fmaxf(acc[co], 0.0f) : acc[co];
  }
}

// ---- conv backward (input): gin[ci][p] = sum_co sum_k W[co][ci][k] gout[co][p-k] ----
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_conv_bwd_in(const float* __restrict__ gout, float* __restrict__ gin,
                                                     const __nv_bfloat16* __restrict__ W, const float* __restrict__ pre,
                                                     int nx, int ny, int nz, long npts) {
  __shared__ float Ws[COUT * CIN * K3];
  for (int i = threadIdx.x; i < COUT * CIN * K3; i += blockDim.x) Ws[i] = __bfloat162float(W[i]);
  __syncthreads();
  const int b = blockIdx.y;
  const long p = blockIdx.x * 256L + threadIdx.x;
  if (p >= npts) return;
  const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((long)nx * ny));
  float acc[CIN];
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.0f;
  const float* g = gout + (long)b * COUT * npts;
  for (int k = 0; k < K3; ++k) {
    const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    const int xx = x - dx, yy = y - dy, zz = z - dz;
    if (xx < 0 || xx >= nx || yy < 0 || yy >= ny || zz < 0 || zz >= nz) continue;
    const long q = p - dx - (long)dy * nx - (long)dz * nx * ny;
#pragma unroll 4
    for (int co = 0; co < COUT; ++co) {
      const float v = g[(long)co * npts + q];
#pragma unroll
      for (int ci = 0; ci < CIN; ++ci) acc[ci] += Ws[(co * CIN + ci) * K3 + k] * v;
    }
  }
  // gradient through the ReLU of the layer that produced the input
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) {
    const long i = ((long)b * CIN + ci) * npts + p;
    gin[i] = (pre == nullptr || pre[i] > 0.0f) ? acc[ci] : 0.0f;
  }
}

// ---- conv backward (weights) ----
// G[co][ci][k] = sum_b sum_p gout[b][co][p] * in[b][ci][p + off_k], bias[co] =
// sum gout[b][co][p].  Work item = 32 consecutive x points of one (b, z, y)
// row; the 3 x 3 x 34 input box and the 32-point gout row are staged in
// shared memory; thread = (co, ci) pair with 27 accumulators.  Each CTA
// writes its partial sums; k_sum_parts adds them in CTA order.
constexpr int WROW = 32;
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_conv_bwd_w(const float* __restrict__ in, const float* __restrict__ gout,
                                                    float* __restrict__ part, int nx, int ny, int nz, long npts,
                                                    int batch) {
  constexpr int NP = CIN * COUT;
  constexpr int NWL = NP * K3 + COUT;
  __shared__ float box[CIN][3][3][WROW + 2];
  __shared__ float grow[COUT][WROW];
  const int nxc = (nx + WROW - 1) / WROW;
  const long items = (long)batch * nz * ny * nxc;
  float acc[K3];
#pragma unroll
  for (int k = 0; k < K3; ++k) acc[k] = 0.0f;
  float bacc = 0.0f;
  const int pair = threadIdx.x;
  const int co = pair / CIN, ci = pair % CIN;
  for (long it = blockIdx.x; it < items; it += gridDim.x) {
    const int xc = (int)(it % nxc);
    const int y = (int)((it / nxc) % ny);
    const int z = (int)((it / ((long)nxc * ny)) % nz);
    const int b = (int)(it / ((long)nxc * ny * nz));
    const int x0 = xc * WROW;
    __syncthreads();
    for (int c = threadIdx.x; c < CIN * 9 * (WROW + 2); c += blockDim.x) {
      const int xx = c % (WROW + 2), dy = (c / (WROW + 2)) % 3, dz = (c / (3 * (WROW + 2))) % 3,
                cc = c / (9 * (WROW + 2));
      const int gx = x0 + xx - 1, gy = y + dy - 1, gz = z + dz - 1;
      float v = 0.0f;
      if (gx >= 0 && gx < nx && gy >= 0 && gy < ny && gz >= 0 && gz < nz)
        v = in[((long)b * CIN + cc) * npts + gx + (long)gy * nx + (long)gz * nx * ny];
      box[cc][dz][dy][xx] = v;
    }
    for (int c = threadIdx.x; c < COUT * WROW; c += blockDim.x) {
      const int xx = c % WROW, oc = c / WROW;
      const int gx = x0 + xx;
      grow[oc][xx] = (gx < nx) ? gout[((long)b * COUT + oc) * npts + gx + (long)y * nx + (long)z * nx * ny] : 0.0f;
    }
    __syncthreads();
    if (pair < NP) {
      for (int xx = 0; xx < WROW; ++xx) {
        const float gv = grow[co][xx];
#pragma unroll
        for (int k = 0; k < K3; ++k) acc[k] += gv * box[ci][k / 9][(k / 3) % 3][xx + k % 3];
        if (ci == 0) bacc += gv;
      }
    }
  }
  if (pair < NP) {
#pragma unroll
    for (int k = 0; k < K3; ++k) part[(long)blockIdx.x * NWL + (co * CIN + ci) * K3 + k] = acc[k];
    if (ci == 0) part[(long)blockIdx.x * NWL + NP * K3 + co] = bacc;
  }
}

__global__ void k_sum_parts(const float* __restrict__ part, int nchunk, int nw, float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < nchunk; ++c) s += part[(long)c * nw + i];
    out[i] = s;
  }
}

// ---- loss: per batch item dots <p,t>, <p,p>, <t,t> (FP64, deterministic) ----
__global__ void __launch_bounds__(256) k_loss_dots(const float* __restrict__ y, const float* __restrict__ off,
                                                   const float* __restrict__ t, long npts, double* __restrict__ part,
                                                   int nblk) {
  __shared__ double red[3][256];
  const int b = blockIdx.y;
  double s[3] = {0.0, 0.0, 0.0};
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)nblk * 256) {
    const double a = (double)y[(long)b * npts + p] + (off ? (double)off[(long)b * npts + p] : 0.0);
    const double c = t[(long)b * npts + p];
    s[0] += a * c;
    s[1] += a * a;
    s[2] += c * c;
  }
  for (int k = 0; k < 3; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[((long)b * nblk + blockIdx.x) * 3 + threadIdx.x] = red[threadIdx.x][0];
}

// dL/dy for L = sum_b 1 - pt^2 / (pp tt): -2 pt/(pp tt) t + 2 pt^2/(pp^2 tt) y
__global__ void k_loss_grad(const float* __restrict__ y, const float* __restrict__ off, const float* __restrict__ t,
                            long npts, const double* __restrict__ part, int nblk, float* __restrict__ gy,
                            double* __restrict__ loss) {
  const int b = blockIdx.y;
  double pt = 0.0, pp = 0.0, tt = 0.0;
  for (int k = 0; k < nblk; ++k) {
    pt += part[((long)b * nblk + k) * 3 + 0];
    pp += part[((long)b * nblk + k) * 3 + 1];
    tt += part[((long)b * nblk + k) * 3 + 2];
  }
  pp = pp > 1e-300 ? pp : 1e-300;
  tt = tt > 1e-300 ? tt : 1e-300;
  const double ca = -2.0 * pt / (pp * tt), cb = 2.0 * pt * pt / (pp * pp * tt);
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)gridDim.x * 256) {
    const double pv = (double)y[(long)b * npts + p] + (off ? (double)off[(long)b * npts + p] : 0.0);
    gy[(long)b * npts + p] = (float)(ca * t[(long)b * npts + p] + cb * pv);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) loss[b] = 1.0 - pt * pt / (pp * tt);
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    m[i] = b1 * m[i] + (1.0f - b1) * g[i];
    v[i] = b2 * v[i] + (1.0f - b2) * g[i] * g[i];
    const float mh = m[i] / c1, vh = v[i] / c2;
    w[i] -= lr * mh / (sqrtf(vh) + eps);
  }
}

__global__ void k_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) wb[i] = __float2bfloat16(w[i]);
}

// CG hook: x0 for every orbital from g (FP64) and V; per-orbital rms first
__global__ void __launch_bounds__(256) k_rms_part(const double* __restrict__ g, long npts, double* __restrict__ part,
                                                  int nblk) {
  __shared__ double red[256];
  const int o = blockIdx.y;
  double s = 0.0;
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)nblk * 256) {
    const double v = g[(long)o * npts + p];
    s += v * v;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(long)o * nblk + blockIdx.x] = red[0];
}

__global__ void k_make_input(const double* __restrict__ g, const double* __restrict__ vloc, long npts,
                             const double* __restrict__ part, int nblk, int o0, float* __restrict__ x0,
                             float* __restrict__ scale) {
  const int b = blockIdx.y, o = o0 + b;
  double s = 0.0;
  for (int k = 0; k < nblk; ++k) s += part[(long)o * nblk + k];
  const double rms = sqrt(s / (double)npts);
  const double inv = rms > 0 ? 1.0 / rms : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[b] = (float)rms;
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)gridDim.x * 256) {
    x0[((long)b * 2 + 0) * npts + p] = (float)(g[(long)o * npts + p] * inv);
    x0[((long)b * 2 + 1) * npts + p] = (float)vloc[p];
  }
}

// corr(o) = rms(g_o) y_o for the orbitals o0 .. o0 + batch - 1
__global__ void k_store_corr(double* __restrict__ corr, const float* __restrict__ y, const float* __restrict__ scale,
                             long npts, int o0) {
  const int b = blockIdx.y;
  const double s = scale[b];
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)gridDim.x * 256)
    corr[(long)(o0 + b) * npts + p] = s * (double)y[(long)b * npts + p];
}

// Partial sums of d0 = <lowpass(g), g> and d1 = <corr, g> per orbital.
__global__ void __launch_bounds__(256) k_dir_dots_part(const double* __restrict__ pre, const double* __restrict__ g,
                                                       const double* __restrict__ corr, long npts,
                                                       double* __restrict__ part, int nblk) {
  __shared__ double r0[256], r1[256];
  const long o = blockIdx.y;
  double s0 = 0.0, s1 = 0.0;
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)nblk * 256) {
    const double gv = g[o * npts + p];
    s0 += pre[o * npts + p] * gv;
    s1 += corr[o * npts + p] * gv;
  }
  r0[threadIdx.x] = s0;
  r1[threadIdx.x] = s1;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      r0[threadIdx.x] += r0[threadIdx.x + st];
      r1[threadIdx.x] += r1[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[(o * nblk + blockIdx.x) * 2 + 0] = r0[0];
    part[(o * nblk + blockIdx.x) * 2 + 1] = r1[0];
  }
}

// The network direction p = lowpass(g) + corr is used only on the side of g
// that keeps <pre, g> clearly positive (the CG's conjugation coefficients are
// ratios of these products): with D = <p, g> and d0 = <lowpass(g), g>,
// pre = p if D >= d0 / 5, pre = -p if D <= -d0 / 5 (the same search line),
// else the low-pass direction alone.
__global__ void k_apply_direction(double* __restrict__ pre, const double* __restrict__ corr,
                                  const double* __restrict__ part, int nblk, long npts) {
  const long o = blockIdx.y;
  double d0 = 0.0, d1 = 0.0;
  for (int k = 0; k < nblk; ++k) {
    d0 += part[(o * nblk + k) * 2 + 0];
    d1 += part[(o * nblk + k) * 2 + 1];
  }
  const double D = d0 + d1;
  double sign;
  if (D >= 0.2 * d0) sign = 1.0;
  else if (D <= -0.2 * d0) sign = -1.0;
  else return;
  for (long p = blockIdx.x * 256L + threadIdx.x; p < npts; p += (long)gridDim.x * 256) {
    const long i = o * npts + p;
    pre[i] = sign * (pre[i] + corr[i]);
  }
}

int gsz(long n) {
  long b = (n + 255) / 256;
  if (b > 148L * 16) b = 148L * 16;
  return (int)(b < 1 ? 1 : b);
}

Net* net_of(sb200_ctx* c) { return (Net*)c->learned; }

int net_ensure(sb200_ctx* c, int batch) {
  Net* n = net_of(c);
  if (!n) {
    n = new Net();
    c->learned = n;
    // d_red holds the loss partials (batch * (64*3 + 1) <= 1024 * 193) and the
    // CG hook's rms partials (norb * 32 <= 65536)
    if (dalloc(&n->d_w, NPARAM) || dalloc(&n->d_wb, NPARAM) || dalloc(&n->d_g, NPARAM) || dalloc(&n->d_m, NPARAM) ||
        dalloc(&n->d_v, NPARAM) || dalloc(&n->d_red, (size_t)1024 * 193 + 65536) || dalloc(&n->d_scale, 4096) ||
        dalloc(&n->d_dots, (size_t)2048 * 32 * 2))
      return SB200_ERR_OOM;
    SB_CUDA(cudaMemset(n->d_w, 0, NPARAM * sizeof(float)));
    SB_CUDA(cudaMemset(n->d_m, 0, NPARAM * sizeof(float)));
    SB_CUDA(cudaMemset(n->d_v, 0, NPARAM * sizeof(float)));
    SB_CUDA(cudaDeviceSynchronize());
  }
  if (n->npts != c->g.npts || n->cap_batch < batch) {
    dfree(n->x0);
    dfree(n->a1);
    dfree(n->a2);
    dfree(n->y);
    dfree(n->gx1);
    dfree(n->gx2);
    dfree(n->gy);
    dfree(n->tgt);
    dfree(n->off);
    n->nx = c->g.nx;
    n->ny = c->g.ny;
    n->nz = c->g.nz;
    n->npts = c->g.npts;
    n->cap_batch = batch;
    const size_t np = (size_t)n->npts * batch;
    if (dalloc(&n->x0, 2 * np) || dalloc(&n->a1, 2 * (size_t)C * np) || dalloc(&n->a2, 2 * (size_t)C * np) ||
        dalloc(&n->y, np) || dalloc(&n->gx1, (size_t)C * np) || dalloc(&n->gx2, (size_t)C * np) ||
        dalloc(&n->gy, np) || dalloc(&n->tgt, np) || dalloc(&n->off, np))
      return SB200_ERR_OOM;
  }
  return SB200_OK;
}

// forward of `batch` items whose x0 is in n->x0; y into n->y
int net_forward(sb200_ctx* c, int batch) {
  Net* n = net_of(c);
  const long np = n->npts;
  float* x1 = n->a1 + (size_t)C * np * batch;  // post-activation halves
  float* x2 = n->a2 + (size_t)C * np * batch;
  dim3 g((unsigned)((np + 255) / 256), batch);
  k_conv_fwd<2, C, true><<<g, 256, 0, c->stream>>>(n->x0, n->a1, x1, n->d_wb + OFF_W1, n->d_w + OFF_B1, n->nx, n->ny,
                                                    n->nz, np);
  k_conv_fwd<C, C, true><<<g, 256, 0, c->stream>>>(x1, n->a2, x2, n->d_wb + OFF_W2, n->d_w + OFF_B2, n->nx, n->ny,
                                                    n->nz, np);
  k_conv_fwd<C, 1, false><<<g, 256, 0, c->stream>>>(x2, nullptr, n->y, n->d_wb + OFF_W3, n->d_w + OFF_B3, n->nx,
                                                     n->ny, n->nz, np);
  SB_LAUNCH_CHECK("k_conv_fwd");
  return SB200_OK;
}

template <int CIN, int COUT>
int weight_grad(sb200_ctx* c, const float* in, const float* gout, int batch, float* gdst) {
  static_assert(CIN * COUT <= 256, "one (co, ci) pair per thread");
  Net* n = net_of(c);
  constexpr int NWL = COUT * CIN * K3 + COUT;
  const long np = n->npts;
  const long items = (long)batch * n->nz * n->ny * ((n->nx + WROW - 1) / WROW);
  int nchunk = (int)(items < 296 ? items : 296);
  const long need = (long)nchunk * NWL;
  if (n->wpart_cap < need) {
    dfree(n->d_wpart);
    if (dalloc(&n->d_wpart, (size_t)need)) return SB200_ERR_OOM;
    n->wpart_cap = need;
  }
  k_conv_bwd_w<CIN, COUT><<<nchunk, 256, 0, c->stream>>>(in, gout, n->d_wpart, n->nx, n->ny, n->nz, np, batch);
  k_sum_parts<<<gsz(NWL), 256, 0, c->stream>>>(n->d_wpart, nchunk, NWL, gdst);
  SB_LAUNCH_CHECK("k_conv_bwd_w");
  return SB200_OK;
}

// loss and gradients for `batch` items (x0 and targets on the device)
int net_loss_grad(sb200_ctx* c, const float* off, const float* target, int batch, double* loss_host) {
  Net* n = net_of(c);
  const long np = n->npts;
  TRY_L(net_forward(c, batch));
  const int nblk = 64;
  dim3 gl(nblk, batch);
  k_loss_dots<<<gl, 256, 0, c->stream>>>(n->y, off, target, np, n->d_red, nblk);
  double* d_loss = n->d_red + (size_t)batch * nblk * 3;
  dim3 gg((unsigned)((np + 255) / 256 < 1024 ? (np + 255) / 256 : 1024), batch);
  k_loss_grad<<<gg, 256, 0, c->stream>>>(n->y, off, target, np, n->d_red, nblk, n->gy, d_loss);
  SB_LAUNCH_CHECK("loss");
  float* x1 = n->a1 + (size_t)C * np * batch;
  float* x2 = n->a2 + (size_t)C * np * batch;
  // layer 3
  TRY_L((weight_grad<C, 1>(c, x2, n->gy, batch, n->d_g + OFF_W3)));
  dim3 g((unsigned)((np + 255) / 256), batch);
  k_conv_bwd_in<C, 1><<<g, 256, 0, c->stream>>>(n->gy, n->gx2, n->d_wb + OFF_W3, n->a2, n->nx, n->ny, n->nz, np);
  // layer 2
  TRY_L((weight_grad<C, C>(c, x1, n->gx2, batch, n->d_g + OFF_W2)));
  k_conv_bwd_in<C, C><<<g, 256, 0, c->stream>>>(n->gx2, n->gx1, n->d_wb + OFF_W2, n->a1, n->nx, n->ny, n->nz, np);
  // layer 1
  TRY_L((weight_grad<2, C>(c, n->x0, n->gx1, batch, n->d_g + OFF_W1)));
  SB_LAUNCH_CHECK("backward");
  if (loss_host) {
    std::vector<double> l(batch);
    SB_CUDA(cudaMemcpyAsync(l.data(), d_loss, batch * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
    double s = 0.0;
    for (int b = 0; b < batch; ++b) s += l[b];
    *loss_host = s;
  }
  return SB200_OK;
}

}  // namespace

int learned_precond_apply(sb200_ctx* c, const double* g, const double* x, double* pre) {
  Net* n = net_of(c);
  if (!n) return set_error(SB200_ERR_STATE, "learned preconditioner weights not set");
  // lowpass part first (the untrained network adds nothing)
  const double alpha = 0.6;
  TRY_L(gs_precond(c, g, pre, alpha));
  const long np = c->g.npts;
  const int norb = c->orb.norb;
  const int nblk = 32;
  if ((long)norb * nblk > (1 << 16)) return set_error(SB200_ERR_BAD_SHAPE, "too many orbitals for the network hook");
  if (n->corr_cap < (size_t)norb * np) {
    dfree(n->d_corr);
    if (dalloc(&n->d_corr, (size_t)norb * np)) return SB200_ERR_OOM;
    n->corr_cap = (size_t)norb * np;
  }
  dim3 gr(nblk, norb);
  k_rms_part<<<gr, 256, 0, c->stream>>>(g, np, n->d_red, nblk);
  const int B = n->cap_batch > 0 ? n->cap_batch : 1;
  for (int o0 = 0; o0 < norb; o0 += B) {
    const int b = (o0 + B <= norb) ? B : norb - o0;
    dim3 gi((unsigned)((np + 255) / 256 < 1024 ? (np + 255) / 256 : 1024), b);
    k_make_input<<<gi, 256, 0, c->stream>>>(g, c->d_vloc, np, n->d_red, nblk, o0, n->x0, n->d_scale);
    TRY_L(net_forward(c, b));
    k_store_corr<<<gi, 256, 0, c->stream>>>(n->d_corr, n->y, n->d_scale, np, o0);
  }
  SB_LAUNCH_CHECK("k_store_corr");
  // the correction lives outside the occupied subspace: its parts along the
  // current orbitals are rotations within the subspace, not progress
  TRY_L(gs_project_out(c, x, norb, n->d_corr, norb));
  k_dir_dots_part<<<dim3(nblk, norb), 256, 0, c->stream>>>(pre, g, n->d_corr, np, n->d_dots, nblk);
  dim3 ga((unsigned)((np + 255) / 256 < 1024 ? (np + 255) / 256 : 1024), norb);
  k_apply_direction<<<ga, 256, 0, c->stream>>>(pre, n->d_corr, n->d_dots, nblk, np);
  SB_LAUNCH_CHECK("learned_precond_apply");
  return SB200_OK;
}

void learned_free(sb200_ctx* c) {
  Net* n = net_of(c);
  if (!n) return;
  dfree(n->d_w);
  dfree(n->d_wb);
  dfree(n->d_g);
  dfree(n->d_m);
  dfree(n->d_v);
  dfree(n->x0);
  dfree(n->a1);
  dfree(n->a2);
  dfree(n->y);
  dfree(n->gx1);
  dfree(n->gx2);
  dfree(n->gy);
  dfree(n->tgt);
  dfree(n->off);
  dfree(n->d_red);
  dfree(n->d_wpart);
  dfree(n->d_scale);
  dfree(n->d_dots);
  dfree(n->d_corr);
  delete n;
  c->learned = nullptr;
  c->learned_set = false;
}

}  // namespace sb200

using namespace sb200;

extern "C" {

int sb200_learned_init(sb200_ctx* c, const float* params, int nparam, int batch) {
  if (!c) return set_error(SB200_ERR_INVALID_ARG, "null ctx");
  if (!c->g.set) return set_error(SB200_ERR_STATE, "set the grid first");
  if (nparam != NPARAM) return set_error(SB200_ERR_INVALID_ARG, "parameter count must be SB200_LEARNED_NPARAM");
  if (batch < 1 || batch > 1024) return set_error(SB200_ERR_INVALID_ARG, "batch out of range");
  TRY_L(net_ensure(c, batch));
  Net* n = net_of(c);
  if (params) SB_CUDA(cudaMemcpy(n->d_w, params, NPARAM * sizeof(float), cudaMemcpyDefault));
  else SB_CUDA(cudaMemset(n->d_w, 0, NPARAM * sizeof(float)));
  SB_CUDA(cudaMemset(n->d_m, 0, NPARAM * sizeof(float)));
  SB_CUDA(cudaMemset(n->d_v, 0, NPARAM * sizeof(float)));
  SB_CUDA(cudaDeviceSynchronize());  // before kernels on the context's non-blocking stream
  n->adam_t = 0;
  k_to_bf16<<<gsz(NPARAM), 256, 0, c->stream>>>(n->d_w, n->d_wb, NPARAM);
  SB_LAUNCH_CHECK("k_to_bf16");
  SB_CUDA(cudaStreamSynchronize(c->stream));
  c->learned_set = true;
  return SB200_OK;
}

int sb200_learned_get_params(sb200_ctx* c, float* params, int nparam) {
  if (!c || !params || nparam != NPARAM) return set_error(SB200_ERR_INVALID_ARG, "bad argument");
  Net* n = net_of(c);
  if (!n) return set_error(SB200_ERR_STATE, "network not initialised");
  SB_CUDA(cudaStreamSynchronize(c->stream));
  SB_CUDA(cudaMemcpy(params, n->d_w, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return SB200_OK;
}

// forward for `batch` inputs x0 [batch][2][npts] (device) -> y [batch][npts] (device)
int sb200_learned_forward(sb200_ctx* c, const float* x0, float* y, int batch) {
  if (!c || !x0 || !y) return set_error(SB200_ERR_INVALID_ARG, "bad argument");
  Net* n = net_of(c);
  if (!n || batch > n->cap_batch) return set_error(SB200_ERR_STATE, "network not initialised for this batch");
  SB_CUDA(cudaMemcpyAsync(n->x0, x0, sizeof(float) * 2 * n->npts * batch, cudaMemcpyDefault, c->stream));
  TRY_L(net_forward(c, batch));
  SB_CUDA(cudaMemcpyAsync(y, n->y, sizeof(float) * n->npts * batch, cudaMemcpyDefault, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

// loss and parameter gradients (host arrays out) for one batch
int sb200_learned_loss_grad(sb200_ctx* c, const float* x0, const float* offset, const float* target, int batch,
                            double* loss, float* grad) {
  if (!c || !x0 || !target) return set_error(SB200_ERR_INVALID_ARG, "bad argument");
  Net* n = net_of(c);
  if (!n || batch > n->cap_batch) return set_error(SB200_ERR_STATE, "network not initialised for this batch");
  SB_CUDA(cudaMemcpyAsync(n->x0, x0, sizeof(float) * 2 * n->npts * batch, cudaMemcpyDefault, c->stream));
  SB_CUDA(cudaMemcpyAsync(n->tgt, target, sizeof(float) * n->npts * batch, cudaMemcpyDefault, c->stream));
  if (offset)
    SB_CUDA(cudaMemcpyAsync(n->off, offset, sizeof(float) * n->npts * batch, cudaMemcpyDefault, c->stream));
  TRY_L(net_loss_grad(c, offset ? n->off : nullptr, n->tgt, batch, loss));
  if (grad) {
    SB_CUDA(cudaMemcpyAsync(grad, n->d_g, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return SB200_OK;
}

// one Adam step on a batch (device inputs); loss (host) optional
int sb200_learned_train_step(sb200_ctx* c, const float* x0, const float* offset, const float* target, int batch,
                             float lr, double* loss) {
  if (!c || !x0 || !target) return set_error(SB200_ERR_INVALID_ARG, "bad argument");
  Net* n = net_of(c);
  if (!n || batch > n->cap_batch) return set_error(SB200_ERR_STATE, "network not initialised for this batch");
  SB_CUDA(cudaMemcpyAsync(n->x0, x0, sizeof(float) * 2 * n->npts * batch, cudaMemcpyDefault, c->stream));
  SB_CUDA(cudaMemcpyAsync(n->tgt, target, sizeof(float) * n->npts * batch, cudaMemcpyDefault, c->stream));
  if (offset)
    SB_CUDA(cudaMemcpyAsync(n->off, offset, sizeof(float) * n->npts * batch, cudaMemcpyDefault, c->stream));
  TRY_L(net_loss_grad(c, offset ? n->off : nullptr, n->tgt, batch, loss));
  n->adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)n->adam_t), c2 = 1.0f - powf(b2, (float)n->adam_t);
  k_adam<<<gsz(NPARAM), 256, 0, c->stream>>>(n->d_w, n->d_g, n->d_m, n->d_v, NPARAM, lr, b1, b2, 1e-8f, c1, c2);
  k_to_bf16<<<gsz(NPARAM), 256, 0, c->stream>>>(n->d_w, n->d_wb, NPARAM);
  SB_LAUNCH_CHECK("k_adam");
  if (!loss) SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

}  // extern "C"
