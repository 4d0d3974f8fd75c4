// sb200_poisson_cg.cu -- Hartree potential of an isolated system by conjugate
// gradients on the 25-point Laplacian with multipole boundary values
// (method_poisson = 'cg', the reference's default for isolated systems).
//
//   poisson_isolated_cg  src/poisson/poisson_isolated.f90:30-221
//   laplacian_poisson    src/poisson/poisson_isolated.f90:223-257
//   poisson_boundary     src/poisson/poisson_isolated.f90:259-690
//   make_corr_pole       src/poisson/init_poisson.f90:23-219 (layouts 2, 3)
//   set_ig_bound         src/poisson/init_poisson.f90:223-299 (face halos)
//   Ylm                  src/math/salmon_math.f90:386-426
//
// Boundary: the density is split into poles (layout 1: one pole at the origin;
// 2: one per atom, each grid point to its nearest atom; 3: box cells of about
// 8 A centred on their charge centroid), the moments
// rholm = sum r^l Ylm(r^) rho hvol of each pole are formed, and the four halo
// layers of the six faces get sum_pole sum_lm Ylm(r^) rholm / r^(l+1).
//
// CG: the reference's iteration (residual zk = -4 pi rho - lap(Vh with the
// boundary halo), then zero halos; ak = (zk.zk) / (zk.lap pk), Vh += ak pk,
// zk -= ak lap pk, stop when hvol zk.zk < threshold * N, pk = zk + ck pk).  Two
// launches per iteration: (A) forms pk = zk + ck pk_old at every point it reads
// (so the direction update needs no launch of its own), writes pk and lap pk
// and the partial sums of zk.lap pk; (B) updates Vh and zk and sums zk.zk.  The
// last block of each launch to finish sums the per-block partials in block
// order (fixed order: the result does not depend on timing) and writes the
// scalars for the next launch; the convergence test sets a device flag after
// which every later launch returns at once.  Called directly, the host checks
// the flag every PCG_CHUNK iterations; inside a CUDA graph capture (the
// self-consistent time loop) the iterations are the body of a conditional
// WHILE node whose condition the convergence test clears, so the loop runs
// without the host.  zk and the two pk buffers are padded by the 4-point halo,
// which stays zero, so the stencil needs no bounds tests.
//
// The default form runs all iterations in ONE cooperative launch
// (k_pcg_solve, at most two blocks of 512 threads per SM, all co-resident):
// (A) and (B) as above, each followed by a grid barrier after which every block
// sums the per-block partials itself, in block order, so all blocks take the
// same decisions.  The barrier's wait is bounded: on expiry it sets an abort
// word that releases the other blocks and the context's error flag, which the
// host turns into SB200_ERR_TIMEOUT.  The two-launch form stays for
// SB200_PCG_PERSISTENT=0 and where a cooperative launch cannot be captured.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "sb200_internal.cuh"

namespace sb200 {
namespace {

constexpr int PT = 256;        // threads per block
constexpr int HALO = 4;        // halo width
constexpr int MCH = 2048;      // points per block of the pole sums
constexpr int NLM_MAX = 25;    // lmax <= 4
constexpr int POLE_W = 32;     // doubles per pole entry: centre (3), itrho, rholm (25)
constexpr int PCG_CHUNK = 16;  // iterations between host checks of the convergence flag
// default iterations per body of the conditional node (SB200_PCG_UNROLL: 1..16;
// on the 64^3 isolated self-consistent loop 8 runs 3 % faster than 2, 16 no faster)
constexpr int PCG_UNROLL = 8;
constexpr double PCG_PI = 3.141592653589793;
constexpr int PTP = 512;                          // threads per block of the one-launch solve
constexpr long long PCG_WAIT_CYCLES = 2000000000LL;  // a grid barrier gives up after ~1 s of SM clocks

// scalars of the iteration (device)
// (SC_NEXT: the iteration the next launch pair performs)
enum { SC_SUM1 = 0, SC_AK, SC_CK, SC_DONE, SC_ITER, SC_NEXT, SC_COUNT };

struct PArgs {
  int nx, ny, nz;
  int px, py;           // padded extents (x, y)
  long N;
  int is[3], odd[3];
  double h[3], hvol;
  double lap0, lapt[12];
  int layout, nlm, npole, nchunk, natom;
  const double* rho;
  double* vh;
  double* vb;           // padded: Vh inside, boundary values in the face halos
  double* zk;           // padded
  double* pk[2];        // padded, alternating per iteration
  double* rlap;         // interior
  double* rho_stage;    // interior: host inputs of the direct call
  double* vh_stage;
  double* part;         // per-block partial sums
  unsigned int* counter;
  double* sc;           // SC_COUNT scalars
  double* pole;         // [npole][POLE_W]
  double* psum;         // [npole][nchunk][NLM_MAX] pole partial sums
  const int* cell;      // layout 3: [npole][6] interior offset boxes (x0, x1, y0, y1, z0, z1)
  int* err;             // the context's device error flag (a bounded wait expired)
  int* owner;           // layout 2: nearest atom of each interior point
  const double* rion;   // [natom][3]
  double threshold;
  int maxiter;
};

__device__ __forceinline__ double coord(const PArgs& a, int d, int off) {  // off: interior offset
  const int i = off + a.is[d];
  return a.odd[d] ? (double)i * a.h[d] : ((double)i - 0.5) * a.h[d];
}
__device__ __forceinline__ long padi(const PArgs& a, int x, int y, int z) {
  return (long)(x + HALO) + (long)a.px * ((long)(y + HALO) + (long)a.py * (long)(z + HALO));
}

// Ylm(x, y, z) of src/math/salmon_math.f90:386-426 for lm = l^2 + l + m < nlm
__device__ __forceinline__ void ylm_all(double x, double y, double z, double (&Y)[NLM_MAX]) {
  const double r2 = x * x + y * y + z * z;
  const double S3 = 1.7320508075688772, S34 = 0.8660254037844386, S58 = 0.7905694150420949,
               S15 = 3.872983346207417, S38 = 0.6123724356957945, S154 = 1.9364916731037085,
               S35_2 = 2.958039891549808, S358 = 2.091650066335189, S5_2 = 1.118033988749895,
               S5_4 = 0.5590169943749475, S35_8 = 0.739509972887452;
  Y[0] = 1.0;
  Y[1] = -y;
  Y[2] = z;
  Y[3] = -x;
  Y[4] = S3 * x * y;
  Y[5] = -S3 * y * z;
  Y[6] = (3.0 * z * z - r2) / 2.0;
  Y[7] = -S3 * x * z;
  Y[8] = S34 * (x * x - y * y);
  Y[9] = -S58 * y * (3 * x * x - y * y);
  Y[10] = S15 * x * y * z;
  Y[11] = -S38 * y * (5.0 * z * z - r2);
  Y[12] = z * (5.0 * z * z - 3 * r2) / 2.0;
  Y[13] = -S38 * x * (5.0 * z * z - r2);
  Y[14] = S154 * z * (x * x - y * y);
  Y[15] = -S58 * x * (x * x - 3.0 * y * y);
  Y[16] = S35_2 * x * y * (x * x - y * y);
  Y[17] = -S358 * y * z * (3.0 * x * x - y * y);
  Y[18] = S5_2 * x * y * (7.0 * z * z - r2);
  Y[19] = -S58 * y * z * (7.0 * z * z - 3.0 * r2);
  Y[20] = (35.0 * z * z * z * z - 30.0 * z * z * r2 + 3.0 * r2 * r2) / 8.0;
  Y[21] = -S58 * x * z * (7.0 * z * z - 3.0 * r2);
  Y[22] = S5_4 * (7.0 * z * z - r2) * (x * x - y * y);
  Y[23] = -S358 * x * z * (x * x - 3.0 * y * y);
  Y[24] = S35_8 * (x * x * x * x + y * y * y * y - 6.0 * x * x * y * y);
}

__device__ __forceinline__ int l_of(int lm) { return lm < 1 ? 0 : lm < 4 ? 1 : lm < 9 ? 2 : lm < 16 ? 3 : 4; }

// block-wide sum of one value per thread; every thread gets the total (fixed order)
template <int NT = PT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (t == 0) {
    for (int i = 0; i < NT / 32; ++i) s += red[i];
    red[NT / 32] = s;
  }
  __syncthreads();
  return red[NT / 32];
}

// The block's partial to part[blockIdx.x]; true in the block that finished last,
// whose threads then see every block's partial.
__device__ __forceinline__ bool post_partial(const PArgs& a, double v, bool* last) {
  if (threadIdx.x == 0) {
    a.part[blockIdx.x] = v;
    __threadfence();
    const unsigned int done = atomicAdd(a.counter, 1u);
    *last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (*last) __threadfence();
  return *last;
}

// sum of part[0 .. gridDim.x) in a fixed order (the last block)
__device__ __forceinline__ double total_of_partials(const PArgs& a, double* red) {
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += PT) v += __ldcg(a.part + i);
  return block_sum(v, red);
}

// ---- poles ---------------------------------------------------------------------

// layout 2: nearest atom of every interior point (first atom on ties, make_corr_pole)
__global__ void __launch_bounds__(PT) k_pcg_owner(PArgs a) {
  for (long q = blockIdx.x * (long)PT + threadIdx.x; q < a.N; q += (long)gridDim.x * PT) {
    const int x = (int)(q % a.nx), y = (int)((q / a.nx) % a.ny), z = (int)(q / ((long)a.nx * a.ny));
    const double cx = coord(a, 0, x), cy = coord(a, 1, y), cz = coord(a, 2, z);
    double rmin = 1e6;
    int amin = 0;
    for (int i = 0; i < a.natom; ++i) {
      const double dx = cx - a.rion[3 * i], dy = cy - a.rion[3 * i + 1], dz = cz - a.rion[3 * i + 2];
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      if (r < rmin) {
        rmin = r;
        amin = i;
      }
    }
    a.owner[q] = amin;
  }
}

// point p of pole `pole`'s enumeration -> interior offset q (false: none / not the pole's)
__device__ __forceinline__ bool pole_point(const PArgs& a, int pole, long p, int& x, int& y, int& z, long& q) {
  if (a.layout == 3) {
    const int* b = a.cell + 6 * pole;
    const int bx = b[1] - b[0] + 1, by = b[3] - b[2] + 1, bz = b[5] - b[4] + 1;
    if (p >= (long)bx * by * bz) return false;
    x = b[0] + (int)(p % bx);
    y = b[2] + (int)((p / bx) % by);
    z = b[4] + (int)(p / ((long)bx * by));
    q = x + (long)a.nx * (y + (long)a.ny * z);
    return true;
  }
  if (p >= a.N) return false;
  q = p;
  if (a.layout == 2 && a.owner[q] != pole) return false;
  x = (int)(q % a.nx);
  y = (int)((q / a.nx) % a.ny);
  z = (int)(q / ((long)a.nx * a.ny));
  return true;
}

// KIND 0 (layout 3): sums rho x, rho y, rho z, rho over the cell; KIND 1: the
// moments r^l Ylm rho hvol about the pole's centre.  Grid (nchunk, npole).
template <int KIND>
__global__ void __launch_bounds__(PT) k_pcg_pole_sum(PArgs a) {
  __shared__ double red[PT / 32 + 1];
  constexpr int NV = KIND == 0 ? 4 : NLM_MAX;
  const int pole = blockIdx.y;
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
  const double* pe = a.pole + (long)pole * POLE_W;
  const bool active = KIND == 0 || pe[3] != 0.0;
  if (active) {
    for (int i = threadIdx.x; i < MCH; i += PT) {
      const long p = (long)blockIdx.x * MCH + i;
      int x, y, z;
      long q;
      if (!pole_point(a, pole, p, x, y, z, q)) continue;
      const double r = a.rho[q];
      if (KIND == 0) {
        acc[0] += r * coord(a, 0, x);
        acc[1] += r * coord(a, 1, y);
        acc[2] += r * coord(a, 2, z);
        acc[NV - 1] += r;
      } else {
        const double xx = coord(a, 0, x) - pe[0], yy = coord(a, 1, y) - pe[1], zz = coord(a, 2, z) - pe[2];
        const double rr = sqrt(xx * xx + yy * yy + zz * zz) + 1e-50;
        double Y[NLM_MAX];
        ylm_all(xx / rr, yy / rr, zz / rr, Y);
        double rl[5];
        rl[0] = 1.0;
        rl[1] = rr;
        rl[2] = rr * rr;
        rl[3] = rr * rr * rr;
        rl[4] = rr * rr * rr * rr;
#pragma unroll
        for (int lm = 0; lm < NV; ++lm)
          if (lm < a.nlm) acc[lm] += rl[l_of(lm)] * Y[lm] * r * a.hvol;
      }
    }
  }
  double* out = a.psum + ((long)pole * a.nchunk + blockIdx.x) * NLM_MAX;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double s = block_sum(acc[v], red);
    if (threadIdx.x == 0) out[v] = s;
  }
}

// pole entries from the partial sums (one thread per pole; chunks in order).
// KIND 0: centroid and itrho of the layout-3 cells; KIND 1: rholm.
template <int KIND>
__global__ void k_pcg_pole_reduce(PArgs a) {
  const int pole = blockIdx.x * blockDim.x + threadIdx.x;
  if (pole >= a.npole) return;
  double* pe = a.pole + (long)pole * POLE_W;
  const double* ps = a.psum + (long)pole * a.nchunk * NLM_MAX;
  if (KIND == 0) {
    double s[4] = {0, 0, 0, 0};
    for (int c = 0; c < a.nchunk; ++c)
      for (int v = 0; v < 4; ++v) s[v] += ps[(long)c * NLM_MAX + v];
    const bool on = s[3] * a.hvol >= 1e-12;
    for (int d = 0; d < 3; ++d) pe[d] = on ? s[d] / s[3] : 0.0;
    pe[3] = on ? 1.0 : 0.0;
  } else {
    for (int lm = 0; lm < NLM_MAX; ++lm) {
      double s = 0.0;
      if (lm < a.nlm)
        for (int c = 0; c < a.nchunk; ++c) s += ps[(long)c * NLM_MAX + lm];
      pe[4 + lm] = s;
    }
  }
}

// boundary values in the four halo layers of the six faces of vb
__global__ void __launch_bounds__(PT) k_pcg_boundary(PArgs a) {
  const long fx = (long)HALO * a.ny * a.nz, fy = (long)HALO * a.nx * a.nz, fz = (long)HALO * a.nx * a.ny;
  const long total = 2 * (fx + fy + fz);
  for (long i = blockIdx.x * (long)PT + threadIdx.x; i < total; i += (long)gridDim.x * PT) {
    int x, y, z;
    long r = i;
    if (r < 2 * fx) {
      const int side = (int)(r / fx);
      r %= fx;
      const int h = (int)(r % HALO);
      y = (int)((r / HALO) % a.ny);
      z = (int)(r / ((long)HALO * a.ny));
      x = side == 0 ? -HALO + h : a.nx + h;
    } else if ((r -= 2 * fx) < 2 * fy) {
      const int side = (int)(r / fy);
      r %= fy;
      x = (int)(r % a.nx);
      const int h = (int)((r / a.nx) % HALO);
      z = (int)(r / ((long)a.nx * HALO));
      y = side == 0 ? -HALO + h : a.ny + h;
    } else {
      r -= 2 * fy;
      const int side = (int)(r / fz);
      r %= fz;
      x = (int)(r % a.nx);
      y = (int)((r / a.nx) % a.ny);
      const int h = (int)(r / ((long)a.nx * a.ny));
      z = side == 0 ? -HALO + h : a.nz + h;
    }
    const double gx = coord(a, 0, x), gy = coord(a, 1, y), gz = coord(a, 2, z);
    double v = 0.0;
    for (int c = 0; c < a.npole; ++c) {
      const double* pe = a.pole + (long)c * POLE_W;
      if (pe[3] == 0.0) continue;
      const double xx = gx - pe[0], yy = gy - pe[1], zz = gz - pe[2];
      const double rinv = 1.0 / (sqrt(xx * xx + yy * yy + zz * zz) + 1e-50);
      double Y[NLM_MAX];
      ylm_all(xx * rinv, yy * rinv, zz * rinv, Y);
      double rp[5];
      rp[0] = rinv;
      rp[1] = rinv * rinv;
      rp[2] = rp[1] * rinv;
      rp[3] = rp[2] * rinv;
      rp[4] = rp[3] * rinv;
      double s1 = 0.0;
#pragma unroll
      for (int lm = 0; lm < NLM_MAX; ++lm)
        if (lm < a.nlm) s1 += Y[lm] * rp[l_of(lm)] * pe[4 + lm];
      v += s1;
    }
    a.vb[padi(a, x, y, z)] = v;
  }
}

// ---- CG ------------------------------------------------------------------------

// 25-point Laplacian of laplacian_poisson at padded index c of array f (the
// reference's association: the 12 pair terms summed in x, y, z order, then added
// to -2 lap0 f)
template <typename F>
__device__ __forceinline__ double lap_at(const PArgs& a, long c, F f) {
  const long sy = a.px, sz = (long)a.px * a.py;
  double t = a.lapt[0] * (f(c + 1) + f(c - 1));
  t += a.lapt[1] * (f(c + 2) + f(c - 2));
  t += a.lapt[2] * (f(c + 3) + f(c - 3));
  t += a.lapt[3] * (f(c + 4) + f(c - 4));
  t += a.lapt[4] * (f(c + sy) + f(c - sy));
  t += a.lapt[5] * (f(c + 2 * sy) + f(c - 2 * sy));
  t += a.lapt[6] * (f(c + 3 * sy) + f(c - 3 * sy));
  t += a.lapt[7] * (f(c + 4 * sy) + f(c - 4 * sy));
  t += a.lapt[8] * (f(c + sz) + f(c - sz));
  t += a.lapt[9] * (f(c + 2 * sz) + f(c - 2 * sz));
  t += a.lapt[10] * (f(c + 3 * sz) + f(c - 3 * sz));
  t += a.lapt[11] * (f(c + 4 * sz) + f(c - 4 * sz));
  return -2.0 * a.lap0 * f(c) + t;
}

__global__ void __launch_bounds__(PT) k_pcg_fill(PArgs a) {
  for (long q = blockIdx.x * (long)PT + threadIdx.x; q < a.N; q += (long)gridDim.x * PT) {
    const int x = (int)(q % a.nx), y = (int)((q / a.nx) % a.ny), z = (int)(q / ((long)a.nx * a.ny));
    a.vb[padi(a, x, y, z)] = a.vh[q];
  }
}

// zk = -4 pi rho - lap(vb); sum1 = sum zk^2 hvol
__global__ void __launch_bounds__(PT) k_pcg_first(PArgs a) {
  __shared__ double red[PT / 32 + 1];
  __shared__ bool last;
  const double* vb = a.vb;
  double s = 0.0;
  for (long q = blockIdx.x * (long)PT + threadIdx.x; q < a.N; q += (long)gridDim.x * PT) {
    const int x = (int)(q % a.nx), y = (int)((q / a.nx) % a.ny), z = (int)(q / ((long)a.nx * a.ny));
    const long c = padi(a, x, y, z);
    const double lv = lap_at(a, c, [&](long i) { return __ldg(vb + i); });
    const double zv = -4.0 * PCG_PI * a.rho[q] - lv;
    a.zk[c] = zv;
    s += zv * zv * a.hvol;
  }
  s = block_sum(s, red);
  if (post_partial(a, s, &last)) {
    const double tot = total_of_partials(a, red);
    if (threadIdx.x == 0) {
      a.sc[SC_SUM1] = tot;
      a.sc[SC_AK] = 0.0;
      a.sc[SC_CK] = 0.0;
      a.sc[SC_DONE] = 0.0;
      a.sc[SC_ITER] = 0.0;
      a.sc[SC_NEXT] = 1.0;
      *a.counter = 0u;
      a.counter[1] = 0u;  // grid barrier of k_pcg_solve: arrivals
      a.counter[3] = 0u;  // and its abort word
    }
  }
}

// (A) of the iteration it = SC_NEXT: pk = zk + ck pk_old (pk = zk at it = 1),
// lap pk, zk.lap pk
__global__ void __launch_bounds__(PT) k_pcg_direction(PArgs a) {
  __shared__ double red[PT / 32 + 1];
  __shared__ bool last;
  if (a.sc[SC_DONE] != 0.0) return;
  const int it = (int)a.sc[SC_NEXT];
  const double ck = a.sc[SC_CK];
  const double* zk = a.zk;
  const double* po = a.pk[(it + 1) & 1];
  double* pn = a.pk[it & 1];
  const bool first = it == 1;
  auto pk_new = [&](long i) { return first ? __ldg(zk + i) : __ldg(zk + i) + ck * __ldg(po + i); };
  double s = 0.0;
  for (long q = blockIdx.x * (long)PT + threadIdx.x; q < a.N; q += (long)gridDim.x * PT) {
    const int x = (int)(q % a.nx), y = (int)((q / a.nx) % a.ny), z = (int)(q / ((long)a.nx * a.ny));
    const long c = padi(a, x, y, z);
    const double lv = lap_at(a, c, pk_new);
    pn[c] = pk_new(c);
    a.rlap[q] = lv;
    s += __ldg(zk + c) * lv;
  }
  s = block_sum(s, red);
  if (post_partial(a, s, &last)) {
    const double tot = total_of_partials(a, red);
    if (threadIdx.x == 0) {
      a.sc[SC_AK] = a.sc[SC_SUM1] / tot / a.hvol;
      *a.counter = 0u;
    }
  }
}

// (B) of the iteration it = SC_NEXT: Vh += ak pk, zk -= ak lap pk, convergence
// test, ck; with use_cond the test also clears the condition of the graph's
// WHILE node
__global__ void __launch_bounds__(PT) k_pcg_update(PArgs a, cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ double red[PT / 32 + 1];
  __shared__ bool last;
  if (a.sc[SC_DONE] != 0.0) return;
  const int it = (int)a.sc[SC_NEXT];
  const double ak = a.sc[SC_AK];
  const double* pk = a.pk[it & 1];
  double s = 0.0;
  for (long q = blockIdx.x * (long)PT + threadIdx.x; q < a.N; q += (long)gridDim.x * PT) {
    const int x = (int)(q % a.nx), y = (int)((q / a.nx) % a.ny), z = (int)(q / ((long)a.nx * a.ny));
    const long c = padi(a, x, y, z);
    a.vh[q] = a.vh[q] + ak * pk[c];
    const double zv = a.zk[c] - ak * a.rlap[q];
    a.zk[c] = zv;
    s += zv * zv;
  }
  s = block_sum(s, red);
  if (post_partial(a, s, &last)) {
    const double sum2 = total_of_partials(a, red) * a.hvol;
    if (threadIdx.x == 0) {
      if (fabs(sum2) < a.threshold * (double)a.N) {
        a.sc[SC_DONE] = 1.0;
        a.sc[SC_ITER] = (double)it;
      } else {
        a.sc[SC_CK] = sum2 / a.sc[SC_SUM1];
        a.sc[SC_SUM1] = sum2;
        if (it >= a.maxiter) {
          a.sc[SC_DONE] = 2.0;
          a.sc[SC_ITER] = (double)(a.maxiter + 1);
        }
      }
      a.sc[SC_NEXT] = (double)(it + 1);
      if (use_cond && a.sc[SC_DONE] != 0.0) cudaGraphSetConditional(cond, 0u);
      *a.counter = 0u;
    }
  }
}

// Grid barrier of k_pcg_solve (every block resident: cooperative launch).
// counter[1] counts arrivals over the whole solve (k_pcg_first zeroes it), so
// barrier k of a block waits for k * gridDim.x arrivals; counter[3] is the
// abort word.  After the block barrier, thread 0 arrives with a release
// reduction (publishing the block's writes at GPU scope) and polls the count
// with acquire loads; the wait is bounded by the SM clock, and on expiry it
// sets the abort word and the context's error flag.  False: leave the solve.
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_gpu(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool grid_barrier(const PArgs& a, unsigned int& target) {
  __shared__ int ok;
  target += gridDim.x;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* abort_word = a.counter + 3;
    int good = 1;
    red_release_gpu(a.counter + 1, 1u);
    const long long t0 = clock64();
    unsigned int polls = 0;
    while ((int)(ld_acquire_gpu(a.counter + 1) - target) < 0) {
      if ((++polls & 63u) == 0u) {
        if (*abort_word != 0u) {
          good = 0;
          break;
        }
        if (clock64() - t0 > PCG_WAIT_CYCLES) {
          atomicExch(a.counter + 3, 1u);
          atomicExch(a.err, 1);
          a.sc[SC_DONE] = 3.0;
          good = 0;
          break;
        }
      }
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// the sum of the nb per-block partials p[0 .. nb) in block order, in every block
__device__ __forceinline__ double grid_total(const double* p, int nb, double* red) {
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += PTP) v += __ldcg(p + i);
  return block_sum<PTP>(v, red);
}

// All CG iterations of one solve in one launch (after k_pcg_first): the
// iteration of k_pcg_direction + k_pcg_update with the scalars kept in
// registers; block 0 writes them back at the end.  The arrays written during
// the launch (zk, pk, rlap, vh) are read with coherent loads, not __ldg.
__global__ void __launch_bounds__(PTP, 2) k_pcg_solve(PArgs a) {
  __shared__ double red[PTP / 32 + 1];
  double* partA = a.part;
  double* partB = a.part + gridDim.x;
  const int nb = (int)gridDim.x;
  // rows (y, z) of the grid: each block an even, contiguous share (its warps
  // take the share's rows in turn, so neighbouring rows meet in one SM's L1
  // and no SM carries more rows than another), the lanes of a warp along x;
  // 32-bit divisions by ny instead of three 64-bit divisions per point
  const int rows = a.ny * a.nz, lane = threadIdx.x & 31;
  const int r_end = (int)(((long)(blockIdx.x + 1) * rows) / nb);
  const int warp0 = (int)(((long)blockIdx.x * rows) / nb) + (int)(threadIdx.x >> 5), nwarps = PTP / 32;
  unsigned int target = 0u;
  double sum1 = a.sc[SC_SUM1], ck = 0.0;
  double done = 0.0, iter = 0.0;
  int it = 1;
  for (; it <= a.maxiter; ++it) {
    const double* zk = a.zk;
    const double* po = a.pk[(it + 1) & 1];
    double* pn = a.pk[it & 1];
    const bool first = it == 1;
    auto pk_new = [&](long i) { return first ? zk[i] : zk[i] + ck * po[i]; };
    double s = 0.0;
    // one loop over this lane's points: x steps by 32 along a row, then the
    // next row of the warp (a nested loop would let the compiler hoist the 50
    // neighbour addresses of a row into registers)
    for (int r = warp0, x = lane; r < r_end;) {
      if (x < a.nx) {
        const long c = padi(a, x, r % a.ny, r / a.ny);
        const double lv = lap_at(a, c, pk_new);
        pn[c] = pk_new(c);
        a.rlap[(long)r * a.nx + x] = lv;
        s += zk[c] * lv;
      }
      x += 32;
      if (x >= a.nx) {
        x = lane;
        r += nwarps;
      }
    }
    s = block_sum<PTP>(s, red);
    if (threadIdx.x == 0) partA[blockIdx.x] = s;
    if (!grid_barrier(a, target)) return;
    const double ak = sum1 / grid_total(partA, nb, red) / a.hvol;
    s = 0.0;
    for (int r = warp0, x = lane; r < r_end;) {
      if (x < a.nx) {
        const long c = padi(a, x, r % a.ny, r / a.ny), q = (long)r * a.nx + x;
        a.vh[q] = a.vh[q] + ak * pn[c];
        const double zv = a.zk[c] - ak * a.rlap[q];
        a.zk[c] = zv;
        s += zv * zv;
      }
      x += 32;
      if (x >= a.nx) {
        x = lane;
        r += nwarps;
      }
    }
    s = block_sum<PTP>(s, red);
    if (threadIdx.x == 0) partB[blockIdx.x] = s;
    if (!grid_barrier(a, target)) return;
    const double sum2 = grid_total(partB, nb, red) * a.hvol;
    if (fabs(sum2) < a.threshold * (double)a.N) {
      done = 1.0;
      iter = (double)it;
      break;
    }
    ck = sum2 / sum1;
    sum1 = sum2;
    if (it >= a.maxiter) {
      done = 2.0;
      iter = (double)(a.maxiter + 1);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.sc[SC_SUM1] = sum1;
    a.sc[SC_CK] = ck;
    a.sc[SC_DONE] = done;
    a.sc[SC_ITER] = iter;
    a.sc[SC_NEXT] = (double)(done == 1.0 ? it + 1 : it);
  }
}

// Check of the grid barrier: `rounds` barriers over the solve's cooperative
// grid.  With withhold != 0 block 0 leaves without arriving, so the other
// blocks' bounded waits expire (about a second of SM clock) and set the abort
// word and the context's error flag, as a stalled solve would.
__global__ void __launch_bounds__(PTP, 2) k_barrier_check(PArgs a, int rounds, int withhold) {
  unsigned int target = 0u;
  if (withhold && blockIdx.x == 0) return;
  for (int r = 0; r < rounds; ++r)
    if (!grid_barrier(a, target)) return;
}

// Vh extrapolation of the isolated time step (time_evolution_step.f90:187-190,
// 196-198): with the global step itt = (device step counter, itt + 1 after
// finalize) - 1 + offset not 1, Vh = 2 stock1 - stock2 and stock2 = stock1
// before the solve (before = 1), stock1 = Vh after it (before = 0)
__global__ void k_vh_stock(const int* step, int offset, double* vh, double* s1, double* s2, long n, int before) {
  if (*step + offset == 2) return;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (before) {
      const double a1 = s1[i];
      vh[i] = 2.0 * a1 - s2[i];
      s2[i] = a1;
    } else {
      s1[i] = vh[i];
    }
  }
}

struct PcgState {
  size_t cap = 0;       // bytes of the arena
  void* arena = nullptr;
  double* host_sc = nullptr;  // pinned: the scalars read back by the host
  PArgs base{};               // the configured solve (rho, vh set per call)
  bool configured = false;
  cudaStream_t side = nullptr;  // captures the body of the conditional node
  int unroll = PCG_UNROLL;      // CG iterations per body of the conditional node
  int solve_grid = 0;           // blocks of k_pcg_solve (0: the two-launch form)
};

PcgState* pcg_of(sb200_ctx* c) { return static_cast<PcgState*>(c->pcg); }

// blocks of the CG launches: one point per thread up to bps blocks per SM
// (SB200_PCG_BLOCKS_PER_SM, 1..8), then grid-stride loops.  Default 4: on the
// 64^3 isolated self-consistent loop 13 % faster than 8 (fewer partial sums
// for the last block, two points per thread), 2 and 1 slower.
int grid_blocks(long n) {
  static const int bps = [] {
    const char* v = std::getenv("SB200_PCG_BLOCKS_PER_SM");
    const int b = v ? std::atoi(v) : 4;
    return (b >= 1 && b <= 8) ? b : 4;
  }();
  long b = (n + PT - 1) / PT;
  if (b > 148L * bps) b = 148L * bps;
  return (int)(b < 1 ? 1 : b);
}

// One cooperative launch of a kernel of PTP threads per block on st (captured or not).
template <typename... Args>
cudaError_t launch_coop(void (*kernel)(PArgs, Args...), int grid, cudaStream_t st, const PArgs& a, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(PTP);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, a, args...);
}

cudaError_t launch_solve(const PArgs& a, int grid, cudaStream_t st) { return launch_coop(k_pcg_solve, grid, st, a); }

// Blocks of the one-launch solve: at most two per SM (one with
// SB200_PCG_SOLVE_BLOCKS_PER_SM=1) and no more than the points need, within
// what the device keeps resident; 0 when disabled
// (SB200_PCG_PERSISTENT=0), when the kernel cannot be resident, or when a
// cooperative launch cannot be captured into a graph on this driver (checked
// once by capturing one on the side stream; the probe graph never runs).
int solve_grid_for(long n, cudaStream_t side, int device) {
  if (const char* v = std::getenv("SB200_PCG_PERSISTENT"))
    if (v[0] == '0') return 0;
  int coop = 0, sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_solve, PTP, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    return 0;
  }
  int bps = 2;  // SB200_PCG_SOLVE_BLOCKS_PER_SM: 1 or 2 (default 2)
  if (const char* v = std::getenv("SB200_PCG_SOLVE_BLOCKS_PER_SM")) bps = (std::atoi(v) == 1) ? 1 : 2;
  long g = (long)sms * (per_sm < bps ? per_sm : bps);
  const long need = (n + PTP - 1) / PTP;
  if (g > need) g = need;
  if (g < 1) return 0;
  PArgs probe{};
  if (cudaStreamBeginCapture(side, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const cudaError_t le = launch_solve(probe, (int)g, side);
  cudaGraph_t pg = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(side, &pg);
  if (pg) cudaGraphDestroy(pg);
  cudaGetLastError();
  return (le == cudaSuccess && ee == cudaSuccess) ? (int)g : 0;
}

}  // namespace

void pcg_free(sb200_ctx* c) {
  PcgState* s = pcg_of(c);
  if (!s) return;
  if (s->arena) cudaFree(s->arena);
  if (s->host_sc) cudaFreeHost(s->host_sc);
  if (s->side) cudaStreamDestroy(s->side);
  delete s;
  c->pcg = nullptr;
}

// Cells of layout 3 per axis when none are given: int((al + s) / s - 1e-8) with
// s = 8 A and al = num h (src/poisson/init_poisson.f90:112-115).
void pcg_default_cells(const sb200_ctx* c, int out[3]) {
  const double sp = 8.0 / 0.52917721067;
  const int num[3] = {c->g.nx, c->g.ny, c->g.nz};
  for (int d = 0; d < 3; ++d) out[d] = (int)((num[d] * c->g.hgs[d] + sp) / sp - 1e-8);
}

bool pcg_is_device(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Sizes the work arrays for the context's grid and the given boundary, uploads
// the pole tables and (layout 2) forms the nearest-atom map; the arrays whose
// halos must stay zero are cleared here, once.
int pcg_configure(sb200_ctx* c, int layout, int lmax, const double* rion, int natom, const int npole_xyz[3],
                  double threshold, int maxiter) {
  if (layout < 1 || layout > 3) return set_error(SB200_ERR_INVALID_ARG, "layout_multipole must be 1, 2 or 3");
  if (lmax < 0 || lmax > 4) return set_error(SB200_ERR_UNSUPPORTED, "lmax_multipole must be 0..4");
  if (maxiter < 1) return set_error(SB200_ERR_INVALID_ARG, "maxiter must be at least 1");
  if (layout == 2 && (natom < 1 || !rion))
    return set_error(SB200_ERR_INVALID_ARG, "layout_multipole 2 needs the atom positions");
  const int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  PArgs a{};
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.px = nx + 2 * HALO;
  a.py = ny + 2 * HALO;
  a.N = (long)nx * ny * nz;
  const long P = (long)a.px * a.py * (nz + 2 * HALO);
  for (int d = 0; d < 3; ++d) {
    a.is[d] = c->g.is[d];
    a.odd[d] = c->g.lg_num[d] % 2;
    a.h[d] = c->g.hgs[d];
  }
  a.hvol = c->g.hvol;
  a.lap0 = c->g.coef_lap0;
  for (int i = 0; i < 12; ++i) a.lapt[i] = c->g.coef_lap[i];
  a.layout = layout;
  a.nlm = (lmax + 1) * (lmax + 1);
  a.natom = natom;
  a.threshold = threshold;
  a.maxiter = maxiter;
  // poles (host tables)
  std::vector<double> pole_h;
  std::vector<int> cell_h;
  long pole_pts = a.N;
  if (layout == 1) {
    a.npole = 1;
    pole_h.assign(POLE_W, 0.0);
    pole_h[3] = 1.0;
  } else if (layout == 2) {
    a.npole = natom;
    pole_h.assign((size_t)natom * POLE_W, 0.0);
    for (int i = 0; i < natom; ++i) {
      for (int d = 0; d < 3; ++d) pole_h[(size_t)i * POLE_W + d] = rion[3 * i + d];
      pole_h[(size_t)i * POLE_W + 3] = 1.0;
    }
  } else {
    int n3[3];
    if (npole_xyz && (npole_xyz[0] || npole_xyz[1] || npole_xyz[2])) {
      for (int d = 0; d < 3; ++d) n3[d] = npole_xyz[d];
    } else {
      pcg_default_cells(c, n3);
    }
    const int num[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d)
      if (n3[d] < 1 || n3[d] > num[d])
        return set_error(SB200_ERR_INVALID_ARG, "num_multipole_xyz: every axis needs 1..num cells");
    a.npole = n3[0] * n3[1] * n3[2];
    cell_h.resize((size_t)a.npole * 6);
    pole_pts = 0;
    for (int j3 = 0; j3 < n3[2]; ++j3)
      for (int j2 = 0; j2 < n3[1]; ++j2)
        for (int j1 = 0; j1 < n3[0]; ++j1) {
          const int ib = j1 + n3[0] * (j2 + n3[1] * j3);
          const int j[3] = {j1, j2, j3};
          long vol = 1;
          for (int d = 0; d < 3; ++d) {
            cell_h[6 * ib + 2 * d] = j[d] * num[d] / n3[d];
            cell_h[6 * ib + 2 * d + 1] = (j[d] + 1) * num[d] / n3[d] - 1;
            vol *= cell_h[6 * ib + 2 * d + 1] - cell_h[6 * ib + 2 * d] + 1;
          }
          if (vol > pole_pts) pole_pts = vol;
        }
    pole_h.assign((size_t)a.npole * POLE_W, 0.0);
  }
  a.nchunk = (int)((pole_pts + MCH - 1) / MCH);
  // device arena
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  PcgState* s = pcg_of(c);
  if (!s) {
    s = new PcgState();
    if (const char* v = std::getenv("SB200_PCG_UNROLL")) {
      const int u = std::atoi(v);
      if (u >= 1 && u <= 16) s->unroll = u;
    }
    c->pcg = s;
    SB_CUDA(cudaMallocHost((void**)&s->host_sc, 8 * sizeof(double)));
    SB_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    s->solve_grid = solve_grid_for(a.N, s->side, c->device);
  }
  const int nblk = grid_blocks(a.N);
  const long n_part = nblk > 2L * s->solve_grid ? nblk : 2L * s->solve_grid;  // k_pcg_solve: two partial arrays
  const size_t b_pad = al(P * sizeof(double)), b_int = al(a.N * sizeof(double));
  const size_t b_part = al((size_t)n_part * sizeof(double)), b_sc = al(8 * sizeof(double) + sizeof(unsigned int) * 8);
  const size_t b_pole = al((size_t)a.npole * POLE_W * sizeof(double));
  const size_t b_psum = al((size_t)a.npole * a.nchunk * NLM_MAX * sizeof(double));
  const size_t b_cell = al(cell_h.size() * sizeof(int) + 4);
  const size_t b_owner = layout == 2 ? al(a.N * sizeof(int)) : 0;
  const size_t b_rion = al((size_t)(natom > 0 ? natom : 1) * 3 * sizeof(double));
  const size_t need = 4 * b_pad + 3 * b_int + b_part + b_sc + b_pole + b_psum + b_cell + b_owner + b_rion;
  s->configured = false;
  if (s->cap < need) {
    if (s->arena) cudaFree(s->arena);
    s->arena = nullptr;
    s->cap = 0;
    char* p = nullptr;
    if (dalloc(&p, need) != SB200_OK) return SB200_ERR_OOM;
    s->arena = p;
    s->cap = need;
  }
  char* p = static_cast<char*>(s->arena);
  a.vb = (double*)p;
  p += b_pad;
  a.zk = (double*)p;
  p += b_pad;
  a.pk[0] = (double*)p;
  p += b_pad;
  a.pk[1] = (double*)p;
  p += b_pad;
  a.rlap = (double*)p;
  p += b_int;
  a.rho_stage = (double*)p;
  p += b_int;
  a.vh_stage = (double*)p;
  p += b_int;
  a.part = (double*)p;
  p += b_part;
  a.sc = (double*)p;
  a.counter = (unsigned int*)(a.sc + 8);
  p += b_sc;
  a.pole = (double*)p;
  p += b_pole;
  a.psum = (double*)p;
  p += b_psum;
  a.cell = (const int*)p;
  int* cell_d = (int*)p;
  p += b_cell;
  a.owner = layout == 2 ? (int*)p : nullptr;
  p += b_owner;
  double* rion_d = (double*)p;
  a.rion = rion_d;
  a.err = c->d_err;
  cudaStream_t st = c->stream;
  // the padded arrays start at zero (their halos stay zero; vb's face halos are
  // rewritten by every solve), the block counter and the grid barrier at zero
  SB_CUDA(cudaMemsetAsync(a.vb, 0, 4 * b_pad, st));
  SB_CUDA(cudaMemsetAsync(a.counter, 0, 8 * sizeof(unsigned int), st));
  SB_CUDA(cudaMemcpyAsync(a.pole, pole_h.data(), pole_h.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  if (!cell_h.empty())
    SB_CUDA(cudaMemcpyAsync(cell_d, cell_h.data(), cell_h.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  if (layout == 2) {
    SB_CUDA(cudaMemcpyAsync(rion_d, rion, (size_t)natom * 3 * sizeof(double), cudaMemcpyHostToDevice, st));
    k_pcg_owner<<<grid_blocks(a.N), PT, 0, st>>>(a);
    SB_LAUNCH_CHECK("k_pcg_owner");
  }
  SB_CUDA(cudaStreamSynchronize(st));  // the host tables above are temporaries
  s->base = a;
  s->configured = true;
  return SB200_OK;
}

// One solve of the configured kind: Vh (device, start value in, solution out)
// of rho (device).  Outside a stream capture the host checks convergence every
// PCG_CHUNK iterations and *iterations gets poisson%iterVh; inside one the
// iterations become a conditional WHILE node of the captured graph and
// *iterations is left alone.
int pcg_issue(sb200_ctx* c, const double* d_rho, double* d_vh, int* iterations) {
  PcgState* s = pcg_of(c);
  if (!s || !s->configured) return set_error(SB200_ERR_STATE, "the CG Hartree solve is not configured");
  PArgs a = s->base;
  a.rho = d_rho;
  a.vh = d_vh;
  cudaStream_t st = c->stream;
  const int gb = grid_blocks(a.N);
  const dim3 gpole(a.nchunk, a.npole);
  const int gred = (a.npole + 127) / 128;
  if (a.layout == 3) {
    k_pcg_pole_sum<0><<<gpole, PT, 0, st>>>(a);
    k_pcg_pole_reduce<0><<<gred, 128, 0, st>>>(a);
  }
  k_pcg_pole_sum<1><<<gpole, PT, 0, st>>>(a);
  k_pcg_pole_reduce<1><<<gred, 128, 0, st>>>(a);
  const long nface = 2L * HALO * ((long)a.ny * a.nz + (long)a.nx * a.nz + (long)a.nx * a.ny);
  k_pcg_boundary<<<grid_blocks(nface), PT, 0, st>>>(a);
  k_pcg_fill<<<gb, PT, 0, st>>>(a);
  k_pcg_first<<<gb, PT, 0, st>>>(a);
  SB_LAUNCH_CHECK("k_pcg boundary / first residual");
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  SB_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
  if (s->solve_grid > 0) {  // every iteration in one cooperative launch
    const cudaError_t le = launch_solve(a, s->solve_grid, st);
    if (le != cudaSuccess) return cuda_error(le, "k_pcg_solve (cooperative launch)");
    if (cs == cudaStreamCaptureStatusActive) return SB200_OK;
    SB_CUDA(cudaMemcpyAsync(s->host_sc, a.sc, SC_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    if (s->host_sc[SC_DONE] == 3.0) {
      SB_CUDA(cudaMemset(a.err, 0, sizeof(int)));
      return set_error(SB200_ERR_TIMEOUT, "k_pcg_solve: a grid barrier wait expired");
    }
    if (iterations) *iterations = (int)s->host_sc[SC_ITER];
    return SB200_OK;
  }
  if (cs == cudaStreamCaptureStatusActive) {
    cudaGraphConditionalHandle h;
    SB_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    SB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    SB_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    SB_CUDA(cudaStreamBeginCaptureToGraph(s->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    for (int u = 0; u < s->unroll; ++u) {
      k_pcg_direction<<<gb, PT, 0, s->side>>>(a);
      k_pcg_update<<<gb, PT, 0, s->side>>>(a, h, 1);
    }
    const cudaError_t le = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s->side, &captured);
    if (le != cudaSuccess) return cuda_error(le, "k_pcg_direction / k_pcg_update (graph body)");
    if (ee != cudaSuccess) return cuda_error(ee, "cudaStreamEndCapture (graph body)");
    return SB200_OK;
  }
  for (int it0 = 1; it0 <= a.maxiter; it0 += PCG_CHUNK) {
    const int it1 = it0 + PCG_CHUNK - 1 < a.maxiter ? it0 + PCG_CHUNK - 1 : a.maxiter;
    for (int it = it0; it <= it1; ++it) {
      k_pcg_direction<<<gb, PT, 0, st>>>(a);
      k_pcg_update<<<gb, PT, 0, st>>>(a, cudaGraphConditionalHandle{}, 0);
    }
    SB_LAUNCH_CHECK("k_pcg_direction / k_pcg_update");
    SB_CUDA(cudaMemcpyAsync(s->host_sc, a.sc, SC_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    if (s->host_sc[SC_DONE] != 0.0) break;
  }
  if (iterations) *iterations = (int)s->host_sc[SC_ITER];
  return SB200_OK;
}

int pcg_vh_stock(sb200_ctx* c, const int* d_step, int offset, double* d_vh, double* d_s1, double* d_s2,
                 bool before) {
  const long n = c->g.npts;
  k_vh_stock<<<grid_blocks(n), PT, 0, c->stream>>>(d_step, offset, d_vh, d_s1, d_s2, n, before ? 1 : 0);
  SB_LAUNCH_CHECK("k_vh_stock");
  return SB200_OK;
}

int hartree_isolated_cg(sb200_ctx* c, const double* rho, double* vh, int layout, int lmax, const double* rion,
                        int natom, const int npole_xyz[3], double threshold, int maxiter, int* iterations) {
  int r = pcg_configure(c, layout, lmax, rion, natom, npole_xyz, threshold, maxiter);
  if (r != SB200_OK) return r;
  PcgState* s = pcg_of(c);
  const long n = s->base.N;
  cudaStream_t st = c->stream;
  const bool rho_dev = pcg_is_device(rho), vh_dev = pcg_is_device(vh);
  if (!rho_dev) SB_CUDA(cudaMemcpyAsync(s->base.rho_stage, rho, n * sizeof(double), cudaMemcpyHostToDevice, st));
  if (!vh_dev) SB_CUDA(cudaMemcpyAsync(s->base.vh_stage, vh, n * sizeof(double), cudaMemcpyHostToDevice, st));
  double* d_vh = vh_dev ? vh : s->base.vh_stage;
  r = pcg_issue(c, rho_dev ? rho : s->base.rho_stage, d_vh, iterations);
  if (r != SB200_OK) return r;
  if (!vh_dev) {
    SB_CUDA(cudaMemcpyAsync(vh, d_vh, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
  }
  return SB200_OK;
}

}  // namespace sb200

namespace sb200 {
namespace {
int check_grid_barrier(sb200_ctx* c, int withhold) {
  PcgState* s = pcg_of(c);
  if (!s || !s->configured) return set_error(SB200_ERR_STATE, "the CG Hartree solve is not configured");
  if (s->solve_grid < 1) return set_error(SB200_ERR_UNSUPPORTED, "the one-launch CG solve is not in use");
  const PArgs& a = s->base;
  cudaStream_t st = c->stream;
  SB_CUDA(cudaMemsetAsync(a.counter + 1, 0, 3 * sizeof(unsigned int), st));
  const cudaError_t le = launch_coop(k_barrier_check, s->solve_grid, st, a, 8, withhold ? 1 : 0);
  if (le != cudaSuccess) return cuda_error(le, "k_barrier_check (cooperative launch)");
  SB_CUDA(cudaStreamSynchronize(st));
  int flag = 0;
  SB_CUDA(cudaMemcpy(&flag, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  SB_CUDA(cudaMemsetAsync(a.counter + 1, 0, 3 * sizeof(unsigned int), st));
  SB_CUDA(cudaStreamSynchronize(st));
  if (flag != 0) {
    SB_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
    return set_error(SB200_ERR_TIMEOUT, "grid barrier: a bounded wait expired (a block did not arrive)");
  }
  return SB200_OK;
}
}  // namespace
}  // namespace sb200

extern "C" int sb200_check_grid_barrier(sb200_ctx* c, int withhold) {
  if (!c) return sb200::set_error(SB200_ERR_INVALID_ARG, "null ctx");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != c->device) cudaSetDevice(c->device);
  const int r = sb200::check_grid_barrier(c, withhold);
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  return r;
}

extern "C" int sb200_hartree_isolated_cg(sb200_ctx* c, const double* rho, double* Vh, int layout_multipole,
                                         int lmax_multipole, const double* Rion, int natom,
                                         const int num_multipole_xyz[3], double threshold_cg, int maxiter,
                                         int* iterations) {
  if (!c) return sb200::set_error(SB200_ERR_INVALID_ARG, "null ctx");
  if (!c->g.set) return sb200::set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  if (c->g.periodic)
    return sb200::set_error(SB200_ERR_UNSUPPORTED, "sb200_hartree_isolated_cg needs an isolated grid");
  if (!rho || !Vh) return sb200::set_error(SB200_ERR_INVALID_ARG, "null argument");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != c->device) cudaSetDevice(c->device);
  const int r = sb200::hartree_isolated_cg(c, rho, Vh, layout_multipole, lmax_multipole, Rion, natom,
                                           num_multipole_xyz, threshold_cg, maxiter, iterations);
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  return r;
}
