// sb200_scf.cu -- per-step potential update of the self-consistent RT path:
// PZ-LDA exchange-correlation (nspin = 1), the periodic Hartree potential and
// update_vlocal, on the device, so that V_local can follow the density every
// time step without a host round trip.
//
//   sb200_exc_cor_pz        exchange_correlation, xc = 'PZ' (src/xc/salmon_xc.f90:58-343,
//                           src/xc/builtin_pz.f90:23-83)
//   sb200_hartree_periodic  hartree -> poisson_ft (src/poisson/hartree.f90:20-128,
//                           src/poisson/poisson_periodic.f90:23-242)
//   sb200_update_vlocal     update_vlocal (src/common/hamiltonian.f90:813-843)
//
// The Hartree solve keeps the reference's method: separable discrete Fourier
// transforms with the exp(+-i 2 pi j k / n) tables (forward along z, y, x;
// division by the number of points and multiplication by 4 pi / |G|^2; inverse
// along z, y, x; real part).  Each pass is one launch in which a thread forms
// one output value as the ordered sum over the transformed axis, so the result
// does not depend on the launch shape.  The grids of this path (16^3 to 128^3)
// make each pass a few microseconds to tens of microseconds; the tables
// (3 n^2 complex) and 4 pi / |G|^2 stay resident across steps.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sb200_internal.cuh"

namespace sb200 {
namespace {

constexpr double SCF_PI = 3.141592653589793;
constexpr int SCF_THREADS = 256;
constexpr int SCF_XC_BLOCKS = 296;  // fixed: the E_xc partial sums have a fixed order
constexpr int SCF_DFT_THREADS = 64;  // small blocks: a 16^3 pass spreads over 64 SMs

// NCCL entry points, resolved at run time from the process's libnccl.so.2
// (the one the host's torch / MPI stack already loaded, else the system's), so
// the library carries no link-time NCCL dependency.
struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                             cudaStream_t) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};

const NcclApi* nccl_api() {
  static NcclApi api;
  static bool ok = false;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
    api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
    api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(dlsym(h, "ncclAllReduce"));
    api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
    api.error_string = reinterpret_cast<decltype(api.error_string)>(dlsym(h, "ncclGetErrorString"));
    ok = api.get_unique_id && api.comm_init_rank && api.all_reduce && api.comm_destroy && api.error_string;
  });
  return ok ? &api : nullptr;
}

struct ScfState {
  long npts = 0;
  int num[3] = {0, 0, 0};
  double2* d_a = nullptr;     // [npts] complex work
  double2* d_b = nullptr;     // [npts] complex work
  double* d_coef = nullptr;   // [npts] 4 pi / |G|^2, x fastest
  double2* d_tab = nullptr;   // egx [nx][nx], egy [ny][ny], egz [nz][nz]
  double* d_in = nullptr;     // staging of host inputs: up to (3 + nspin) * npts
  size_t in_cap = 0;
  double* d_out = nullptr;    // staging of host outputs: nspin * npts
  size_t out_cap = 0;
  double* d_part = nullptr;   // [SCF_XC_BLOCKS + 1]
  bool have_coef = false;
  double brl[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  // self-consistent time loop (sb200_set_self_consistent)
  bool rt_on = false;
  double* d_vpsl = nullptr;   // [npts]
  double* d_rho = nullptr;    // [npts]
  double* d_vh = nullptr;     // [npts]
  double* d_vxc = nullptr;    // [npts]
  // density sum over k-point shards (sb200_set_density_comm)
  ncclComm_t comm = nullptr;
  // isolated grids: transforms on the doubled box (sb200_hartree_isolated_ft)
  double2* d_ia = nullptr;    // [8 npts] complex work
  double2* d_ib = nullptr;    // [8 npts] complex work
  double* d_icoef = nullptr;  // [8 npts] 4 pi / |G|^2 of the doubled cell
  double2* d_itab = nullptr;  // tables of length 2nx, 2ny, 2nz
  bool have_icoef = false;
  double ibrl[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  // isolated grids, method_poisson = 'cg' (sb200_set_hartree_cg): d_vh carries
  // Vh from step to step as the CG start value, with the two stored potentials
  // of the extrapolation
  bool cg_on = false;
  int* d_step0 = nullptr;     // a zero step counter (the restart's stock update)
  double* d_rho_tot = nullptr;  // [npts] rho_up + rho_dn (nspin = 2)
  size_t spin_cap = 0;          // spins d_rho / d_vxc hold
  double* d_stock1 = nullptr;
  double* d_stock2 = nullptr;
};

ScfState* scf_of(sb200_ctx* c) { return static_cast<ScfState*>(c->scf); }

#define TRY_S(x)                   \
  do {                             \
    int _r = (x);                  \
    if (_r != SB200_OK) return _r; \
  } while (0)

struct ScfDevGuard {
  int prev = -1;
  explicit ScfDevGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~ScfDevGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

bool scf_is_device(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int scf_ready(sb200_ctx* c) {
  if (!c) return set_error(SB200_ERR_INVALID_ARG, "null ctx");
  if (!c->g.set) return set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  if (!c->orb.set) return set_error(SB200_ERR_STATE, "sb200_set_orbitals has not been called");
  return SB200_OK;
}

int scf_ensure(sb200_ctx* c) {
  ScfState* s = scf_of(c);
  if (s && s->npts == c->g.npts && s->num[0] == c->g.nx && s->num[1] == c->g.ny && s->num[2] == c->g.nz)
    return SB200_OK;
  scf_free(c);
  s = new ScfState();
  c->scf = s;
  s->npts = c->g.npts;
  s->num[0] = c->g.nx;
  s->num[1] = c->g.ny;
  s->num[2] = c->g.nz;
  TRY_S(dalloc(&s->d_part, (size_t)SCF_XC_BLOCKS + 1));
  return SB200_OK;
}

int scf_stage_in(sb200_ctx* c, size_t count) {
  ScfState* s = scf_of(c);
  if (s->in_cap >= count) return SB200_OK;
  dfree(s->d_in);
  s->in_cap = 0;
  TRY_S(dalloc(&s->d_in, count));
  s->in_cap = count;
  return SB200_OK;
}

int scf_stage_out(sb200_ctx* c, size_t count) {
  ScfState* s = scf_of(c);
  if (s->out_cap >= count) return SB200_OK;
  dfree(s->d_out);
  s->out_cap = 0;
  TRY_S(dalloc(&s->d_out, count));
  s->out_cap = count;
  return SB200_OK;
}

// device view of a caller array: the array itself when it is device memory,
// else a copy in the staging slot
int scf_input(sb200_ctx* c, const double* p, size_t count, double* slot, const double** dev) {
  if (scf_is_device(p)) {
    *dev = p;
    return SB200_OK;
  }
  SB_CUDA(cudaMemcpyAsync(slot, p, count * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  *dev = slot;
  return SB200_OK;
}

int scf_grid_blocks(long n) {
  long b = (n + SCF_THREADS - 1) / SCF_THREADS;
  const long cap = 148L * 8;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

// ---- kernels -----------------------------------------------------------------

// PZxc, src/xc/builtin_pz.f90:51-83 (Perdew-Zunger 1981: Slater exchange and
// the Ceperley-Alder correlation fit, high-density branch for rs <= 1).
__device__ __forceinline__ void pzxc_dev(double trho, double cst, double& exc, double& dexc) {
  const double gammaU = -0.1423, beta1U = 1.0529, beta2U = 0.3334, AU = 0.0311, BU = -0.048, CU = 0.002,
               DU = -0.0116;
  const double ttrho = trho + 1e-10;
  const double rs = pow(3.0 / (4.0 * SCF_PI * ttrho), 1.0 / 3.0);
  double e = -cst / rs;
  double de = e / (3.0 * ttrho);
  if (rs > 1.0) {
    const double rssq = sqrt(rs);
    const double den = 1.0 + beta1U * rssq + beta2U * rs;
    e = e + gammaU / den;
    de = de + gammaU * (0.5 * beta1U * rssq + beta2U * rs) / (3.0 * ttrho) / (den * den);
  } else {
    const double rsln = log(rs);
    e = e + AU * rsln + BU + CU * rs * rsln + DU * rs;
    de = de - rs / (3.0 * ttrho) * (AU / rs + CU * (rsln + 1.0) + DU);
  }
  exc = e;
  dexc = de;
}

// Vxc = e_xc + trho de_xc/drho per point (rho_s = rho/2, trho = 2 rho_s as
// calc_xc forms them, salmon_xc.f90:778 and builtin_pz.f90:39-44); per-block
// partial sums of e_xc * trho in a fixed tree order.
__global__ void __launch_bounds__(SCF_THREADS) k_exc_pz(const double* __restrict__ rho, double* __restrict__ vxc,
                                                        long n, double cst, double* __restrict__ part) {
  __shared__ double red[SCF_THREADS];
  double s = 0.0;
  for (long i = blockIdx.x * (long)SCF_THREADS + threadIdx.x; i < n; i += (long)gridDim.x * SCF_THREADS) {
    const double rho_s = rho[i] * 0.5;
    const double trho = 2.0 * rho_s;
    double e, de;
    pzxc_dev(trho, cst, e, de);
    vxc[i] = e + trho * de;
    s += e * trho;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = SCF_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// PZxc_sp, src/xc/builtin_pz_sp.f90:43-95: Slater exchange with the spin
// interpolation f(zeta) between the unpolarised and polarised Perdew-Zunger
// 1981 correlation fits; v[0] spin up (sign +1), v[1] spin down (-1).
__device__ __forceinline__ void pzxc_sp_dev(double trho, double tu, double td, double& exc, double (&v)[2]) {
  const double gammaU = -0.1423, gammaP = -0.0843, beta1U = 1.0529, beta2U = 0.3334, beta1P = 1.3981,
               beta2P = 0.2611, AU = 0.0311, BU = -0.048, CU = 0.002, DU = -0.0116, AP = 0.01555, BP = -0.0269,
               CP = 0.0007, DP = -0.0048;
  const double rs = pow(3.0 / (4.0 * SCF_PI * trho), 1.0 / 3.0);
  const double zeta = (tu - td) / trho;
  const double fden = pow(2.0, 4.0 / 3.0) - 2.0;
  const double sf = (pow(1.0 + zeta, 4.0 / 3.0) + pow(1.0 - zeta, 4.0 / 3.0) - 2.0) / fden;
  const double dsf = 4.0 / 3.0 * (pow(1.0 + zeta, 1.0 / 3.0) - pow(1.0 - zeta, 1.0 / 3.0)) / fden;
  const double cx = 3.0 / 4.0 * pow(3.0 / (2 * SCF_PI), 2.0 / 3.0);
  const double a = -pow(2.0, 1.0 / 3.0) + 1.0;
  double e = -cx / rs + a * cx / rs * sf;
  const double sgn[2] = {1.0, -1.0};
#pragma unroll
  for (int js = 0; js < 2; ++js)
    v[js] = e - 1.0 / 3.0 * cx / rs + 1.0 / 3.0 * a * cx / rs * sf + a * cx / rs * (sgn[js] - zeta) * dsf;
  double ecu, ecp, vcu, vcp;
  if (rs > 1.0) {
    const double q = sqrt(rs);
    const double du = 1.0 + beta1U * q + beta2U * rs, dp = 1.0 + beta1P * q + beta2P * rs;
    ecu = gammaU / du;
    ecp = gammaP / dp;
    vcu = gammaU * (1.0 + 7.0 / 6.0 * beta1U * q + 4.0 / 3.0 * beta2U * rs) / (du * du);
    vcp = gammaP * (1.0 + 7.0 / 6.0 * beta1P * q + 4.0 / 3.0 * beta2P * rs) / (dp * dp);
  } else {
    const double l = log(rs);
    ecu = AU * l + BU + CU * rs * l + DU * rs;
    ecp = AP * l + BP + CP * rs * l + DP * rs;
    vcu = AU * l + (BU - AU / 3.0) + 2.0 / 3.0 * CU * rs * l + (2.0 * DU - CU) / 3.0 * rs;
    vcp = AP * l + (BP - AP / 3.0) + 2.0 / 3.0 * CP * rs * l + (2.0 * DP - CP) / 3.0 * rs;
  }
  e = e + ecu + sf * (ecp - ecu);
#pragma unroll
  for (int js = 0; js < 2; ++js) v[js] = v[js] + vcu + sf * (vcp - vcu) + (ecp - ecu) * (sgn[js] - zeta) * dsf;
  exc = e;
}

// exc_cor_pz_sp (builtin_pz_sp.f90:23-40): rho_s(n, 2) -> vxc_s(n, 2), per-block
// partial sums of e_xc * trho (trho = rho_up + rho_dn + 1e-20, each spin
// density + 5e-21) in a fixed tree order.
__global__ void __launch_bounds__(SCF_THREADS) k_exc_pz_sp(const double* __restrict__ rho, double* __restrict__ vxc,
                                                           long n, double* __restrict__ part) {
  __shared__ double red[SCF_THREADS];
  double s = 0.0;
  for (long i = blockIdx.x * (long)SCF_THREADS + threadIdx.x; i < n; i += (long)gridDim.x * SCF_THREADS) {
    const double trho = rho[i] + rho[n + i] + 1e-20;
    double e, v[2];
    pzxc_sp_dev(trho, rho[i] + 5e-21, rho[n + i] + 5e-21, e, v);
    vxc[i] = v[0];
    vxc[n + i] = v[1];
    s += e * trho;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = SCF_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// predictor_corrector's V_local = 0.5 (V_tmp + V_new), V_new = Vpsl + Vh + Vxc(is)
// (update_vlocal) or the fixed v0
__global__ void k_pc_vloc(const double* __restrict__ vtmp, const double* __restrict__ vpsl,
                          const double* __restrict__ vh, const double* __restrict__ vxc,
                          const double* __restrict__ v0, double* __restrict__ v, float* __restrict__ v32, long n,
                          int nspin) {
  const long tot = n * nspin;
  for (long i = blockIdx.x * (long)SCF_THREADS + threadIdx.x; i < tot; i += (long)gridDim.x * SCF_THREADS) {
    const long p = i % n;
    const double vn = v0 ? v0[i] : vpsl[p] + vh[p] + vxc[i];
    const double val = 0.5 * (vtmp[i] + vn);
    v[i] = val;
    v32[i] = (float)val;
  }
}

// rho = rho_up + rho_dn (time_evolution_step.f90:160-170: rho%f summed over spins)
__global__ void k_rho_total(const double* __restrict__ rho_s, double* __restrict__ rho, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    rho[i] = (0.0 + rho_s[i]) + rho_s[n + i];
}

// E_xc = hvol * sum of the block partials, in block order (one thread).
__global__ void k_exc_final(double* __restrict__ part, int nblk, double hvol) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < nblk; ++b) t += part[b];
    part[nblk] = t * hvol;
  }
}

// One separable transform pass along `axis` (0 x, 1 y, 2 z):
//   out(k) = sum_j T(k, j) * in(j)   (sg = -1: the conjugate table)
// for every line of the grid, x fastest.  in_real: the input is the real array
// in_real (first forward pass).  coef: the forward x pass ends with
// coef * (sum / ntot) as poisson_ft does.  out_real: keep the real part (last
// inverse pass).
__global__ void __launch_bounds__(SCF_DFT_THREADS) k_dft_pass(const double2* __restrict__ in,
                                                          const double* __restrict__ in_real,
                                                          double2* __restrict__ out, double* __restrict__ out_real,
                                                          const double2* __restrict__ T, double sg, int nx, int ny,
                                                          int nz, int axis, const double* __restrict__ coef,
                                                          double ntot) {
  const long npts = (long)nx * ny * nz;
  for (long p = blockIdx.x * (long)SCF_DFT_THREADS + threadIdx.x; p < npts; p += (long)gridDim.x * SCF_DFT_THREADS) {
    const int x = (int)(p % nx);
    const long r = p / nx;
    const int y = (int)(r % ny);
    const int z = (int)(r / ny);
    int k, n;
    long stride;
    if (axis == 0) {
      k = x;
      n = nx;
      stride = 1;
    } else if (axis == 1) {
      k = y;
      n = ny;
      stride = nx;
    } else {
      k = z;
      n = nz;
      stride = (long)nx * ny;
    }
    const long base = p - (long)k * stride;
    const double2* Tk = T + (long)k * n;
    double re = 0.0, im = 0.0;
#pragma unroll 4
    for (int j = 0; j < n; ++j) {
      const double2 t = Tk[j];
      const double ti = sg * t.y;
      double vr, vi;
      if (in_real) {
        vr = in_real[base + (long)j * stride];
        vi = 0.0;
      } else {
        const double2 v = in[base + (long)j * stride];
        vr = v.x;
        vi = v.y;
      }
      re = re + (t.x * vr - ti * vi);
      im = im + (t.x * vi + ti * vr);
    }
    if (coef) {
      const double cf = coef[p];
      re = cf * (re / ntot);
      im = cf * (im / ntot);
    }
    if (out_real)
      out_real[p] = re;
    else
      out[p] = make_double2(re, im);
  }
}

// One pass of the isolated solve on the doubled (mx, my, mz) box: outputs on
// the corner box [0,bx) x [0,by) x [0,bz), each the ordered sum over the first
// nsum inputs along `axis` of T(k, j) * in(j), T the exp(+-2 pi i jk / ma) table
// of the axis (sg = -1: conjugate).  in_real / out_real: the (rx, ry, .) interior
// array (the density in, Vh out) instead of the doubled complex one.
__global__ void __launch_bounds__(SCF_DFT_THREADS) k_dft_box(const double2* __restrict__ in,
                                                         const double* __restrict__ in_real,
                                                         double2* __restrict__ out, double* __restrict__ out_real,
                                                         const double2* __restrict__ T, double sg, int mx, int my,
                                                         int bx, int by, int bz, int axis, int nsum, int ma,
                                                         const double* __restrict__ coef, double ntot, int rx,
                                                         int ry) {
  const long nb = (long)bx * by * bz;
  for (long p = blockIdx.x * (long)SCF_DFT_THREADS + threadIdx.x; p < nb; p += (long)gridDim.x * SCF_DFT_THREADS) {
    const int x = (int)(p % bx);
    const long r = p / bx;
    const int y = (int)(r % by);
    const int z = (int)(r / by);
    const int k = axis == 0 ? x : axis == 1 ? y : z;
    // input index of j = 0 along the axis, and the stride along it
    const int ix = axis == 0 ? 0 : x, iy = axis == 1 ? 0 : y, iz = axis == 2 ? 0 : z;
    long base, stride;
    if (in_real) {
      base = ix + (long)rx * (iy + (long)ry * iz);
      stride = axis == 0 ? 1 : axis == 1 ? rx : (long)rx * ry;
    } else {
      base = ix + (long)mx * (iy + (long)my * iz);
      stride = axis == 0 ? 1 : axis == 1 ? mx : (long)mx * my;
    }
    const double2* Tk = T + (long)k * ma;
    double re = 0.0, im = 0.0;
#pragma unroll 4
    for (int j = 0; j < nsum; ++j) {
      const double2 t = Tk[j];
      const double ti = sg * t.y;
      double vr, vi;
      if (in_real) {
        vr = in_real[base + (long)j * stride];
        vi = 0.0;
      } else {
        const double2 v = in[base + (long)j * stride];
        vr = v.x;
        vi = v.y;
      }
      re = re + (t.x * vr - ti * vi);
      im = im + (t.x * vi + ti * vr);
    }
    if (coef) {
      const double cf = coef[x + (long)mx * (y + (long)my * z)];
      re = cf * (re / ntot);
      im = cf * (im / ntot);
    }
    if (out_real)
      out_real[x + (long)rx * (y + (long)ry * z)] = re;
    else
      out[x + (long)mx * (y + (long)my * z)] = make_double2(re, im);
  }
}

// V_local(is) = Vpsl + Vh + Vxc(is), FP64 and its FP32 copy.
__global__ void k_update_vlocal(const double* __restrict__ vpsl, const double* __restrict__ vh,
                                const double* __restrict__ vxc, double* __restrict__ v, float* __restrict__ v32,
                                long n, int nspin) {
  const long tot = n * nspin;
  for (long i = blockIdx.x * (long)SCF_THREADS + threadIdx.x; i < tot; i += (long)gridDim.x * SCF_THREADS) {
    const long p = i % n;
    const double val = vpsl[p] + vh[p] + vxc[i];
    v[i] = val;
    v32[i] = (float)val;
  }
}

// ---- host tables (the same expressions as initialization.f90:690-776) -------

int fold_index(int m, int n) { return (m - (n + 1) / 2 >= 0) ? m - n : m; }

int scf_tables(sb200_ctx* c, const double brl[9]) {
  ScfState* s = scf_of(c);
  const int nx = s->num[0], ny = s->num[1], nz = s->num[2];
  if (!s->d_tab) {
    const size_t nt = (size_t)nx * nx + (size_t)ny * ny + (size_t)nz * nz;
    TRY_S(dalloc(&s->d_tab, nt));
    std::vector<double2> tab(nt);
    size_t o = 0;
    for (int n : {nx, ny, nz}) {
      for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) {
          const double a = 2.0 * SCF_PI * (double)(i * k) / (double)n;
          tab[o + (size_t)k * n + i] = make_double2(std::cos(a), std::sin(a));
        }
      o += (size_t)n * n;
    }
    SB_CUDA(cudaMemcpyAsync(s->d_tab, tab.data(), nt * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (s->have_coef && std::memcmp(s->brl, brl, sizeof(s->brl)) == 0) return SB200_OK;
  if (!s->d_coef) TRY_S(dalloc(&s->d_coef, (size_t)s->npts));
  if (!s->d_a) TRY_S(dalloc(&s->d_a, (size_t)s->npts));
  if (!s->d_b) TRY_S(dalloc(&s->d_b, (size_t)s->npts));
  std::vector<double> coef((size_t)s->npts);
  for (int kz = 0; kz < nz; ++kz)
    for (int ky = 0; ky < ny; ++ky)
      for (int kx = 0; kx < nx; ++kx) {
        const long p = kx + (long)nx * (ky + (long)ny * kz);
        const int iix = fold_index(kx, nx), iiy = fold_index(ky, ny), iiz = fold_index(kz, nz);
        double g[3];
        for (int d = 0; d < 3; ++d)
          g[d] = (double)iix * brl[d + 0] + (double)iiy * brl[d + 3] + (double)iiz * brl[d + 6];
        const double G2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
        coef[p] = (kx == 0 && ky == 0 && kz == 0) ? 0.0 : 4.0 * SCF_PI / G2;
      }
  SB_CUDA(cudaMemcpyAsync(s->d_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  std::memcpy(s->brl, brl, sizeof(s->brl));
  s->have_coef = true;
  return SB200_OK;
}

// Doubled-box tables of init_reciprocal_grid_isolated_ft
// (src/common/initialization.f90:823-1077): exp(i 2 pi j k / 2n) per axis and
// 4 pi / |G|^2 with G_d = fold(k_d, 2n_d) b_d / 2 (zero at G = 0).  The
// reference's tables repeat the first n columns in the second n; those columns
// only multiply the zero half of the box, so the plain table is used.
int scf_itables(sb200_ctx* c, const double brl[9]) {
  ScfState* s = scf_of(c);
  const int mx = 2 * s->num[0], my = 2 * s->num[1], mz = 2 * s->num[2];
  const size_t M = (size_t)mx * my * mz;
  if (!s->d_itab) {
    const size_t nt = (size_t)mx * mx + (size_t)my * my + (size_t)mz * mz;
    TRY_S(dalloc(&s->d_itab, nt));
    std::vector<double2> tab(nt);
    size_t o = 0;
    for (int n : {mx, my, mz}) {
      for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) {
          const double a = 2.0 * SCF_PI * (double)(i * k) / (double)n;
          tab[o + (size_t)k * n + i] = make_double2(std::cos(a), std::sin(a));
        }
      o += (size_t)n * n;
    }
    SB_CUDA(cudaMemcpyAsync(s->d_itab, tab.data(), nt * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (!s->d_ia) TRY_S(dalloc(&s->d_ia, M));
  if (!s->d_ib) TRY_S(dalloc(&s->d_ib, M));
  if (s->have_icoef && std::memcmp(s->ibrl, brl, sizeof(s->ibrl)) == 0) return SB200_OK;
  if (!s->d_icoef) TRY_S(dalloc(&s->d_icoef, M));
  std::vector<double> coef(M);
  for (int kz = 0; kz < mz; ++kz)
    for (int ky = 0; ky < my; ++ky)
      for (int kx = 0; kx < mx; ++kx) {
        const int iix = fold_index(kx, mx), iiy = fold_index(ky, my), iiz = fold_index(kz, mz);
        const double g0 = (double)iix * brl[0] / 2.0, g1 = (double)iiy * brl[4] / 2.0, g2 = (double)iiz * brl[8] / 2.0;
        const double G2 = g0 * g0 + g1 * g1 + g2 * g2;
        coef[kx + (size_t)mx * (ky + (size_t)my * kz)] =
            (iix == 0 && iiy == 0 && iiz == 0) ? 0.0 : 4.0 * SCF_PI / G2;
      }
  SB_CUDA(cudaMemcpyAsync(s->d_icoef, coef.data(), M * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  std::memcpy(s->ibrl, brl, sizeof(s->ibrl));
  s->have_icoef = true;
  return SB200_OK;
}

// ---- launch sequences (no host synchronisation: also issued inside the
// CUDA graph of the time loop) ---------------------------------------------------

// kind >= 0: each launch bracketed for sb200_kernel_times
int scf_mark(sb200_ctx* c, int kind, bool start) { return kind >= 0 ? kernel_timing_mark(c, kind, start) : SB200_OK; }

int scf_launch_hartree(sb200_ctx* c, const double* d_rho, double* d_vh, int kind) {
  ScfState* s = scf_of(c);
  const long n = s->npts;
  const int nx = s->num[0], ny = s->num[1], nz = s->num[2];
  const double2* tx = s->d_tab;
  const double2* ty = tx + (size_t)nx * nx;
  const double2* tz = ty + (size_t)ny * ny;
  long gbl = (n + SCF_DFT_THREADS - 1) / SCF_DFT_THREADS;
  if (gbl > 148L * 16) gbl = 148L * 16;
  const int gb = (int)gbl;
  const double ntot = (double)n;
  // forward: z, y, x (conjugate tables), the x pass dividing by the point count
  // and multiplying by 4 pi / |G|^2; inverse: z, y, x, the last keeping the real part
  struct Pass {
    const double2* in;
    const double* in_real;
    double2* out;
    double* out_real;
    const double2* T;
    double sg;
    int axis;
    const double* coef;
  } passes[6] = {{nullptr, d_rho, s->d_a, nullptr, tz, -1.0, 2, nullptr},
                 {s->d_a, nullptr, s->d_b, nullptr, ty, -1.0, 1, nullptr},
                 {s->d_b, nullptr, s->d_a, nullptr, tx, -1.0, 0, s->d_coef},
                 {s->d_a, nullptr, s->d_b, nullptr, tz, 1.0, 2, nullptr},
                 {s->d_b, nullptr, s->d_a, nullptr, ty, 1.0, 1, nullptr},
                 {s->d_a, nullptr, nullptr, d_vh, tx, 1.0, 0, nullptr}};
  for (const Pass& p : passes) {
    TRY_S(scf_mark(c, kind, true));
    k_dft_pass<<<gb, SCF_DFT_THREADS, 0, c->stream>>>(p.in, p.in_real, p.out, p.out_real, p.T, p.sg, nx, ny, nz,
                                                       p.axis, p.coef, ntot);
    TRY_S(scf_mark(c, kind, false));
  }
  return SB200_OK;
}

// poisson_isolated_ft's six passes on the doubled box (only the corner rows
// that carry data formed, as the reference's loop bounds)
int scf_launch_hartree_isolated(sb200_ctx* c, const double* d_rho, double* d_vh, int kind) {
  ScfState* s = scf_of(c);
  const int nx = s->num[0], ny = s->num[1], nz = s->num[2];
  const int mx = 2 * nx, my = 2 * ny, mz = 2 * nz;
  const double2* tx = s->d_itab;
  const double2* ty = tx + (size_t)mx * mx;
  const double2* tz = ty + (size_t)my * my;
  const double ntot = 8.0 * (double)nx * ny * nz;
  struct Pass {
    const double2* in;
    const double* in_real;
    double2* out;
    double* out_real;
    const double2* T;
    double sg;
    int bx, by, bz, axis, nsum, ma;
    const double* coef;
  } passes[6] = {{nullptr, d_rho, s->d_ia, nullptr, tz, -1.0, nx, ny, mz, 2, nz, mz, nullptr},
                 {s->d_ia, nullptr, s->d_ib, nullptr, ty, -1.0, nx, my, mz, 1, ny, my, nullptr},
                 {s->d_ib, nullptr, s->d_ia, nullptr, tx, -1.0, mx, my, mz, 0, nx, mx, s->d_icoef},
                 {s->d_ia, nullptr, s->d_ib, nullptr, tz, 1.0, mx, my, nz, 2, mz, mz, nullptr},
                 {s->d_ib, nullptr, s->d_ia, nullptr, ty, 1.0, mx, ny, nz, 1, my, my, nullptr},
                 {s->d_ia, nullptr, nullptr, d_vh, tx, 1.0, nx, ny, nz, 0, mx, mx, nullptr}};
  for (const Pass& p : passes) {
    long nb = ((long)p.bx * p.by * p.bz + SCF_DFT_THREADS - 1) / SCF_DFT_THREADS;
    if (nb > 148L * 16) nb = 148L * 16;
    TRY_S(scf_mark(c, kind, true));
    k_dft_box<<<(int)nb, SCF_DFT_THREADS, 0, c->stream>>>(p.in, p.in_real, p.out, p.out_real, p.T, p.sg, mx, my,
                                                           p.bx, p.by, p.bz, p.axis, p.nsum, p.ma, p.coef, ntot,
                                                           nx, ny);
    TRY_S(scf_mark(c, kind, false));
  }
  return SB200_OK;
}

// Vxc of d_rho; with total, E_xc lands in d_part[SCF_XC_BLOCKS] (the time loop
// does not use it and skips the final sum)
int scf_launch_xc(sb200_ctx* c, const double* d_rho, double* d_vxc, int kind, bool total = true) {
  ScfState* s = scf_of(c);
  const double cst = 0.75 * std::pow(3.0 / (2.0 * SCF_PI), 2.0 / 3.0);
  TRY_S(scf_mark(c, kind, true));
  if (c->orb.nspin == 2)
    k_exc_pz_sp<<<SCF_XC_BLOCKS, SCF_THREADS, 0, c->stream>>>(d_rho, d_vxc, s->npts, s->d_part);
  else
    k_exc_pz<<<SCF_XC_BLOCKS, SCF_THREADS, 0, c->stream>>>(d_rho, d_vxc, s->npts, cst, s->d_part);
  TRY_S(scf_mark(c, kind, false));
  if (!total) return SB200_OK;
  TRY_S(scf_mark(c, kind, true));
  k_exc_final<<<1, 32, 0, c->stream>>>(s->d_part, SCF_XC_BLOCKS, c->g.hvol);
  return scf_mark(c, kind, false);
}

int scf_launch_update(sb200_ctx* c, const double* vpsl, const double* vh, const double* vxc, int kind) {
  const long n = scf_of(c)->npts;
  const int nspin = c->orb.nspin;
  TRY_S(scf_mark(c, kind, true));
  // in a length-gauge loop the update is the field-free base the next step adds E.r to
  double* target = c->lg_active ? c->d_vloc_base : c->d_vloc;
  k_update_vlocal<<<scf_grid_blocks(n * nspin), SCF_THREADS, 0, c->stream>>>(vpsl, vh, vxc, target, c->d_vloc32,
                                                                            n, nspin);
  return scf_mark(c, kind, false);
}

// the density the Hartree solve takes: rho itself (nspin = 1) or rho_up + rho_dn
const double* scf_total_density(sb200_ctx* c, int kind) {
  ScfState* s = scf_of(c);
  if (c->orb.nspin != 2) return s->d_rho;
  const long n = s->npts;
  scf_mark(c, kind, true);
  k_rho_total<<<scf_grid_blocks(n), SCF_THREADS, 0, c->stream>>>(s->d_rho, s->d_rho_tot, n);
  scf_mark(c, kind, false);
  return s->d_rho_tot;
}

}  // namespace

int scf_rt_prepare(sb200_ctx* c) {
  ScfState* s = scf_of(c);
  if (!s || !s->rt_on) return SB200_OK;
  if (s->npts != c->g.npts || s->num[0] != c->g.nx || s->num[1] != c->g.ny || s->num[2] != c->g.nz)
    return set_error(SB200_ERR_STATE, "grid changed since sb200_set_self_consistent");
  return density_prepare(c);
}

int scf_density_allreduce(sb200_ctx* c, double* d_rho) {
  ScfState* s = scf_of(c);
  if (!s || !s->comm) return SB200_OK;
  const NcclApi* api = nccl_api();
  const ncclResult_t r = api->all_reduce(d_rho, d_rho, (size_t)c->g.npts * c->orb.nspin, ncclFloat64, ncclSum,
                                         s->comm, c->stream);
  if (r != ncclSuccess) return set_error(SB200_ERR_CUDA, std::string("ncclAllReduce: ") + api->error_string(r));
  return SB200_OK;
}

bool shard_comm_set(const sb200_ctx* c) {
  const ScfState* s = c->scf ? static_cast<const ScfState*>(c->scf) : nullptr;
  return s != nullptr && s->comm != nullptr;
}

int shard_sum(sb200_ctx* c, double* d, size_t n) {
  ScfState* s = scf_of(c);
  if (!s || !s->comm) return SB200_OK;
  const NcclApi* api = nccl_api();
  const ncclResult_t r = api->all_reduce(d, d, n, ncclFloat64, ncclSum, s->comm, c->stream);
  if (r != ncclSuccess) return set_error(SB200_ERR_CUDA, std::string("ncclAllReduce: ") + api->error_string(r));
  return SB200_OK;
}

int scf_rt_issue(sb200_ctx* c, const double2* psi) {
  ScfState* s = scf_of(c);
  if (!s || !s->rt_on) return SB200_OK;
  TRY_S(launch_density(c, psi, s->d_rho, SB200_KIND_POTENTIAL));
  TRY_S(scf_density_allreduce(c, s->d_rho));
  const double* rho_h = scf_total_density(c, SB200_KIND_POTENTIAL);
  if (c->g.periodic) {
    TRY_S(scf_launch_hartree(c, rho_h, s->d_vh, SB200_KIND_POTENTIAL));
  } else if (s->cg_on) {  // time_evolution_step.f90:186-198 with method_poisson = 'cg'
    TRY_S(scf_mark(c, SB200_KIND_POTENTIAL, true));
    TRY_S(pcg_vh_stock(c, c->rt.d_step, c->rt.loop_mit0, s->d_vh, s->d_stock1, s->d_stock2, true));
    TRY_S(pcg_issue(c, rho_h, s->d_vh, nullptr));
    TRY_S(pcg_vh_stock(c, c->rt.d_step, c->rt.loop_mit0, s->d_vh, s->d_stock1, s->d_stock2, false));
    TRY_S(scf_mark(c, SB200_KIND_POTENTIAL, false));
  } else {
    TRY_S(scf_launch_hartree_isolated(c, rho_h, s->d_vh, SB200_KIND_POTENTIAL));
  }
  TRY_S(scf_launch_xc(c, s->d_rho, s->d_vxc, SB200_KIND_POTENTIAL, false));
  TRY_S(scf_launch_update(c, s->d_vpsl, s->d_vh, s->d_vxc, SB200_KIND_POTENTIAL));
  SB_LAUNCH_CHECK("self-consistent potential update");
  return SB200_OK;
}

// predictor_corrector (time_evolution_step.f90:374-428) after the predicted
// Taylor step: the density of psi, with yn_fix_func = 'n' its Hartree (the
// hartree call from the current Vh, no extrapolation) and exchange-correlation
// potentials, update_vlocal, then V_local = (V_tmp + V_local) / 2; with a
// fixed potential update_vlocal gives v0
int scf_pc_potential(sb200_ctx* c, const double2* psi, const double* vtmp, const double* v0) {
  ScfState* s = scf_of(c);
  const long n = c->g.npts;
  const int nspin = c->orb.nspin;
  const bool scf = s && s->rt_on;
  if (scf) {
    TRY_S(launch_density(c, psi, s->d_rho, SB200_KIND_POTENTIAL));
    TRY_S(scf_density_allreduce(c, s->d_rho));
    const double* rho_h = scf_total_density(c, SB200_KIND_POTENTIAL);
    if (c->g.periodic) {
      TRY_S(scf_launch_hartree(c, rho_h, s->d_vh, SB200_KIND_POTENTIAL));
    } else if (s->cg_on) {
      TRY_S(scf_mark(c, SB200_KIND_POTENTIAL, true));
      TRY_S(pcg_issue(c, rho_h, s->d_vh, nullptr));
      TRY_S(scf_mark(c, SB200_KIND_POTENTIAL, false));
    } else {
      TRY_S(scf_launch_hartree_isolated(c, rho_h, s->d_vh, SB200_KIND_POTENTIAL));
    }
    TRY_S(scf_launch_xc(c, s->d_rho, s->d_vxc, SB200_KIND_POTENTIAL, false));
  }
  TRY_S(scf_mark(c, SB200_KIND_POTENTIAL, true));
  k_pc_vloc<<<scf_grid_blocks(n * nspin), SCF_THREADS, 0, c->stream>>>(
      vtmp, scf ? s->d_vpsl : nullptr, scf ? s->d_vh : nullptr, scf ? s->d_vxc : nullptr, scf ? nullptr : v0,
      c->d_vloc, c->d_vloc32, n, nspin);
  TRY_S(scf_mark(c, SB200_KIND_POTENTIAL, false));
  SB_LAUNCH_CHECK("k_pc_vloc");
  return SB200_OK;
}

bool scf_cg_on(const sb200_ctx* c) {
  const ScfState* s = c->scf ? static_cast<const ScfState*>(c->scf) : nullptr;
  return s != nullptr && s->cg_on;
}

bool scf_vh_stock(sb200_ctx* c, double** vh, double** s1, double** s2) {
  ScfState* s = scf_of(c);
  if (!s || !s->cg_on) return false;
  *vh = s->d_vh;
  *s1 = s->d_stock1;
  *s2 = s->d_stock2;
  return true;
}

// initialization_rt.f90:268-283 with yn_restart = 'y': Vh = 2 stock1 - stock2,
// stock2 = stock1, Vh of the density of psi (CG from that start), Vxc,
// V_local, stock1 = Vh
int scf_restart_potential(sb200_ctx* c, const double2* psi) {
  ScfState* s = scf_of(c);
  if (!s || !s->rt_on || !s->cg_on) return SB200_OK;
  if (!s->d_step0) {
    TRY_S(dalloc(&s->d_step0, 1));
    SB_CUDA(cudaMemsetAsync(s->d_step0, 0, sizeof(int), c->stream));
  }
  TRY_S(density_prepare(c));
  TRY_S(launch_density(c, psi, s->d_rho));
  TRY_S(scf_density_allreduce(c, s->d_rho));
  const double* rho_h = scf_total_density(c, -1);
  TRY_S(pcg_vh_stock(c, s->d_step0, 0, s->d_vh, s->d_stock1, s->d_stock2, true));
  TRY_S(pcg_issue(c, rho_h, s->d_vh, nullptr));
  TRY_S(scf_launch_xc(c, s->d_rho, s->d_vxc, -1, false));
  TRY_S(scf_launch_update(c, s->d_vpsl, s->d_vh, s->d_vxc, -1));
  TRY_S(pcg_vh_stock(c, s->d_step0, 0, s->d_vh, s->d_stock1, s->d_stock2, false));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

void scf_free(sb200_ctx* c) {
  ScfState* s = scf_of(c);
  if (!s) return;
  dfree(s->d_a);
  dfree(s->d_b);
  dfree(s->d_coef);
  dfree(s->d_tab);
  dfree(s->d_in);
  dfree(s->d_out);
  dfree(s->d_part);
  dfree(s->d_vpsl);
  dfree(s->d_rho);
  dfree(s->d_vh);
  dfree(s->d_vxc);
  if (s->comm) nccl_api()->comm_destroy(s->comm);
  dfree(s->d_ia);
  dfree(s->d_ib);
  dfree(s->d_icoef);
  dfree(s->d_itab);
  dfree(s->d_stock1);
  dfree(s->d_step0);
  dfree(s->d_rho_tot);
  dfree(s->d_stock2);
  delete s;
  c->scf = nullptr;
}

}  // namespace sb200

using namespace sb200;

extern "C" {

int sb200_exc_cor_pz(sb200_ctx* c, const double* rho, double* Vxc, double* E_xc) {
  TRY_S(scf_ready(c));
  if (!rho || !Vxc) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  ScfDevGuard dg(c->device);
  TRY_S(scf_ensure(c));
  ScfState* s = scf_of(c);
  const long n = s->npts;
  const size_t m = (size_t)n * c->orb.nspin;  // rho_s / Vxc_s of every spin
  TRY_S(scf_stage_in(c, m));
  const double* d_rho = nullptr;
  TRY_S(scf_input(c, rho, m, s->d_in, &d_rho));
  const bool out_dev = scf_is_device(Vxc);
  if (!out_dev) TRY_S(scf_stage_out(c, m));
  double* d_v = out_dev ? Vxc : s->d_out;
  TRY_S(scf_launch_xc(c, d_rho, d_v, -1));
  SB_LAUNCH_CHECK("k_exc_pz");
  if (!out_dev) SB_CUDA(cudaMemcpyAsync(Vxc, d_v, m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  double e = 0.0;
  SB_CUDA(cudaMemcpyAsync(&e, s->d_part + SCF_XC_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  if (E_xc) *E_xc = e;
  return SB200_OK;
}

int sb200_hartree_periodic(sb200_ctx* c, const double primitive_b[9], const double* rho, double* Vh) {
  TRY_S(scf_ready(c));
  if (!primitive_b || !rho || !Vh) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  if (!c->g.periodic)
    return set_error(SB200_ERR_UNSUPPORTED, "sb200_hartree_periodic needs a periodic grid");
  ScfDevGuard dg(c->device);
  TRY_S(scf_ensure(c));
  TRY_S(scf_tables(c, primitive_b));
  ScfState* s = scf_of(c);
  const long n = s->npts;
  TRY_S(scf_stage_in(c, (size_t)n));
  const double* d_rho = nullptr;
  TRY_S(scf_input(c, rho, (size_t)n, s->d_in, &d_rho));
  const bool out_dev = scf_is_device(Vh);
  if (!out_dev) TRY_S(scf_stage_out(c, (size_t)n));
  double* d_v = out_dev ? Vh : s->d_out;
  TRY_S(scf_launch_hartree(c, d_rho, d_v, -1));
  SB_LAUNCH_CHECK("k_dft_pass");
  if (!out_dev) SB_CUDA(cudaMemcpyAsync(Vh, d_v, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

int sb200_hartree_isolated_ft(sb200_ctx* c, const double primitive_b[9], const double* rho, double* Vh) {
  TRY_S(scf_ready(c));
  if (!primitive_b || !rho || !Vh) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  if (c->g.periodic)
    return set_error(SB200_ERR_UNSUPPORTED, "sb200_hartree_isolated_ft needs an isolated grid");
  ScfDevGuard dg(c->device);
  TRY_S(scf_ensure(c));
  TRY_S(scf_itables(c, primitive_b));
  ScfState* s = scf_of(c);
  const long n = s->npts;
  TRY_S(scf_stage_in(c, (size_t)n));
  const double* d_rho = nullptr;
  TRY_S(scf_input(c, rho, (size_t)n, s->d_in, &d_rho));
  const bool out_dev = scf_is_device(Vh);
  if (!out_dev) TRY_S(scf_stage_out(c, (size_t)n));
  double* d_v = out_dev ? Vh : s->d_out;
  TRY_S(scf_launch_hartree_isolated(c, d_rho, d_v, -1));
  SB_LAUNCH_CHECK("k_dft_box");
  if (!out_dev) SB_CUDA(cudaMemcpyAsync(Vh, d_v, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

int sb200_update_vlocal(sb200_ctx* c, const double* Vpsl, const double* Vh, const double* Vxc) {
  TRY_S(scf_ready(c));
  if (!Vpsl || !Vh || !Vxc) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  ScfDevGuard dg(c->device);
  TRY_S(scf_ensure(c));
  ScfState* s = scf_of(c);
  const long n = s->npts;
  const int nspin = c->orb.nspin;
  if (!c->d_vloc) TRY_S(dalloc(&c->d_vloc, (size_t)n * nspin));
  if (!c->d_vloc32) TRY_S(dalloc(&c->d_vloc32, (size_t)n * nspin));
  TRY_S(scf_stage_in(c, (size_t)n * (2 + nspin)));
  const double *a = nullptr, *b = nullptr, *x = nullptr;
  TRY_S(scf_input(c, Vpsl, (size_t)n, s->d_in, &a));
  TRY_S(scf_input(c, Vh, (size_t)n, s->d_in + n, &b));
  TRY_S(scf_input(c, Vxc, (size_t)n * nspin, s->d_in + 2 * n, &x));
  TRY_S(scf_launch_update(c, a, b, x, -1));
  SB_LAUNCH_CHECK("k_update_vlocal");
  SB_CUDA(cudaStreamSynchronize(c->stream));
  c->vloc_set = true;
  return SB200_OK;
}

int sb200_nccl_unique_id(unsigned char id[128]) {
  if (!id) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique id size");
  const NcclApi* api = nccl_api();
  if (!api) return set_error(SB200_ERR_UNSUPPORTED, "libnccl.so.2 could not be loaded");
  ncclUniqueId u;
  const ncclResult_t r = api->get_unique_id(&u);
  if (r != ncclSuccess) return set_error(SB200_ERR_CUDA, std::string("ncclGetUniqueId: ") + api->error_string(r));
  std::memcpy(id, &u, sizeof(u));
  return SB200_OK;
}

int sb200_set_density_comm(sb200_ctx* c, int nranks, int rank, const unsigned char id[128]) {
  TRY_S(scf_ready(c));
  ScfDevGuard dg(c->device);
  TRY_S(scf_ensure(c));
  ScfState* s = scf_of(c);
  const NcclApi* api = nccl_api();
  if (s->comm) {
    SB_CUDA(cudaStreamSynchronize(c->stream));
    api->comm_destroy(s->comm);
    s->comm = nullptr;
  }
  if (nranks <= 0) return SB200_OK;
  if (!id || rank < 0 || rank >= nranks) return set_error(SB200_ERR_INVALID_ARG, "bad rank or null id");
  if (!api) return set_error(SB200_ERR_UNSUPPORTED, "libnccl.so.2 could not be loaded");
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof(u));
  const ncclResult_t r = api->comm_init_rank(&s->comm, nranks, u, rank);
  if (r != ncclSuccess) {
    s->comm = nullptr;
    return set_error(SB200_ERR_CUDA, std::string("ncclCommInitRank: ") + api->error_string(r));
  }
  return SB200_OK;
}

int sb200_set_self_consistent(sb200_ctx* c, int enable, const double* Vpsl, const double primitive_b[9]) {
  TRY_S(scf_ready(c));
  ScfDevGuard dg(c->device);
  if (!enable) {
    if (scf_of(c)) scf_of(c)->rt_on = false;
    return SB200_OK;
  }
  if (!Vpsl || !primitive_b) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  if (!c->vloc_set) return set_error(SB200_ERR_STATE, "set V_local (sb200_set_vlocal / sb200_update_vlocal) first");
  TRY_S(scf_ensure(c));
  if (c->g.periodic)
    TRY_S(scf_tables(c, primitive_b));
  else
    TRY_S(scf_itables(c, primitive_b));
  ScfState* s = scf_of(c);
  const size_t n = (size_t)s->npts;
  const size_t ns = (size_t)c->orb.nspin;
  if (s->spin_cap < ns) {  // the per-spin arrays (rho_s, Vxc_s)
    dfree(s->d_rho);
    dfree(s->d_vxc);
    s->spin_cap = 0;
  }
  if (!s->d_vpsl) TRY_S(dalloc(&s->d_vpsl, n));
  if (!s->d_rho) TRY_S(dalloc(&s->d_rho, n * ns));
  if (!s->d_vh) TRY_S(dalloc(&s->d_vh, n));
  if (!s->d_vxc) TRY_S(dalloc(&s->d_vxc, n * ns));
  s->spin_cap = ns;
  if (ns == 2 && !s->d_rho_tot) TRY_S(dalloc(&s->d_rho_tot, n));
  SB_CUDA(cudaMemcpyAsync(s->d_vpsl, Vpsl, n * sizeof(double), cudaMemcpyDefault, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  TRY_S(density_prepare(c));
  s->rt_on = true;
  return SB200_OK;
}

int sb200_set_hartree_cg(sb200_ctx* c, const double* Vh0, int layout_multipole, int lmax_multipole,
                         const double* Rion, int natom, const int num_multipole_xyz[3], double threshold_cg,
                         int maxiter) {
  TRY_S(scf_ready(c));
  if (c->g.periodic) return set_error(SB200_ERR_UNSUPPORTED, "sb200_set_hartree_cg needs an isolated grid");
  ScfDevGuard dg(c->device);
  TRY_S(scf_ensure(c));
  ScfState* s = scf_of(c);
  if (!Vh0) {
    s->cg_on = false;
    return SB200_OK;
  }
  TRY_S(pcg_configure(c, layout_multipole, lmax_multipole, Rion, natom, num_multipole_xyz, threshold_cg, maxiter));
  const size_t n = (size_t)s->npts;
  if (!s->d_vh) TRY_S(dalloc(&s->d_vh, n));
  if (!s->d_stock1) TRY_S(dalloc(&s->d_stock1, n));
  if (!s->d_stock2) TRY_S(dalloc(&s->d_stock2, n));
  // initialization_rt.f90:277-286 (no restart): Vh of the initial density, both
  // stored potentials equal to it
  SB_CUDA(cudaMemcpyAsync(s->d_vh, Vh0, n * sizeof(double), cudaMemcpyDefault, c->stream));
  SB_CUDA(cudaMemcpyAsync(s->d_stock1, s->d_vh, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  SB_CUDA(cudaMemcpyAsync(s->d_stock2, s->d_vh, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  s->cg_on = true;
  return SB200_OK;
}

}  // extern "C"
