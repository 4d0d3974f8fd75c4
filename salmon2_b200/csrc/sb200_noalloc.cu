// sb200_noalloc.cu -- H psi for callers that cannot allocate device memory.
//
// Some hosts run this library where cudaMalloc is not available to them: a
// host code whose device memory is owned by another runtime (an OpenACC or
// OpenMP-offload program that maps its arrays itself), a memory-capped
// sandbox, or code that must not allocate in the middle of a time loop.
// sb200_hpsi_noalloc computes the same H psi as sb200_hpsi from arrays the
// caller already holds on the device and allocates nothing: no context, no
// cudaMalloc / cudaFree, no allocating library call.  Its only scratch -- the
// Kleinman-Bylander projections <beta|psi> of every orbital -- lives in the
// file-scope device array below, of fixed size, which every GPU that loads
// this library keeps until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "sb200_internal.cuh"

namespace sb200 {
namespace {

// Projection scratch: norb * nlma complex values at most (4 MiB).
constexpr long NOALLOC_MAX_PROJ = SB200_NOALLOC_MAX_PROJECTIONS;
static __device__ __align__(256) double2 g_noalloc_proj[NOALLOC_MAX_PROJ];

// Device address of g_noalloc_proj per device, resolved once per device on
// the host (the host-side symbol is a stand-in, not a device address).
constexpr int MAX_DEVICES = 64;
double2* g_proj_ptr[MAX_DEVICES] = {nullptr};
std::mutex g_proj_mu;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

struct NAArgs {
  int nx, ny, nz, periodic, nspin, nspin_no, norb, natom, nps, nlma;
  int is[3];
  long npts;
  double coef_lap0, lapt[12], nab[12];
  const double* kAc;      // device (3, nk)
  const double* vloc;     // device [nspin][npts]
  const int *mps, *jxyz, *ia_tbl;
  const double *rxyz, *uv, *rinv;
};

// Flat grid index of sphere point j of atom ia, or -1 when the table entry lies
// outside is..is+n-1 (the caller's table is checked here, on the device, since
// the host never sees it).
__device__ __forceinline__ long pt_index(const NAArgs& a, int j, int ia) {
  const int* c = a.jxyz + 3L * (j + (long)a.nps * ia);
  const int x = c[0] - a.is[0], y = c[1] - a.is[1], z = c[2] - a.is[2];
  if (x < 0 || x >= a.nx || y < 0 || y >= a.ny || z < 0 || z >= a.nz) return -1;
  return x + (long)a.nx * (y + (long)a.ny * z);
}

// Atom of projector ilma and its sphere size, or -1 when ia_tbl / mps are out
// of range.
__device__ __forceinline__ int atom_of(const NAArgs& a, int ilma, int* m) {
  const int ia = a.ia_tbl[ilma] - 1;
  if (ia < 0 || ia >= a.natom) return -1;
  const int mm = a.mps[ia];
  if (mm < 0 || mm > a.nps) return -1;
  *m = mm;
  return ia;
}

__device__ __forceinline__ void flag_bad_table(int* status) {
  if (status != nullptr) atomicExch(status, SB200_ERR_BAD_SHAPE);
}

// zekr_uV(j, ilma, k) = conj(exp(i kAc.r_j)) * uV(j, ilma) (hamiltonian.f90:883-894;
// isolated: uV, prep_pp.f90:618-619)
__device__ __forceinline__ double2 zekr(const NAArgs& a, int j, int ia, int ilma, int ik) {
  const double uv = a.uv[j + (long)a.nps * ilma];
  if (!a.periodic) return make_double2(uv, 0.0);
  const double* r = a.rxyz + 3L * (j + (long)a.nps * ia);
  const double* k = a.kAc + 3L * ik;
  double s, c;
  sincos(k[0] * r[0] + k[1] * r[1] + k[2] * r[2], &s, &c);
  return make_double2(c * uv, -s * uv);
}

// projections: one warp per (orbital, ilma), fixed butterfly reduction
__global__ void k_na_project(const double2* __restrict__ psi, double2* __restrict__ proj, NAArgs a,
                             int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  if (w >= (long)a.norb * a.nlma) return;
  const int o = (int)(w / a.nlma), ilma = (int)(w % a.nlma);
  int m = 0;
  const int ia = atom_of(a, ilma, &m);
  if (ia < 0) {
    if (lane == 0) {
      flag_bad_table(status);
      proj[w] = make_double2(0.0, 0.0);
    }
    return;
  }
  const int ik = o / a.nspin_no;
  const double2* p = psi + (long)o * a.npts;
  double2 acc = make_double2(0.0, 0.0);
  for (int j = lane; j < m; j += 32) {
    const long q = pt_index(a, j, ia);
    if (q < 0) {
      flag_bad_table(status);
      continue;
    }
    const double2 z = zekr(a, j, ia, ilma, ik);
    acc = cadd(acc, cmul(make_double2(z.x, -z.y), p[q]));
  }
  for (int off = 16; off > 0; off >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
  }
  if (lane == 0) proj[w] = make_double2(a.rinv[ilma] * acc.x, a.rinv[ilma] * acc.y);
}

// local part: 25-point stencil + k+A gradient + V_local (seq.f90:65-122).
// Orbitals beyond gridDim.y (at most 65535) are taken by a grid-stride loop.
// The first block clears the caller's status word; the kernels after it in
// the stream only ever raise it.
__global__ void k_na_local(const double2* __restrict__ in, double2* __restrict__ out, NAArgs a,
                           int* __restrict__ status) {
  if (status != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *status = SB200_OK;
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= a.npts) return;
  const int x = (int)(p % a.nx), y = (int)((p / a.nx) % a.ny), z = (int)(p / ((long)a.nx * a.ny));
  const int c3[3] = {x, y, z}, n3[3] = {a.nx, a.ny, a.nz};
  const long st3[3] = {1, a.nx, (long)a.nx * a.ny};
  for (int o = blockIdx.y; o < a.norb; o += gridDim.y) {
    const double2* src = in + (long)o * a.npts;
    const int ik = o / a.nspin_no;
    double kac[3] = {0.0, 0.0, 0.0};
    if (a.periodic)
      for (int d = 0; d < 3; ++d) kac[d] = a.kAc[3 * ik + d];
    double2 v = make_double2(0.0, 0.0), w = v;
    for (int d = 0; d < 3; ++d) {
      double2 vd = make_double2(0.0, 0.0), wd = vd;
      for (int s = 1; s <= ND; ++s) {
        double2 tp = make_double2(0.0, 0.0), tm = tp;
        int qp = c3[d] + s, qm = c3[d] - s;
        if (a.periodic) {
          qp = qp >= n3[d] ? qp - n3[d] : qp;
          qm = qm < 0 ? qm + n3[d] : qm;
        }
        if (qp < n3[d]) tp = src[p + (qp - c3[d]) * st3[d]];
        if (qm >= 0) tm = src[p + (qm - c3[d]) * st3[d]];
        const double l = a.lapt[4 * d + s - 1], nb = kac[d] * a.nab[4 * d + s - 1];
        vd = make_double2(vd.x + l * (tp.x + tm.x), vd.y + l * (tp.y + tm.y));
        wd = make_double2(wd.x + nb * (tp.x - tm.x), wd.y + nb * (tp.y - tm.y));
      }
      v = cadd(vd, v);
      w = cadd(wd, w);
    }
    const double lap0 = a.periodic ? a.coef_lap0 + 0.5 * (kac[0] * kac[0] + kac[1] * kac[1] + kac[2] * kac[2])
                                   : a.coef_lap0;
    const double2 c = src[p];
    const double vl = a.vloc[(long)(o % a.nspin) * a.npts + p];
    out[(long)o * a.npts + p] =
        make_double2(vl * c.x + lap0 * c.x - 0.5 * v.x + w.y, vl * c.y + lap0 * c.y - 0.5 * v.y - w.x);
  }
}

// nonlocal scatter: one warp per orbital walks the projectors in ilma order
// and each projector's sphere points in j order, 32 at a time (the order of
// nonlocal_potential.f90:368-375).  A sphere wider than half a periodic cell
// reaches some grid points through two images, so two lanes of one chunk can
// hold the same grid point: the lanes of such a group are found with a match
// and the lowest of them adds the group's values to h in lane (= j) order, so
// no update is lost and the result does not depend on timing.  Chunks and
// projectors follow one another in program order within the warp.
__global__ void k_na_scatter(const double2* __restrict__ proj, double2* __restrict__ out, NAArgs a,
                             int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const long o = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  if (o >= a.norb) return;  // uniform over the warp
  const int ik = (int)(o / a.nspin_no);
  double2* h = out + o * a.npts;
  for (int ilma = 0; ilma < a.nlma; ++ilma) {
    int m = 0;
    const int ia = atom_of(a, ilma, &m);
    if (ia < 0) continue;  // flagged by the projection kernel
    const double2 P = proj[o * a.nlma + ilma];
    for (int j0 = 0; j0 < m; j0 += 32) {
      const int j = j0 + lane;
      long q = -1;
      double2 c = make_double2(0.0, 0.0);
      if (j < m) {
        q = pt_index(a, j, ia);
        if (q < 0) flag_bad_table(status);
        else c = cmul(P, zekr(a, j, ia, ilma, ik));
      }
      const unsigned same = __match_any_sync(0xffffffffu, q);
      if (!__any_sync(0xffffffffu, q >= 0 && __popc(same) > 1)) {
        if (q >= 0) h[q] = cadd(h[q], c);
      } else {
        const bool lead = q >= 0 && lane == __ffs(same) - 1;
        double2 s = lead ? h[q] : make_double2(0.0, 0.0);
        for (int l = 0; l < 32; ++l) {
          const double vx = __shfl_sync(0xffffffffu, c.x, l);
          const double vy = __shfl_sync(0xffffffffu, c.y, l);
          if (lead && ((same >> l) & 1u)) s = make_double2(s.x + vx, s.y + vy);
        }
        if (lead) h[q] = s;
      }
      __syncwarp();
    }
  }
}

int proj_scratch(int dev, double2** out) {
  if (dev < 0 || dev >= MAX_DEVICES) return set_error(SB200_ERR_INVALID_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_proj_mu);
  if (g_proj_ptr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_proj);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_proj)");
    g_proj_ptr[dev] = (double2*)p;
  }
  *out = g_proj_ptr[dev];
  return SB200_OK;
}

}  // namespace
}  // namespace sb200

using namespace sb200;

extern "C" int sb200_hpsi_noalloc(int nx, int ny, int nz, int periodic, int nspin, int no, int nk, const int is[3],
                                  double coef_lap0, const double coef_lap[12], const double coef_nab[12],
                                  const double* kAc, const double* V_local, int natom, int nps, int nlma,
                                  const int* mps, const int* jxyz, const double* rxyz, const double* uv,
                                  const int* ia_tbl, const double* rinv_uvu, const double* tpsi, double* htpsi,
                                  int* status, void* stream) {
  if (nx < ND || ny < ND || nz < ND || nspin < 1 || nspin > 2 || no < 1 || nk < 1 || !is || !coef_lap ||
      !coef_nab || !V_local || !tpsi || !htpsi || tpsi == htpsi || (periodic && !kAc))
    return set_error(SB200_ERR_INVALID_ARG, "sb200_hpsi_noalloc: bad sizes or null / aliased pointer");
  if (nlma > 0 && (natom < 1 || nps < 1 || !mps || !jxyz || !uv || !ia_tbl || !rinv_uvu || (periodic && !rxyz)))
    return set_error(SB200_ERR_INVALID_ARG, "sb200_hpsi_noalloc: null projector table");
  const long norb = (long)nspin * no * nk;
  if (norb > 0x7fffffffL)
    return set_error(SB200_ERR_BAD_SHAPE, "sb200_hpsi_noalloc: more than 2^31-1 orbitals");
  if (nlma > 0 && norb * nlma > NOALLOC_MAX_PROJ)
    return set_error(SB200_ERR_BAD_SHAPE,
                     "sb200_hpsi_noalloc: norb*nlma exceeds SB200_NOALLOC_MAX_PROJECTIONS (262144); "
                     "use sb200_hpsi");
  int dev = 0;
  SB_CUDA(cudaGetDevice(&dev));
  double2* proj = nullptr;
  if (nlma > 0) {
    int r = proj_scratch(dev, &proj);
    if (r != SB200_OK) return r;
  }
  NAArgs a;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.periodic = periodic ? 1 : 0;
  a.nspin = nspin;
  a.nspin_no = nspin * no;
  a.norb = (int)norb;
  a.natom = natom;
  a.nps = nps;
  a.nlma = nlma > 0 ? nlma : 0;
  for (int d = 0; d < 3; ++d) a.is[d] = is[d];
  a.npts = (long)nx * ny * nz;
  a.coef_lap0 = coef_lap0;
  for (int i = 0; i < 12; ++i) {
    a.lapt[i] = coef_lap[i];
    a.nab[i] = coef_nab[i];
  }
  a.kAc = kAc;
  a.vloc = V_local;
  a.mps = mps;
  a.jxyz = jxyz;
  a.ia_tbl = ia_tbl;
  a.rxyz = rxyz;
  a.uv = uv;
  a.rinv = rinv_uvu;
  cudaStream_t st = (cudaStream_t)stream;
  const double2* in = (const double2*)tpsi;
  double2* out = (double2*)htpsi;
  // orbitals on grid y (at most 65535 blocks; the kernel loops over the rest)
  dim3 lg((unsigned)((a.npts + 255) / 256), (unsigned)(norb < 65535 ? norb : 65535));
  k_na_local<<<lg, 256, 0, st>>>(in, out, a, status);
  SB_LAUNCH_CHECK("k_na_local");
  if (a.nlma > 0) {
    const long warps = norb * a.nlma;
    k_na_project<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(in, proj, a, status);
    SB_LAUNCH_CHECK("k_na_project");
    // one warp per orbital, four orbitals per block
    k_na_scatter<<<(unsigned)((norb + 3) / 4), 128, 0, st>>>(proj, out, a, status);
    SB_LAUNCH_CHECK("k_na_scatter");
  }
  return SB200_OK;
}
