// sb200_restart.cu -- restart data in the reference's file layouts: the
// ground-state orbitals that start a time propagation and the checkpoints of a
// propagation (host I/O; one kernel widens real orbitals to complex).
//
//   write_bin / read_bin         src/io/checkpoint_restart.f90:310-534
//     info.bin        Fortran sequential records: nk, no, iter, nprocs, if_real_orbital
//     occupation.bin  one record: rocc(mo, mk, nspin)
//     Vh_stock.bin    two records: Vh_stock1, Vh_stock2 (isolated grids)
//   write_wavefunction /
//   read_wavefunction            src/io/checkpoint_restart.f90:539-677,1149-1305
//     'single' wfn.bin            stream: per (ik, io, ispin), ispin fastest, the
//                                 grid block (x fastest), real(8) or complex(8)
//     'slice'  k_IK_ob_NB/wfn_ob_IO.dat   stream: the nspin blocks of one orbital,
//                                 NB the first orbital of its block of
//                                 min(mo, nblock_wf_distribute) orbitals
//   write_rtdata / read_rtdata   src/io/checkpoint_restart.f90:1925-1993
//     rtdata.bin      ('lo' only) records Ac_tot(:,itt:itt+1), Ac_ind(:,itt:itt+1), Ac_ind(:,0)
//   restart_rt                   src/io/checkpoint_restart.f90:277-306 and the
//                                restart branch of initialization_rt.f90:244-283
//
// Sequential records carry 4-byte length markers before and after the data
// (gfortran's layout; a negative leading marker continues the record in the
// next subrecord).  Integers of 4 or 8 bytes are accepted on reading.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sb200_internal.cuh"

#define RS_CHECK_CTX(c)                                                     \
  do {                                                                      \
    if ((c) == nullptr) return set_error(SB200_ERR_INVALID_ARG, "null ctx"); \
  } while (0)
#define RS_TRY(x)                  \
  do {                             \
    int _r = (x);                  \
    if (_r != SB200_OK) return _r; \
  } while (0)

namespace sb200 {
namespace {

struct RsDevGuard {
  int prev = -1;
  explicit RsDevGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~RsDevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

__global__ void k_widen_real(const double* __restrict__ in, double2* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = make_double2(in[i], 0.0);
}

struct File {
  FILE* f = nullptr;
  File(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

std::string join(const std::string& dir, const std::string& name) {
  if (dir.empty() || dir.back() == '/') return dir + name;
  return dir + "/" + name;
}

bool put_record(FILE* f, const void* data, size_t bytes) {
  if (bytes > 0x7fffffffu) return false;
  const int32_t m = (int32_t)bytes;
  return std::fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes) &&
         std::fwrite(&m, 4, 1, f) == 1;
}

bool get_record(FILE* f, std::vector<char>& out) {
  out.clear();
  for (;;) {
    int32_t lead = 0, tail = 0;
    if (std::fread(&lead, 4, 1, f) != 1) return false;
    const size_t len = (size_t)(lead < 0 ? -(int64_t)lead : lead);
    const size_t at = out.size();
    out.resize(at + len);
    if (len && std::fread(out.data() + at, 1, len, f) != len) return false;
    if (std::fread(&tail, 4, 1, f) != 1) return false;
    if (lead >= 0) return true;
  }
}

bool get_int(FILE* f, long* v) {
  std::vector<char> r;
  if (!get_record(f, r)) return false;
  if (r.size() == 4) {
    int32_t x;
    std::memcpy(&x, r.data(), 4);
    *v = x;
    return true;
  }
  if (r.size() == 8) {
    int64_t x;
    std::memcpy(&x, r.data(), 8);
    *v = (long)x;
    return true;
  }
  return false;
}

bool get_doubles(FILE* f, double* v, size_t n) {
  std::vector<char> r;
  if (!get_record(f, r) || r.size() < n * sizeof(double)) return false;
  std::memcpy(v, r.data(), n * sizeof(double));
  return true;
}

int make_dir(const std::string& d) {
  if (::mkdir(d.c_str(), 0755) != 0 && errno != EEXIST)
    return set_error(SB200_ERR_INVALID_ARG, "cannot create directory " + d);
  return SB200_OK;
}

std::string slice_path(const std::string& dir, int ik, int nb, int io) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "k_%06d_ob_%06d", ik, nb);
  std::string d = join(dir, buf);
  std::snprintf(buf, sizeof(buf), "wfn_ob_%06d.dat", io);
  return join(d, buf);
}

std::string slice_dir(const std::string& dir, int ik, int nb) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), "k_%06d_ob_%06d", ik, nb);
  return join(dir, buf);
}

}  // namespace
}  // namespace sb200

using namespace sb200;

extern "C" {

int sb200_write_restart(sb200_ctx* c, const char* dir, int method_wf_distributor, int nblock_wf_distribute,
                        const double* psi, int if_real_orbital, int iter, int trans_longi) {
  RS_CHECK_CTX(c);
  if (!c->g.set || !c->orb.set) return set_error(SB200_ERR_STATE, "grid and orbitals must be set");
  if (!dir || !psi || (method_wf_distributor != 0 && method_wf_distributor != 1) ||
      (if_real_orbital != 0 && if_real_orbital != 1))
    return set_error(SB200_ERR_INVALID_ARG, "sb200_write_restart: bad argument");
  RsDevGuard dg(c->device);
  const std::string d(dir);
  RS_TRY(make_dir(d));
  const OrbInfo& o = c->orb;
  const size_t npts = (size_t)c->g.npts;
  const size_t esz = if_real_orbital ? sizeof(double) : 2 * sizeof(double);
  {  // info.bin
    File f(join(d, "info.bin"), "wb");
    const int32_t v[5] = {o.nk, o.no, iter, 1, if_real_orbital ? 1 : 0};
    bool ok = f.f != nullptr;
    for (int i = 0; i < 5 && ok; ++i) ok = put_record(f.f, &v[i], 4);
    if (!ok) return set_error(SB200_ERR_INVALID_ARG, "cannot write " + join(d, "info.bin"));
  }
  {  // occupation.bin
    File f(join(d, "occupation.bin"), "wb");
    if (!f.f || !put_record(f.f, o.rocc.data(), o.rocc.size() * sizeof(double)))
      return set_error(SB200_ERR_INVALID_ARG, "cannot write " + join(d, "occupation.bin"));
  }
  std::vector<char> host(npts * esz);
  const char* src = reinterpret_cast<const char*>(psi);
  auto block = [&](int ik, int io, int is) -> int {  // orbital block (1-based ik, io, is) to host
    const size_t orb = (size_t)(is - 1) + (size_t)o.nspin * ((size_t)(io - 1) + (size_t)o.no * (ik - 1));
    SB_CUDA(cudaMemcpyAsync(host.data(), src + orb * npts * esz, npts * esz, cudaMemcpyDefault, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
    return SB200_OK;
  };
  if (method_wf_distributor == 0) {  // 'single': wfn.bin
    File f(join(d, "wfn.bin"), "wb");
    if (!f.f) return set_error(SB200_ERR_INVALID_ARG, "cannot write " + join(d, "wfn.bin"));
    for (int ik = 1; ik <= o.nk; ++ik)
      for (int io = 1; io <= o.no; ++io)
        for (int is = 1; is <= o.nspin; ++is) {
          RS_TRY(block(ik, io, is));
          if (std::fwrite(host.data(), 1, host.size(), f.f) != host.size())
            return set_error(SB200_ERR_INVALID_ARG, "short write to wfn.bin");
        }
  } else {  // 'slice'
    const int nbo = nblock_wf_distribute < o.no ? (nblock_wf_distribute > 0 ? nblock_wf_distribute : 1) : o.no;
    for (int ik = 1; ik <= o.nk; ++ik)
      for (int io = 1; io <= o.no; ++io) {
        const int nb = ((io - 1) / nbo) * nbo + 1;
        RS_TRY(make_dir(slice_dir(d, ik, nb)));
        File f(slice_path(d, ik, nb, io), "wb");
        if (!f.f) return set_error(SB200_ERR_INVALID_ARG, "cannot write " + slice_path(d, ik, nb, io));
        for (int is = 1; is <= o.nspin; ++is) {
          RS_TRY(block(ik, io, is));
          if (std::fwrite(host.data(), 1, host.size(), f.f) != host.size())
            return set_error(SB200_ERR_INVALID_ARG, "short write to " + slice_path(d, ik, nb, io));
        }
      }
  }
  double *vh, *s1, *s2;
  if (scf_vh_stock(c, &vh, &s1, &s2)) {  // Vh_stock.bin (write_Vh_stock, non-self form)
    std::vector<double> a(npts), b(npts);
    SB_CUDA(cudaMemcpyAsync(a.data(), s1, npts * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaMemcpyAsync(b.data(), s2, npts * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
    File f(join(d, "Vh_stock.bin"), "wb");
    if (!f.f || !put_record(f.f, a.data(), npts * sizeof(double)) ||
        !put_record(f.f, b.data(), npts * sizeof(double)))
      return set_error(SB200_ERR_INVALID_ARG, "cannot write " + join(d, "Vh_stock.bin"));
  }
  if (trans_longi == SB200_TRANS_LO) {  // rtdata.bin (write_rtdata)
    double tot[6], ind[6];
    const double zero[3] = {0.0, 0.0, 0.0};
    int mit = 0;
    RS_TRY(sb200_rt_get_state(c, &mit, tot, ind));
    File f(join(d, "rtdata.bin"), "wb");
    if (!f.f || !put_record(f.f, tot, sizeof(tot)) || !put_record(f.f, ind, sizeof(ind)) ||
        !put_record(f.f, zero, sizeof(zero)))
      return set_error(SB200_ERR_INVALID_ARG, "cannot write " + join(d, "rtdata.bin"));
  }
  return SB200_OK;
}

int sb200_read_restart(sb200_ctx* c, const char* dir, int method_wf_distributor, int nblock_wf_distribute,
                       int yn_restart, int ik_s, int io_s, double* psi, int* iter, double* rocc_out) {
  RS_CHECK_CTX(c);
  if (!c->g.set || !c->orb.set) return set_error(SB200_ERR_STATE, "grid and orbitals must be set");
  if (!dir || !psi || (method_wf_distributor != 0 && method_wf_distributor != 1) || ik_s < 1 || io_s < 1)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_read_restart: bad argument");
  RsDevGuard dg(c->device);
  const std::string d(dir);
  OrbInfo& o = c->orb;
  const size_t npts = (size_t)c->g.npts;
  long mk = 0, mo = 0, itt = 0, nprocs = 0, lreal = 0;
  {
    File f(join(d, "info.bin"), "rb");
    if (!f.f || !get_int(f.f, &mk) || !get_int(f.f, &mo) || !get_int(f.f, &itt) || !get_int(f.f, &nprocs) ||
        !get_int(f.f, &lreal))
      return set_error(SB200_ERR_INVALID_ARG, "cannot read " + join(d, "info.bin"));
  }
  const bool is_real = lreal != 0;
  if (ik_s - 1 + o.nk > mk || io_s - 1 + o.no > mo)
    return set_error(SB200_ERR_BAD_SHAPE, "restart data hold fewer k-points or orbitals than the context");
  {  // occupation.bin: rocc(1:no,1:nk,1:nspin) = roccbox(...) of the mo x mk x nspin box
    std::vector<double> box((size_t)mo * mk * o.nspin);
    File f(join(d, "occupation.bin"), "rb");
    if (!f.f || !get_doubles(f.f, box.data(), box.size()))
      return set_error(SB200_ERR_INVALID_ARG, "cannot read " + join(d, "occupation.bin"));
    std::vector<double> rocc((size_t)o.no * o.nk * o.nspin);
    for (int is = 0; is < o.nspin; ++is)
      for (int ik = 0; ik < o.nk; ++ik)
        for (int io = 0; io < o.no; ++io)
          rocc[io + (size_t)o.no * (ik + (size_t)o.nk * is)] =
              box[(io + io_s - 1) + (size_t)mo * ((ik + ik_s - 1) + (size_t)mk * is)];
    const std::vector<double> vk = o.vec_k, wtk = o.wtk;
    RS_TRY(sb200_set_orbitals(c, o.nspin, o.no, o.nk, vk.data(), rocc.data(), wtk.data()));
    if (rocc_out) std::memcpy(rocc_out, rocc.data(), rocc.size() * sizeof(double));
  }
  const size_t esz = is_real ? sizeof(double) : 2 * sizeof(double);
  std::vector<char> host(npts * esz);
  double* d_real = nullptr;
  if (is_real) RS_TRY(dalloc(&d_real, npts));
  int rc = SB200_OK;
  auto store = [&](int ik, int io, int is) -> int {  // host block of global (ik, io, is) to psi
    const size_t orb = (size_t)(is - 1) + (size_t)o.nspin * ((size_t)(io - io_s) + (size_t)o.no * (ik - ik_s));
    double2* dst = reinterpret_cast<double2*>(psi) + orb * npts;
    // copies and the widening kernel in order on the context's stream, finished
    // before the host buffer is refilled
    if (!is_real) {
      SB_CUDA(cudaMemcpyAsync(dst, host.data(), npts * esz, cudaMemcpyHostToDevice, c->stream));
      SB_CUDA(cudaStreamSynchronize(c->stream));
      return SB200_OK;
    }
    SB_CUDA(cudaMemcpyAsync(d_real, host.data(), npts * esz, cudaMemcpyHostToDevice, c->stream));
    long nb = ((long)npts + 255) / 256;
    if (nb > 148L * 8) nb = 148L * 8;
    k_widen_real<<<(unsigned)nb, 256, 0, c->stream>>>(d_real, dst, (long)npts);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(c->stream));
    return SB200_OK;
  };
  auto wanted = [&](int ik, int io) {
    return ik >= ik_s && ik < ik_s + o.nk && io >= io_s && io < io_s + o.no;
  };
  if (method_wf_distributor == 0) {  // read_all
    File f(join(d, "wfn.bin"), "rb");
    if (!f.f) rc = set_error(SB200_ERR_INVALID_ARG, "cannot read " + join(d, "wfn.bin"));
    for (int ik = 1; ik <= mk && rc == SB200_OK; ++ik)
      for (int io = 1; io <= mo && rc == SB200_OK; ++io)
        for (int is = 1; is <= o.nspin && rc == SB200_OK; ++is) {
          if (!wanted(ik, io)) {
            if (std::fseek(f.f, (long)(npts * esz), SEEK_CUR) != 0)
              rc = set_error(SB200_ERR_INVALID_ARG, "short wfn.bin");
            continue;
          }
          if (std::fread(host.data(), 1, host.size(), f.f) != host.size())
            rc = set_error(SB200_ERR_INVALID_ARG, "short wfn.bin");
          else
            rc = store(ik, io, is);
        }
  } else {  // read_sliced
    const long nbo = nblock_wf_distribute < mo ? (nblock_wf_distribute > 0 ? nblock_wf_distribute : 1) : mo;
    for (int ik = ik_s; ik < ik_s + o.nk && rc == SB200_OK; ++ik)
      for (int io = io_s; io < io_s + o.no && rc == SB200_OK; ++io) {
        const int nb = (int)(((io - 1) / nbo) * nbo + 1);
        File f(slice_path(d, ik, nb, io), "rb");
        if (!f.f) {
          rc = set_error(SB200_ERR_INVALID_ARG, "cannot read " + slice_path(d, ik, nb, io));
          break;
        }
        for (int is = 1; is <= o.nspin && rc == SB200_OK; ++is) {
          if (std::fread(host.data(), 1, host.size(), f.f) != host.size())
            rc = set_error(SB200_ERR_INVALID_ARG, "short " + slice_path(d, ik, nb, io));
          else
            rc = store(ik, io, is);
        }
      }
  }
  dfree(d_real);
  if (rc != SB200_OK) return rc;
  if (iter) *iter = yn_restart ? (int)itt : 0;
  if (!yn_restart) return SB200_OK;
  // restart_rt: Mit, the stored potentials, the fields of 'lo'
  double tot[6], ind[6];
  bool seeds = false;
  {
    File f(join(d, "rtdata.bin"), "rb");
    if (f.f) {
      if (!get_doubles(f.f, tot, 6) || !get_doubles(f.f, ind, 6))
        return set_error(SB200_ERR_INVALID_ARG, "cannot read " + join(d, "rtdata.bin"));
      seeds = true;
    }
  }
  RS_TRY(sb200_rt_set_start(c, (int)itt, seeds ? tot : nullptr, seeds ? ind : nullptr));
  double *vh, *s1, *s2;
  if (scf_vh_stock(c, &vh, &s1, &s2)) {
    File f(join(d, "Vh_stock.bin"), "rb");
    if (f.f) {
      std::vector<double> a(npts), b(npts);
      if (!get_doubles(f.f, a.data(), npts) || !get_doubles(f.f, b.data(), npts))
        return set_error(SB200_ERR_INVALID_ARG, "cannot read " + join(d, "Vh_stock.bin"));
      SB_CUDA(cudaMemcpyAsync(s1, a.data(), npts * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      SB_CUDA(cudaMemcpyAsync(s2, b.data(), npts * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      SB_CUDA(cudaStreamSynchronize(c->stream));
      RS_TRY(scf_restart_potential(c, reinterpret_cast<const double2*>(psi)));
    }
  }
  return SB200_OK;
}

}  // extern "C"
