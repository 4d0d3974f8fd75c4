/*
 * salmon_b200.hpp -- C++ host side above the C ABI (salmon_b200.h).
 *
 * SALMON's hot path is compiled Fortran; where no Fortran compiler is at hand
 * this header is the host mirror of its call surface: the derived types the
 * path reads (src/common/structures.f90), a context that holds their device
 * copies, and hpsi / taylor / calc_* with the reference's names and argument
 * meaning.  Where the reference stops the program on an invalid call, the
 * mirror throws salmon_b200::error carrying the library's status code and
 * message.  Orbitals (s_orbital) live on the device in the library's resident
 * layout; from_ref / to_ref convert from / to the reference's zwf arrays.
 *
 * Header-only; link with libsalmon_b200.so and the CUDA runtime.
 */
#ifndef SALMON_B200_HPP
#define SALMON_B200_HPP

#include <cuda_runtime.h>

#include <complex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "salmon_b200.h"

namespace salmon_b200 {

class error : public std::runtime_error {
 public:
  error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int status, const char* where) {
  if (status != SB200_OK) throw error(status, std::string(where) + ": " + sb200_last_error());
}

// ---- mirrors of the reference's derived types (the fields the path reads) --

// s_rgrid (structures.f90:198-203) of one r-space domain holding the whole
// grid, plus lg%num.  idx/idy/idz cover is-4 .. ie+4 (Fortran mg%idx).
struct s_rgrid {
  int is[3], ie[3], is_array[3], ie_array[3], lg_num[3];
  std::vector<int> idx, idy, idz;
};

// s_stencil (structures.f90:86-94): coef_lap(4,3), coef_nab(4,3), Fortran order.
struct s_stencil {
  double coef_lap0;
  double coef_lap[12];
  double coef_nab[12];
};

// s_dft_system (structures.f90:126-203): the fields of the orbital block.
struct s_dft_system {
  int nspin, no, nk;
  double hgs[3], hvol;
  std::vector<double> vec_k;  // (3, nk)
  std::vector<double> rocc;   // (no, nk, nspin)
  std::vector<double> wtk;    // (nk)
  double vec_Ac[3];           // A/c of the current step
};

// s_pp_grid (structures.f90:254-319): Kleinman-Bylander tables.
struct s_pp_grid {
  int natom = 0, nps = 0, nlma = 0;
  std::vector<int> mps;         // (natom)
  std::vector<int> jxyz;        // (3, nps, natom)
  std::vector<double> rxyz;     // (3, nps, natom)
  std::vector<double> uv;       // (nps, nlma)
  std::vector<int> ia_tbl;      // (nlma), 1-based
  std::vector<double> rinv_uvu; // (nlma)
};

// s_scalar (structures.f90): V_local(ispin)%f on the interior points.
struct s_scalar {
  std::vector<double> f;
};

// rt%zc (initialization_rt.f90:492-507): the n_hamil Taylor coefficients.
struct s_rt {
  std::vector<std::complex<double>> zc;
};

// ---- context: device copies of grid, stencil, orbitals' k-points, V, KB ----
class context {
 public:
  context(int device, const s_rgrid& mg, const s_stencil& stencil, const s_dft_system& system,
          const std::vector<s_scalar>& V_local, const s_pp_grid& ppg) {
    check(sb200_ctx_create(device, &h_), "sb200_ctx_create");
    try {
      check(sb200_set_grid(h_, mg.is, mg.ie, mg.is_array, mg.ie_array, mg.idx.data(), mg.idy.data(), mg.idz.data(),
                           mg.lg_num, system.hgs, system.hvol, stencil.coef_lap0, stencil.coef_lap,
                           stencil.coef_nab),
            "sb200_set_grid");
      check(sb200_set_orbitals(h_, system.nspin, system.no, system.nk, system.vec_k.data(), system.rocc.data(),
                               system.wtk.data()),
            "sb200_set_orbitals");
      std::vector<double> v;
      for (const s_scalar& s : V_local) v.insert(v.end(), s.f.begin(), s.f.end());
      check(sb200_set_vlocal(h_, v.data()), "sb200_set_vlocal");
      check(sb200_set_pp(h_, ppg.natom, ppg.nps, ppg.nlma, ppg.mps.data(), ppg.jxyz.data(), ppg.rxyz.data(),
                         ppg.uv.data(), ppg.ia_tbl.data(), ppg.rinv_uvu.data()),
            "sb200_set_pp");
      check(sb200_set_vec_Ac(h_, system.vec_Ac), "sb200_set_vec_Ac");
      for (int d = 0; d < 3; ++d) ac_[d] = system.vec_Ac[d];
    } catch (...) {
      sb200_ctx_destroy(h_);
      throw;
    }
  }
  ~context() { sb200_ctx_destroy(h_); }
  context(const context&) = delete;
  context& operator=(const context&) = delete;

  sb200_ctx* get() const { return h_; }
  void sync() { check(sb200_ctx_sync(h_), "sb200_ctx_sync"); }
  // system%vec_Ac as hpsi reads it: the k+A coefficients and projector phases
  // follow the caller's system each call (update_kvector_nonlocalpt)
  void follow(const s_dft_system& system) {
    if (system.vec_Ac[0] != ac_[0] || system.vec_Ac[1] != ac_[1] || system.vec_Ac[2] != ac_[2]) {
      check(sb200_set_vec_Ac(h_, system.vec_Ac), "sb200_set_vec_Ac");
      for (int d = 0; d < 3; ++d) ac_[d] = system.vec_Ac[d];
    }
  }

 private:
  sb200_ctx* h_ = nullptr;
  double ac_[3] = {0.0, 0.0, 0.0};
};

// s_orbital: one orbital block on the device (resident layout).
class s_orbital {
 public:
  explicit s_orbital(const context& ctx) : ctx_(ctx.get()), bytes_(sb200_orbital_block_bytes(ctx.get())) {
    const cudaError_t e = cudaMalloc(&d_, bytes_);
    if (e != cudaSuccess) throw error(SB200_ERR_OOM, std::string("s_orbital: ") + cudaGetErrorString(e));
    cudaMemset(d_, 0, bytes_);
  }
  ~s_orbital() { cudaFree(d_); }
  s_orbital(const s_orbital&) = delete;
  s_orbital& operator=(const s_orbital&) = delete;

  double* data() { return static_cast<double*>(d_); }
  const double* data() const { return static_cast<const double*>(d_); }
  // zwf(is_array:ie_array, nspin, no, nk) of the reference <-> device block
  void from_ref(const std::complex<double>* zwf) {
    check(sb200_orbitals_from_ref(ctx_, reinterpret_cast<const double*>(zwf), data()), "sb200_orbitals_from_ref");
  }
  void to_ref(std::complex<double>* zwf) const {
    check(sb200_orbitals_to_ref(ctx_, data(), reinterpret_cast<double*>(zwf)), "sb200_orbitals_to_ref");
  }

 private:
  sb200_ctx* ctx_;
  size_t bytes_;
  void* d_ = nullptr;
};

// ---- the call surface --------------------------------------------------------

// hpsi(tpsi,htpsi,info,mg,V_local,system,stencil,srg,ppg) (hamiltonian.f90:27)
inline void hpsi(context& ctx, const s_orbital& tpsi, s_orbital& htpsi, const s_dft_system& system) {
  ctx.follow(system);
  check(sb200_hpsi(ctx.get(), tpsi.data(), htpsi.data()), "hpsi");
}

// hpsi(..., ttpsi) with the optional kinetic output (hamiltonian.f90:364-414)
inline void hpsi(context& ctx, const s_orbital& tpsi, s_orbital& htpsi, s_orbital& ttpsi,
                 const s_dft_system& system) {
  ctx.follow(system);
  check(sb200_hpsi_tt(ctx.get(), tpsi.data(), htpsi.data(), ttpsi.data()), "hpsi");
}

// taylor(mg,system,info,stencil,srg,tspsi_in,tspsi_out,sshtpsi,ppg,V_local,rt)
// (taylor.f90:21); tspsi_in and sshtpsi are scratch on return.
inline void taylor(context& ctx, const s_dft_system& system, s_orbital& tspsi_in, s_orbital& tspsi_out,
                   s_orbital& sshtpsi, const s_rt& rt) {
  ctx.follow(system);
  check(sb200_taylor(ctx.get(), tspsi_in.data(), tspsi_out.data(), sshtpsi.data(),
                     reinterpret_cast<const double*>(rt.zc.data()), static_cast<int>(rt.zc.size())),
        "taylor");
}

// calc_density(system,rho,psi,info,mg) (density_matrix.f90:26): rho(ispin)%f
inline void calc_density(context& ctx, std::vector<s_scalar>& rho, const s_orbital& psi) {
  std::vector<double> r;
  size_t n = rho.empty() ? 0 : rho[0].f.size();
  r.resize(n * rho.size());
  check(sb200_calc_density(ctx.get(), psi.data(), r.data()), "calc_density");
  for (size_t s = 0; s < rho.size(); ++s) std::copy(r.begin() + s * n, r.begin() + (s + 1) * n, rho[s].f.begin());
}

// calc_current (density_matrix.f90:240-463): curr(3, nspin) for A/c = vec_Ac
inline void calc_current(context& ctx, const s_orbital& psi, const double vec_Ac[3], double* curr) {
  check(sb200_calc_current(ctx.get(), psi.data(), vec_Ac, curr), "calc_current");
}

// calc_eigen_energy (total_energy.f90:505): esp(no,nk,nspin), E_kin, E_ion_nloc
inline void calc_eigen_energy(context& ctx, const s_orbital& tpsi, s_orbital& htpsi, s_orbital& ttpsi,
                              const s_dft_system& system, std::vector<double>& esp, double& e_kin,
                              double& e_ion_nloc) {
  ctx.follow(system);
  esp.assign(static_cast<size_t>(system.no) * system.nk * system.nspin, 0.0);
  check(sb200_calc_eigen_energy(ctx.get(), tpsi.data(), htpsi.data(), ttpsi.data(), esp.data(), &e_kin,
                                &e_ion_nloc),
        "calc_eigen_energy");
}

// hartree(lg,mg,info,system,fg,poisson,srg_scalar,stencil,rho,Vh) (hartree.f90:20) on
// a periodic grid: poisson_ft (poisson_periodic.f90:23); primitive_b = system%primitive_b
inline void hartree(context& ctx, const double primitive_b[9], const s_scalar& rho, s_scalar& Vh) {
  Vh.f.resize(rho.f.size());
  check(sb200_hartree_periodic(ctx.get(), primitive_b, rho.f.data(), Vh.f.data()), "hartree");
}

// the same call on an isolated system with method_poisson = 'ft': poisson_isolated_ft
// (poisson_isolated.f90:692)
inline void hartree_isolated_ft(context& ctx, const double primitive_b[9], const s_scalar& rho, s_scalar& Vh) {
  Vh.f.resize(rho.f.size());
  check(sb200_hartree_isolated_ft(ctx.get(), primitive_b, rho.f.data(), Vh.f.data()), "hartree");
}

// exchange_correlation(system,xc_func,mg,srg_scalar,srg,rho_s,ppn,info,spsi,stencil,Vxc,E_xc)
// (salmon_xc.f90:58) with xc = 'PZ' and nspin = 1
inline void exchange_correlation(context& ctx, const s_scalar& rho, std::vector<s_scalar>& Vxc, double& E_xc) {
  Vxc.resize(1);
  Vxc[0].f.resize(rho.f.size());
  check(sb200_exc_cor_pz(ctx.get(), rho.f.data(), Vxc[0].f.data(), &E_xc), "exchange_correlation");
}

// update_vlocal(mg,nspin,Vh,Vpsl,Vxc,Vlocal) (hamiltonian.f90:813): V_local of the
// context (its device copy, used by hpsi / taylor) becomes Vpsl + Vh + Vxc(ispin)
inline void update_vlocal(context& ctx, const s_scalar& Vh, const s_scalar& Vpsl, const std::vector<s_scalar>& Vxc) {
  const size_t n = Vpsl.f.size();
  std::vector<double> x(n * Vxc.size());
  for (size_t s = 0; s < Vxc.size(); ++s) std::copy(Vxc[s].f.begin(), Vxc[s].f.end(), x.begin() + s * n);
  check(sb200_update_vlocal(ctx.get(), Vpsl.f.data(), Vh.f.data(), x.data()), "update_vlocal");
}

// yn_fix_func = 'n' (time_evolution_step.f90:160-207): sb200_rt_propagate recomputes
// V_local = Vpsl + Vh[rho] + Vxc[rho] after every step; enable = false: fixed potential
inline void set_self_consistent(context& ctx, bool enable, const s_scalar& Vpsl, const double primitive_b[9]) {
  check(sb200_set_self_consistent(ctx.get(), enable ? 1 : 0, enable ? Vpsl.f.data() : nullptr,
                                  enable ? primitive_b : nullptr),
        "set_self_consistent");
}

// rho summed over the processes that share the k-points (comm_summation over
// icomm_ko, density_matrix.f90:223): id from sb200_nccl_unique_id on rank 0
inline void set_density_comm(context& ctx, int nranks, int rank, const unsigned char id[128]) {
  check(sb200_set_density_comm(ctx.get(), nranks, rank, id), "set_density_comm");
}

// gram_schmidt(system, mg, info, psi) for complex orbitals (gram_schmidt_orth.f90:1069)
inline void gram_schmidt(context& ctx, s_orbital& psi) {
  check(sb200_gram_schmidt_complex(ctx.get(), psi.data()), "gram_schmidt");
}

}  // namespace salmon_b200

#endif  // SALMON_B200_HPP
