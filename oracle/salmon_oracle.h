/*
 * salmon_oracle.h -- CPU oracle for the SALMON RT-TDDFT propagation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++/OpenMP restatement of the
 * reference's Fortran algorithms (SALMON v2.2.0), used as the parity checker
 * for the CUDA library and as the timed CPU baseline ("port").  The product
 * library (salmon2_b200/csrc) never links, loads or calls it.
 *
 * Parity status of this oracle:
 *   - zpseudo (KB nonlocal) and the local part of calc_current are pinned
 *     against the reference's own CUDA kernels (src/common/zpseudo.cu,
 *     src/common/stencil_current.cu) compiled from the reference sources into
 *     oracle/_ref and run on the GPU; their outputs are committed as golden
 *     fixtures in tests/golden/.
 *   - zstencil (with the k+A coefficients and V_local of hpsi) is pinned
 *     against the reference's own hand-vectorised AVX-512 stencil
 *     (src/common/zstencil_core/avx512/seq.c, built with gcc into oracle/_ref)
 *     on periodic grids; golden fixture in tests/golden/.
 *   - taylor / calc_density / calc_dip / calc_emfields and the
 *     ground-state CG are pinned only by analytic known-answer tests
 *     (plane-wave eigenvalues of the finite-difference operator, exact Taylor
 *     polynomials of diagonal systems, Hermiticity, conservation laws): the
 *     Fortran reference cannot be compiled here (no Fortran compiler), so
 *     those parts are "parity unpinned" against reference outputs.
 *
 * Memory layout follows the reference exactly: Fortran column-major arrays,
 * x fastest, complex(8) stored as interleaved (re, im) doubles, with the
 * reference's array bounds (is_array:ie_array, halo of 4 for isolated grids,
 * +1 padding on the y extent when the caller asks for it).
 */
#ifndef SALMON_ORACLE_H
#define SALMON_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of the subset of s_rgrid / s_stencil / s_dft_system / s_pp_grid the
 * hot path reads (src/common/structures.f90:86-203,254-319). */
typedef struct {
  /* s_rgrid (structures.f90:86-94): interior and allocated bounds */
  int is[3], ie[3], is_array[3], ie_array[3];
  /* idx/idy/idz(is-4:ie+4): neighbour index maps (initialization.f90:570-600) */
  const int *idx, *idy, *idz;
  int lg_num[3];            /* global grid size (dip.f90:128 parity switch)  */
  /* s_stencil (initialization.f90:241-256) */
  double coef_lap0;
  double coef_lap[12];      /* (4,3) column-major                            */
  double coef_nab[12];      /* (4,3) column-major                            */
  /* s_dft_system */
  int periodic;             /* 0 isolated, 1 periodic (yn_periodic)           */
  int nspin, no, nk;        /* io = 1..no, ik = 1..nk, im = 1                 */
  double hgs[3], hvol;
  int ngrid;                /* system%ngrid                                   */
  const double *vec_k;      /* (3,nk)                                         */
  double vec_Ac[3];         /* system%vec_Ac (A/c)                            */
  const double *rocc;       /* (no,nk,nspin)                                  */
  const double *wtk;        /* (nk)                                           */
  double BT[9];             /* transpose(rmatrix_B), (3,3) column-major       */
  const double *V_local;    /* (is:ie, nspin) interior                        */
  /* s_pp_grid (structures.f90:254-319) */
  int natom, nps, nlma;
  const int *mps;           /* (natom)                                        */
  const int *jxyz;          /* (3,nps,natom)                                  */
  const double *rxyz;       /* (3,nps,natom)                                  */
  const double *uv;         /* (nps,nlma)                                     */
  const int *ia_tbl;        /* (nlma), 1-based atom index                     */
  const double *rinv_uvu;   /* (nlma)                                         */
  double *zekr;             /* (nps,nlma,nk) complex; written by update_kvector */
  /* OpenMP mode: 1 = grid-parallel stencil (>=32^3), 0 = orbital-parallel   */
  int stencil_rgrid_mode;
  /* non-orthogonal lattice (stencil%if_orthogonal = .false.): system%rmatrix_B
   * and stencil%coef_F of init_lattice (lattice.f90:23-75)                    */
  int nonorth;
  double rmatrix_B[9];      /* (3,3) column-major                            */
  double coef_F[6];
  /* single-scale Maxwell-TDDFT: system%Ac_micro%v (3, is:ie) and
   * system%div_Ac%f (is:ie), or NULL (hamiltonian.f90:236-298)              */
  const double *ac_micro;
  const double *div_ac;
  /* yn_symmetrized_stencil = 'y': zstencil_microAc_symmetrized (div_ac unused) */
  int symmetrized;
  /* absorbing_boundary = 'z' (hamiltonian.f90:760-807): imagnary_potential_w0,
   * imagnary_potential_dr, al(3) */
  int cap_on;
  double cap_w0, cap_dr, cap_al;
  /* isolated grid, pulse in the length gauge (ae_shape1 /= 'impulse'):
   * V_local + E_ext(itt).r in each step's Taylor expansion                  */
  int length_gauge;
  /* propagator = 'aetrs' (time_evolution_step.f90:117-147, 430-470): half
   * steps (zc of -i dt/2) around the extrapolated potential                  */
  int aetrs;
  /* yn_predictor_corrector = 'y' (time_evolution_step.f90:374-428)           */
  int pred_corr;
  /* gram_schmidt_interval >= 1: gram_schmidt of psi(t+dt) every N steps
   * (time_evolution_step.f90:149-152)                                        */
  int gs_interval;
} sbo_system;

void sbo_set_threads(int n);
int  sbo_get_threads(void);

/* impulse kick of the initial orbitals (initialization_rt.f90:382-423) */
void sbo_impulse_kick(const sbo_system* s, double* psi, double e_impulse, const double epdir[3]);

/* Real-space stencil kernels */
void sbo_zstencil(const sbo_system* s, const double* tpsi, double* htpsi,
                  const double* V_local, double lap0, const double* lapt,
                  const double* nabt);
void sbo_dstencil(const sbo_system* s, const double* tpsi, double* htpsi,
                  const double* V_local, double lap0, const double* lapt);

/* update_kvector_nonlocalpt (hamiltonian.f90:847-903); isolated: zekr = uV */
void sbo_update_kvector_nonlocalpt(sbo_system* s);

/* zpseudo / dpseudo over all orbitals of the block (nonlocal_potential.f90) */
void sbo_zpseudo(const sbo_system* s, const double* tpsi, double* htpsi);
void sbo_dpseudo(const sbo_system* s, const double* tpsi, double* htpsi);
/* Projections uVpsi(ilma, orbital) = rinv_uvu * <zekr|psi> (diagnostics) */
void sbo_zprojections(const sbo_system* s, const double* tpsi, double* uvpsi);

/* hpsi, complex orbitals, orthogonal lattice (hamiltonian.f90:27-235,424-435) */
void sbo_hpsi(const sbo_system* s, const double* tpsi, double* htpsi);
/* hpsi with the optional ttpsi: the kinetic part, stencil output minus V psi
 * before the nonlocal term (hamiltonian.f90:364-414).                           */
void sbo_hpsi_tt(const sbo_system* s, const double* tpsi, double* htpsi, double* ttpsi);
/* calc_eigen_energy, complex orbitals (total_energy.f90:505-775):
 * esp(no,nk,nspin), e[0] = E_kin, e[1] = E_ion_nloc.                            */
void sbo_calc_eigen_energy(const sbo_system* s, const double* tpsi, double* htpsi, double* ttpsi, double* esp,
                           double* e);
/* hpsi, real orbitals (hamiltonian.f90:88-125) */
void sbo_hpsi_real(const sbo_system* s, const double* tpsi, double* htpsi);

/* taylor (taylor.f90:21-121); zc = complex(n_hamil) interleaved */
void sbo_taylor(const sbo_system* s, double* tspsi_in, double* tspsi_out,
                double* sshtpsi, const double* zc, int n_hamil);

/* calc_density (density_matrix.f90:150-232) -> rho(is:ie, nspin) */
void sbo_calc_density(const sbo_system* s, const double* psi, double* rho);
/* calc_current (density_matrix.f90:240-463), curr(3,nspin); uses vec_Ac for
 * the local term and zekr (as last updated) for the nonlocal term.          */
void sbo_calc_current(const sbo_system* s, const double* psi, double* curr);
/* per-orbital pieces of calc_current: out(10, norb) =
 * [rtmp, Im-sums*2 (x,y,z) (before BT), jw(3) nonlocal, j_total(3) weighted] */
void sbo_current_parts(const sbo_system* s, const double* psi, double* out);
/* calc_microscopic_current (density_matrix.f90:726-845) -> curr(3, is:ie) */
void sbo_calc_microscopic_current(const sbo_system* s, const double* psi, double* curr);
/* calc_dip (dip.f90:114-225): rbox(4) */
void sbo_calc_dip(const sbo_system* s, const double* rho, double* rbox);

/* calc_Ac_ext_t shapes (em_field.f90:86-306): shape 0 = impulse,
 * 1 = Asin2cos, 2 = Acos2.  Ac(3, is:ie) at t = t0 + i*delta_t.            */
void sbo_calc_Ac_ext_t(int shape, double t0, double delta_t, int is, int ie,
                       const double* epdir, double f0, double omega,
                       double tw, double phi_cep, double t1_start,
                       double e_impulse, double* Ac);

/* Time loop: nt steps of time_evolution_step (time_evolution_step.f90:102-312)
 * for the linear-response path (fixed V_local, no Hartree/XC update).
 *   psi_a holds psi(0) on entry; on exit the final orbitals are returned in
 *   the buffer *which_out (0 -> psi_a, 1 -> psi_b).
 *   Ac_ext(3,0:nt+1) and Ac_ind(3,0:nt+1) / Ac_tot(3,0:nt+1) in/out.
 *   trans_longi: 0 = 'tr', 1 = 'lo'.
 *   Outputs per step itt=1..nt: curr(3,nt) (periodic), rbox(4,nt) (calc_dip).
 */
int sbo_rt_run(sbo_system* s, double* psi_a, double* psi_b, double* work,
               int nt, double dt, const double* zc, int n_hamil,
               const double* Ac_ext, double* Ac_ind, double* Ac_tot,
               int trans_longi, double* curr, double* rbox, double* rho_work);

/* Ground state, real orbitals, one k (salmon_oracle_gs.cpp).
 * dstencil_preconditioning (src/gs/preconditioning.f90:25-77) on every orbital */
void sbo_precond_real(const sbo_system* s, const double* gk, double* pre_gk, double alpha);
/* gscg_rwf (src/gs/conjugate_gradient.f90:21-466); work = 7 orbital blocks;
 * esp_out(nspin*no) = final Rayleigh quotients.                              */
void sbo_gscg_rwf(const sbo_system* s, int ncg, double* psi, double* work, int precondition,
                  double alpha_pre, double* esp_out);
/* classical Gram-Schmidt (src/gs/gram_schmidt_orth.f90:59-230, 1069-1242)     */
void sbo_gram_schmidt_real(const sbo_system* s, double* psi);
void sbo_gram_schmidt_complex(const sbo_system* s, double* psi);
/* ssdg_rwf (src/gs/subspace_diagonalization.f90:62-238) with a Jacobi
 * eigensolver instead of LAPACK dsyev; work = one orbital block.             */
void sbo_subspace_diag_real(const sbo_system* s, double* psi, double* work, double* evals);
void sbo_inner_product_real(const sbo_system* s, const double* x, const double* y, double* out);

/* Per-step potential update (salmon_oracle_scf.cpp): PZ-LDA exchange-correlation
 * for nspin = 1 (src/xc/builtin_pz.f90, src/xc/salmon_xc.f90:86-254), the
 * periodic Hartree potential by separable DFTs (poisson_ft,
 * src/poisson/poisson_periodic.f90:23-242) and update_vlocal
 * (src/common/hamiltonian.f90:813-843).  Interior arrays, x fastest.           */
void sbo_exc_cor_pz(long n, const double* rho, double hvol, double* vxc, double* E_xc);
/* exchange_correlation, nspin = 2, xc = 'PZ' (exc_cor_pz_sp / PZxc_sp,
 * builtin_pz_sp.f90:23-95): rho_s(n, 2) -> vxc_s(n, 2), E_xc               */
void sbo_exc_cor_pz_sp(long n, const double* rho_s, double hvol, double* vxc_s, double* E_xc);
void sbo_poisson_coef(const int num[3], const double brl[9], double* coef);
void sbo_dft_table(int n, double* eg);
void sbo_poisson_ft(const int num[3], const double brl[9], const double* rho, double* vh);
void sbo_poisson_isolated_ft(const int num[3], const double brl[9], const double* rho, double* vh);
void sbo_update_vlocal(long n, int nspin, const double* vpsl, const double* vh, const double* vxc, double* vloc);
/* poisson_isolated_cg with the multipole boundary (src/poisson/poisson_isolated.f90:
 * 30-690; pole tables of src/poisson/init_poisson.f90:23-299): layout 1 / 2 / 3,
 * lmax <= 4, rion [natom][3], npole_xyz the cells of layout 3.  vh: start value
 * in, solution out (interior, x fastest).                                       */
void sbo_poisson_isolated_cg(const sbo_system* s, const double* rho, double* vh, int layout, int lmax,
                             const double* rion, int natom, const int npole_xyz[3], double threshold,
                             int maxiter, int* iterations);
/* sbo_rt_run_scf on an isolated grid with the Hartree potential by
 * poisson_isolated_cg (method_poisson = 'cg') and the Vh extrapolation of
 * time_evolution_step.f90:186-198: vh holds the potential of the initial density
 * on entry (initialization_rt.f90:277-286) and the last step's on exit;
 * iters[nt] the iterations of each solve.  Returns -1 for nspin 2 or periodic. */
int sbo_rt_run_scf_cg(sbo_system* s, double* psi_a, double* psi_b, double* work, int nt, double dt,
                      const double* zc, int n_hamil, const double* Ac_ext, double* Ac_ind, double* Ac_tot,
                      int trans_longi, double* curr, double* rbox, double* rho_work, const double* vpsl,
                      double* vloc, double* vh, int layout, int lmax, const double* rion, int natom,
                      const int npole_xyz[3], double threshold, int maxiter, int* iters);
/* Ylm (src/math/salmon_math.f90:386-426), lm = l^2 + l + m, l <= 4            */
double sbo_ylm(double x, double y, double z, int lm);
/* sbo_rt_run with the self-consistent potential update every step (nspin = 1;
 * periodic or isolated Hartree by transforms): vloc holds V_local on entry and
 * is rewritten each step as Vpsl + Vh[rho] + Vxc[rho]; returns -1 for nspin 2. */
int sbo_rt_run_scf(sbo_system* s, double* psi_a, double* psi_b, double* work, int nt, double dt,
                   const double* zc, int n_hamil, const double* Ac_ext, double* Ac_ind,
                   double* Ac_tot, int trans_longi, double* curr, double* rbox, double* rho_work,
                   const double* vpsl, const double brl[9], double* vloc);

#ifdef __cplusplus
}
#endif
#endif
