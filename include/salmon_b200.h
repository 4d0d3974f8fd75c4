/*
 * salmon_b200.h -- C ABI of the B200-native RT-TDDFT propagation library.
 *
 * Drop-in boundary for SALMON's hpsi / taylor hot path (SALMON v2.2.0).  The
 * entry points take plain pointers and sizes only.  Host arrays use the
 * reference's own layout (Fortran column-major, x fastest, the caller's
 * is_array:ie_array bounds, complex(8) as interleaved re/im doubles).  Orbital
 * arrays that the compute entry points read and write are DEVICE arrays in the
 * library's resident layout ("orbital block"):
 *
 *     psi[o][iz][iy][ix]  complex double, o = ispin-1 + nspin*((io-1) + no*(ik-1)),
 *     ix in 0..nx-1 fastest (interior points only, no halo, no padding),
 *
 * sized by sb200_orbital_block_bytes().  sb200_orbitals_from_ref /
 * sb200_orbitals_to_ref convert between the two layouts.
 *
 * Every function returns 0 on success or one of the SB200_ERR_* codes; a
 * description of the last failure on the calling thread is returned by
 * sb200_last_error().  A context is used from one host thread at a time; all
 * work is ordered on the context's stream.  Compute entry points are
 * asynchronous unless stated otherwise.
 */
#ifndef SALMON_B200_H
#define SALMON_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB200_OK 0
#define SB200_ERR_INVALID_ARG 1  /* null pointer, bad enum, inconsistent sizes          */
#define SB200_ERR_BAD_SHAPE 2    /* grid / orbital / table shape the path cannot take   */
#define SB200_ERR_UNSUPPORTED 3  /* valid reference input outside this path's scope     */
#define SB200_ERR_OOM 4          /* device allocation failed                           */
#define SB200_ERR_CUDA 5         /* CUDA runtime / launch error                        */
#define SB200_ERR_TIMEOUT 6      /* a bounded device wait expired                       */
#define SB200_ERR_STATE 7        /* call order: e.g. hpsi before set_grid               */

#define SB200_PREC_FP64 0  /* plain FP64 form                                          */
#define SB200_PREC_MIXED 1 /* FP32 stencil for Taylor terms n >= 2, FP64 accumulation  */

#define SB200_PRECOND_NONE 0    /* gscg without preconditioner (yn_preconditioning='n')  */
#define SB200_PRECOND_LOWPASS 1 /* preconditioning_rgk low-pass filter, alpha_pre         */
#define SB200_PRECOND_LEARNED 2 /* learned 3-D convolutional preconditioner               */

#define SB200_TRANS_TR 0 /* trans_longi = 'tr': no induced field                      */
#define SB200_TRANS_LO 1 /* trans_longi = 'lo': A_ind from the current                  */

typedef struct sb200_ctx sb200_ctx;

/* Kernel classes reported by sb200_kernel_times.                              */
#define SB200_KIND_PREP 0      /* k+A coefficients and projector phases        */
#define SB200_KIND_PROJECT 1   /* KB projections <beta|psi>                     */
#define SB200_KIND_HPSI 2      /* fused stencil + V + KB scatter + Taylor term  */
#define SB200_KIND_OBS 3       /* density / current / dipole partial sums       */
#define SB200_KIND_MOMENTS 4   /* nonlocal current projections                  */
#define SB200_KIND_FINAL 5     /* per-step reduction and field update           */
#define SB200_KIND_POTENTIAL 6 /* self-consistent update: rho, Hartree, XC, V    */
#define SB200_KIND_COUNT 8

/* ---- context ------------------------------------------------------------ */

/* New context on CUDA device `device`, with its own non-blocking stream.      */
int sb200_ctx_create(int device, sb200_ctx** out);
int sb200_ctx_destroy(sb200_ctx* ctx);
/* Replace the context's stream by a caller-owned cudaStream_t (NULL restores
 * the context's own stream).                                                   */
int sb200_ctx_set_stream(sb200_ctx* ctx, void* stream);
/* Block until all work of the context has finished; reports deferred errors.  */
int sb200_ctx_sync(sb200_ctx* ctx);
/* Message of the last failure on this thread ("" if none).                    */
const char* sb200_last_error(void);
/* Library version string.                                                     */
const char* sb200_version(void);
/* Device-time accounting: with enable = 1, every kernel the context launches
 * is bracketed by CUDA events on its stream and sb200_rt_propagate runs its
 * steps without graph capture (one stream synchronisation per step); the
 * accumulated milliseconds and launch counts per SB200_KIND_* are read with
 * sb200_kernel_times (reset = 1 clears them).  Off by default.              */
int sb200_set_timing(sb200_ctx* ctx, int enable);
int sb200_kernel_times(sb200_ctx* ctx, double ms[SB200_KIND_COUNT], long count[SB200_KIND_COUNT], int reset);

/* ---- set-up (replaces the device-side data SALMON's init builds) -------- */

/* s_rgrid + s_stencil of one r-space domain holding the whole grid.
 * Replaces: init_grid_parallel (src/common/initialization.f90:508-611) and the
 * stencil coefficients (src/common/initialization.f90:241-256).
 *   is, ie, is_array, ie_array : mg%is, mg%ie, mg%is_array, mg%ie_array (3 each)
 *   idx, idy, idz : mg%idx(is-4:ie+4) etc.; must be the identity map with a
 *                   4-deep halo (isolated, zero Dirichlet halo) or the modular
 *                   map of a periodic grid (anything else: SB200_ERR_UNSUPPORTED)
 *   lg_num        : lg%num (global grid size; selects calc_dip's coordinate shift)
 *   hgs           : system%Hgs;  hvol : system%Hvol
 *   coef_lap0, coef_lap(4,3), coef_nab(4,3) : stencil%coef_lap0 / coef_lap / coef_nab */
int sb200_set_grid(sb200_ctx* ctx, const int is[3], const int ie[3], const int is_array[3],
                   const int ie_array[3], const int* idx, const int* idy, const int* idz,
                   const int lg_num[3], const double hgs[3], double hvol, double coef_lap0,
                   const double coef_lap[12], const double coef_nab[12]);

/* Orbital block: nspin, io = 1..no, ik = 1..nk (info%io_s..io_e, ik_s..ik_e
 * re-based to 1; im = 1), the k-points system%vec_k(3,nk), occupations
 * system%rocc(no,nk,nspin) and weights system%wtk(nk) (src/common/structures.f90:126-203). */
int sb200_set_orbitals(sb200_ctx* ctx, int nspin, int no, int nk, const double* vec_k,
                       const double* rocc, const double* wtk);

/* V_local(is:ie, nspin) interior values, host pointer (s_scalar%f per spin;
 * src/common/hamiltonian.f90:813-843 builds it).                               */
int sb200_set_vlocal(sb200_ctx* ctx, const double* V_local);

/* Kleinman-Bylander projector tables of s_pp_grid (src/common/structures.f90:254-319;
 * built by init_ps, src/atom/pp/prep_pp.f90:280-525): mps(natom),
 * jxyz(3,nps,natom) (grid indices in is..ie), rxyz(3,nps,natom),
 * uv(nps,nlma), ia_tbl(nlma) (1-based), rinv_uvu(nlma).  Host pointers.
 * natom = 0 / nlma = 0 disables the nonlocal term.                              */
int sb200_set_pp(sb200_ctx* ctx, int natom, int nps, int nlma, const int* mps, const int* jxyz,
                 const double* rxyz, const double* uv, const int* ia_tbl, const double* rinv_uvu);

/* Host-side set-up (no device, no context): the Kleinman-Bylander tables of
 * s_pp_grid and, on an isolated grid, the local pseudopotential Vpsl, from
 * Yabana-Bertsch pseudopotential files (`_rps.dat`, ps_format = 'KY'; angstrom
 * and eV as written).  files[nelem] the element files, lmax_ps[nelem] (Lmax_ps;
 * NULL or -1: the file's), lloc_ps[nelem] (Lloc_ps, the local channel); the
 * grid as for sb200_set_grid (lg%num, lg%is, system%hgs, system%hvol; orthogonal
 * cell); natom atoms of element kion[a] (1-based) at Rion(3, natom) (bohr).
 * Call once with mps ... rinv_uvu NULL: *nps and *nlma return the sizes; then
 * with arrays mps(natom), jxyz(3,nps,natom), rxyz(3,nps,natom), uv(nps,nlma),
 * ia_tbl(nlma), rinv_uvu(nlma) (the layout sb200_set_pp takes) and Vpsl(is:ie)
 * or NULL (isolated grids: the local channel interpolated at each atom's
 * distance; periodic: form factors, structure sum, inverse transforms).
 * Replaces: read_ps_KY and the radial set-up of input_pp
 * (src/atom/pp/input_pp.f90:96-341), making_ps_without_masking (:1111-1240),
 * init_ps with calc_nps / calc_jxyz / set_lma / calc_uv
 * (src/atom/pp/prep_pp.f90:22-525), calc_Vpsl_isolated (:550-620) and
 * calc_Vpsl_periodic (:798-974).                                                */
int sb200_init_ps_ky(int nelem, const char* const* files, const int* lmax_ps, const int* lloc_ps, int periodic,
                     const int num[3], const int is[3], const double hgs[3], double hvol, int natom,
                     const int* kion, const double* Rion, int* nps, int* nlma, int* mps, int* jxyz, double* rxyz,
                     double* uv, int* ia_tbl, double* rinv_uvu, double* Vpsl);

/* sb200_init_ps_ky for the pseudopotential formats with one projector per
 * angular momentum, the format chosen by the file name as init_pp does:
 * `_rps.dat` Yabana-Bertsch ('KY'), `.pspnc` ABINIT format 1 ('ABINIT',
 * Troullier-Martins tables on ABINIT's fixed logarithmic grid), `.fhi` the FHI
 * files of the ABINIT tables ('ABINITFHI'), `.cpi` FHI98PP ('FHI'); Hartree
 * atomic units in the last three.  The core-correction block of an `.fhi` file
 * is read past (no nonlinear core correction on this path); `.psp8`, `.vps`
 * and `.upf` (several projectors per l or given beta projectors) return
 * SB200_ERR_UNSUPPORTED.  Arguments, two-call protocol and outputs as
 * sb200_init_ps_ky.
 * Replaces: read_pslfile / init_pp's format selection
 * (src/atom/pp/salmon_pp.f90:22-100), read_ps_abinit, read_ps_abinitfhi and
 * read_ps_fhi (src/atom/pp/input_pp.f90:343-496,614-684) with the rest of
 * input_pp and init_ps as above.                                               */
int sb200_init_ps(int nelem, const char* const* files, const int* lmax_ps, const int* lloc_ps, int periodic,
                  const int num[3], const int is[3], const double hgs[3], double hvol, int natom,
                  const int* kion, const double* Rion, int* nps, int* nlma, int* mps, int* jxyz, double* rxyz,
                  double* uv, int* ia_tbl, double* rinv_uvu, double* Vpsl);

/* yn_psmask (1 = 'y', 0 = 'n', the default) and alpha_mask, gamma_mask,
 * eta_mask (the reference's defaults 0.8, 1.8, 15) for the following
 * sb200_init_ps / sb200_init_ps_ky calls, process-wide as the reference's
 * input variables: the radial KB functions u_l (v_l - v_lloc) are divided by
 * the normalized mask function on the cut-off widened to gamma_mask rps,
 * Fourier-filtered below alpha_mask pi / max(h) (spherical Bessel transforms
 * on 1000 k points) and multiplied by the mask again.
 * Replaces: making_ps_with_masking, ps_masking and make_mask_function
 * (src/atom/pp/input_pp.f90:848-1016,1302-1542).                               */
int sb200_set_psmask(int yn_psmask, double alpha_mask, double gamma_mask, double eta_mask);

/* system%vec_Ac (A/c) used by sb200_hpsi: recomputes k+A stencil coefficients
 * and the projector phases (update_kvector_nonlocalpt,
 * src/common/hamiltonian.f90:847-903).  Isolated grids ignore it.              */
int sb200_set_vec_Ac(sb200_ctx* ctx, const double vec_Ac[3]);

/* Non-orthogonal periodic cell: rmatrix_B(3,3) (system%rmatrix_B, the
 * inverse of the unit lattice vectors [u v w]) and coef_F(6) (stencil%coef_F:
 * F = B B^T, (f_uu, f_vv, f_ww, f_vw, f_uw, f_uv)) of init_lattice; the grid of
 * sb200_set_grid then runs along the lattice vectors and its coef_lap0 is the
 * F-weighted one.  hpsi and everything built on it (taylor, rt_propagate) take
 * the non-orthogonal stencil: lattice-axis Laplacian and B (k+A) gradient,
 * then the mixed second derivatives from the stored first derivatives; the
 * current's gradient sums are taken to Cartesian components by B^T.  Periodic
 * grids, FP64 only (no mixed form, no ttpsi).  NULL arguments return to the
 * orthogonal stencil.
 * Replaces: hpsi's non-orthogonal branch (src/common/hamiltonian.f90:306-357)
 * -> zstencil_nonorthogonal (src/common/stencil.f90:120-214); the B^T of
 * calc_current (src/common/density_matrix.f90:313,413); the tables of
 * init_lattice (src/common/lattice.f90:23-75).                                */
int sb200_set_lattice(sb200_ctx* ctx, const double rmatrix_B[9], const double coef_F[6]);

/* Single-scale Maxwell-TDDFT: the microscopic vector potential Ac_micro(3, is:ie)
 * (system%Ac_micro%v) and its divergence div_Ac(is:ie) (system%div_Ac%f), host
 * or device, copied into the context.  hpsi and sb200_taylor then take the
 * micro-A stencil: per point k + A(r) in the gradient term and in |k + A(r)|^2 / 2,
 * plus -i div A / 2 (the deviation from the Coulomb gauge); the KB term as set
 * by sb200_set_vec_Ac.  Call again whenever the field changes (the Maxwell
 * update is the caller's).  Orthogonal lattices, FP64; Ac_micro = NULL turns it
 * off; div_Ac = NULL stands for a zero divergence (the symmetrized form below
 * does not use it).
 * Replaces: hpsi's single-scale branch (src/common/hamiltonian.f90:236-298)
 * -> zstencil_microAc / zstencil_microAc_typical_seq
 * (src/common/stencil.f90:295-315, src/common/zstencil_microac_core/typical/seq.f90). */
int sb200_set_micro_ac(sb200_ctx* ctx, const double* Ac_micro, const double* div_Ac);

/* gram_schmidt_interval (the reference's default -1: never; values below 1
 * leave the loop without it): with N >= 1 every step of sb200_rt_propagate
 * whose global step itt is a multiple of N orthonormalises psi(t+dt)
 * (sb200_gram_schmidt_complex) before its density and current, inside the
 * loop's CUDA graph as a conditional node.
 * Replaces: the gram_schmidt call of time_evolution_step
 * (src/rt/time_evolution_step.f90:149-152).                                   */
int sb200_set_gram_schmidt_interval(sb200_ctx* ctx, int gram_schmidt_interval);

/* yn_predictor_corrector (1 = 'y', 0 = 'n', the default; the middle-point
 * propagator): every step of sb200_rt_propagate first propagates a copy of the
 * orbitals, takes the potential of the predicted density (with
 * sb200_set_self_consistent: Hartree from the current Vh, exchange-
 * correlation, update_vlocal; with a fixed potential the loop's initial
 * V_local), sets V_local = (V_step + V_predicted) / 2 and then propagates the
 * orbitals with it.
 * Replaces: predictor_corrector (src/rt/time_evolution_step.f90:139-143,
 * 374-428).                                                                    */
int sb200_set_predictor_corrector(sb200_ctx* ctx, int yn);

/* propagator (0 = 'middlepoint', the default; 1 = 'aetrs'): with AETRS every
 * step of sb200_rt_propagate is two half steps with the zc the caller passes
 * (those of -i dt/2): the first with A(itt) and V_local, then V_local
 * extrapolated as 3 V - 3 V_old1 + V_old2 (the stored potentials start as the
 * loop's initial V_local) and A(itt+1) predicted as Ac_ext(itt+1) +
 * 2 Ac_ind(itt) - Ac_ind(itt-1), the second half step; the current, the
 * fields, the density and the self-consistent update as for the middle point.
 * Replaces: the propagator = 'aetrs' branch of time_evolution_step and
 * time_evolution_half_step_etrs (src/rt/time_evolution_step.f90:117-147,
 * 430-470), with vloc_old of initialization_rt (:287-292).                    */
int sb200_set_propagator(sb200_ctx* ctx, int aetrs);

/* An isolated system driven by a pulse in the length gauge (ae_shape1 /=
 * 'impulse'; on = 1, 0 = off, the default): every step of sb200_rt_propagate
 * takes V_local + E_ext(itt).r (lg%coordinate) for its Taylor expansion, with
 * E_ext(itt) = -(Ac_ext(itt+1) - Ac_ext(itt)) / dt from the loop's Ac_ext,
 * and leaves the field-free V_local (with the self-consistent update, that of
 * the last step) behind.  Isolated grids only (periodic ones take A(t)).
 * Replaces: calcVbox (src/rt/em_field.f90:422-548), the E_ext table of
 * initialization_rt (src/rt/initialization_rt.f90:180-183) and V_local +
 * Vbox of time_evolution_step (src/rt/time_evolution_step.f90:95-116).       */
int sb200_set_length_gauge(sb200_ctx* ctx, int on);

/* absorbing_boundary = 'z' (yn_z = 1; 0 = 'none', the default): hpsi adds
 * -i w(z) psi with w = w0 (dr - z) / dr for z <= dr and w0 (z - (al_z - dr)) / dr
 * for z >= al_z - dr (z = iz * hgs(3) of the global plane index, al_z = al(3)
 * the cell length, w0 = imagnary_potential_w0, dr = imagnary_potential_dr),
 * after the stencil and before the nonlocal term; ttpsi includes it.  Taken by
 * sb200_hpsi, sb200_taylor and sb200_rt_propagate through the per-point
 * kernels (orthogonal cells, FP64; the mixed form refuses it).
 * Replaces: add_imaginary_potential_for_absorbing_boundary_z
 * (src/common/hamiltonian.f90:760-807) as hpsi calls it (:231-234, :300-303). */
int sb200_set_absorbing_boundary(sb200_ctx* ctx, int yn_z, double imagnary_potential_w0,
                                 double imagnary_potential_dr, double al_z);

/* yn_symmetrized_stencil (1 = 'y', 0 = 'n', the default): the single-scale
 * hpsi takes the symmetrized form, h = (V + lap0) psi - lap psi / 2
 * + |k + A(r)|^2 psi / 2 - (i/2) ((k + A(r)).grad psi + div((k + A) psi)), the
 * divergence formed with A at the neighbour points.
 * Replaces: zstencil_microAc_symmetrized (src/common/stencil.f90:319-411), as
 * hamiltonian.f90:239-256 selects it.                                          */
int sb200_set_symmetrized_stencil(sb200_ctx* ctx, int yn);

/* Electron-number current density of the orbitals psi (device), without the
 * rho A / c term and without a nonlocal part: curr(3, is:ie) = sum_{k,o,s}
 * rocc wtk (Im(conj(psi) grad psi) + vec_k |psi|^2), grad by coef_nab, into a
 * host or device array; summed over the k-point shards when a communicator is
 * set.  Synchronous.
 * Replaces: calc_microscopic_current / micro_current
 * (src/common/density_matrix.f90:726-845), called by time_evolution_step
 * (src/rt/time_evolution_step.f90:175-182) for rt%j_e.                        */
int sb200_calc_microscopic_current(sb200_ctx* ctx, const double* psi, double* curr);

/* Impulse kick of the initial orbitals: psi <- exp(i e_impulse epdir.r) psi
 * at every interior point of every orbital of the resident block psi (device
 * pointer), r the grid coordinate lg%coordinate of set_gridcoordinate.
 * Replaces: the ae_shape1 = 'impulse' branch of initialization_rt
 * (src/rt/initialization_rt.f90:382-423; coordinates
 * src/common/initialization.f90:1125-1190).                                    */
int sb200_impulse_kick(sb200_ctx* ctx, void* psi, double e_impulse, const double epdir[3]);

/* Arithmetic form of sb200_taylor / sb200_rt_propagate (SB200_PREC_*).          */
int sb200_set_precision(sb200_ctx* ctx, int mode);

/* ---- orbital blocks ------------------------------------------------------ */

/* Bytes of one orbital block in the resident layout (norb*nx*ny*nz*16).       */
size_t sb200_orbital_block_bytes(const sb200_ctx* ctx);
/* zwf(is_array:ie_array, nspin, no, nk) in the reference layout (host or
 * device memory) -> resident device block.  Synchronous with respect to the
 * source buffer (it may be reused when the call returns).                     */
int sb200_orbitals_from_ref(sb200_ctx* ctx, const double* zwf_ref, double* psi_dev);
/* Resident device block -> zwf in the reference layout (host or device);
 * halo and padding points of zwf are written as zero.  Synchronous.          */
int sb200_orbitals_to_ref(sb200_ctx* ctx, const double* psi_dev, double* zwf_ref);

/* ---- the hot path --------------------------------------------------------- */

/* htpsi = H tpsi for every orbital of the block: 25-point Laplacian, Bloch
 * k+A gradient, V_local and the KB nonlocal term.
 * Replaces: hpsi (src/common/hamiltonian.f90:27-235 orthogonal branch,
 * :424-435 nonlocal), zstencil_typical_* (src/common/zstencil_core/typical/seq.f90:17-127)
 * and zpseudo / zpseudo_cuda (src/common/nonlocal_potential.f90:175-390,
 * src/common/zpseudo.cu:132-191).  tpsi and htpsi are distinct device blocks. */
int sb200_hpsi(sb200_ctx* ctx, const double* tpsi, double* htpsi);

/* hpsi with its optional argument ttpsi: htpsi = H tpsi as sb200_hpsi, and
 * ttpsi = the kinetic part, the stencil output minus V_local tpsi before the
 * nonlocal term is added (-1/2 (nabla + i(k+A))^2 tpsi).
 * Replaces: hpsi(tpsi,htpsi,...,ttpsi) (src/common/hamiltonian.f90:27,364-414).
 * Three distinct device blocks.                                                 */
int sb200_hpsi_tt(sb200_ctx* ctx, const double* tpsi, double* htpsi, double* ttpsi);

/* Band energies of the orbital block psi: esp(no,nk,nspin) (host, Fortran
 * order) = Re <psi|H|psi> hvol per orbital, *e_kin = sum rocc wtk Re <psi|T|psi>
 * hvol, *e_nloc = sum rocc wtk hvol Re <psi|H - T - V_local|psi> (the KB
 * energy).  htpsi and ttpsi are device work blocks that receive H psi and T psi.
 * Replaces: calc_eigen_energy (src/common/total_energy.f90:505-775, complex
 * branch), energy%esp / E_kin / E_ion_nloc.  Synchronous.                       */
int sb200_calc_eigen_energy(sb200_ctx* ctx, const double* psi, double* htpsi, double* ttpsi, double* esp,
                            double* e_kin, double* e_nloc);

/* tspsi_out = sum_{n=0}^{n_hamil} zc(n) H^n tspsi_in, zc(0) = 1, with zc the
 * complex(n_hamil) array rt%zc (interleaved re/im, host pointer).
 * Replaces: taylor (src/rt/taylor.f90:21-121).  tspsi_in and sshtpsi are
 * scratch on return (the reference also leaves intermediate H^n psi there).  */
int sb200_taylor(sb200_ctx* ctx, double* tspsi_in, double* tspsi_out, double* sshtpsi,
                 const double* zc, int n_hamil);

/* rho(is:ie, nspin) = sum_{k,o} rocc*wtk*|psi|^2 into a host or device array.
 * Replaces: calc_density (src/common/density_matrix.f90:26-236).  Synchronous. */
int sb200_calc_density(sb200_ctx* ctx, const double* psi, double* rho);

/* curr(3,nspin) (host) for the current A = vec_Ac; the nonlocal part uses the
 * projector phases of the last sb200_set_vec_Ac, as the reference's
 * calc_current reads the zekr_uV of the step.  Periodic grids only.
 * Replaces: calc_current (src/common/density_matrix.f90:240-463) and
 * stencil_current_core_gpu (src/common/stencil_current.cu:81-142).  Synchronous. */
int sb200_calc_current(sb200_ctx* ctx, const double* psi, const double vec_Ac[3], double* curr);

/* rbox(4) of calc_dip (src/rt/dip.f90:114-225) for rho(is:ie,nspin) (host or
 * device).  Synchronous.                                                       */
int sb200_calc_dip(sb200_ctx* ctx, const double* rho, double rbox[4]);

/* nt steps of time_evolution_step (src/rt/time_evolution_step.f90:102-312) for
 * the fixed-potential linear-response path with the middlepoint propagator:
 * per step A_mid = (Ac_tot(itt)+Ac_tot(itt-1))/2, update_kvector_nonlocalpt,
 * taylor, calc_current with Ac_tot(itt) and calc_emfields (periodic), calc_dip
 * (both), all on the device.
 *   psi_a      : device block holding psi(itt0-1... ) on entry
 *   psi_b, work: device blocks (scratch)
 *   *psi_final : set to psi_a or psi_b, whichever holds the result
 *   zc         : complex(n_hamil), host
 *   Ac_ext     : (3, 0:nt+1) host, Ac_ext(:,i) at t = i*dt
 *   trans_longi: SB200_TRANS_TR or SB200_TRANS_LO
 *   curr_out   : (3, nt) host or NULL; J(itt) summed over spin
 *   rbox_out   : (4, nt) host or NULL; calc_dip rbox for rho(itt)
 *   Ac_tot_out : (3, 0:nt+1) host or NULL
 * The whole loop is issued as CUDA graphs; synchronous on return.            */
int sb200_rt_propagate(sb200_ctx* ctx, double* psi_a, double* psi_b, double* work, int nt,
                       double dt, const double* zc, int n_hamil, const double* Ac_ext,
                       int trans_longi, double* curr_out, double* rbox_out,
                       double* Ac_tot_out, double** psi_final);

/* Continuation of the time loop: the next sb200_rt_propagate runs the global
 * steps itt = Mit + 1 .. Mit + nt (main_tddft.f90:89) instead of 1 .. nt, its
 * Ac_ext(:, 0:nt+1) taken as the global Ac_ext(:, Mit:Mit+nt+1); with Ac_tot /
 * Ac_ind (3,2) given (steps Mit and Mit + 1, host; Ac_ind may be NULL = zero),
 * the loop's field history starts from them ('lo'), else from Ac_ext; the
 * isolated CG potential is extrapolated from the first step on (itt /= 1).
 * Used once, by the next loop.  Mit = 0 with NULLs is a fresh start.
 * Replaces: Mit of restart_rt and read_rtdata
 * (src/io/checkpoint_restart.f90:277-306,1959-1993).                         */
int sb200_rt_set_start(sb200_ctx* ctx, int Mit, const double Ac_tot[6], const double Ac_ind[6]);
/* After a loop: *Mit = the global step it reached, Ac_tot / Ac_ind (3,2) at
 * that step and the next (host; either may be NULL); what sb200_rt_set_start
 * takes to continue it exactly.  SB200_ERR_STATE before any loop.
 * Replaces: the rt%Ac_tot / rt%Ac_ind entries write_rtdata stores
 * (src/io/checkpoint_restart.f90:1925-1957).                                  */
int sb200_rt_get_state(sb200_ctx* ctx, int* Mit, double Ac_tot[6], double Ac_ind[6]);

/* Restart data in the reference's file layouts, in directory dir:
 * info.bin, occupation.bin, the orbitals (method_wf_distributor 0 = 'single':
 * wfn.bin; 1 = 'slice': k_IK_ob_NB/wfn_ob_IO.dat in blocks of
 * nblock_wf_distribute orbitals), Vh_stock.bin when the context runs the
 * isolated CG self-consistent loop, rtdata.bin when trans_longi = 'lo' (the
 * state of the last loop, sb200_rt_get_state).  psi: the context's orbital
 * block (device), complex, or real with if_real_orbital = 1 (ground state);
 * iter: the iteration or step number recorded.  Synchronous.
 * Replaces: checkpoint_rt / checkpoint_gs -> write_bin, write_wavefunction,
 * write_Vh_stock, write_rtdata (src/io/checkpoint_restart.f90:88-123,231-396,
 * 539-677,897-967,1925-1957) for one process.                                 */
int sb200_write_restart(sb200_ctx* ctx, const char* dir, int method_wf_distributor, int nblock_wf_distribute,
                        const double* psi, int if_real_orbital, int iter, int trans_longi);
/* Reads restart data written by the reference (one or many processes: the
 * 'single' layout is the same) or by sb200_write_restart into the context's
 * complex orbital block psi (device): the orbitals ik_s .. ik_s+nk-1 and
 * io_s .. io_s+no-1 of the file's mk x mo (real ground-state orbitals are
 * widened to complex on the device); the occupations become the context's
 * (and go to rocc_out(no,nk,nspin) unless NULL).  yn_restart = 1 continues a
 * propagation: *iter = the stored step, sb200_rt_set_start with the stored
 * fields ('lo'), and on an isolated CG self-consistent context the stored
 * potentials with the restart's Hartree solve and V_local update; yn_restart
 * = 0 (ground-state data starting a propagation): *iter = 0.  Synchronous.
 * Replaces: restart_rt / restart_gs -> read_bin, read_wavefunction,
 * read_Vh_stock, read_rtdata (src/io/checkpoint_restart.f90:125-154,277-306,
 * 400-534,1149-1305,1959-1993) and the yn_restart branch of initialization_rt
 * (src/rt/initialization_rt.f90:244-283).                                     */
int sb200_read_restart(sb200_ctx* ctx, const char* dir, int method_wf_distributor, int nblock_wf_distribute,
                       int yn_restart, int ik_s, int io_s, double* psi, int* iter, double* rocc_out);

/* ---- ground state: real orbitals, one k-point ------------------------------- */

/* The context's orbital block (sb200_set_orbitals with nk = 1) holds real
 * orbitals psi[o][z][y][x] (double, o = ispin + nspin*io) for these calls.
 * rwf(is_array:ie_array, nspin, no) in the reference layout <-> device block.  */
int sb200_gs_from_ref(sb200_ctx* ctx, const double* rwf_ref, double* psi_dev);
int sb200_gs_to_ref(sb200_ctx* ctx, const double* psi_dev, double* rwf_ref);
/* htpsi = H tpsi, real orbitals: dstencil + dpseudo.
 * Replaces: hpsi real branch (src/common/hamiltonian.f90:88-125),
 * dstencil (src/common/stencil.f90:30-80), dpseudo (src/common/nonlocal_potential.f90:26-171). */
int sb200_hpsi_real(sb200_ctx* ctx, const double* tpsi, double* htpsi);
/* ncg iterations of the band-by-band CG with 2x2 Rayleigh-Ritz per orbital;
 * precondition = SB200_PRECOND_*; esp (host, nspin*no) gets <x|H|x>/<x|x>.
 * With SB200_PRECOND_LEARNED the conjugation restarts every iteration.
 * Replaces: gscg_rwf (src/gs/conjugate_gradient.f90:21-466) and
 * preconditioning_rgk / dstencil_preconditioning (src/gs/preconditioning.f90:25-77). */
int sb200_gscg(sb200_ctx* ctx, double* psi, int ncg, int precondition, double alpha_pre, double* esp);
/* Classical column Gram-Schmidt.
 * Replaces: gram_schmidt_col_real8 (src/gs/gram_schmidt_orth.f90:59-230).          */
int sb200_gram_schmidt_real(sb200_ctx* ctx, double* psi);
/* Classical column Gram-Schmidt of complex orbitals, every (k, spin) group of
 * the resident block (any number of k-points), orbitals in order.
 * Replaces: gram_schmidt_col_complex8 (src/gs/gram_schmidt_orth.f90:1069-1242),
 * called on the RT path every gram_schmidt_interval steps
 * (src/rt/time_evolution_step.f90:154-155).  Synchronous.                       */
int sb200_gram_schmidt_complex(sb200_ctx* ctx, double* psi);
/* Subspace diagonalisation (nspin = 1); evals (host, no) ascending.
 * Replaces: ssdg_rwf (src/gs/subspace_diagonalization.f90:62-238) with
 * eigen_dsyev (src/gs/eigen_subdiag_lapack.f90:23-38).                          */
int sb200_subspace_diag_real(sb200_ctx* ctx, double* psi, double* evals);

/* ---- learned preconditioner for sb200_gscg ------------------------------------ */

/* A 3-layer 3-D convolutional network (3x3x3 kernels, SB200_LEARNED_CHANNELS
 * hidden channels, BF16 weights in the forward pass with FP32 accumulation)
 * maps the normalised residual g/rms(g) and V_local of an orbital to a
 * correction of the low-pass preconditioner: pre_g = lowpass(g) + rms(g) * y.
 * It takes the place of preconditioning_rgk (src/gs/conjugate_gradient.f90:427-464)
 * when sb200_gscg is called with SB200_PRECOND_LEARNED.
 * Parameters (FP32, SB200_LEARNED_NPARAM): W1(C,2,27) b1(C) W2(C,C,27) b2(C)
 * W3(1,C,27) b3(1); NULL initialises them to zero (= plain low-pass).
 * batch = orbitals per network pass (activation buffers are sized for it).   */
#define SB200_LEARNED_CHANNELS 16
#define SB200_LEARNED_NPARAM 8241
int sb200_learned_init(sb200_ctx* ctx, const float* params, int nparam, int batch);
int sb200_learned_get_params(sb200_ctx* ctx, float* params, int nparam);
/* Training / checking interfaces on device (or host) float arrays:
 * x0 (batch, 2, npts) network inputs, offset and target (batch, npts),
 * y (batch, npts).                                                             */
int sb200_learned_forward(sb200_ctx* ctx, const float* x0, float* y, int batch);
/* loss = sum_b 1 - <p,t>^2/(<p,p><t,t>) with p = offset + y (offset may be
 * NULL); grad (host, NPARAM) may be NULL.                                      */
int sb200_learned_loss_grad(sb200_ctx* ctx, const float* x0, const float* offset, const float* target,
                            int batch, double* loss, float* grad);
/* One Adam step (beta 0.9 / 0.999) with learning rate lr.                     */
int sb200_learned_train_step(sb200_ctx* ctx, const float* x0, const float* offset, const float* target,
                             int batch, float lr, double* loss);

/* ---- batches of independent isolated systems ------------------------------- */

/* No single counterpart in the reference, which runs one system per process;
 * each system here is one fully set-up context (sb200_set_grid, _orbitals,
 * _vlocal and optionally _pp) of an isolated grid, and a batch advances all of
 * them together through the loop of sb200_rt_propagate (time_evolution_step,
 * src/rt/time_evolution_step.f90:102-264, 'tr', no external field): per Taylor
 * term one launch of the KB projections and one persistent hpsi launch over
 * the tiles of every system, per step one observable and one final launch,
 * two steps captured as a CUDA graph.  Every system's results (psi, rbox
 * history) equal those of its own sb200_rt_propagate.  All contexts must live
 * on one device with one precision; work runs on the first context's stream.
 * The batch keeps pointers to the contexts: destroy it before them.          */
typedef struct sb200_batch sb200_batch;
#define SB200_TILE_32x8 0     /* 32 x 8 tiles, register-prefetch z sweep            */
#define SB200_TILE_16x16 1    /* 16 x 16 tiles, register-prefetch z sweep           */
#define SB200_TILE_32x8_TMA 2 /* 32 x 8 tiles fed by tensor copies (all systems or none;
                                 the default where every system can take it)         */
int sb200_batch_create(sb200_ctx* const* systems, int nsys, sb200_batch** out);
int sb200_batch_destroy(sb200_batch* batch);
/* Per-system hpsi tiling: shape SB200_TILE_* and z planes per work item.
 * Autotuning searches the z chunk (and, for the register sweep, the shape)
 * within the family of the current tiles.                                    */
int sb200_batch_set_tiles(sb200_batch* batch, const int* shape, const int* zchunk);
int sb200_batch_get_tiles(sb200_batch* batch, int* shape, int* zchunk);
/* Time every tiling candidate of every system at full occupancy (`reps`
 * launches each) and keep the fastest; psi[s] is read, work[s] overwritten.
 * shape_out / zchunk_out (nsys entries each) may be NULL.                    */
int sb200_batch_autotune(sb200_batch* batch, const double* const* psi, double* const* work, int reps,
                         int* shape_out, int* zchunk_out);
/* nt steps of every system: per system s the buffers psi_a[s] (input),
 * psi_b[s], work[s] as in sb200_rt_propagate; rbox_out[s] (4, nt) host or
 * device, may be NULL; psi_final[s] receives the buffer holding psi(nt).     */
int sb200_batch_propagate(sb200_batch* batch, double* const* psi_a, double* const* psi_b, double* const* work,
                          int nt, double dt, const double* zc, int n_hamil, double* const* rbox_out,
                          double** psi_final);

/* ---- per-step potential update (self-consistent path) ---------------------- *
 * The three steps time_evolution_step takes after the density when the
 * functional is not fixed (src/rt/time_evolution_step.f90:184-207): Hartree,
 * exchange-correlation, update_vlocal.  Density and potentials are interior
 * arrays (is:ie), x fastest, host or device pointers; all three calls are
 * synchronous.                                                                 */

/* Vxc and E_xc = hvol * sum rho*eps_xc of the Perdew-Zunger LDA: for nspin = 1
 * rho(is:ie) -> Vxc(is:ie); for nspin = 2 the spin densities rho_s(is:ie, 2) ->
 * Vxc_s(is:ie, 2) of the spin-polarised form.  E_xc may be NULL.
 * Replaces: exchange_correlation with xc = 'PZ' (src/xc/salmon_xc.f90:58-343,
 * calc_xc :667-812) -> exc_cor_pz / PZxc (src/xc/builtin_pz.f90:23-83) and
 * exc_cor_pz_sp / PZxc_sp (src/xc/builtin_pz_sp.f90:23-95).                   */
int sb200_exc_cor_pz(sb200_ctx* ctx, const double* rho, double* Vxc, double* E_xc);

/* Vh(is:ie) of rho on a periodic grid by separable discrete Fourier transforms
 * with 4 pi / |G|^2 (G = 0 dropped).  primitive_b(3,3), column j = b_j
 * (system%primitive_b, host).  Isolated grids: SB200_ERR_UNSUPPORTED.
 * Replaces: hartree (src/poisson/hartree.f90:20-128) -> poisson_ft
 * (src/poisson/poisson_periodic.f90:23-242) with fg%coef and the egx/egy/egz
 * tables of src/common/initialization.f90:632-776.                             */
int sb200_hartree_periodic(sb200_ctx* ctx, const double primitive_b[9], const double* rho, double* Vh);

/* Vh(is:ie) of rho on an isolated grid: the density placed in the corner of a
 * doubled box, separable transforms of length 2n, 4 pi / |G|^2 of the doubled
 * cell (G = 0 dropped), inverse transforms, the corner kept.  primitive_b of the
 * box (orthogonal: 2 pi / L_d on the diagonal).  Periodic grids:
 * SB200_ERR_UNSUPPORTED.  Replaces: hartree with method_poisson = 'ft' on an
 * isolated system -> poisson_isolated_ft (src/poisson/poisson_isolated.f90:692-836;
 * tables init_reciprocal_grid_isolated_ft, src/common/initialization.f90:823-1077). */
int sb200_hartree_isolated_ft(sb200_ctx* ctx, const double primitive_b[9], const double* rho, double* Vh);

/* Vh(is:ie) of rho on an isolated grid by conjugate gradients on the 25-point
 * Laplacian (the reference's default method_poisson = 'cg').  Vh holds the
 * start value on entry (the previous step's potential, or zeros) and the
 * solution on exit.  Boundary values in the four halo layers of each face come
 * from multipole expansions (l <= lmax_multipole <= 4) of the density about
 * poles: layout_multipole 1 one pole at the origin, 2 one pole per atom over
 * its nearest grid points (Rion(3, natom) needed), 3 box cells
 * (num_multipole_xyz per axis; NULL or zeros: about 8 A each) centred on their
 * charge centroid.  Stops when hvol sum |r|^2 < threshold_cg * (grid points),
 * at most maxiter iterations; *iterations = poisson%iterVh (maxiter + 1 when
 * not converged; may be NULL).  rho, Vh host or device, synchronous.  Periodic
 * grids: SB200_ERR_UNSUPPORTED.
 * Replaces: hartree with method_poisson = 'cg' on an isolated system ->
 * poisson_isolated_cg / laplacian_poisson / poisson_boundary
 * (src/poisson/poisson_isolated.f90:30-690) with the pole tables of
 * make_corr_pole and set_ig_bound (src/poisson/init_poisson.f90:23-299).      */
int sb200_hartree_isolated_cg(sb200_ctx* ctx, const double* rho, double* Vh, int layout_multipole,
                              int lmax_multipole, const double* Rion, int natom, const int num_multipole_xyz[3],
                              double threshold_cg, int maxiter, int* iterations);

/* Check of the bounded grid barrier that the one-launch CG solve uses
 * between the halves of each iteration: eight barriers over the solve's
 * cooperative grid.  withhold = 0: SB200_OK.  withhold != 0: one block leaves
 * without arriving, the others' waits expire after about a second of SM clock,
 * and the call returns SB200_ERR_TIMEOUT with the context still usable (the
 * failure report a stalled solve gives).  Needs the CG solve configured (a
 * prior sb200_hartree_isolated_cg or sb200_set_hartree_cg); SB200_ERR_UNSUPPORTED
 * when the two-launch form is in use.  No reference counterpart: failure
 * detection of this library's own device wait.                                 */
int sb200_check_grid_barrier(sb200_ctx* ctx, int withhold);

/* Selects the CG Hartree solve (sb200_hartree_isolated_cg, same arguments) for
 * the isolated self-consistent time loop (sb200_set_self_consistent) in place
 * of the doubled-box transforms, the reference's default for isolated systems.
 * Vh0(is:ie) is the potential of the initial density (the Vh of
 * initialization_rt; host or device); it starts the first step's CG and both
 * stored potentials of the extrapolation.  Every later step starts its CG from
 * 2 Vh_stock1 - Vh_stock2 as the reference does.  The iterations run inside the
 * loop's CUDA graph with the convergence test on the device.  Vh0 = NULL goes
 * back to the transforms.  Periodic grids: SB200_ERR_UNSUPPORTED.
 * Replaces: the Vh extrapolation and hartree call of time_evolution_step
 * (src/rt/time_evolution_step.f90:184-198) with method_poisson = 'cg', and the
 * Vh_stock set-up of src/rt/initialization_rt.f90:277-286.                     */
int sb200_set_hartree_cg(sb200_ctx* ctx, const double* Vh0, int layout_multipole, int lmax_multipole,
                         const double* Rion, int natom, const int num_multipole_xyz[3], double threshold_cg,
                         int maxiter);

/* V_local(is) = Vpsl + Vh + Vxc(is) written into the context's device copy of
 * V_local (FP64 and the FP32 copy of the mixed form); Vpsl, Vh (is:ie), Vxc
 * (is:ie, nspin).  Also serves as the first sb200_set_vlocal.
 * Replaces: update_vlocal (src/common/hamiltonian.f90:813-843).               */
int sb200_update_vlocal(sb200_ctx* ctx, const double* Vpsl, const double* Vh, const double* Vxc);

/* Self-consistent time loop.  With enable = 1 every step of sb200_rt_propagate
 * ends with calc_density, hartree, exchange_correlation (PZ) and update_vlocal
 * with this Vpsl(is:ie) (host or device; copied), in the order of
 * time_evolution_step with yn_fix_func = 'n', inside the loop's CUDA graph; the
 * next step's Taylor expansion uses the updated V_local.  The first step uses
 * the V_local already set (sb200_set_vlocal, or sb200_update_vlocal from
 * rho(t=0)).  The Hartree solve (poisson_ft on periodic grids,
 * poisson_isolated_ft on isolated ones) uses the cell of the latest call that
 * passed primitive_b.  nspin = 2: the Hartree potential of rho_up + rho_dn,
 * the spin-polarised PZ and V_local per spin (exc_cor_pz_sp);
 * enable = 0 returns to the fixed-potential loop (Vpsl, primitive_b unused).
 * The density is that of the context's own orbitals, summed over the k-point
 * shards of other processes when sb200_set_density_comm gave the context a
 * communicator.
 * Replaces: the yn_fix_func = 'n' branch of time_evolution_step
 * (src/rt/time_evolution_step.f90:160-207).                                    */
int sb200_set_self_consistent(sb200_ctx* ctx, int enable, const double* Vpsl, const double primitive_b[9]);

/* Sums over k-point shards.  A job that gives each process (one per GPU) a
 * share of the k-points needs the density and the current of all of them:
 * with a communicator set, sb200_calc_density and the self-consistent loop
 * all-reduce rho (NCCL, in the loop's CUDA graph) over the nranks processes,
 * and every step of sb200_rt_propagate (and sb200_calc_current) all-reduces
 * J(t) and the dipole sums before calc_emfields updates the induced field,
 * so trans_longi = 'lo' sees the current of the whole k-mesh.  id: 128 bytes from
 * sb200_nccl_unique_id on rank 0, passed to every rank by the host (MPI_Bcast,
 * torch.distributed).  nranks <= 0 removes the communicator.  NCCL is the
 * process's libnccl.so.2, loaded at run time (absent: SB200_ERR_UNSUPPORTED).
 * Replaces: comm_summation of rho over info%icomm_ko in calc_density
 * (src/common/density_matrix.f90:223) and of the current over info%icomm_rko
 * in calc_current (src/common/density_matrix.f90:448).                          */
int sb200_nccl_unique_id(unsigned char id[128]);
int sb200_set_density_comm(sb200_ctx* ctx, int nranks, int rank, const unsigned char id[128]);

/* ---- H psi without device allocation ---------------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory themselves -- hosts whose device arrays belong to another runtime
 * (OpenACC / OpenMP-offload programs that map their own arrays), memory-capped
 * or pre-sized environments, and code that must not allocate inside a time
 * loop -- this computes the same H psi as sb200_hpsi without a context and
 * without any allocation (no cudaMalloc, cudaFree or allocating library call).
 * Every array is caller-owned device memory, in the resident orbital layout
 * for tpsi / htpsi and in the reference's layout for the projector tables:
 *   V_local (nx*ny*nz, nspin); kAc (3, nk) = vec_k + vec_Ac (periodic only);
 *   mps(natom), jxyz(3,nps,natom) (grid indices in is..ie), rxyz(3,nps,natom),
 *   uv(nps,nlma), ia_tbl(nlma) (1-based), rinv_uvu(nlma); host values for
 *   is[3], coef_lap0, coef_lap(4,3), coef_nab(4,3).  periodic = 0 means the
 *   zero Dirichlet boundary of an isolated grid.  Work is queued on `stream`
 *   (a cudaStream_t, NULL for the legacy default stream).
 * The projector tables are checked on the device, since the host never sees
 * them: a jxyz entry outside is..is+n-1, an ia_tbl entry outside 1..natom or
 * an mps entry outside 0..nps is skipped (it adds nothing) instead of being
 * read or written, and the call's `status` word (caller-owned device int, may
 * be NULL) is set to SB200_ERR_BAD_SHAPE; otherwise the call sets it to
 * SB200_OK.  Read it after the stream's work has finished.  Spheres that
 * reach one grid point twice through two periodic images are added in the
 * reference's order (ilma, then j) without lost updates.
 * Its only scratch, the projections <beta|psi> of all orbitals, is a fixed
 * device array inside the library of SB200_NOALLOC_MAX_PROJECTIONS complex
 * values (4 MiB), held by every GPU that loads the library until the process
 * exits; norb*nlma above that limit returns SB200_ERR_BAD_SHAPE.  The first
 * call on each device looks up that array's device address; make the first
 * call before any stream capture.  All calls share the array and every call
 * overwrites the entries it uses, so calls whose GPU work overlaps (other
 * streams, other host threads) race and must be serialised by the caller.    */
#define SB200_NOALLOC_MAX_PROJECTIONS 262144
int sb200_hpsi_noalloc(int nx, int ny, int nz, int periodic, int nspin, int no, int nk, const int is[3],
                       double coef_lap0, const double coef_lap[12], const double coef_nab[12],
                       const double* kAc, const double* V_local, int natom, int nps, int nlma,
                       const int* mps, const int* jxyz, const double* rxyz, const double* uv,
                       const int* ia_tbl, const double* rinv_uvu, const double* tpsi, double* htpsi,
                       int* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SALMON_B200_H */
