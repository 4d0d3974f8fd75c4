!
! salmon_b200.f90 -- ISO_C_BINDING interface to libsalmon_b200 (the B200
! RT-TDDFT propagation library), for SALMON's Fortran host.
!
! Every routine binds one entry point of include/salmon_b200.h.  Integer
! status codes are returned as c_int (0 = success); salmon_b200_check turns a
! non-zero status into SALMON's usual `stop` with the library's message.
!
! This module is shipped as source; it is not compiled in this repository
! (the build machines have no Fortran compiler).  Its argument lists follow
! the C prototypes one to one.
!
module salmon_b200
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: SB200_OK = 0
  integer(c_int), parameter :: SB200_PREC_FP64 = 0, SB200_PREC_MIXED = 1
  integer(c_int), parameter :: SB200_TRANS_TR = 0, SB200_TRANS_LO = 1
  integer(c_int), parameter :: SB200_PRECOND_NONE = 0, SB200_PRECOND_LOWPASS = 1, SB200_PRECOND_LEARNED = 2
  integer(c_int), parameter :: SB200_TILE_32x8 = 0, SB200_TILE_16x16 = 1, SB200_TILE_32x8_TMA = 2
  integer(c_int), parameter :: SB200_LEARNED_NPARAM = 8241

  interface
    integer(c_int) function sb200_ctx_create(device, ctx) bind(c, name="sb200_ctx_create")
      import
      integer(c_int), value :: device
      type(c_ptr) :: ctx
    end function

    integer(c_int) function sb200_ctx_destroy(ctx) bind(c, name="sb200_ctx_destroy")
      import
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function sb200_ctx_sync(ctx) bind(c, name="sb200_ctx_sync")
      import
      type(c_ptr), value :: ctx
    end function

    type(c_ptr) function sb200_last_error() bind(c, name="sb200_last_error")
      import
    end function

    type(c_ptr) function sb200_version() bind(c, name="sb200_version")
      import
    end function

    ! a caller-owned cudaStream_t (c_null_ptr: the context's own stream)
    integer(c_int) function sb200_ctx_set_stream(ctx, stream) bind(c, name="sb200_ctx_set_stream")
      import
      type(c_ptr), value :: ctx, stream
    end function

    ! device-time accounting per kernel class (SB200_KIND_*, 8 slots)
    integer(c_int) function sb200_set_timing(ctx, enable) bind(c, name="sb200_set_timing")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
    end function

    integer(c_int) function sb200_kernel_times(ctx, ms, count, reset) bind(c, name="sb200_kernel_times")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: ms(8)
      integer(c_long), intent(inout) :: count(8)
      integer(c_int), value :: reset
    end function

    ! s_rgrid + s_stencil (initialization.f90:241-256,508-611)
    integer(c_int) function sb200_set_grid(ctx, is, ie, is_array, ie_array, idx, idy, idz, lg_num, hgs, hvol, &
                                           coef_lap0, coef_lap, coef_nab) bind(c, name="sb200_set_grid")
      import
      type(c_ptr), value :: ctx
      integer(c_int), intent(in) :: is(3), ie(3), is_array(3), ie_array(3)
      integer(c_int), intent(in) :: idx(*), idy(*), idz(*)
      integer(c_int), intent(in) :: lg_num(3)
      real(c_double), intent(in) :: hgs(3)
      real(c_double), value :: hvol, coef_lap0
      real(c_double), intent(in) :: coef_lap(4,3), coef_nab(4,3)
    end function

    integer(c_int) function sb200_set_orbitals(ctx, nspin, no, nk, vec_k, rocc, wtk) &
        bind(c, name="sb200_set_orbitals")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nspin, no, nk
      real(c_double), intent(in) :: vec_k(3,*), rocc(*), wtk(*)
    end function

    integer(c_int) function sb200_set_vlocal(ctx, V_local) bind(c, name="sb200_set_vlocal")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: V_local(*)
    end function

    integer(c_int) function sb200_set_pp(ctx, natom, nps, nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu) &
        bind(c, name="sb200_set_pp")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: natom, nps, nlma
      integer(c_int), intent(in) :: mps(*), jxyz(3,nps,*), ia_tbl(*)
      real(c_double), intent(in) :: rxyz(3,nps,*), uv(nps,*), rinv_uvu(*)
    end function

    integer(c_int) function sb200_set_vec_Ac(ctx, vec_Ac) bind(c, name="sb200_set_vec_Ac")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: vec_Ac(3)
    end function

    integer(c_int) function sb200_set_lattice(ctx, rmatrix_B, coef_F) bind(c, name="sb200_set_lattice")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: rmatrix_B(3, 3), coef_F(6)
    end function

    integer(c_int) function sb200_init_ps_ky(nelem, files, lmax_ps, lloc_ps, periodic, num, is, hgs, hvol, &
        natom, kion, Rion, nps, nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl) bind(c, name="sb200_init_ps_ky")
      import
      integer(c_int), value :: nelem, periodic, natom
      type(c_ptr), intent(in) :: files(*)       ! c_loc of NUL-terminated file names
      integer(c_int), intent(in) :: lmax_ps(*), lloc_ps(*), num(3), is(3), kion(*)
      real(c_double), intent(in) :: hgs(3), Rion(3, *)
      real(c_double), value :: hvol
      integer(c_int), intent(inout) :: nps, nlma
      type(c_ptr), value :: mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl
    end function

    integer(c_int) function sb200_rt_set_start(ctx, Mit, Ac_tot, Ac_ind) bind(c, name="sb200_rt_set_start")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: Mit
      real(c_double), intent(in) :: Ac_tot(3, 2), Ac_ind(3, 2)
    end function

    integer(c_int) function sb200_rt_get_state(ctx, Mit, Ac_tot, Ac_ind) bind(c, name="sb200_rt_get_state")
      import
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: Mit
      real(c_double), intent(out) :: Ac_tot(3, 2), Ac_ind(3, 2)
    end function

    integer(c_int) function sb200_write_restart(ctx, dir, method_wf_distributor, nblock_wf_distribute, psi, &
        if_real_orbital, iter, trans_longi) bind(c, name="sb200_write_restart")
      import
      type(c_ptr), value :: ctx, psi
      character(kind=c_char), intent(in) :: dir(*)   ! NUL-terminated
      integer(c_int), value :: method_wf_distributor, nblock_wf_distribute, if_real_orbital, iter, trans_longi
    end function

    integer(c_int) function sb200_read_restart(ctx, dir, method_wf_distributor, nblock_wf_distribute, &
        yn_restart, ik_s, io_s, psi, iter, rocc_out) bind(c, name="sb200_read_restart")
      import
      type(c_ptr), value :: ctx, psi
      character(kind=c_char), intent(in) :: dir(*)   ! NUL-terminated
      integer(c_int), value :: method_wf_distributor, nblock_wf_distribute, yn_restart, ik_s, io_s
      integer(c_int), intent(out) :: iter
      real(c_double), intent(inout) :: rocc_out(*)
    end function

    integer(c_int) function sb200_set_psmask(yn_psmask, alpha_mask, gamma_mask, eta_mask) &
        bind(c, name="sb200_set_psmask")
      import
      integer(c_int), value :: yn_psmask
      real(c_double), value :: alpha_mask, gamma_mask, eta_mask
    end function

    integer(c_int) function sb200_init_ps(nelem, files, lmax_ps, lloc_ps, periodic, num, is, hgs, hvol, &
        natom, kion, Rion, nps, nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl) bind(c, name="sb200_init_ps")
      import
      integer(c_int), value :: nelem, periodic, natom
      type(c_ptr), intent(in) :: files(*)       ! c_loc of NUL-terminated file names
      integer(c_int), intent(in) :: lmax_ps(*), lloc_ps(*), num(3), is(3), kion(*)
      real(c_double), intent(in) :: hgs(3), Rion(3, *)
      real(c_double), value :: hvol
      integer(c_int), intent(inout) :: nps, nlma
      type(c_ptr), value :: mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl
    end function

    integer(c_int) function sb200_set_micro_ac(ctx, Ac_micro, div_Ac) bind(c, name="sb200_set_micro_ac")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: Ac_micro(3, *), div_Ac(*)
    end function

    integer(c_int) function sb200_set_gram_schmidt_interval(ctx, gram_schmidt_interval) &
        bind(c, name="sb200_set_gram_schmidt_interval")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: gram_schmidt_interval
    end function

    integer(c_int) function sb200_set_predictor_corrector(ctx, yn) bind(c, name="sb200_set_predictor_corrector")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: yn
    end function

    integer(c_int) function sb200_set_propagator(ctx, aetrs) bind(c, name="sb200_set_propagator")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: aetrs
    end function

    integer(c_int) function sb200_set_length_gauge(ctx, on) bind(c, name="sb200_set_length_gauge")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: on
    end function

    integer(c_int) function sb200_set_absorbing_boundary(ctx, yn_z, imagnary_potential_w0, imagnary_potential_dr, &
        al_z) bind(c, name="sb200_set_absorbing_boundary")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: yn_z
      real(c_double), value :: imagnary_potential_w0, imagnary_potential_dr, al_z
    end function

    integer(c_int) function sb200_set_symmetrized_stencil(ctx, yn) bind(c, name="sb200_set_symmetrized_stencil")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: yn
    end function

    integer(c_int) function sb200_calc_microscopic_current(ctx, psi, curr) &
        bind(c, name="sb200_calc_microscopic_current")
      import
      type(c_ptr), value :: ctx, psi
      real(c_double), intent(inout) :: curr(3, *)
    end function

    integer(c_int) function sb200_set_precision(ctx, mode) bind(c, name="sb200_set_precision")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: mode
    end function

    integer(c_size_t) function sb200_orbital_block_bytes(ctx) bind(c, name="sb200_orbital_block_bytes")
      import
      type(c_ptr), value :: ctx
    end function

    ! zwf(is_array:ie_array, nspin, io_s:io_e, ik_s:ik_e, 1) <-> resident device block
    integer(c_int) function sb200_orbitals_from_ref(ctx, zwf, psi_dev) bind(c, name="sb200_orbitals_from_ref")
      import
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(in) :: zwf(*)
      type(c_ptr), value :: psi_dev
    end function

    integer(c_int) function sb200_orbitals_to_ref(ctx, psi_dev, zwf) bind(c, name="sb200_orbitals_to_ref")
      import
      type(c_ptr), value :: ctx
      type(c_ptr), value :: psi_dev
      complex(c_double_complex), intent(inout) :: zwf(*)
    end function

    ! hpsi (hamiltonian.f90:27) on resident device blocks
    integer(c_int) function sb200_hpsi(ctx, tpsi, htpsi) bind(c, name="sb200_hpsi")
      import
      type(c_ptr), value :: ctx, tpsi, htpsi
    end function

    ! hpsi with its optional ttpsi (hamiltonian.f90:27,364-414)
    integer(c_int) function sb200_hpsi_tt(ctx, tpsi, htpsi, ttpsi) bind(c, name="sb200_hpsi_tt")
      import
      type(c_ptr), value :: ctx, tpsi, htpsi, ttpsi
    end function

    ! calc_eigen_energy (total_energy.f90:505): esp(no,nk,nspin), E_kin, E_ion_nloc
    integer(c_int) function sb200_calc_eigen_energy(ctx, psi, htpsi, ttpsi, esp, e_kin, e_nloc) &
        bind(c, name="sb200_calc_eigen_energy")
      import
      type(c_ptr), value :: ctx, psi, htpsi, ttpsi
      real(c_double) :: esp(*)
      real(c_double) :: e_kin, e_nloc
    end function

    ! taylor (taylor.f90:21) on resident device blocks; zc = rt%zc
    integer(c_int) function sb200_taylor(ctx, tspsi_in, tspsi_out, sshtpsi, zc, n_hamil) &
        bind(c, name="sb200_taylor")
      import
      type(c_ptr), value :: ctx, tspsi_in, tspsi_out, sshtpsi
      complex(c_double_complex), intent(in) :: zc(*)
      integer(c_int), value :: n_hamil
    end function

    integer(c_int) function sb200_calc_density(ctx, psi, rho) bind(c, name="sb200_calc_density")
      import
      type(c_ptr), value :: ctx, psi
      real(c_double), intent(inout) :: rho(*)
    end function

    integer(c_int) function sb200_calc_current(ctx, psi, vec_Ac, curr) bind(c, name="sb200_calc_current")
      import
      type(c_ptr), value :: ctx, psi
      real(c_double), intent(in) :: vec_Ac(3)
      real(c_double), intent(inout) :: curr(3,*)
    end function

    integer(c_int) function sb200_calc_dip(ctx, rho, rbox) bind(c, name="sb200_calc_dip")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: rho(*)
      real(c_double), intent(inout) :: rbox(4)
    end function

    ! initialization_rt.f90:382-423: psi <- exp(i e_impulse epdir.r) psi (psi: device block)
    integer(c_int) function sb200_impulse_kick(ctx, psi, e_impulse, epdir) bind(c, name="sb200_impulse_kick")
      import
      type(c_ptr), value :: ctx, psi
      real(c_double), value :: e_impulse
      real(c_double), intent(in) :: epdir(3)
    end function

    ! H psi without any allocation: every array is caller-owned device memory
    ! (passed as addresses) except is, coef_lap0, coef_lap, coef_nab; status is
    ! a device integer (or c_null_ptr) set to SB200_ERR_BAD_SHAPE when a table
    ! entry lies outside the grid
    integer(c_int) function sb200_hpsi_noalloc(nx, ny, nz, periodic, nspin, no, nk, is, coef_lap0, coef_lap, &
                                               coef_nab, kAc, V_local, natom, nps, nlma, mps, jxyz, rxyz, uv, &
                                               ia_tbl, rinv_uvu, tpsi, htpsi, status, stream) &
        bind(c, name="sb200_hpsi_noalloc")
      import
      integer(c_int), value :: nx, ny, nz, periodic, nspin, no, nk
      integer(c_int), intent(in) :: is(3)
      real(c_double), value :: coef_lap0
      real(c_double), intent(in) :: coef_lap(12), coef_nab(12)
      type(c_ptr), value :: kAc, V_local
      integer(c_int), value :: natom, nps, nlma
      type(c_ptr), value :: mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, tpsi, htpsi, status, stream
    end function

    ! time_evolution_step.f90:184-207: hartree (periodic), exchange_correlation (PZ,
    ! nspin = 1), update_vlocal; rho, Vh, Vxc, Vpsl: s_scalar%f(mg%is:mg%ie) host arrays
    integer(c_int) function sb200_exc_cor_pz(ctx, rho, Vxc, E_xc) bind(c, name="sb200_exc_cor_pz")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: rho(*)
      real(c_double), intent(inout) :: Vxc(*)
      real(c_double), intent(out) :: E_xc
    end function

    integer(c_int) function sb200_hartree_periodic(ctx, primitive_b, rho, Vh) &
        bind(c, name="sb200_hartree_periodic")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: primitive_b(3, 3)
      real(c_double), intent(in) :: rho(*)
      real(c_double), intent(inout) :: Vh(*)
    end function

    integer(c_int) function sb200_hartree_isolated_ft(ctx, primitive_b, rho, Vh) &
        bind(c, name="sb200_hartree_isolated_ft")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: primitive_b(3, 3)
      real(c_double), intent(in) :: rho(*)
      real(c_double), intent(inout) :: Vh(*)
    end function

    integer(c_int) function sb200_hartree_isolated_cg(ctx, rho, Vh, layout_multipole, lmax_multipole, Rion, &
        natom, num_multipole_xyz, threshold_cg, maxiter, iterations) bind(c, name="sb200_hartree_isolated_cg")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: rho(*)
      real(c_double), intent(inout) :: Vh(*)
      integer(c_int), value :: layout_multipole, lmax_multipole, natom, maxiter
      real(c_double), intent(in) :: Rion(3, *)
      integer(c_int), intent(in) :: num_multipole_xyz(3)
      real(c_double), value :: threshold_cg
      integer(c_int), intent(out) :: iterations
    end function

    integer(c_int) function sb200_check_grid_barrier(ctx, withhold) bind(c, name="sb200_check_grid_barrier")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: withhold
    end function

    integer(c_int) function sb200_set_hartree_cg(ctx, Vh0, layout_multipole, lmax_multipole, Rion, natom, &
        num_multipole_xyz, threshold_cg, maxiter) bind(c, name="sb200_set_hartree_cg")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: Vh0(*)
      integer(c_int), value :: layout_multipole, lmax_multipole, natom, maxiter
      real(c_double), intent(in) :: Rion(3, *)
      integer(c_int), intent(in) :: num_multipole_xyz(3)
      real(c_double), value :: threshold_cg
    end function

    integer(c_int) function sb200_update_vlocal(ctx, Vpsl, Vh, Vxc) bind(c, name="sb200_update_vlocal")
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: Vpsl(*), Vh(*), Vxc(*)
    end function

    ! yn_fix_func = 'n' inside sb200_rt_propagate (enable = 1); Vpsl(mg%is:mg%ie)
    integer(c_int) function sb200_set_self_consistent(ctx, enable, Vpsl, primitive_b) &
        bind(c, name="sb200_set_self_consistent")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
      real(c_double), intent(in) :: Vpsl(*)
      real(c_double), intent(in) :: primitive_b(3, 3)
    end function

    ! rho summed over the k-point processes (comm_summation over icomm_ko)
    integer(c_int) function sb200_nccl_unique_id(id) bind(c, name="sb200_nccl_unique_id")
      import
      integer(c_signed_char), intent(inout) :: id(128)
    end function

    integer(c_int) function sb200_set_density_comm(ctx, nranks, rank, id) bind(c, name="sb200_set_density_comm")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nranks, rank
      integer(c_signed_char), intent(in) :: id(128)
    end function

    integer(c_int) function sb200_rt_propagate(ctx, psi_a, psi_b, work, nt, dt, zc, n_hamil, Ac_ext, &
                                               trans_longi, curr, rbox, Ac_tot, psi_final) &
        bind(c, name="sb200_rt_propagate")
      import
      type(c_ptr), value :: ctx, psi_a, psi_b, work
      integer(c_int), value :: nt, n_hamil, trans_longi
      real(c_double), value :: dt
      complex(c_double_complex), intent(in) :: zc(*)
      real(c_double), intent(in) :: Ac_ext(3,0:*)
      real(c_double), intent(inout) :: curr(3,*), rbox(4,*), Ac_tot(3,0:*)
      type(c_ptr) :: psi_final
    end function

    ! ---- ground state (real orbitals) ----
    integer(c_int) function sb200_gs_from_ref(ctx, rwf_ref, psi_dev) bind(c, name="sb200_gs_from_ref")
      import
      type(c_ptr), value :: ctx, psi_dev
      real(c_double), intent(in) :: rwf_ref(*)
    end function

    integer(c_int) function sb200_gs_to_ref(ctx, psi_dev, rwf_ref) bind(c, name="sb200_gs_to_ref")
      import
      type(c_ptr), value :: ctx, psi_dev
      real(c_double), intent(inout) :: rwf_ref(*)
    end function

    integer(c_int) function sb200_hpsi_real(ctx, tpsi, htpsi) bind(c, name="sb200_hpsi_real")
      import
      type(c_ptr), value :: ctx, tpsi, htpsi
    end function

    integer(c_int) function sb200_gscg(ctx, psi, ncg, precondition, alpha_pre, esp) bind(c, name="sb200_gscg")
      import
      type(c_ptr), value :: ctx, psi
      integer(c_int), value :: ncg, precondition
      real(c_double), value :: alpha_pre
      real(c_double), intent(inout) :: esp(*)
    end function

    integer(c_int) function sb200_gram_schmidt_real(ctx, psi) bind(c, name="sb200_gram_schmidt_real")
      import
      type(c_ptr), value :: ctx, psi
    end function

    ! gram_schmidt_col_complex8 (gram_schmidt_orth.f90:1069); RT path every gram_schmidt_interval steps
    integer(c_int) function sb200_gram_schmidt_complex(ctx, psi) bind(c, name="sb200_gram_schmidt_complex")
      import
      type(c_ptr), value :: ctx, psi
    end function

    integer(c_int) function sb200_subspace_diag_real(ctx, psi, evals) bind(c, name="sb200_subspace_diag_real")
      import
      type(c_ptr), value :: ctx, psi
      real(c_double), intent(inout) :: evals(*)
    end function

    integer(c_int) function sb200_learned_init(ctx, params, nparam, batch) bind(c, name="sb200_learned_init")
      import
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: params(*)
      integer(c_int), value :: nparam, batch
    end function

    integer(c_int) function sb200_learned_get_params(ctx, params, nparam) bind(c, name="sb200_learned_get_params")
      import
      type(c_ptr), value :: ctx
      real(c_float), intent(inout) :: params(*)
      integer(c_int), value :: nparam
    end function

    ! network inputs x0(npts, 2, batch), outputs y / offset / target (npts, batch):
    ! host or device arrays, passed as addresses
    integer(c_int) function sb200_learned_forward(ctx, x0, y, batch) bind(c, name="sb200_learned_forward")
      import
      type(c_ptr), value :: ctx, x0, y
      integer(c_int), value :: batch
    end function

    integer(c_int) function sb200_learned_loss_grad(ctx, x0, offset, target, batch, loss, grad) &
        bind(c, name="sb200_learned_loss_grad")
      import
      type(c_ptr), value :: ctx, x0, offset, target
      integer(c_int), value :: batch
      real(c_double), intent(out) :: loss
      type(c_ptr), value :: grad
    end function

    integer(c_int) function sb200_learned_train_step(ctx, x0, offset, target, batch, lr, loss) &
        bind(c, name="sb200_learned_train_step")
      import
      type(c_ptr), value :: ctx, x0, offset, target
      integer(c_int), value :: batch
      real(c_float), value :: lr
      real(c_double), intent(out) :: loss
    end function

    ! ---- batches of independent isolated systems ----
    integer(c_int) function sb200_batch_create(systems, nsys, batch) bind(c, name="sb200_batch_create")
      import
      type(c_ptr), intent(in) :: systems(*)
      integer(c_int), value :: nsys
      type(c_ptr) :: batch
    end function

    integer(c_int) function sb200_batch_destroy(batch) bind(c, name="sb200_batch_destroy")
      import
      type(c_ptr), value :: batch
    end function

    integer(c_int) function sb200_batch_set_tiles(batch, shape, zchunk) bind(c, name="sb200_batch_set_tiles")
      import
      type(c_ptr), value :: batch
      integer(c_int), intent(in) :: shape(*), zchunk(*)
    end function

    integer(c_int) function sb200_batch_get_tiles(batch, shape, zchunk) bind(c, name="sb200_batch_get_tiles")
      import
      type(c_ptr), value :: batch
      integer(c_int), intent(inout) :: shape(*), zchunk(*)
    end function

    integer(c_int) function sb200_batch_autotune(batch, psi, work, reps, shape, zchunk) &
        bind(c, name="sb200_batch_autotune")
      import
      type(c_ptr), value :: batch
      type(c_ptr), intent(in) :: psi(*), work(*)
      integer(c_int), value :: reps
      integer(c_int), intent(inout) :: shape(*), zchunk(*)
    end function

    integer(c_int) function sb200_batch_propagate(batch, psi_a, psi_b, work, nt, dt, zc, n_hamil, rbox, psi_final) &
        bind(c, name="sb200_batch_propagate")
      import
      type(c_ptr), value :: batch
      type(c_ptr), intent(in) :: psi_a(*), psi_b(*), work(*), rbox(*)
      integer(c_int), value :: nt, n_hamil
      real(c_double), value :: dt
      complex(c_double_complex), intent(in) :: zc(*)
      type(c_ptr), intent(inout) :: psi_final(*)
    end function
  end interface

contains

  subroutine salmon_b200_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    character(len=512) :: text
    integer :: i
    if (rc == SB200_OK) return
    call c_f_pointer(sb200_last_error(), msg, [512])
    text = ''
    do i = 1, 512
      if (msg(i) == c_null_char) exit
      text(i:i) = msg(i)
    end do
    write(*,*) 'salmon_b200 error in ', where, ': ', trim(text)
    stop 'salmon_b200'
  end subroutine salmon_b200_check

end module salmon_b200
