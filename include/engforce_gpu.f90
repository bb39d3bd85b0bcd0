! engforce_gpu.f90 -- Fortran shim that makes the B200 engine the body of
! MDFF's engforce (src/engforce_driver.f90:102-190) through iso_c_binding.
!
! A maintainer adds this module to the reference's src/ and links with
! -L<repo>/mdff_b200 -lmdff_gpu -lcudart.  The bind(c) derived types mirror
! mdff_params and mdff_result of include/mdff_gpu.h field by field (the
! layout is checked against the library on the CPU); the C tables are
! [it][jt] (0-based) = Fortran (it+1, jt+1), so a bind(c) array A(NT,NT)
! holds the transpose of the namelist table, and the 3-index damping tables
! are reshaped with order=[3,2,1].  Status codes replace STOP inside the
! library; the shim prints the reference's message and STOPs itself.
MODULE engforce_gpu
  USE iso_c_binding
  implicit none
  integer, parameter :: NT = 16
  TYPE, bind(c) :: mdff_params
    integer(c_int) :: natm, ntype, natmi(NT)
    integer(c_int) :: lcoulomb, lbmhft, lbmhftd, lnmlj, lsurf, lreduced, calc
    real(c_double) :: cutshortrange, cutlongrange, skindiff
    real(c_double) :: qch(NT), dip(3,NT)
    integer(c_int) :: trunc, symmetric_pot_nb
    real(c_double) :: epslj(NT,NT), sigmalj(NT,NT), plj(NT,NT), qlj(NT,NT)
    real(c_double) :: Abmhftd(NT,NT), Bbmhftd(NT,NT), Cbmhftd(NT,NT), Dbmhftd(NT,NT), BDbmhftd(NT,NT)
    real(c_double) :: alphaES
    integer(c_int) :: kES(3), lautoES
    real(c_double) :: epsw
    integer(c_int) :: ldip_polar(NT)
    real(c_double) :: poldip(3,3,NT)
    integer(c_int) :: ldip_damping(NT,NT,NT)
    real(c_double) :: pol_damp_b(NT,NT,NT), pol_damp_c(NT,NT,NT)
    integer(c_int) :: pol_damp_k(NT,NT,NT)
    real(c_double) :: conv_tol_ind
    integer(c_int) :: min_scf_pol_iter, max_scf_pol_iter, extrapolate_order, symmetric_pot_pim
    integer(c_int) :: precision, solver
    real(c_double) :: cg_tol
    integer(c_int) :: cg_max_iter, fail_on_nonconvergence, device
    real(c_double) :: wall24(NT,NT)
    integer(c_int) :: thole_type              ! 0 = off, 1..4 = linear, expon1, expon2, gauss
    real(c_double) :: thole_param(NT,NT)
    integer(c_int) :: algo_moment_from_pola   ! 0 scf, 1 scf_kO_v1, 2 scf_kO_v2, 4 scf_kO_v4_1
    integer(c_int) :: algo_ext_dipole         ! 0 aspc, 1 poly
    real(c_double) :: omegakO
    integer(c_int) :: lwfc(NT), ldip_wfc       ! Wannier centres: lwfc < 0 marks a centre type
    real(c_double) :: rcut_wfc
  END TYPE
  TYPE, bind(c) :: mdff_result
    type(c_ptr) :: fx, fy, fz, mu, ef
    real(c_double) :: u_lj, vir_lj, u_bmhft, vir_bmhft, u_coul, u_pol, pvirial_coul
    real(c_double) :: tau_nonb(3,3), tau_coul(3,3), tau(3,3)   ! C [a][b] = transpose
  END TYPE
  TYPE, bind(c) :: mdff_stats
    integer(c_int) :: n_pol_iter, converged
    real(c_double) :: rmsd
    integer(c_int) :: list_rebuilds, list_capacity, list_needed, nk
    real(c_double) :: alphaES
    integer(c_int) :: kES(3)
    real(c_double) :: cutlongrange
    integer(c_int) :: n_launches
    real(c_double) :: ms_last, rmsd_initial
    integer(c_int) :: n_fp64_residuals
    integer(c_int) :: n_kardir                 ! in-place kardir/dirkar round trips of the call
  END TYPE
  INTERFACE
    integer(c_int) FUNCTION mdff_gpu_create(p, cellA, h) bind(c)
      import; type(mdff_params) :: p; real(c_double) :: cellA(9); type(c_ptr) :: h
    END FUNCTION
    integer(c_int) FUNCTION mdff_gpu_engforce(h, rx, ry, rz, itime, res) bind(c)
      import; type(c_ptr), value :: h; real(c_double) :: rx(*), ry(*), rz(*)
      integer(c_int), value :: itime; type(mdff_result) :: res
    END FUNCTION
    integer(c_int) FUNCTION mdff_gpu_set_cell(h, cellA) bind(c)
      import; type(c_ptr), value :: h; real(c_double) :: cellA(9)
    END FUNCTION
    integer(c_int) FUNCTION mdff_gpu_get_stats(h, st) bind(c)
      import; type(c_ptr), value :: h; type(mdff_stats) :: st
    END FUNCTION
    integer(c_int) FUNCTION mdff_gpu_kardir_roundtrips(h, rx, ry, rz, count) bind(c)
      import; type(c_ptr), value :: h; real(c_double) :: rx(*), ry(*), rz(*)
      integer(c_int), value :: count
    END FUNCTION
    type(c_ptr) FUNCTION mdff_gpu_strerror(s) bind(c)
      import; integer(c_int), value :: s
    END FUNCTION
  END INTERFACE
  type(c_ptr), save :: handle = c_null_ptr
  ! .true.: after each call rx, ry, rz hold what the reference's engforce
  ! leaves in them, its in-place kardir/dirkar round trips included
  ! (ewald_dir.f90:138,739, non_bonded.f90:1113,1221, moment_from_pola.f90:685,803)
  logical, save :: mimic_kardir = .false.
  real(c_double), allocatable, target, save :: mu_buf(:,:), ef_buf(:,:)
CONTAINS
  SUBROUTINE engforce   ! replaces engforce_driver.f90:102-190
    USE config, ONLY : natm, rx, ry, rz, fx, fy, fz, tau, tau_nonb, tau_coul, simu_cell
    USE thermodynamic, ONLY : u_lj, vir_lj, u_bmhft, vir_bmhft, u_coul, u_pol, pvirial_coul
    USE coulomb, ONLY : mu_t, ef_t
    USE md, ONLY : itime
    type(mdff_params) :: p
    type(mdff_result) :: res
    type(mdff_stats) :: stats
    real(c_double), target :: cA(9)
    integer(c_int) :: st
    if ( .not. c_associated(handle) ) then
      CALL fill_params(p)                     ! from the namelist modules (transposes)
      cA = reshape(transpose(simu_cell%A), [9])
      st = mdff_gpu_create(p, cA, handle)
      if ( st .ne. 0 ) STOP 'mdff_gpu_create failed'
      allocate(mu_buf(3,natm), ef_buf(3,natm))
    endif
    res%fx = c_loc(fx); res%fy = c_loc(fy); res%fz = c_loc(fz)
    res%mu = c_loc(mu_buf); res%ef = c_loc(ef_buf)
    st = mdff_gpu_engforce(handle, rx, ry, rz, int(itime, c_int), res)
    if ( st .eq. 3 ) then                     ! moment_from_pola.f90:176-216
      WRITE(*,'(a)') ' ERROR : POLARIZATION CATASTROPH'
      STOP
    else if ( st .ne. 0 ) then
      STOP 'mdff_gpu_engforce failed'
    endif
    u_lj = res%u_lj; vir_lj = res%vir_lj; u_bmhft = res%u_bmhft; vir_bmhft = res%vir_bmhft
    u_coul = res%u_coul; u_pol = res%u_pol; pvirial_coul = res%pvirial_coul
    tau_nonb = transpose(res%tau_nonb); tau_coul = transpose(res%tau_coul)
    tau = transpose(res%tau)                  ! = tau_nonb + 2 tau_coul, as the reference
    mu_t = mu_buf; ef_t = ef_buf
    if ( mimic_kardir ) then
      st = mdff_gpu_get_stats(handle, stats)
      if ( stats%n_kardir .gt. 0 ) st = mdff_gpu_kardir_roundtrips(handle, rx, ry, rz, stats%n_kardir)
    endif
  END SUBROUTINE engforce

  ! the namelist modules after their *_init routines (tables already
  ! symmetrised there, so symmetric_pot_* = 0 here); C [a][b] tables are the
  ! Fortran transposes, C [a][b][c] tables reshape(..., order=[3,2,1])
  SUBROUTINE fill_params(p)
    USE config, ONLY : natm, ntype, natmi
    USE control, ONLY : lcoulomb, lbmhft, lbmhftd, lnmlj, lsurf, lreduced, calc, &
                        cutshortrange, cutlongrange, skindiff
    USE non_bonded, ONLY : trunc, epslj, sigmalj, plj, qlj, Abmhftd, Bbmhftd, Cbmhftd, Dbmhftd, BDbmhftd
    USE coulomb, ONLY : qch, dip, alphaES, kES, lautoES, epsw, thole_functions, &
                        thole_function_type, thole_param
    USE pim, ONLY : ldip_polar, poldip, ldip_damping, pol_damp_b, pol_damp_c, pol_damp_k, &
                    conv_tol_ind, min_scf_pol_iter, max_scf_pol_iter, extrapolate_order, &
                    algo_moment_from_pola, algo_ext_dipole, omegakO, lwfc, ldip_wfc, rcut_wfc
    type(mdff_params), intent(out) :: p
    integer, parameter :: o3(3) = [3, 2, 1]
    character(len=6), parameter :: thole_names(4) = ['linear', 'expon1', 'expon2', 'gauss ']
    integer :: it
    p%natm = natm; p%ntype = ntype; p%natmi = natmi(1:NT)
    p%lcoulomb = merge(1, 0, lcoulomb); p%lbmhft = merge(1, 0, lbmhft)
    p%lbmhftd = merge(1, 0, lbmhftd); p%lnmlj = merge(1, 0, lnmlj)
    p%lsurf = merge(1, 0, lsurf); p%lreduced = merge(1, 0, lreduced)
    p%calc = 2
    if ( calc .eq. 'md' ) p%calc = 0
    if ( calc .eq. 'opt' ) p%calc = 1
    p%cutshortrange = cutshortrange; p%cutlongrange = cutlongrange; p%skindiff = skindiff
    p%qch = qch; p%dip = transpose(dip)
    p%trunc = trunc; p%symmetric_pot_nb = 0
    p%epslj = transpose(epslj); p%sigmalj = transpose(sigmalj)
    p%plj = transpose(plj); p%qlj = transpose(qlj)
    p%Abmhftd = transpose(Abmhftd); p%Bbmhftd = transpose(Bbmhftd); p%Cbmhftd = transpose(Cbmhftd)
    p%Dbmhftd = transpose(Dbmhftd); p%BDbmhftd = transpose(BDbmhftd)
    p%alphaES = alphaES; p%kES = kES; p%lautoES = merge(1, 0, lautoES); p%epsw = epsw
    p%ldip_polar = merge(1, 0, ldip_polar)
    p%poldip = reshape(poldip, [3, 3, NT], order=o3)
    p%ldip_damping = reshape(merge(1, 0, ldip_damping), [NT, NT, NT], order=o3)
    p%pol_damp_b = reshape(pol_damp_b, [NT, NT, NT], order=o3)
    p%pol_damp_c = reshape(pol_damp_c, [NT, NT, NT], order=o3)
    p%pol_damp_k = reshape(pol_damp_k, [NT, NT, NT], order=o3)
    p%conv_tol_ind = conv_tol_ind; p%min_scf_pol_iter = min_scf_pol_iter
    p%max_scf_pol_iter = max_scf_pol_iter; p%extrapolate_order = extrapolate_order
    p%symmetric_pot_pim = 0
    p%precision = 0; p%solver = 0; p%cg_tol = 0.0_c_double; p%cg_max_iter = 200   ! &gputag defaults
    p%fail_on_nonconvergence = 0; p%device = 0
    p%wall24 = 0.0_c_double
    p%thole_type = 0
    if ( thole_functions ) then
      do it = 1, 4
        if ( thole_function_type .eq. thole_names(it) ) p%thole_type = it
      enddo
    endif
    p%thole_param = transpose(thole_param)
    p%algo_moment_from_pola = 0
    if ( algo_moment_from_pola .eq. 'scf_kO_v1' ) p%algo_moment_from_pola = 1
    if ( algo_moment_from_pola .eq. 'scf_kO_v2' ) p%algo_moment_from_pola = 2
    if ( algo_moment_from_pola .eq. 'scf_kO_v3' ) p%algo_moment_from_pola = 3
    if ( algo_moment_from_pola .eq. 'scf_kO_v4_1' ) p%algo_moment_from_pola = 4
    if ( algo_moment_from_pola .eq. 'scf_kO_v4_2' ) p%algo_moment_from_pola = 5
    p%algo_ext_dipole = merge(1, 0, algo_ext_dipole .eq. 'poly')
    p%omegakO = omegakO
    p%lwfc = lwfc; p%ldip_wfc = merge(1, 0, ldip_wfc); p%rcut_wfc = rcut_wfc
  END SUBROUTINE fill_params
END MODULE engforce_gpu
