! Fortran twin of include/half.h (libhalf ABI v1, B200 build) plus the
! additive entry points of include/half_b200.h.
!
! The names, constant values, derived-type layouts and argument lists are
! those of the reference's include/half_api.f90:1-163, because Fortran hosts
! (VASP's half_vasp_init.F) `use half_api` and call through these interfaces
! unchanged.  Every interface binds the C symbol of the same name; strings
! passed in must be NUL-terminated (c_null_char), error buffers are
! character(c_char) arrays of error_capacity elements.
module half_api
  use iso_c_binding
  implicit none

  ! status codes (half.h enum half_status)
  integer(c_int), parameter :: HALF_SUCCESS = 0
  integer(c_int), parameter :: HALF_ERROR_INVALID_ARGUMENT = 1
  integer(c_int), parameter :: HALF_ERROR_IO = 2
  integer(c_int), parameter :: HALF_ERROR_INVALID_HANDLE = 3
  integer(c_int), parameter :: HALF_ERROR_CAPACITY = 4
  integer(c_int), parameter :: HALF_ERROR_UNAVAILABLE = 5
  integer(c_int), parameter :: HALF_ERROR_INTERNAL = 6

  ! selectors (half.h enums half_xc, half_backend, half_solver)
  integer(c_int), parameter :: HALF_XC_LDA = 1
  integer(c_int), parameter :: HALF_XC_PBE = 2
  integer(c_int), parameter :: HALF_BACKEND_AUTO = 0
  integer(c_int), parameter :: HALF_BACKEND_CPU = 1
  integer(c_int), parameter :: HALF_BACKEND_CUDA = 2
  integer(c_int), parameter :: HALF_SOLVER_EVD = 1
  integer(c_int), parameter :: HALF_SOLVER_EVJ = 2
  integer(c_int), parameter :: HALF_SOLVER_VASP = 3
  integer(c_int), parameter :: HALF_SOLVER_ACC = 4

  ! capability bits (half.h enum half_capability)
  integer(c_int), parameter :: HALF_CAP_CPU = 1
  integer(c_int), parameter :: HALF_CAP_CUDA = 2
  integer(c_int), parameter :: HALF_CAP_MPI = 4
  integer(c_int), parameter :: HALF_CAP_HDF5 = 8
  integer(c_int), parameter :: HALF_CAP_SPGLIB = 16
  integer(c_int), parameter :: HALF_CAP_ESCN_API = 32

  integer(c_int32_t), parameter :: HALF_ESCN_INCLUDE_UNCERTAINTY = 1_c_int32_t
  integer(c_int), parameter :: HALF_DENSITY_RAW = 0
  integer(c_int), parameter :: HALF_DENSITY_NORMALIZE_VALENCE = 1

  ! precision selectors of half_set_acc_controls (half_b200.h enum half_precision)
  integer(c_int), parameter :: HALF_PRECISION_FP64 = 0
  integer(c_int), parameter :: HALF_PRECISION_MIXED = 1
  integer(c_int), parameter :: HALF_PRECISION_FP64_GUARDED = 2

  ! half.h struct half_request_geometry_v1
  type, bind(C) :: half_request_geometry_v1
    integer(c_int32_t) :: struct_size = 0
    integer(c_int32_t) :: flags = 0
    integer(c_int32_t) :: nions = 0
    integer(c_int32_t) :: ntypes = 0
    integer(c_int32_t) :: grid(3) = 0
    integer(c_int32_t) :: reserved_i32 = 0
    real(c_double) :: lattice(9) = 0.0_c_double
    type(c_ptr) :: species = c_null_ptr
    type(c_ptr) :: positions_fractional = c_null_ptr
    integer(c_int64_t) :: reserved(8) = 0_c_int64_t
  end type half_request_geometry_v1

  ! half.h struct half_escn_request_v1
  type, bind(C) :: half_escn_request_v1
    integer(c_int32_t) :: struct_size = 0
    integer(c_int32_t) :: flags = 0
    integer(c_int32_t) :: nions = 0
    integer(c_int32_t) :: grid(3) = 0
    integer(c_int32_t) :: reserved_i32 = 0
    real(c_double) :: cell(9) = 0.0_c_double
    type(c_ptr) :: atomic_numbers = c_null_ptr
    type(c_ptr) :: positions_cartesian = c_null_ptr
    integer(c_int64_t) :: reserved(8) = 0_c_int64_t
  end type half_escn_request_v1

  ! half.h struct half_escn_result_v1
  type, bind(C) :: half_escn_result_v1
    integer(c_int32_t) :: struct_size = 0
    integer(c_int32_t) :: flags = 0
    integer(c_int32_t) :: grid(3) = 0
    integer(c_int32_t) :: reserved_i32 = 0
    integer(c_int64_t) :: capacity = 0_c_int64_t
    type(c_ptr) :: density = c_null_ptr
    type(c_ptr) :: nu = c_null_ptr
    type(c_ptr) :: alpha = c_null_ptr
    type(c_ptr) :: beta = c_null_ptr
    type(c_ptr) :: risk = c_null_ptr
    real(c_double) :: elapsed_seconds = 0.0_c_double
    integer(c_int64_t) :: reserved(8) = 0_c_int64_t
  end type half_escn_result_v1

  ! half_b200.h struct half_solve_info_v1
  type, bind(C) :: half_solve_info_v1
    integer(c_int32_t) :: struct_size = 0
    integer(c_int32_t) :: iterations = 0
    integer(c_int32_t) :: fp64_iterations = 0
    integer(c_int32_t) :: converged = 0
    integer(c_int64_t) :: npw = 0_c_int64_t
    integer(c_int64_t) :: operator_applications = 0_c_int64_t
    real(c_double) :: max_residual_eV = 0.0_c_double
    real(c_double) :: setup_ms = 0.0_c_double
    real(c_double) :: solve_ms = 0.0_c_double
    real(c_double) :: operator_ms = 0.0_c_double
    real(c_double) :: device_ms = 0.0_c_double
    real(c_double) :: local_ms = 0.0_c_double
    real(c_double) :: local_bytes = 0.0_c_double
    integer(c_int64_t) :: local_columns = 0_c_int64_t
    integer(c_int64_t) :: kernel_launches = 0_c_int64_t
    real(c_double) :: sweep_ms = 0.0_c_double
    integer(c_int64_t) :: sweep_columns = 0_c_int64_t
    real(c_double) :: adjoint_ms = 0.0_c_double
    real(c_double) :: tensor_ms = 0.0_c_double
    real(c_double) :: tensor_flops = 0.0_c_double
    integer(c_int64_t) :: tensor_launches = 0_c_int64_t
    integer(c_int64_t) :: reserved(1) = 0_c_int64_t
  end type half_solve_info_v1

  interface

    ! ------------------------------------------------------------ ABI v1 (half.h)

    function half_get_abi_version() bind(C, name="half_get_abi_version") result(v)
      import :: c_int
      integer(c_int) :: v
    end function half_get_abi_version

    function half_get_version_string() bind(C, name="half_get_version_string") result(p)
      import :: c_ptr
      type(c_ptr) :: p
    end function half_get_version_string

    function half_get_capabilities() bind(C, name="half_get_capabilities") result(v)
      import :: c_int
      integer(c_int) :: v
    end function half_get_capabilities

    function half_escn_health(base_url, timeout, error, error_capacity) &
        bind(C, name="half_escn_health") result(status)
      import :: c_char, c_int
      character(c_char), intent(in) :: base_url(*)
      integer(c_int), value :: timeout
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_escn_health

    function half_escn_predict(base_url, request, result_, timeout, error, error_capacity) &
        bind(C, name="half_escn_predict") result(status)
      import :: c_char, c_int, c_ptr
      character(c_char), intent(in) :: base_url(*)
      type(c_ptr), value :: request
      type(c_ptr), value :: result_
      integer(c_int), value :: timeout
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_escn_predict

    function half_create_from_files(charge, potential, encut, xc, use_uspp, handle, error, error_capacity) &
        bind(C, name="half_create_from_files") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      character(c_char), intent(in) :: charge(*), potential(*)
      real(c_double), value :: encut
      integer(c_int), value :: xc, use_uspp
      integer(c_int64_t), intent(out) :: handle
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_create_from_files

    function half_create_from_files_backend(charge, potential, encut, xc, use_uspp, backend, solver, handle, &
        error, error_capacity) bind(C, name="half_create_from_files_backend") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      character(c_char), intent(in) :: charge(*), potential(*)
      real(c_double), value :: encut
      integer(c_int), value :: xc, use_uspp, backend, solver
      integer(c_int64_t), intent(out) :: handle
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_create_from_files_backend

    function half_create_from_escn(base_url, potential, geometry, encut, xc, use_uspp, backend, solver, &
        normalization, timeout, handle, error, error_capacity) bind(C, name="half_create_from_escn") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      character(c_char), intent(in) :: base_url(*), potential(*)
      type(c_ptr), value :: geometry
      real(c_double), value :: encut
      integer(c_int), value :: xc, use_uspp, backend, solver, normalization, timeout
      integer(c_int64_t), intent(out) :: handle
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_create_from_escn

    function half_destroy(handle, error, error_capacity) bind(C, name="half_destroy") result(status)
      import :: c_char, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_destroy

    function half_set_request_geometry(handle, geometry, error, error_capacity) &
        bind(C, name="half_set_request_geometry") result(status)
      import :: c_char, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      type(c_ptr), value :: geometry
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_set_request_geometry

    function half_get_request_geometry(handle, nions, ntypes, grid, lattice, species_capacity, species, &
        positions_capacity, positions, error, error_capacity) bind(C, name="half_get_request_geometry") result(status)
      import :: c_char, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      type(c_ptr), value :: nions, ntypes, grid, lattice
      integer(c_int64_t), value :: species_capacity
      type(c_ptr), value :: species
      integer(c_int64_t), value :: positions_capacity
      type(c_ptr), value :: positions
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_get_request_geometry

    function half_get_system_info(handle, nions, ntypes, grid, lattice, volume, error, error_capacity) &
        bind(C, name="half_get_system_info") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      integer(c_int), intent(out) :: nions, ntypes, grid(3)
      real(c_double), intent(out) :: lattice(9), volume
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_get_system_info

    function half_get_basis_size(handle, kpoint, npw, error, error_capacity) &
        bind(C, name="half_get_basis_size") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int64_t), intent(out) :: npw
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_get_basis_size

    function half_get_basis(handle, kpoint, capacity, gvec, kinetic, error, error_capacity) &
        bind(C, name="half_get_basis") result(status)
      import :: c_char, c_double, c_int, c_int32_t, c_int64_t
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int64_t), value :: capacity
      integer(c_int32_t), intent(out) :: gvec(*)
      real(c_double), intent(out) :: kinetic(*)
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_get_basis

    function half_assemble_hs(handle, kpoint, ld, h, s, error, error_capacity) &
        bind(C, name="half_assemble_hs") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: h, s
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_assemble_hs

    function half_apply_hs(handle, kpoint, nstates, ld, psi, hpsi, spsi, error, error_capacity) &
        bind(C, name="half_apply_hs") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int), value :: nstates
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: psi, hpsi, spsi
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_apply_hs

    function half_solve_kpoint(handle, kpoint, nbands, eigenvalues, eigenvectors, ld, smin, smax, &
        error, error_capacity) bind(C, name="half_solve_kpoint") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int), value :: nbands
      real(c_double), intent(out) :: eigenvalues(*)
      type(c_ptr), value :: eigenvectors
      integer(c_int64_t), value :: ld
      real(c_double), intent(out) :: smin, smax
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_solve_kpoint

    function half_solve_kpoint_mapped(handle, kpoint, nbands, host_npw, host_gvec, eigenvalues, eigenvectors, &
        ld, smin, smax, error, error_capacity) bind(C, name="half_solve_kpoint_mapped") result(status)
      import :: c_char, c_double, c_int, c_int32_t, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int), value :: nbands
      integer(c_int64_t), value :: host_npw
      integer(c_int32_t), intent(in) :: host_gvec(*)
      real(c_double), intent(out) :: eigenvalues(*)
      type(c_ptr), value :: eigenvectors
      integer(c_int64_t), value :: ld
      real(c_double), intent(out) :: smin, smax
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_solve_kpoint_mapped

    ! ------------------------------------------------ additive extensions (half_b200.h)

    function half_set_acc_controls(handle, tolerance_eV, max_iterations, block_size, precision, &
        error, error_capacity) bind(C, name="half_set_acc_controls") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      real(c_double), value :: tolerance_eV
      integer(c_int), value :: max_iterations, block_size, precision
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_set_acc_controls

    function half_get_last_solve_info(handle, info, error, error_capacity) &
        bind(C, name="half_get_last_solve_info") result(status)
      import :: c_char, c_int, c_int64_t, half_solve_info_v1
      integer(c_int64_t), value :: handle
      type(half_solve_info_v1), intent(inout) :: info
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_get_last_solve_info

    function half_solve_kpoints(handle, nk, kpoints, nbands, eigenvalues, error, error_capacity) &
        bind(C, name="half_solve_kpoints") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      integer(c_int), value :: nk
      real(c_double), intent(in) :: kpoints(*)
      integer(c_int), value :: nbands
      real(c_double), intent(out) :: eigenvalues(*)
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_solve_kpoints

    function half_solve_kpoints_device(handle, nk, kpoints, nbands, eigenvalues_device, vectors_device, ld, &
        error, error_capacity) bind(C, name="half_solve_kpoints_device") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      integer(c_int), value :: nk
      real(c_double), intent(in) :: kpoints(*)
      integer(c_int), value :: nbands
      type(c_ptr), value :: eigenvalues_device, vectors_device
      integer(c_int64_t), value :: ld
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_solve_kpoints_device

    function half_set_positions(handle, positions_fractional, error, error_capacity) &
        bind(C, name="half_set_positions") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: positions_fractional(*)
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_set_positions

    function half_set_positions_noalloc(handle, positions_fractional, error, error_capacity) &
        bind(C, name="half_set_positions_noalloc") result(status)
      import :: c_char, c_double, c_int, c_int64_t
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: positions_fractional(*)
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_set_positions_noalloc

    function half_nonlocal_forces(handle, kpoint, nbands, ld, vectors, eigenvalues, occupations, kweight, &
        forces, error, error_capacity) bind(C, name="half_nonlocal_forces") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      real(c_double), intent(in) :: kpoint(3)
      integer(c_int), value :: nbands
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: vectors
      real(c_double), intent(in) :: eigenvalues(*), occupations(*)
      real(c_double), value :: kweight
      real(c_double), intent(inout) :: forces(*)
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_nonlocal_forces

    function half_band_forces(handle, nk, kpoints, kweights, nbands, nelect, sigma, ismear, forces, &
        eigenvalues, occupations, energies, error, error_capacity) bind(C, name="half_band_forces") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      integer(c_int), value :: nk
      real(c_double), intent(in) :: kpoints(*), kweights(*)
      integer(c_int), value :: nbands
      real(c_double), value :: nelect, sigma
      integer(c_int), value :: ismear
      real(c_double), intent(out) :: forces(*)
      type(c_ptr), value :: eigenvalues, occupations, energies
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_band_forces

    function half_ionic_forces(handle, output_density, n, ewald, local, nlcc, harris, energies, &
        error, error_capacity) bind(C, name="half_ionic_forces") result(status)
      import :: c_char, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      type(c_ptr), value :: output_density
      integer(c_int64_t), value :: n
      type(c_ptr), value :: ewald, local, nlcc, harris, energies
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_ionic_forces

    function half_output_density(handle, nk, kpoints, kweights, nbands, ld, vectors, occupations, density, n, &
        augmentation_charge, error, error_capacity) bind(C, name="half_output_density") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      integer(c_int), value :: nk
      real(c_double), intent(in) :: kpoints(*), kweights(*)
      integer(c_int), value :: nbands
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: vectors
      real(c_double), intent(in) :: occupations(*)
      type(c_ptr), value :: density
      integer(c_int64_t), value :: n
      type(c_ptr), value :: augmentation_charge
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_output_density

    function half_forces(handle, nk, kpoints, kweights, nbands, nelect, sigma, ismear, forces, components, &
        output_density, energies, error, error_capacity) bind(C, name="half_forces") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      integer(c_int), value :: nk
      real(c_double), intent(in) :: kpoints(*), kweights(*)
      integer(c_int), value :: nbands
      real(c_double), value :: nelect, sigma
      integer(c_int), value :: ismear
      real(c_double), intent(out) :: forces(*)
      type(c_ptr), value :: components, output_density, energies
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_forces

    function half_pack_vasp_waves(handle, nk, kpoints, nbands, ld, vectors, packed, capacity, npws, offsets, &
        error, error_capacity) bind(C, name="half_pack_vasp_waves") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      integer(c_int64_t), value :: handle
      integer(c_int), value :: nk
      real(c_double), intent(in) :: kpoints(*)
      integer(c_int), value :: nbands
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: vectors, packed
      integer(c_int64_t), value :: capacity
      integer(c_int), intent(out) :: npws(*)
      integer(c_int64_t), intent(out) :: offsets(*)
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_pack_vasp_waves

    function half_occupations(nk, nbands, eigenvalues, kweights, nelect, sigma, ismear, occupations, energies, &
        error, error_capacity) bind(C, name="half_occupations") result(status)
      import :: c_char, c_double, c_int, c_ptr
      integer(c_int), value :: nk, nbands
      real(c_double), intent(in) :: eigenvalues(*), kweights(*)
      real(c_double), value :: nelect, sigma
      integer(c_int), value :: ismear
      real(c_double), intent(out) :: occupations(*)
      type(c_ptr), value :: energies
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_occupations

    function half_get_allocation_counts(requests, driver_allocations, error, error_capacity) &
        bind(C, name="half_get_allocation_counts") result(status)
      import :: c_char, c_int, c_int64_t
      integer(c_int64_t), intent(out) :: requests, driver_allocations
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_get_allocation_counts

    function half_tc_cgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, c_fp64, &
        error, error_capacity) bind(C, name="half_tc_cgemm") result(status)
      import :: c_char, c_double, c_int, c_int64_t, c_ptr
      character(c_char), value :: op_a, op_b
      integer(c_int), value :: m, n, k
      real(c_double), intent(in) :: alpha(2)
      type(c_ptr), value :: a
      integer(c_int64_t), value :: lda
      type(c_ptr), value :: b
      integer(c_int64_t), value :: ldb
      real(c_double), intent(in) :: beta(2)
      type(c_ptr), value :: c
      integer(c_int64_t), value :: ldc
      integer(c_int), value :: c_fp64
      character(c_char), intent(out) :: error(*)
      integer(c_int), value :: error_capacity
      integer(c_int) :: status
    end function half_tc_cgemm

  end interface

end module half_api
