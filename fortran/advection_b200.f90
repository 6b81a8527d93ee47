!> ---------------------------------------------------------------------------
!!  ICAR's advection module on the B200 library (libicar_adv.so, C ABI in
!!  include/icar_adv.h).
!!
!!  Two modules:
!!    icar_adv_c  ISO_C_BINDING interfaces of the C entry points this file
!!                uses, and the two option/description structs;
!!    advection   a drop-in for src/physics/advection_driver.f90 (module
!!                advection, public :: advect, adv_init, adv_var_request):
!!                the same three names and arguments, the state kept on the
!!                GPU, every failure reported with the library's message and
!!                then stopped, as the reference stops.
!!
!!  Not compiled here: no Fortran compiler exists on the build machine.  The
!!  names bound below are checked against the C header by
!!  tests/test_fortran_binding.py.
!! ---------------------------------------------------------------------------
module icar_adv_c
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: ICAR_ADV_OK = 0
    integer(c_int), parameter :: ICAR_ADV_STD = 1, ICAR_ADV_MPDATA = 2
    integer(c_int), parameter :: ICAR_F_U = 1, ICAR_F_V = 2, ICAR_F_W = 3, ICAR_F_DENSITY = 39
    integer(c_int), parameter :: ICAR_F_JACOBIAN = 1001, ICAR_F_JACOBIAN_U = 1002, &
                                 ICAR_F_JACOBIAN_V = 1003, ICAR_F_JACOBIAN_W = 1004, &
                                 ICAR_F_ADVECTION_DZ = 1005
    integer(c_int), parameter :: ICAR_ADV_MAX_SPECIES = 32

    !> icar_adv_desc (include/icar_adv.h): one image's domain
    type, bind(C) :: icar_adv_desc
        integer(c_int32_t) :: nx, ny, nz
        real(c_float)      :: dx
        integer(c_int32_t) :: n_species
        integer(c_int32_t) :: species(ICAR_ADV_MAX_SPECIES)   ! kVARS ids, adv_vars order
        integer(c_int32_t) :: north_boundary, south_boundary, east_boundary, west_boundary
        integer(c_int32_t) :: device
    end type

    !> icar_adv_opts: the advection subset of options_t, field for field
    type, bind(C) :: icar_adv_opts
        integer(c_int32_t) :: advection, mpdata_fct, mpdata_order, flux_corr
        integer(c_int32_t) :: h_order, v_order, rk3, advect_density, debug, boundary_buffer
    end type

    interface
        integer(c_int) function icar_adv_default_opts(opts) bind(C, name="icar_adv_default_opts")
            import; type(icar_adv_opts), intent(out) :: opts
        end function
        integer(c_int) function icar_adv_var_request(opts, alloc_vars, n_alloc, advect_vars, n_advect) &
                bind(C, name="icar_adv_var_request")
            import; type(icar_adv_opts), intent(in) :: opts
            integer(c_int32_t), intent(out) :: alloc_vars(*), advect_vars(*)
            integer(c_int32_t), intent(inout) :: n_alloc, n_advect
        end function
        integer(c_int) function icar_adv_restart_vars(opts, vars, n) bind(C, name="icar_adv_restart_vars")
            import; type(icar_adv_opts), intent(in) :: opts
            integer(c_int32_t), intent(out) :: vars(*); integer(c_int32_t), intent(inout) :: n
        end function
        integer(c_int) function icar_adv_create(desc, opts, h) bind(C, name="icar_adv_create")
            import; type(icar_adv_desc), intent(in) :: desc; type(icar_adv_opts), intent(in) :: opts
            type(c_ptr), intent(out) :: h
        end function
        integer(c_int) function icar_adv_destroy(h) bind(C, name="icar_adv_destroy")
            import; type(c_ptr), value :: h
        end function
        integer(c_int) function icar_adv_set_field(h, field, host, strides) bind(C, name="icar_adv_set_field")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: field
            type(c_ptr), value :: host, strides
        end function
        integer(c_int) function icar_adv_get_field(h, field, host, strides) bind(C, name="icar_adv_get_field")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: field
            type(c_ptr), value :: host, strides
        end function
        integer(c_int) function icar_adv_advect(h, dt) bind(C, name="icar_adv_advect")
            import; type(c_ptr), value :: h; real(c_float), value :: dt
        end function
        integer(c_int) function icar_adv_sync(h) bind(C, name="icar_adv_sync")
            import; type(c_ptr), value :: h
        end function
        type(c_ptr) function icar_adv_last_error(h) bind(C, name="icar_adv_last_error")
            import; type(c_ptr), value :: h
        end function
        integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
            import; type(c_ptr), value :: s
        end function
    end interface
end module icar_adv_c


module advection
    use iso_c_binding
    use icar_adv_c
    use icar_constants,           only : kADV_STD, kADV_MPDATA, kVARS
    use options_interface,        only : options_t
    use domain_interface,         only : domain_t
    use variable_interface,       only : variable_t

    implicit none
    private

    public :: advect, adv_init, adv_var_request

    type(c_ptr), save :: h = c_null_ptr                ! the library handle of this image's domain
    integer, save :: n_adv = 0
    integer(c_int32_t), save :: adv_ids(ICAR_ADV_MAX_SPECIES)
    character(len=32), save :: adv_names(ICAR_ADV_MAX_SPECIES)

contains

    !> Stop with the library's message when a call failed (the reference
    !! stops on errors; the library itself never aborts).
    subroutine check(ierr, what)
        integer(c_int), intent(in) :: ierr
        character(len=*), intent(in) :: what
        character(kind=c_char), pointer :: msg(:)
        type(c_ptr) :: p
        integer :: n, i
        character(len=512) :: text
        if (ierr == ICAR_ADV_OK) return
        text = ""
        p = icar_adv_last_error(h)
        if (c_associated(p)) then
            n = int(min(c_strlen(p), int(len(text), c_size_t)))
            call c_f_pointer(p, msg, [n])
            do i = 1, n
                text(i:i) = msg(i)
            end do
        endif
        write(*,*) "advection (B200 library): ", trim(what), " failed, status ", ierr, ": ", trim(text)
        error stop
    end subroutine

    !> kVARS id of an adv_vars name (domain_obj.f90:68-89 adds them by name)
    integer(c_int32_t) function var_id(name) result(id)
        character(len=*), intent(in) :: name
        select case (trim(name))
        case ("qv");          id = kVARS%water_vapor
        case ("theta");       id = kVARS%potential_temperature
        case ("qc");          id = kVARS%cloud_water
        case ("qr");          id = kVARS%rain_in_air
        case ("qs");          id = kVARS%snow_in_air
        case ("qi");          id = kVARS%cloud_ice
        case ("qg");          id = kVARS%graupel_in_air
        case ("ni");          id = kVARS%ice_number_concentration
        case ("nr");          id = kVARS%rain_number_concentration
        case ("ns");          id = kVARS%snow_number_concentration
        case ("ng");          id = kVARS%graupel_number_concentration
        case ("nc");          id = kVARS%cloud_number_concentration
        case ("ice1_a");      id = kVARS%ice1_a
        case ("ice1_c");      id = kVARS%ice1_c
        case ("ice2_mass");   id = kVARS%ice2_mass
        case ("ice2_number"); id = kVARS%ice2_number
        case ("ice2_a");      id = kVARS%ice2_a
        case ("ice2_c");      id = kVARS%ice2_c
        case ("ice3_mass");   id = kVARS%ice3_mass
        case ("ice3_number"); id = kVARS%ice3_number
        case ("ice3_a");      id = kVARS%ice3_a
        case ("ice3_c");      id = kVARS%ice3_c
        case default
            write(*,*) "advection (B200 library): no kVARS id for advected variable ", trim(name)
            error stop
        end select
    end function

    !> options_t -> icar_adv_opts (adv_options_type, opt_types.f90:119-127)
    subroutine fill_opts(options, opts)
        type(options_t), intent(in) :: options
        type(icar_adv_opts), intent(out) :: opts
        call check(icar_adv_default_opts(opts), "icar_adv_default_opts")
        opts%advection = merge(ICAR_ADV_MPDATA, ICAR_ADV_STD, options%physics%advection == kADV_MPDATA)
        opts%mpdata_fct = merge(1, 0, options%adv_options%MPDATA_FCT)
        opts%mpdata_order = options%adv_options%mpdata_order
        opts%flux_corr = options%adv_options%flux_corr
        opts%h_order = options%adv_options%h_order
        opts%v_order = options%adv_options%v_order
        opts%rk3 = merge(1, 0, options%time_options%RK3)
        opts%advect_density = merge(1, 0, options%parameters%advect_density)
        opts%debug = merge(1, 0, options%parameters%debug)
        opts%boundary_buffer = 0
    end subroutine

    !> adv_init(domain, options), advection_driver.f90:26-44: create the
    !! handle for this image's domain and upload the fields that stay fixed
    !! (jacobians and advection_dz); winds, density and the species are
    !! uploaded by every advect call.
    subroutine adv_init(domain, options)
        type(domain_t), intent(inout), target :: domain
        type(options_t), intent(in) :: options
        type(icar_adv_desc) :: desc
        type(icar_adv_opts) :: opts
        type(variable_t) :: var
        character(len=32) :: name

        if (this_image() == 1) write(*,*) ""
        if (this_image() == 1) write(*,*) "Initializing Advection (B200 library)"
        call fill_opts(options, opts)
        desc%nx = domain%ime - domain%ims + 1
        desc%ny = domain%jme - domain%jms + 1
        desc%nz = domain%kme - domain%kms + 1
        desc%dx = domain%dx
        desc%north_boundary = 1; desc%south_boundary = 1; desc%east_boundary = 1; desc%west_boundary = 1
        desc%device = 0
        n_adv = 0
        desc%species = 0
        call domain%adv_vars%reset_iterator()
        do while (domain%adv_vars%has_more_elements())
            var = domain%adv_vars%next(name)
            n_adv = n_adv + 1
            if (n_adv > ICAR_ADV_MAX_SPECIES) then
                write(*,*) "advection (B200 library): more than 32 advected variables"
                error stop
            endif
            adv_names(n_adv) = name
            adv_ids(n_adv) = var_id(name)
            desc%species(n_adv) = adv_ids(n_adv)
        enddo
        desc%n_species = n_adv
        if (c_associated(h)) call check(icar_adv_destroy(h), "icar_adv_destroy")
        call check(icar_adv_create(desc, opts, h), "icar_adv_create")
        call check(icar_adv_set_field(h, ICAR_F_JACOBIAN, c_loc(domain%jacobian), c_null_ptr), "set jacobian")
        call check(icar_adv_set_field(h, ICAR_F_JACOBIAN_U, c_loc(domain%jacobian_u), c_null_ptr), "set jacobian_u")
        call check(icar_adv_set_field(h, ICAR_F_JACOBIAN_V, c_loc(domain%jacobian_v), c_null_ptr), "set jacobian_v")
        call check(icar_adv_set_field(h, ICAR_F_JACOBIAN_W, c_loc(domain%jacobian_w), c_null_ptr), "set jacobian_w")
        call check(icar_adv_set_field(h, ICAR_F_ADVECTION_DZ, c_loc(domain%advection_dz), c_null_ptr), &
                   "set advection_dz")
    end subroutine adv_init

    !> adv_var_request(options), advection_driver.f90:46-57 ->
    !! adv_std_var_request, advect.f90:94-108: the library returns the same
    !! lists the reference registers.
    subroutine adv_var_request(options)
        type(options_t), intent(inout) :: options
        type(icar_adv_opts) :: opts
        integer(c_int32_t) :: alloc_ids(32), adv_list(32), restart_ids(32)
        integer(c_int32_t) :: n_alloc, n_advect, n_restart
        call fill_opts(options, opts)
        n_alloc = 32; n_advect = 32; n_restart = 32
        call check(icar_adv_var_request(opts, alloc_ids, n_alloc, adv_list, n_advect), "icar_adv_var_request")
        call check(icar_adv_restart_vars(opts, restart_ids, n_restart), "icar_adv_restart_vars")
        call options%alloc_vars(int(alloc_ids(1:n_alloc)))
        call options%advect_vars(int(adv_list(1:n_advect)))
        call options%restart_vars(int(restart_ids(1:n_restart)))
    end subroutine adv_var_request

    !> advect(domain, options, dt), advection_driver.f90:59-126: upload the
    !! fields CPU code may have changed since the last call (winds and
    !! density after the wind update, the species after the other physics),
    !! advance every advected variable on the GPU, and bring the species
    !! back into domain_t.
    subroutine advect(domain, options, dt)
        type(domain_t), intent(inout), target :: domain
        type(options_t), intent(in) :: options
        real, intent(in) :: dt
        type(variable_t) :: var
        character(len=32) :: name
        integer :: s

        if (.not. c_associated(h)) then
            write(*,*) "advection (B200 library): advect called before adv_init"
            error stop
        endif
        call check(icar_adv_set_field(h, ICAR_F_U, c_loc(domain%u%data_3d), c_null_ptr), "set u")
        call check(icar_adv_set_field(h, ICAR_F_V, c_loc(domain%v%data_3d), c_null_ptr), "set v")
        call check(icar_adv_set_field(h, ICAR_F_W, c_loc(domain%w%data_3d), c_null_ptr), "set w")
        call check(icar_adv_set_field(h, ICAR_F_DENSITY, c_loc(domain%density%data_3d), c_null_ptr), "set density")
        s = 0
        call domain%adv_vars%reset_iterator()
        do while (domain%adv_vars%has_more_elements())
            var = domain%adv_vars%next(name)
            s = s + 1
            call check(icar_adv_set_field(h, adv_ids(s), c_loc(var%data_3d), c_null_ptr), "set "//trim(name))
        enddo
        call check(icar_adv_advect(h, real(dt, c_float)), "icar_adv_advect")
        s = 0
        call domain%adv_vars%reset_iterator()
        do while (domain%adv_vars%has_more_elements())
            var = domain%adv_vars%next(name)
            s = s + 1
            ! get_field returns once the data has arrived in host memory
            call check(icar_adv_get_field(h, adv_ids(s), c_loc(var%data_3d), c_null_ptr), "get "//trim(name))
        enddo
    end subroutine advect

end module advection
