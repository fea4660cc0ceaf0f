! robinsolver_b200 -- Fortran 2008 binding of librobin_b200.so (include/robin_b200.h).
!
! Keeps the reference's public names and calls (robin_tree%factor, robin_tree%solve,
! get_solution and the types elliptic_operator, solve_opts, elliptic_rhs, bndry_rhs,
! leaf_solution) so that a program written against robin_tree_module/robin_output_module
! switches by changing its `use` lines.  Callbacks stay scalar `pure` functions of a point; this
! module evaluates them on the host at the points the library reports and hands the samples to
! the C-ABI.  A non-zero status becomes `stop` with the library's message, as the reference stops.
!
! Not compiled in this repository's build (the image has no Fortran compiler); the Python
! binding (robinsolver_b200/_lib.py) exercises the same C-ABI in the tests.
module robinsolver_b200
    use, intrinsic :: iso_c_binding
    implicit none
    private

    integer, parameter :: dp = kind(1.0d0)

    public :: elliptic_operator, solve_opts, debug_opts, elliptic_rhs, bndry_rhs, leaf_solution, &
              robin_tree, get_solution, scalar_proc, coeff_proc, b200_opts

    abstract interface
        pure function coeff_proc(x) result(c)
            import dp
            real(dp), dimension(:), intent(in) :: x
            complex(dp), dimension(1:3,1:3) :: c
        end function
        pure function scalar_proc(x) result(r)
            import dp
            real(dp), dimension(:), intent(in) :: x
            complex(dp) :: r
        end function
    end interface

    type elliptic_operator
        integer :: d
        real(dp), dimension(1:2,1:3) :: domain
        procedure(coeff_proc), pointer, nopass :: coeff => null()
        procedure(scalar_proc), pointer, nopass :: k => null()
        complex(dp), dimension(1:6,1:2) :: robin_coeff
    end type

    type bndry_rhs
        procedure(scalar_proc), pointer, nopass :: g_face => null()
    end type

    type elliptic_rhs
        integer :: d
        procedure(scalar_proc), pointer, nopass :: f => null()
        type(bndry_rhs), dimension(1:6) :: g
    end type

    type debug_opts
        logical :: txt_output = .false.
        logical :: no_delete = .false.
    end type

    type solve_opts
        real(dp) :: h_tgt
        real(dp), dimension(1:3) :: h
        integer :: ordering = 1
        character(len=2) :: disc = 'fd'
        character(len=3) :: local_mode = 'LU'
        character(len=3) :: R_mode = 'LU'
        real(dp) :: kb = 1.0d0
        type(debug_opts) :: debug
    end type

    type leaf_solution
        real(dp), dimension(1:2,1:3) :: box
        complex(dp), dimension(:), allocatable :: u
    end type

    ! Extensions of this library, kept out of solve_opts so that it stays the reference's type:
    ! precision 'fp64' (RB_PREC_FP64) or 'mixed' (RB_PREC_MIXED: int8 tensor-core GEMMs on the
    ! lower merge levels, every solve refined against the FP64 residual to tol); int8_top: the
    ! mixed factor's top two levels on the tensor cores too (RB_FLAG_MIXED_INT8_TOP).
    type b200_opts
        character(len=5) :: precision = 'fp64'
        real(dp) :: tol = 1.0d-10
        integer :: max_iter = 8
        logical :: int8_top = .false.
    end type

    type robin_tree
        integer :: nlvls
        type(elliptic_operator) :: ell_op
        type(solve_opts) :: opts
        complex(dp), dimension(1:2,1:2) :: bndry_params
        logical :: factored = .false.
        real(dp) :: f_time, s_time
        type(b200_opts) :: b200
        type(c_ptr) :: handle = c_null_ptr
    contains
        procedure :: factor => robin_tree_factor
        procedure :: solve => robin_tree_solve
    end type

    ! ---- C-ABI (include/robin_b200.h) -----------------------------------------------------------
    type, bind(c) :: rb_geom
        integer(c_int32_t) :: d, L
        real(c_double) :: domain(6)
        real(c_double) :: h_tgt, kb
        real(c_double) :: bndry_params(8)
        integer(c_int32_t) :: ordering, flags
        integer(c_int64_t) :: device_budget
    end type

    type, bind(c) :: rb_info
        integer(c_int32_t) :: nleaves, leaf_a, leaf_b, leaf_n, leaf_nb, root_nb, root_a, root_b
        real(c_double) :: h_last(3)
        integer(c_int64_t) :: n_interior, device_bytes
        integer(c_int32_t) :: factored, nrhs
        integer(c_int32_t) :: d, leaf_c, root_c, reserved
    end type

    integer(c_int), parameter :: RB_POINTS_POTENTIAL = 0, RB_POINTS_SOURCE = 1, RB_POINTS_BOUNDARY = 2

    interface
        integer(c_int) function rb_tree_create(geom, out) bind(c, name='rb_tree_create')
            import :: c_int, c_ptr, rb_geom
            type(rb_geom), intent(in) :: geom
            type(c_ptr), intent(out) :: out
        end function
        integer(c_int) function rb_tree_destroy(t) bind(c, name='rb_tree_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: t
        end function
        type(c_ptr) function rb_last_error(t) bind(c, name='rb_last_error')
            import :: c_ptr
            type(c_ptr), value :: t
        end function
        integer(c_int) function rb_tree_info(t, info) bind(c, name='rb_tree_info')
            import :: c_int, c_ptr, rb_info
            type(c_ptr), value :: t
            type(rb_info), intent(out) :: info
        end function
        integer(c_int) function rb_tree_sample_points(t, which, xyz) bind(c, name='rb_tree_sample_points')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: t
            integer(c_int), value :: which
            real(c_double), intent(out) :: xyz(*)
        end function
        integer(c_int) function rb_tree_factor(t, k, precision) bind(c, name='rb_tree_factor')
            import :: c_int, c_ptr, c_double_complex
            type(c_ptr), value :: t
            complex(c_double_complex), intent(in) :: k(*)
            integer(c_int), value :: precision
        end function
        integer(c_int) function rb_tree_solve(t, nrhs, f, g) bind(c, name='rb_tree_solve')
            import :: c_int, c_ptr, c_double_complex
            type(c_ptr), value :: t
            integer(c_int), value :: nrhs
            complex(c_double_complex), intent(in) :: f(*), g(*)
        end function
        integer(c_int) function rb_get_solution(t, irhs, u, boxes) bind(c, name='rb_get_solution')
            import :: c_int, c_ptr, c_double, c_double_complex
            type(c_ptr), value :: t
            integer(c_int), value :: irhs
            complex(c_double_complex), intent(out) :: u(*)
            real(c_double), intent(out) :: boxes(*)
        end function
        integer(c_int) function rb_tree_times(t, f_time, s_time) bind(c, name='rb_tree_times')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: t
            real(c_double), intent(out) :: f_time, s_time
        end function
        integer(c_int) function rb_tree_set_refinement(t, tol, max_iter) bind(c, name='rb_tree_set_refinement')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: t
            real(c_double), value :: tol
            integer(c_int), value :: max_iter
        end function
    end interface

contains

    subroutine check(rc, t)
        integer(c_int), intent(in) :: rc
        type(c_ptr), intent(in) :: t
        character(kind=c_char), pointer :: msg(:)
        character(len=512) :: text
        integer :: i
        if (rc == 0) return
        call c_f_pointer(rb_last_error(t), msg, [512])
        text = ''
        do i = 1, 512
            if (msg(i) == c_null_char) exit
            text(i:i) = msg(i)
        end do
        write(*, '(A)') trim(text)
        stop
    end subroutine

    subroutine robin_tree_factor(T, L, ell_op, opts)
        class(robin_tree), intent(inout) :: T
        integer, intent(in) :: L
        type(elliptic_operator), intent(in) :: ell_op
        type(solve_opts), intent(in) :: opts
        type(rb_geom) :: g
        type(rb_info) :: info
        real(c_double), allocatable :: xyz(:)
        complex(c_double_complex), allocatable :: k(:)
        integer :: j, p
        if (c_associated(T%handle)) call check(rb_tree_destroy(T%handle), c_null_ptr)
        T%nlvls = L
        T%ell_op = ell_op
        T%opts = opts
        g%d = ell_op%d
        g%L = L
        do j = 1, 3
            g%domain(2*j-1) = ell_op%domain(1,j)
            g%domain(2*j) = ell_op%domain(2,j)
        end do
        g%h_tgt = opts%h_tgt
        g%kb = opts%kb
        g%bndry_params = [real(T%bndry_params(1,1)), aimag(T%bndry_params(1,1)), &
                          real(T%bndry_params(2,1)), aimag(T%bndry_params(2,1)), &
                          real(T%bndry_params(1,2)), aimag(T%bndry_params(1,2)), &
                          real(T%bndry_params(2,2)), aimag(T%bndry_params(2,2))]
        g%ordering = opts%ordering
        g%flags = merge(2, 0, opts%debug%txt_output) + merge(32, 0, T%b200%int8_top)
        g%device_budget = 0
        call check(rb_tree_create(g, T%handle), c_null_ptr)
        call check(rb_tree_info(T%handle, info), T%handle)
        allocate(xyz(3*info%n_interior), k(info%n_interior))
        call check(rb_tree_sample_points(T%handle, RB_POINTS_POTENTIAL, xyz), T%handle)
        do p = 1, int(info%n_interior)
            k(p) = ell_op%k(xyz(3*p-2:3*p))
        end do
        call check(rb_tree_set_refinement(T%handle, real(T%b200%tol, c_double), int(T%b200%max_iter, c_int)), &
                   T%handle)
        call check(rb_tree_factor(T%handle, k, merge(1_c_int, 0_c_int, T%b200%precision == 'mixed')), T%handle)
        call check(rb_tree_info(T%handle, info), T%handle)
        T%opts%h = info%h_last
        call check(rb_tree_times(T%handle, T%f_time, T%s_time), T%handle)
        T%factored = .true.
    end subroutine

    subroutine robin_tree_solve(T, rhs)
        class(robin_tree), intent(inout) :: T
        type(elliptic_rhs), intent(in) :: rhs
        type(rb_info) :: info
        real(c_double), allocatable :: xf(:), xg(:)
        complex(c_double_complex), allocatable :: f(:), g(:)
        integer :: p, face, first, last, nfaces
        integer :: bounds(7), pf(6)
        if (.not. T%factored) stop 'Error: Robin Tree must be factored first.'
        if (T%ell_op%d /= rhs%d) stop 'Error: Dimensions of Robin Tree and RHS do not match.'
        call check(rb_tree_info(T%handle, info), T%handle)
        allocate(xf(3*info%n_interior), f(info%n_interior), xg(3*info%root_nb), g(info%root_nb))
        call check(rb_tree_sample_points(T%handle, RB_POINTS_SOURCE, xf), T%handle)
        call check(rb_tree_sample_points(T%handle, RB_POINTS_BOUNDARY, xg), T%handle)
        do p = 1, int(info%n_interior)
            f(p) = rhs%f(xf(3*p-2:3*p))
        end do
        ! points per root face (get_pt_face, fd_module.f90:1033-1049), faces x1 x2 y1 y2 (z1 z2)
        nfaces = 2*info%d
        if (info%d == 2) then
            pf(1:4) = [info%root_b, info%root_b, info%root_a, info%root_a]
        else
            pf = [info%root_b*info%root_c, info%root_b*info%root_c, info%root_a*info%root_c, &
                  info%root_a*info%root_c, info%root_a*info%root_b, info%root_a*info%root_b]
        end if
        bounds(1) = 0
        do face = 1, nfaces
            bounds(face + 1) = bounds(face) + pf(face)
        end do
        do face = 1, nfaces
            first = bounds(face) + 1
            last = bounds(face + 1)
            do p = first, last
                g(p) = rhs%g(face)%g_face(xg(3*p-2:3*p))
            end do
        end do
        call check(rb_tree_solve(T%handle, 1_c_int, f, g), T%handle)
        call check(rb_tree_times(T%handle, T%f_time, T%s_time), T%handle)
    end subroutine

    subroutine get_solution(T, sol)
        type(robin_tree), intent(in) :: T
        type(leaf_solution), dimension(:), allocatable, intent(inout) :: sol
        type(rb_info) :: info
        complex(c_double_complex), allocatable :: u(:)
        real(c_double), allocatable :: boxes(:)
        integer :: i, n
        if (.not. T%factored) stop 'Error in GET_SOLUTION: Robin Tree not factored.'
        call check(rb_tree_info(T%handle, info), T%handle)
        n = info%leaf_n
        allocate(u(info%nleaves * n), boxes(6 * info%nleaves), sol(info%nleaves))
        call check(rb_get_solution(T%handle, 0_c_int, u, boxes), T%handle)
        do i = 1, info%nleaves
            sol(i)%box = reshape(boxes(6*i-5:6*i), [2, 3])
            allocate(sol(i)%u(n))
            sol(i)%u = u((i-1)*n+1:i*n)
        end do
    end subroutine

end module robinsolver_b200
