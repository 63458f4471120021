!> ISO_C_BINDING interface to libptrans_b200.so (include/ptrans_gpu.h).
!!
!! A Fortran host of the RTMC solver uses this module to replace the body of
!! TransmissionFunction (src/RTMCphon.f90:1544-1604): flatten vgrain / anphon
!! once with ptg_setup_from_rtmc (below), then call ptg_transmission once per
!! mean free path; MPI_Allreduce of transmit stays where it is.
!! No Fortran compiler exists on the machines this library was built on, so
!! this file is provided as source for the maintainer's build.
module ptrans_gpu
  use iso_c_binding
  implicit none
  private

  integer(c_int), parameter, public :: PTG_OK = 0
  integer(c_int32_t), parameter, public :: PTG_PREC_FP32 = 0, PTG_PREC_FP64 = 1

  type, bind(C), public :: ptg_geometry
    real(c_double) :: box(3), scope(2)
    integer(c_int32_t) :: face_kind(6)
    integer(c_int32_t) :: kind_grain, ngrain, igrain_fill, nmaterial
    integer(c_int32_t) :: ngrain_total, nsurf, nvertex_total
    type(c_ptr) :: grain_begin, grain_incident, grain_generatrix
    type(c_ptr) :: shape, nvertex, vertex_begin, vertex, normal, tangent, center, radius
    type(c_ptr) :: kind_trans, specularity, trans_param, grain_inside, grain_outside
    type(c_ptr) :: internal, incident, material1, material2
  end type ptg_geometry

  type, bind(C), public :: ptg_spectrum
    integer(c_int32_t) :: nbranch, nkpoint
    real(c_double) :: rtemp, vol
    type(c_ptr) :: omega, tau, vel, mfp, weight
  end type ptg_spectrum

  type, bind(C), public :: ptg_options
    integer(c_int32_t) :: device = 0, block_size = 0, blocks_per_sm = 0
    integer(c_int32_t) :: regen_threshold = 0, ref_quirks = 1, bvh_leaf = 0
    integer(c_int64_t) :: max_flights = 0
    real(c_double) :: lost_limit = 0.0d0
    integer(c_int64_t) :: chunk = 0
    integer(c_int32_t) :: tune_flags = 0, fast_steps = 0, coop_lanes = 0, reserved = 0
  end type ptg_options

  public :: ptg_create, ptg_destroy, ptg_transmission, ptg_strerror_f

  interface
    integer(c_int) function ptg_create(geom, spec, opt, handle) bind(C, name="ptg_create")
      import :: c_int, c_ptr, ptg_geometry, ptg_spectrum, ptg_options
      type(ptg_geometry), intent(in) :: geom
      type(ptg_spectrum), intent(in) :: spec
      type(ptg_options), intent(in) :: opt
      type(c_ptr), intent(out) :: handle
    end function ptg_create

    subroutine ptg_destroy(handle) bind(C, name="ptg_destroy")
      import :: c_ptr
      type(c_ptr), value :: handle
    end subroutine ptg_destroy

    integer(c_int) function ptg_transmission(handle, mfp_nm, nangle, np, rank, nranks, seed, &
        precision, transmit, stderr_opt) bind(C, name="ptg_transmission")
      import :: c_int, c_ptr, c_double, c_int32_t, c_int64_t
      type(c_ptr), value :: handle
      real(c_double), value :: mfp_nm
      integer(c_int32_t), value :: nangle
      integer(c_int64_t), value :: np
      integer(c_int32_t), value :: rank, nranks
      integer(c_int64_t), value :: seed          ! uint64_t on the C side
      integer(c_int32_t), value :: precision
      real(c_double), intent(inout) :: transmit(*)
      type(c_ptr), value :: stderr_opt           ! c_null_ptr when not wanted
    end function ptg_transmission

    type(c_ptr) function ptg_strerror(status) bind(C, name="ptg_strerror")
      import :: c_ptr, c_int
      integer(c_int), value :: status
    end function ptg_strerror
  end interface

contains

  !> Message text of a status code.
  function ptg_strerror_f(status) result(msg)
    integer(c_int), intent(in) :: status
    character(len=64) :: msg
    character(kind=c_char), pointer :: p(:)
    integer :: i
    call c_f_pointer(ptg_strerror(status), p, [64])
    msg = ' '
    do i = 1, 64
      if (p(i) == c_null_char) exit
      msg(i:i) = p(i)
    end do
  end function ptg_strerror_f

end module ptrans_gpu
