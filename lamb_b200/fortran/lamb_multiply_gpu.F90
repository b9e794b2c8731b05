! lamb_multiply_gpu.F90 -- single-rank body of lamb_multiply that runs the
! multiply on the B200 through liblamb_b200.so.
!
! Replaces the sector-pair loop and the exchange of lamb_multiply
! (src/lamb_multiplication.F90:116-204): at one rank every sector is local,
! so the market / window calls of service_schedule (:227-320) are not made,
! and the loop over sector triples (:180-201) with its sector_multiply stub
! (:206-225) becomes ONE lamb_gpu_multiply over all triples.  The
! distribution checks of :136-146 stay with the caller.
!
! upload:   every matrix%sectors(s) crosses as a lamb_c_sector (subset
!           positions, block sizes, row_p, col_i, data_stores(1)%d); the
!           extents are repacked into a contiguous int64 (2, n_blks) array
!           because lamb_blk_info_type is not BIND(C)
!           (src/lamb_index_types.F90:86-91).
! download: two-phase size -> fill: lamb_gpu_matrix_query gives each C
!           sector's block count and data length, the Fortran side sizes its
!           own storage (index arrays; lamb_data_ensure_length,
!           src/lamb_data_X_methods.F90:138-162), then lamb_gpu_matrix_download
!           fills it and the extents are copied back into blk_info.
!
! Not compiled in this repository's containers (no Fortran compiler).  It
! uses the reference's generic names (lamb_matrix_types etc., generated by
! make_interface.py) and its kinds (blkn_k int64, locatm_k int16,
! dataptr_k int64, blksz_k int8: src/lamb_kinds.F90:155-179).
module lamb_multiply_gpu
  use iso_c_binding
  use lamb_gpu_bindings
  use lamb_kinds
  use lamb_error
  use lamb_matrix_types
  use lamb_sector_types
  use lamb_index_types
  use lamb_data_methods
  implicit none
  private

  public :: lamb_multiply_on_gpu, lamb_gpu_finalize

  type(c_ptr), save :: ctx = c_null_ptr

  ! Host copies that must live while a call runs (extents repacked, sector
  ! descriptors).
  type sector_staging
     integer(c_int64_t), allocatable :: extents(:, :)
     integer(c_int8_t), allocatable :: rbs(:), cbs(:)
  end type sector_staging

contains

  subroutine check(st, what, error)
    integer(c_int32_t), intent(in) :: st
    character(len=*), intent(in) :: what
    type(lamb_error_type), intent(inout) :: error
    character(kind=c_char) :: msg(512)
    character(len=512) :: text
    integer :: i, rc
    if (st == 0) return
    rc = lamb_gpu_last_error(ctx, msg, 512_c_int32_t)
    text = ' '
    do i = 1, 512
       if (msg(i) == c_null_char) exit
       text(i:i) = msg(i)
    end do
    call lamb_error_throw(error, int(lamb_gpu_status_level(st)), int(lamb_gpu_status_type(st)), &
         what//': '//trim(text), lamb_here('lamb_multiply_gpu', what, __LINE__))
  end subroutine check

  subroutine upload(matrix, handle, staging, error)
    type(lamb_matrix_d_type), intent(in), target :: matrix
    integer(c_int64_t), intent(out) :: handle
    type(sector_staging), allocatable, intent(inout) :: staging(:)
    type(lamb_error_type), intent(inout) :: error
    type(lamb_c_sector), allocatable :: cs(:)
    integer :: s, nb
    allocate(cs(size(matrix%sectors)), staging(size(matrix%sectors)))
    do s = 1, size(matrix%sectors)
       associate (sec => matrix%sectors(s))
         nb = int(sec%index%row_p(sec%index%n_rows + 1))
         allocate(staging(s)%extents(2, max(nb, 1)))
         if (nb > 0) then
            staging(s)%extents(1, 1:nb) = sec%index%blk_info(1:nb)%extent(1)
            staging(s)%extents(2, 1:nb) = sec%index%blk_info(1:nb)%extent(2)
         end if
         staging(s)%rbs = int(sec%subsets(1)%p%blksizes, c_int8_t)
         staging(s)%cbs = int(sec%subsets(2)%p%blksizes, c_int8_t)
         cs(s)%subset_row = int(sec%subsets(1)%p%pos, c_int32_t)
         cs(s)%subset_col = int(sec%subsets(2)%p%pos, c_int32_t)
         cs(s)%n_rows = int(sec%subsets(1)%p%n, c_int32_t)
         cs(s)%n_cols = int(sec%subsets(2)%p%n, c_int32_t)
         cs(s)%row_blk_sizes = c_loc(staging(s)%rbs)
         cs(s)%col_blk_sizes = c_loc(staging(s)%cbs)
         cs(s)%row_p = c_loc(sec%index%row_p)
         cs(s)%col_i = c_loc(sec%index%col_i)
         cs(s)%extents = c_loc(staging(s)%extents)
         cs(s)%data = c_loc(sec%data_stores(1)%d)
         cs(s)%n_blks = int(nb, c_int64_t)
         cs(s)%data_len = int(sec%data_stores(1)%data_len, c_int64_t)
       end associate
    end do
    call check(lamb_gpu_matrix_upload(ctx, cs, int(size(cs), c_int32_t), handle), 'lamb_gpu_matrix_upload', error)
  end subroutine upload

  subroutine download(handle, matrix, error)
    integer(c_int64_t), intent(in) :: handle
    type(lamb_matrix_d_type), intent(inout), target :: matrix
    type(lamb_error_type), intent(inout) :: error
    integer(c_int32_t) :: n
    type(lamb_c_sector_sizes), allocatable :: sz(:)
    type(lamb_c_sector), allocatable :: cs(:)
    type(sector_staging), allocatable :: staging(:)
    integer :: s, t, nb
    call check(lamb_gpu_matrix_n_sectors(ctx, handle, n), 'lamb_gpu_matrix_n_sectors', error)
    allocate(sz(n), cs(n), staging(n))
    call check(lamb_gpu_matrix_query(ctx, handle, sz, n), 'lamb_gpu_matrix_query', error)
    do s = 1, n
       ! C's sectors come in the same (subset_row, subset_col) order as the
       ! matrix's own sectors (fill_my_sectors, src/lamb_plexus_operations.F90:454-488)
       associate (sec => matrix%sectors(s))
         nb = int(sz(s)%n_blks)
         if (allocated(sec%index%col_i)) deallocate(sec%index%col_i)
         if (allocated(sec%index%blk_info)) deallocate(sec%index%blk_info)
         allocate(sec%index%col_i(max(nb, 1)), sec%index%blk_info(max(nb, 1)))
         call lamb_data_ensure_length(sec%data_stores(1), int(sz(s)%data_len, dataptr_k), error)
         allocate(staging(s)%extents(2, max(nb, 1)))
         allocate(staging(s)%rbs(max(sz(s)%n_rows, 1)), staging(s)%cbs(max(sz(s)%n_cols, 1)))
         cs(s)%row_blk_sizes = c_loc(staging(s)%rbs)
         cs(s)%col_blk_sizes = c_loc(staging(s)%cbs)
         cs(s)%row_p = c_loc(sec%index%row_p)
         cs(s)%col_i = c_loc(sec%index%col_i)
         cs(s)%extents = c_loc(staging(s)%extents)
         cs(s)%data = c_loc(sec%data_stores(1)%d)
         cs(s)%n_blks = sz(s)%n_blks
         cs(s)%data_len = sz(s)%data_len
       end associate
    end do
    call check(lamb_gpu_matrix_download(ctx, handle, cs, n), 'lamb_gpu_matrix_download', error)
    do s = 1, n
       associate (sec => matrix%sectors(s))
         nb = int(cs(s)%n_blks)
         do t = 1, nb
            sec%index%blk_info(t)%extent(1) = staging(s)%extents(1, t)
            sec%index%blk_info(t)%extent(2) = staging(s)%extents(2, t)
            sec%index%blk_info(t)%store = 1
            sec%index%blk_info(t)%bits = 0
         end do
         sec%index%n_idx_blks = int(nb, blkn_k)
         sec%n_blks = int(nb, blkn_k)
         sec%data_stores(1)%data_len = int(cs(s)%data_len, dataptr_k)
       end associate
    end do
  end subroutine download

  !> C := A . B on the GPU; A, B and C share one distribution (checked by
  !> the caller as lamb_multiply does).  eps is the filter threshold of the
  !> build's product and result filters (eps <= 0 disables both).
  subroutine lamb_multiply_on_gpu(matrix_a, matrix_b, matrix_c, eps, error)
    type(lamb_matrix_d_type), intent(in), target :: matrix_a, matrix_b
    type(lamb_matrix_d_type), intent(inout), target :: matrix_c
    real(c_double), intent(in) :: eps
    type(lamb_error_type), intent(inout) :: error
    integer(c_int64_t) :: ha, hb, hc
    type(lamb_gpu_mult_stats) :: stats
    type(sector_staging), allocatable :: sa(:), sb(:)
    integer(c_int32_t) :: st
    if (.not. c_associated(ctx)) call check(lamb_gpu_ctx_create(0_c_int32_t, ctx), 'lamb_gpu_ctx_create', error)
    call upload(matrix_a, ha, sa, error)
    call upload(matrix_b, hb, sb, error)
    call check(lamb_gpu_matrix_create_like(ctx, ha, hc), 'lamb_gpu_matrix_create_like', error)
    ! LAMB_GPU_ASYNC: the download below copies C row chunk by row chunk
    ! while the numeric phase finishes the rest.
    call check(lamb_gpu_multiply(ctx, ha, hb, hc, eps, lamb_gpu_async, stats), 'lamb_gpu_multiply', error)
    call download(hc, matrix_c, error)
    st = lamb_gpu_matrix_destroy(ctx, hc)
    st = lamb_gpu_matrix_destroy(ctx, hb)
    st = lamb_gpu_matrix_destroy(ctx, ha)
  end subroutine lamb_multiply_on_gpu

  subroutine lamb_gpu_finalize()
    integer(c_int32_t) :: st
    if (c_associated(ctx)) st = lamb_gpu_ctx_destroy(ctx)
    ctx = c_null_ptr
  end subroutine lamb_gpu_finalize

end module lamb_multiply_gpu
