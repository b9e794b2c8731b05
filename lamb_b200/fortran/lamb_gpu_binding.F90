! lamb_gpu_binding.F90 -- ISO_C_BINDING interface to liblamb_b200.so
! (include/lamb_gpu.h) for LAMB's Fortran 2003 sources.
!
! The derived types mirror the C structs field for field (BIND(C));
! lamb_c_sector_out has lamb_c_sector's memory layout, so one type serves
! uploads and downloads.  Status codes: 0 is success, otherwise
! level*100000 + (type + 50000) with LAMB's error levels and types
! (src/lamb_error.F90:120-159); lamb_gpu_status_level / _type decode them.
!
! Not compiled in this repository's containers (no Fortran compiler); the C
! side of every interface below is exercised by the Python and C99 callers.
module lamb_gpu_bindings
  use iso_c_binding
  implicit none
  private

  integer(c_int32_t), parameter, public :: lamb_gpu_fp64 = 0, lamb_gpu_mixed = 1, &
       lamb_gpu_no_product_filter = 2, lamb_gpu_no_result_filter = 4, lamb_gpu_async = 8

  ! One sector in the reference's storage (src/lamb_index_types.F90:86-105,
  ! src/lamb_data_X_types.F90:77-83): row_p int64 exclusive offsets, col_i
  ! int16 1-based, extents int64 (2, n_blks) 1-based inclusive, data real64
  ! column-major blocks, block sizes int8.
  type, bind(c), public :: lamb_c_sector
     integer(c_int32_t) :: subset_row = 0, subset_col = 0, n_rows = 0, n_cols = 0
     type(c_ptr) :: row_blk_sizes = c_null_ptr, col_blk_sizes = c_null_ptr
     type(c_ptr) :: row_p = c_null_ptr, col_i = c_null_ptr, extents = c_null_ptr, data = c_null_ptr
     integer(c_int64_t) :: n_blks = 0, data_len = 0
  end type lamb_c_sector

  type, bind(c), public :: lamb_c_sector_sizes
     integer(c_int32_t) :: subset_row, subset_col, n_rows, n_cols
     integer(c_int64_t) :: n_blks, data_len
  end type lamb_c_sector_sizes

  type, bind(c), public :: lamb_gpu_mult_stats
     integer(c_int64_t) :: n_products, n_products_skipped, n_c_blocks, n_c_blocks_dropped
     real(c_double) :: flops, ms_symbolic, ms_numeric, ms_total
     integer(c_int32_t) :: mixed_slices, kernel_launches
     real(c_double) :: ms_prepare, ms_filter, tensor_ops, ms_kernel
  end type lamb_gpu_mult_stats

  public :: lamb_gpu_ctx_create, lamb_gpu_ctx_destroy, lamb_gpu_last_error, lamb_gpu_status_level, &
       lamb_gpu_status_type, lamb_gpu_matrix_upload, lamb_gpu_matrix_set_positions, &
       lamb_gpu_matrix_create_like, lamb_gpu_matrix_destroy, lamb_gpu_matrix_n_sectors, &
       lamb_gpu_matrix_query, lamb_gpu_matrix_download, lamb_gpu_multiply, lamb_gpu_ctx_synchronize

  interface
     integer(c_int32_t) function lamb_gpu_ctx_create(device, ctx) bind(c, name='lamb_gpu_ctx_create')
       import :: c_int32_t, c_ptr
       integer(c_int32_t), value :: device
       type(c_ptr) :: ctx
     end function lamb_gpu_ctx_create
     integer(c_int32_t) function lamb_gpu_ctx_destroy(ctx) bind(c, name='lamb_gpu_ctx_destroy')
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function lamb_gpu_ctx_destroy
     integer(c_int32_t) function lamb_gpu_ctx_synchronize(ctx) bind(c, name='lamb_gpu_ctx_synchronize')
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function lamb_gpu_ctx_synchronize
     integer(c_int32_t) function lamb_gpu_last_error(ctx, msg, len) bind(c, name='lamb_gpu_last_error')
       import :: c_int32_t, c_ptr, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char) :: msg(*)
       integer(c_int32_t), value :: len
     end function lamb_gpu_last_error
     integer(c_int32_t) function lamb_gpu_status_level(status) bind(c, name='lamb_gpu_status_level')
       import :: c_int32_t
       integer(c_int32_t), value :: status
     end function lamb_gpu_status_level
     integer(c_int32_t) function lamb_gpu_status_type(status) bind(c, name='lamb_gpu_status_type')
       import :: c_int32_t
       integer(c_int32_t), value :: status
     end function lamb_gpu_status_type
     integer(c_int32_t) function lamb_gpu_matrix_upload(ctx, sectors, n_sectors, handle) &
          bind(c, name='lamb_gpu_matrix_upload')
       import :: c_int32_t, c_int64_t, c_ptr, lamb_c_sector
       type(c_ptr), value :: ctx
       type(lamb_c_sector), intent(in) :: sectors(*)
       integer(c_int32_t), value :: n_sectors
       integer(c_int64_t), intent(out) :: handle
     end function lamb_gpu_matrix_upload
     integer(c_int32_t) function lamb_gpu_matrix_set_positions(ctx, handle, xyz, n_rows, box) &
          bind(c, name='lamb_gpu_matrix_set_positions')
       import :: c_int32_t, c_int64_t, c_ptr, c_float
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: handle
       real(c_float), intent(in) :: xyz(3, *)
       integer(c_int32_t), value :: n_rows
       real(c_float), intent(in) :: box(3)
     end function lamb_gpu_matrix_set_positions
     integer(c_int32_t) function lamb_gpu_matrix_create_like(ctx, like, handle) &
          bind(c, name='lamb_gpu_matrix_create_like')
       import :: c_int32_t, c_int64_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: like
       integer(c_int64_t), intent(out) :: handle
     end function lamb_gpu_matrix_create_like
     integer(c_int32_t) function lamb_gpu_matrix_destroy(ctx, handle) bind(c, name='lamb_gpu_matrix_destroy')
       import :: c_int32_t, c_int64_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: handle
     end function lamb_gpu_matrix_destroy
     integer(c_int32_t) function lamb_gpu_matrix_n_sectors(ctx, handle, n) bind(c, name='lamb_gpu_matrix_n_sectors')
       import :: c_int32_t, c_int64_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: handle
       integer(c_int32_t), intent(out) :: n
     end function lamb_gpu_matrix_n_sectors
     integer(c_int32_t) function lamb_gpu_matrix_query(ctx, handle, sizes, n) bind(c, name='lamb_gpu_matrix_query')
       import :: c_int32_t, c_int64_t, c_ptr, lamb_c_sector_sizes
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: handle
       type(lamb_c_sector_sizes), intent(out) :: sizes(*)
       integer(c_int32_t), value :: n
     end function lamb_gpu_matrix_query
     integer(c_int32_t) function lamb_gpu_matrix_download(ctx, handle, sectors, n) &
          bind(c, name='lamb_gpu_matrix_download')
       import :: c_int32_t, c_int64_t, c_ptr, lamb_c_sector
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: handle
       type(lamb_c_sector), intent(inout) :: sectors(*)
       integer(c_int32_t), value :: n
     end function lamb_gpu_matrix_download
     integer(c_int32_t) function lamb_gpu_multiply(ctx, a, b, c, eps, flags, stats) bind(c, name='lamb_gpu_multiply')
       import :: c_int32_t, c_int64_t, c_ptr, c_double, lamb_gpu_mult_stats
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: a, b, c
       real(c_double), value :: eps
       integer(c_int32_t), value :: flags
       type(lamb_gpu_mult_stats), intent(out) :: stats
     end function lamb_gpu_multiply
  end interface
end module lamb_gpu_bindings
