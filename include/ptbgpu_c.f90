! ISO_C_BINDING interface of libptbgpu (include/ptbgpu.h) for the PTB Fortran program.
!
! Built with the reference's flags (-i8: default integers are 8 bytes, source/Makefile:35-37);
! every default-integer argument of the C-ABI is int64_t.  The bind(C) types mirror the
! header's structs field by field (tests/test_abi.py checks the order and kinds).
! Link with -L<repo>/ptb_b200 -lptbgpu -Wl,-rpath,<repo>/ptb_b200.
module ptbgpu_c
   use iso_c_binding
   implicit none
   type(c_ptr), save :: ptbgpu_ctx = c_null_ptr

   type, bind(C) :: ptbgpu_opts
      real(c_double)     :: filter = 0.0_c_double
      integer(c_int64_t) :: precision = 1_c_int64_t
      integer(c_int64_t) :: print_level = 1_c_int64_t
      integer(c_int64_t) :: max_iter = 100_c_int64_t
      real(c_double)     :: electronic_temp = 300.0_c_double
      real(c_double)     :: glob_par15 = 0.0_c_double, glob_par17 = 0.0_c_double
      integer(c_int64_t) :: split3_iters = -1_c_int64_t
      integer(c_int64_t) :: fp64_slices = 8_c_int64_t   ! 0: cuBLAS/cuSOLVER FP64 products
      integer(c_int64_t) :: refine_rounds = 4_c_int64_t  ! cap on the refinement rounds
      real(c_double)     :: refine_tol = 1.0e-7_c_double ! next round while the predicted error exceeds it
   end type
   type, bind(C) :: ptbgpu_stats
      real(c_double)     :: mu, nel, band_energy, idempotency_ref, idempotency_frob
      integer(c_int64_t) :: nsm, sum_dims, max_dim, iterations, mu_iterations, info
      real(c_double)     :: ms_total, ms_h2d, ms_solve, ms_d2h, flops, ms_tc_sp2
      integer(c_int64_t) :: n_tc_sp2
      real(c_double)     :: ms_tc_full
      integer(c_int64_t) :: n_tc_full, kernel_launches
      real(c_double)     :: ms_oz
      integer(c_int64_t) :: n_oz
      real(c_double)     :: oz_ops, tc_flops
      integer(c_int64_t) :: refine_rounds, fp64_fallback
   end type

   type, bind(C) :: ptbgpu_pur_settings      ! POD mirror of tPurificationSet
      integer(c_int64_t) :: mode, type, cycles, prlvl, nel, submatrix_mode, submatrix_columns
      integer(c_int64_t) :: metric_type, metric_cycles, metric_iterative, chempot_cycles
      real(c_double)     :: chempot_guess, chempot_increment
   end type

   interface
      integer(c_int) function ptbgpu_init(device, ctx) bind(C, name="ptbgpu_init")
         import :: c_int, c_ptr
         integer(c_int), value :: device
         type(c_ptr) :: ctx
      end function
      integer(c_int) function ptbgpu_last_error(ctx, buf, len) bind(C, name="ptbgpu_last_error")
         import :: c_int, c_ptr, c_char, c_size_t
         type(c_ptr), value :: ctx
         character(kind=c_char) :: buf(*)
         integer(c_size_t), value :: len
      end function
      integer(c_int) function ptbgpu_sm_density(ctx, ndim, nelref, H, S, P, nat, xyz, aoat, &
            columns, mode, partition, opts, st) bind(C, name="ptbgpu_sm_density")
         import :: c_int, c_int64_t, c_double, c_ptr, ptbgpu_opts, ptbgpu_stats
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: ndim, nelref, nat, columns, mode
         real(c_double) :: H(*), S(*), P(*), xyz(3,*)
         integer(c_int64_t) :: aoat(*)
         type(c_ptr), value :: partition
         type(ptbgpu_opts) :: opts
         type(ptbgpu_stats) :: st
      end function
      integer(c_int) function ptbgpu_purify(ctx, pur, ndim, H, S, P, opts, st) bind(C, name="ptbgpu_purify")
         import :: c_int, c_int64_t, c_double, c_ptr, ptbgpu_pur_settings, ptbgpu_opts, ptbgpu_stats
         type(c_ptr), value :: ctx
         type(ptbgpu_pur_settings) :: pur
         integer(c_int64_t), value :: ndim
         real(c_double) :: H(*), S(*), P(*)
         type(ptbgpu_opts) :: opts
         type(ptbgpu_stats) :: st
      end function
      integer(c_int) function ptbgpu_tc_purify(ctx, ndim, nel, H, S, P, opts, st) &
            bind(C, name="ptbgpu_tc_purify")
         import :: c_int, c_int64_t, c_double, c_ptr, ptbgpu_opts, ptbgpu_stats
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: ndim, nel
         real(c_double) :: H(*), S(*), P(*)
         type(ptbgpu_opts) :: opts
         type(ptbgpu_stats) :: st
      end function
      integer(c_int) function ptbgpu_xc_damping(ctx, nat, ndim, aoat, rab, rad, hao, xdiag, P, H, ms) &
            bind(C, name="ptbgpu_xc_damping")
         import :: c_int, c_int64_t, c_double, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: nat, ndim
         integer(c_int64_t) :: aoat(*)
         real(c_double) :: rab(*), rad(*), hao(*), xdiag(*), P(*), H(*)
         type(c_ptr), value :: ms
      end function
   end interface
end module
