! Shims that keep the reference's entry points and route them to libptbgpu.
!
! Each subroutine replaces the routine of the same name in the contains section of
! module sm (source/sm.f90:34) and of module purification_ (source/purification.f90:28),
! with the same signature, so twoscf (source/pgtb.f90:594-642) calls them unchanged.
! Those modules already use gtb_accuracy (wp) and purification_settings
! (tPurificationSet).  The reference's stop / error stop on failures stays an
! error stop, now with the library's message.

subroutine sm_stupid_simple(ndim,nelref,Hvec,Svec,Pvec,n,xyz,aoat,submatrix_columns,submatrix_mode)
   use ptbgpu_c
   integer, intent(in) :: nelref, ndim, n, submatrix_columns, submatrix_mode
   real(wp), intent(in) :: Hvec(:), Svec(:), xyz(3,n)
   real(wp), intent(inout) :: Pvec(:)
   integer, intent(in) :: aoat(ndim)
   type(ptbgpu_opts) :: opts
   type(ptbgpu_stats) :: st
   character(kind=c_char, len=512) :: msg
   integer(c_int) :: rc
   if (.not. c_associated(ptbgpu_ctx)) then
      rc = ptbgpu_init(0_c_int, ptbgpu_ctx)
      if (rc /= 0) error stop 'ptbgpu_init failed (no usable GPU or library)'
   endif
   rc = ptbgpu_sm_density(ptbgpu_ctx, int(ndim,c_int64_t), int(nelref,c_int64_t), Hvec, Svec, Pvec, &
        int(n,c_int64_t), xyz, aoat, int(submatrix_columns,c_int64_t), int(submatrix_mode,c_int64_t), &
        c_null_ptr, opts, st)
   if (rc /= 0) then
      ! the message is NUL-terminated; the reference's stop on errors becomes error stop with it
      if (ptbgpu_last_error(ptbgpu_ctx, msg, 512_c_size_t) /= 0) msg = 'ptbgpu_sm_density failed' // c_null_char
      error stop msg(1:index(msg, c_null_char) - 1)
   endif
end subroutine

subroutine purification_wrapper(pur, ndim, H, S, P)
   use ptbgpu_c
   type(tPurificationSet) :: pur
   integer, intent(in) :: ndim
   real(wp), intent(in) :: H(ndim*(ndim+1)/2), S(ndim*(ndim+1)/2)
   real(wp), intent(out) :: P(ndim*(ndim+1)/2)
   type(ptbgpu_pur_settings) :: cs
   type(ptbgpu_opts) :: opts
   type(ptbgpu_stats) :: st
   character(kind=c_char, len=512) :: msg
   integer(c_int) :: rc
   cs = ptbgpu_pur_settings(int(pur%mode,c_int64_t), int(pur%type,c_int64_t), int(pur%cycles,c_int64_t), &
        int(pur%prlvl,c_int64_t), int(pur%nel,c_int64_t), int(pur%submatrix_mode,c_int64_t), &
        int(pur%submatrix_columns,c_int64_t), int(pur%metric%type,c_int64_t), &
        int(pur%metric%cycles,c_int64_t), merge(1_c_int64_t, 0_c_int64_t, pur%metric%iterative), &
        int(pur%chempot%cycles,c_int64_t), real(pur%chempot%guess,c_double), &
        real(pur%chempot%increment,c_double))
   opts%print_level = int(pur%prlvl, c_int64_t)
   if (.not. c_associated(ptbgpu_ctx)) then
      rc = ptbgpu_init(0_c_int, ptbgpu_ctx)
      if (rc /= 0) error stop 'ptbgpu_init failed (no usable GPU or library)'
   endif
   rc = ptbgpu_purify(ptbgpu_ctx, cs, int(ndim,c_int64_t), H, S, P, opts, st)
   if (rc /= 0) then
      if (ptbgpu_last_error(ptbgpu_ctx, msg, 512_c_size_t) /= 0) msg = 'ptbgpu_purify failed' // c_null_char
      error stop msg(1:index(msg, c_null_char) - 1)
   endif
end subroutine
