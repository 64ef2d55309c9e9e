! z2_cuda_mod.f90 -- ISO_C_BINDING interface of the B200 DQMC library
! (include/z2dqmc.h) for the reference's Fortran driver.  Every entry point
! of the C header is bound here with the header's arguments; see
! INTEGRATION.md for the calls that replace src/main.f90:72-79 and for the
! module procedures each mirror stands in for.
!
! Compile with the driver:  gfortran -c include/z2_cuda_mod.f90
! Link:  -L<repo>/z2_gauge_zfy_b200 -lz2dqmc -Wl,-rpath,<repo>/z2_gauge_zfy_b200
module z2_cuda_mod
    use iso_c_binding
    implicit none
    type, bind(C) :: z2_chain_params
        real(c_double)  :: RT, J, h, mu, Q
        integer(c_int32_t) :: Nlx, Nly, Ltrot
        real(c_double)  :: beta
        integer(c_int32_t) :: Nwrap, absolute, seed
        type(c_ptr)     :: rt_bond          ! c_null_ptr = uniform RT
    end type
    type, bind(C) :: z2_options
        integer(c_int32_t) :: delay_k, record, device, tau, graph
        type(c_ptr)     :: delay_k_chain    ! c_null_ptr, or c_loc(k(1)) from z2_tune
        type(c_ptr)     :: flush_shape_chain ! c_null_ptr, or c_loc(s(1)) from z2_tune
        integer(c_int32_t) :: stab_exact    ! 1 = the reference's pivoted QR in the wraps
    end type
    interface
        integer(c_int) function z2_create(h, p, n, opt) bind(C, name="z2_create")
            import; type(c_ptr) :: h; type(z2_chain_params) :: p(*)
            integer(c_int32_t), value :: n; type(z2_options) :: opt
        end function
        integer(c_int) function z2_destroy(h) bind(C, name="z2_destroy")
            import; type(c_ptr), value :: h
        end function
        integer(c_int) function z2_pre(h) bind(C, name="z2_pre")
            import; type(c_ptr), value :: h
        end function
        integer(c_int) function z2_sweep(h, nsweep, toggle) bind(C, name="z2_sweep")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: nsweep, toggle
        end function
        integer(c_int) function z2_set_config(h, chain, sigma, iseed) bind(C, name="z2_set_config")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, iseed
            real(c_double) :: sigma(*)
        end function
        integer(c_int) function z2_get_config(h, chain, sigma, iseed) bind(C, name="z2_get_config")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: sigma(*); integer(c_int32_t) :: iseed
        end function
        integer(c_int) function z2_get_obs_equal(h, chain, obs) bind(C, name="z2_get_obs_equal")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: obs(7)
        end function
        integer(c_int) function z2_get_obs_equal_all(h, obs) bind(C, name="z2_get_obs_equal_all")
            import; type(c_ptr), value :: h
            real(c_double) :: obs(7, *)
        end function
        integer(c_int) function z2_get_obs_tau(h, chain, obs) bind(C, name="z2_get_obs_tau")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: obs(*)
        end function
        integer(c_int) function z2_get_stats(h, chain, st) bind(C, name="z2_get_stats")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: st(14)
        end function
        integer(c_int) function z2_opk_mmult_R(h, chain, M, nt, nflag) bind(C, name="z2_opk_mmult_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt, nflag
            real(c_double) :: M(*)
        end function
        integer(c_int) function z2_get_obs_tau_k(h, chain, re, im) bind(C, name="z2_get_obs_tau_k")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: re(*), im(*)
        end function
        integer(c_int) function z2_sweep_global(h, nglobal) bind(C, name="z2_sweep_global")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: nglobal
        end function
        integer(c_int) function z2_get_global_stats(h, chain, g) bind(C, name="z2_get_global_stats")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: g(5)
        end function
        integer(c_int) function z2_tune_delay(p, n, opt, k) bind(C, name="z2_tune_delay")
            import; type(z2_chain_params) :: p(*); integer(c_int32_t), value :: n
            type(z2_options) :: opt; integer(c_int32_t) :: k(*)
        end function
        integer(c_int) function z2_tune(p, n, opt, k, shape) bind(C, name="z2_tune")
            import; type(z2_chain_params) :: p(*); integer(c_int32_t), value :: n
            type(z2_options) :: opt; integer(c_int32_t) :: k(*), shape(*)
        end function
        integer(c_int) function z2_stab_green(h, chain, UR, DR, VR, UL, DL, VL, nt, G) &
                bind(C, name="z2_stab_green")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
            real(c_double) :: UR(*), DR(*), VR(*), UL(*), DL(*), VL(*), G(*)
        end function
        ! ---- the remaining entry points of z2dqmc.h ----
        ! Outputs the header calls optional are bound as type(c_ptr), value:
        ! pass c_loc(x) or c_null_ptr.
        type(c_ptr) function z2_last_error(h) bind(C, name="z2_last_error")
            import; type(c_ptr), value :: h
        end function
        integer(c_int) function z2_chain_dims(h, chain, N, Ltrot, Nst) bind(C, name="z2_chain_dims")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            integer(c_int32_t) :: N, Ltrot, Nst
        end function
        integer(c_int) function z2_sweep_timed(h, nsweep, toggle, ms) bind(C, name="z2_sweep_timed")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: nsweep, toggle
            real(c_float) :: ms
        end function
        integer(c_int) function z2_therm(h, nwarm, acc) bind(C, name="z2_therm")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: nwarm
            type(c_ptr), value :: acc              ! optional real(c_double) acc(nchains)
        end function
        integer(c_int) function z2_get_green(h, chain, G) bind(C, name="z2_get_green")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: G(*)
        end function
        integer(c_int) function z2_get_phase_cycles(h, chain, cyc) bind(C, name="z2_get_phase_cycles")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: cyc(12)
        end function
        integer(c_int) function z2_set_replay(h, chain, r, n) bind(C, name="z2_set_replay")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: r(*); integer(c_size_t), value :: n
        end function
        integer(c_int) function z2_get_decisions(h, chain, dec, ratios, n) &
                bind(C, name="z2_get_decisions")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            type(c_ptr), value :: dec, ratios      ! optional int8 dec(n), real(c_double) ratios(n)
            integer(c_size_t), value :: n
        end function
        integer(c_int) function z2_logdet_grad(h, chain, logdet, dt, dmu) bind(C, name="z2_logdet_grad")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: logdet, dt(*), dmu
        end function
        integer(c_int) function z2_opk_mmult_L(h, chain, M, nt, nflag) bind(C, name="z2_opk_mmult_L")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt, nflag
            real(c_double) :: M(*)
        end function
        integer(c_int) function z2_stab_UR(h, chain, U, D, V) bind(C, name="z2_stab_UR")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: U(*), D(*), V(*)
        end function
        integer(c_int) function z2_stab_UL(h, chain, U, D, V) bind(C, name="z2_stab_UL")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: U(*), D(*), V(*)
        end function
        integer(c_int) function z2_stab_green_big(h, chain, UR, DR, VR, UL, DL, VL, &
                G00, G0t, Gt0, Gtt) bind(C, name="z2_stab_green_big")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            real(c_double) :: UR(*), DR(*), VR(*), UL(*), DL(*), VL(*)
            real(c_double) :: G00(*), G0t(*), Gt0(*), Gtt(*)
        end function
        ! device pointers and a cudaStream_t (c_null_ptr = default stream)
        integer(c_int) function z2_stab_green_noalloc(N, nt, Ltrot, UR, DR, VR, UL, DL, VL, &
                G, stream) bind(C, name="z2_stab_green_noalloc")
            import; integer(c_int32_t), value :: N, nt, Ltrot
            type(c_ptr), value :: UR, DR, VR, UL, DL, VL, G, stream
        end function
        ! ---- module-level mirrors on a chain's resident state (z2dqmc.h):
        !      multiply, stabilization, dynamics, localK, local_sweep,
        !      obser_equal and obser_tau procedures of one chain ----
        integer(c_int) function z2_propK_pre(h, chain, nt) bind(C, name="z2_propK_pre")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_propK_L(h, chain, nt) bind(C, name="z2_propK_L")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_propK_R(h, chain, nt) bind(C, name="z2_propK_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_propgrK_R(h, chain, nt) bind(C, name="z2_propgrK_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_propT_pre(h, chain) bind(C, name="z2_propT_pre")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
        end function
        integer(c_int) function z2_propT_L(h, chain) bind(C, name="z2_propT_L")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
        end function
        integer(c_int) function z2_propT_R(h, chain) bind(C, name="z2_propT_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
        end function
        integer(c_int) function z2_propgrT_R(h, chain) bind(C, name="z2_propgrT_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
        end function
        integer(c_int) function z2_wrap_pre(h, chain, nt) bind(C, name="z2_wrap_pre")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_wrap_L(h, chain, nt, flag) bind(C, name="z2_wrap_L")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt, flag
        end function
        integer(c_int) function z2_wrap_R(h, chain, nt, flag) bind(C, name="z2_wrap_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt, flag
        end function
        integer(c_int) function z2_wrap_tau(h, chain, nt) bind(C, name="z2_wrap_tau")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_dyn_reset(h, chain) bind(C, name="z2_dyn_reset")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
        end function
        integer(c_int) function z2_prop_slice_L(h, chain, nt) bind(C, name="z2_prop_slice_L")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_prop_slice_R(h, chain, nt) bind(C, name="z2_prop_slice_R")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_sweep_reset(h, chain, toggle) bind(C, name="z2_sweep_reset")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, toggle
        end function
        integer(c_int) function z2_obs_equal_calc(h, chain, nt) bind(C, name="z2_obs_equal_calc")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_obs_equal_ave(h, chain, nobs) bind(C, name="z2_obs_equal_ave")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nobs
        end function
        integer(c_int) function z2_obs_tau_calc(h, chain, nt) bind(C, name="z2_obs_tau_calc")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nt
        end function
        integer(c_int) function z2_obs_tau_ave(h, chain, nobst) bind(C, name="z2_obs_tau_ave")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain, nobst
        end function
        ! Propagator / PropGreen transfer: every buffer optional (c_loc(x) or c_null_ptr)
        integer(c_int) function z2_get_prop(h, chain, G, UR, DR, VR, UL, DL, VL) &
                bind(C, name="z2_get_prop")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            type(c_ptr), value :: G, UR, DR, VR, UL, DL, VL
        end function
        integer(c_int) function z2_set_prop(h, chain, G, UR, DR, VR, UL, DL, VL) &
                bind(C, name="z2_set_prop")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            type(c_ptr), value :: G, UR, DR, VR, UL, DL, VL
        end function
        integer(c_int) function z2_get_propgr(h, chain, G00, G0t, Gt0, Gtt) &
                bind(C, name="z2_get_propgr")
            import; type(c_ptr), value :: h; integer(c_int32_t), value :: chain
            type(c_ptr), value :: G00, G0t, Gt0, Gtt
        end function
    end interface
contains
    ! z2_last_error as a Fortran string (the C text is NUL-terminated and
    ! shorter than 512 characters)
    function z2_error_text(h) result(msg)
        type(c_ptr), intent(in) :: h
        character(len=:), allocatable :: msg
        character(kind=c_char), pointer :: s(:)
        integer :: n, i
        call c_f_pointer(z2_last_error(h), s, [512])
        do n = 0, 511
            if (s(n + 1) == c_null_char) exit
        enddo
        allocate(character(len=n) :: msg)
        do i = 1, n
            msg(i:i) = s(i)
        enddo
    end function
end module z2_cuda_mod
