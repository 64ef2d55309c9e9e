"""Argument errors on a live handle, through the C ABI: a null buffer that an
entry point must read or write comes back as Z2_ERR_ARG with the entry
point's name in z2_last_error, nothing is copied, and the handle keeps
working (the reference stops the program on bad input instead)."""
import ctypes as C

import numpy as np
import pytest

from z2_gauge_zfy_b200 import Chain, Z2Batch

pytestmark = pytest.mark.gpu


def test_null_buffers_rejected_and_handle_survives():
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10,
               seed=12345)
    with Z2Batch([ch]) as b:
        lib, h = b.lib, b.h
        b.pre()
        g0 = b.green(0)
        buf = np.zeros(16 * 16)
        p = buf.ctypes.data_as(C.POINTER(C.c_double))
        calls = {
            "z2_set_config": lambda: lib.z2_set_config(h, 0, None, 1),
            "z2_get_green": lambda: lib.z2_get_green(h, 0, None),
            "z2_get_obs_equal": lambda: lib.z2_get_obs_equal(h, 0, None),
            "z2_get_obs_tau": lambda: lib.z2_get_obs_tau(h, 0, None),
            "z2_get_stats": lambda: lib.z2_get_stats(h, 0, None),
            "z2_get_phase_cycles": lambda: lib.z2_get_phase_cycles(h, 0, None),
            "z2_get_global_stats": lambda: lib.z2_get_global_stats(h, 0, None),
            "z2_set_replay": lambda: lib.z2_set_replay(h, 0, None, 4),
            "z2_opk_mmult": lambda: lib.z2_opk_mmult_R(h, 0, None, 1, 1),
            "z2_stab_UR": lambda: lib.z2_stab_UR(h, 0, p, None, p),
            "z2_stab_UL": lambda: lib.z2_stab_UL(h, 0, None, p, p),
            "z2_stab_green": lambda: lib.z2_stab_green(h, 0, p, p, p, None, p, p, 1, p),
            "z2_stab_green_big": lambda: lib.z2_stab_green_big(h, 0, p, p, p, p, p, p, p, p,
                                                               None, p),
        }
        for name, call in calls.items():
            assert call() == 1, name
            assert name in lib.z2_last_error(h).decode(), name
        # nothing was written to the state: the same G, and sweeps still run
        assert np.array_equal(b.green(0), g0)
        b.sweep(1)
        assert np.all(np.isfinite(b.green(0)))


def test_python_mirrors_check_shapes():
    """The Python mirrors reject arrays whose shape does not match the chain
    (the library copies exactly N x N or 2N x Ltrot values)."""
    from z2_gauge_zfy_b200 import Z2Error
    ch = Chain(RT=1.0, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=10, seed=777)
    N = ch.N
    eye, one = np.eye(N), np.ones(N)
    small = np.eye(N - 2)
    with Z2Batch([ch]) as b:
        bad = [
            lambda: b.opk_mmult_R(0, np.ones((N, N - 1)), 1, 1),
            lambda: b.opk_mmult_L(0, small, 1, 1),
            lambda: b.stab_UR(0, eye, np.ones(N - 1), eye),
            lambda: b.stab_green(0, eye, one, eye, small, one, eye, 1),
            lambda: b.stab_green_big(0, eye, one, eye, eye, one, small),
            lambda: b.set_config(0, np.ones((ch.Ltrot, 2 * N)), 1),
        ]
        for i, call in enumerate(bad):
            with pytest.raises(Z2Error) as e:
                call()
            assert e.value.code == 1 and "needs" in str(e.value), i
        # the right shapes still go through
        assert b.opk_mmult_R(0, eye, 1, 1).shape == (N, N)
