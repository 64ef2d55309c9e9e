"""Host logic of the Python mirror without a GPU: the layout conversions
(natural indexing <-> the library's column-major buffers) and the shape
checks, against a stand-in library whose entry points copy nothing.  With
such a library every mirror must hand its inputs back unchanged."""
import numpy as np
import pytest

from z2_gauge_zfy_b200 import api
from z2_gauge_zfy_b200 import Z2Error


class _NoOpLib:
    """z2_chain_dims reports a chain of N sites and L slices; every other
    entry point succeeds without touching its buffers."""

    def __init__(self, N, L):
        self.N, self.L = N, L

    def z2_chain_dims(self, h, chain, N, L, S):
        N._obj.value, L._obj.value, S._obj.value = self.N, self.L, 1
        return 0

    def __getattr__(self, name):
        return lambda *args: 0


def _batch(N=6, L=4):
    b = api.Z2Batch.__new__(api.Z2Batch)   # no z2_create: nothing on a device
    b.lib, b.h, b.chains = _NoOpLib(N, L), None, []
    return b


def test_mirrors_round_trip_layouts():
    N = 6
    b = _batch(N)
    rng = np.random.default_rng(0)
    U, V, M = rng.standard_normal((3, N, N))
    D = rng.standard_normal(N)
    for fn in (b.stab_UR, b.stab_UL):
        u, d, v = fn(0, U, D, V)
        assert np.array_equal(u, U) and np.array_equal(d, D) and np.array_equal(v, V)
        assert d is not D                      # D is returned as a new array
    assert np.array_equal(b.opk_mmult_R(0, M, 1, 1), M)
    assert np.array_equal(b.opk_mmult_L(0, M, 1, -1), M)
    assert b.stab_green(0, U, D, V, U, D, V, 1).shape == (N, N)
    assert [g.shape for g in b.stab_green_big(0, U, D, V, U, D, V)] == [(N, N)] * 4


@pytest.mark.parametrize("call", [
    lambda b: b.opk_mmult_R(0, np.eye(5), 1, 1),
    lambda b: b.stab_UL(0, np.eye(6), np.ones(5), np.eye(6)),
    lambda b: b.stab_green(0, np.eye(6), np.ones(6), np.eye(6), np.eye(6), np.ones(6),
                           np.ones((6, 7)), 1),
    lambda b: b.set_config(0, np.ones((4, 12)), 1),     # transposed sigma(2N, Ltrot)
])
def test_mirrors_reject_wrong_shapes(call):
    with pytest.raises(Z2Error) as e:
        call(_batch())
    assert e.value.code == 1 and "needs" in str(e.value)
