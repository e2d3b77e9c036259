"""CPU checks of the numpy restatement of the learned V-cycle (oracle/mg_oracle.py):
the properties the device network and its training rely on."""
import numpy as np
import pytest

from oracle import mg_oracle as MO


_random_faces = MO.random_faces
_weights = MO.random_weights


@pytest.mark.parametrize("dim,n", [(2, (12, 10)), (3, (6, 6, 5))])
def test_vcycle_is_symmetric(dim, n):
    dims, f = MO.kernel_faces(dim, n, _random_faces(dim, n, 1))
    H = MO.hierarchy(dims, f, dim)
    k, c = _weights(dim, 2, 2)
    V = MO.VCycle(dim, H, k, c, nu=2, coarse_sweeps=7)
    rng = np.random.default_rng(3)
    a, b = rng.normal(size=(2, int(np.prod(n))))
    assert abs(a @ V.apply(b) - b @ V.apply(a)) <= 1e-10 * abs(a @ V.apply(a))


def test_hierarchy_shapes_follow_the_stop_rule():
    dims, f = MO.kernel_faces(2, (40, 36), _random_faces(2, (40, 36), 4))
    H = MO.hierarchy(dims, f, 2)
    # 5 x 5 = 25 cells <= 64: the coarsest level
    assert [L.dims for L in H] == [(40, 1, 36), (20, 1, 18), (10, 1, 9), (5, 1, 5)]
    # a coarse x-face carries the fine faces at the even x positions it covers
    for F, C in zip(H[:2], H[1:3]):
        assert np.isclose(C.fx.sum(), F.fx[:, :, 0::2].sum())


def test_default_network_contracts():
    dims, f = MO.kernel_faces(2, (32, 32), _random_faces(2, (32, 32), 5))
    H = MO.hierarchy(dims, f, 2)
    k = np.zeros((1, 27))
    k[0, 13] = 0.8
    V = MO.VCycle(2, H, k, [1.0])
    e = np.random.default_rng(6).normal(size=32 * 32)
    assert 0.0 < V.loss(e, pin=0) < 0.5
