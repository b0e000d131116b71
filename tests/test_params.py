"""Region parameter tables on the host (CPU only): the inter-region exchange
LUT with the reference's ScaleExchange / InterExchange semantics
(engine/exchange.go:136-164: lut = scale * average + inter)."""
import numpy as np

from umagnus_b200.engine import exch_average, exchange_lut, pair_tables, symmidx


def test_scale_and_inter_tables():
    aex = np.zeros(256)
    aex[:4] = (13e-12, 10e-12, 20e-12, 5e-12)
    sc, it = pair_tables({(1, 2): -1.0, (3, 0): 0.5}, {(2, 3): 7e-12})
    lut = exchange_lut(aex, sc, it)
    plain = exchange_lut(aex)
    assert lut[symmidx(1, 2)] == np.float32(-1.0) * exch_average(10e-12, 20e-12)
    assert lut[symmidx(2, 1)] == lut[symmidx(1, 2)]
    assert lut[symmidx(0, 3)] == np.float32(0.5) * exch_average(13e-12, 5e-12)
    assert lut[symmidx(2, 3)] == np.float32(7e-12)
    changed = {symmidx(1, 2), symmidx(0, 3), symmidx(2, 3)}
    keep = np.array([k not in changed for k in range(lut.size)])
    assert np.array_equal(lut[keep], plain[keep])
    assert pair_tables(None, None) == (None, None)


def test_inter_overrides_scale_for_the_same_pair():
    sc, it = pair_tables({(4, 5): 2.0}, {(5, 4): 1e-12})
    k = symmidx(4, 5)
    assert sc[k] == 0 and it[k] == np.float32(1e-12)


def test_shapes_and_configurations():
    """Host-side shapes and configurations (engine/shape.go, engine/config.go)
    on the cell centres of a mesh centred on the origin."""
    from umagnus_b200 import config
    N, c = (128, 64, 1), 5e-9
    cell = (c, c, c)
    centred = config.rect(N, cell, 64 * c, 32 * c)
    shifted = config.rect(N, cell, 64 * c, 32 * c, repeat=(128 * c, 64 * c, 0), transl=(64 * c, 32 * c, 0))
    assert centred.sum() == shifted.sum() == 64 * 32
    assert shifted[0, 0, 0] == 1 and shifted[0, 32, 64] == 0 and centred[0, 32, 64] == 1
    # two domains rotated by 90 degrees: down below y = 0, up above, the wall along x
    f = config.rot_z(config.two_domain_fn(cell, (0, 0, -1), (1, 1, 0), (0, 0, 1)), np.pi / 2)
    m = config.sample((16, 16, 1), cell, f)
    assert m.dtype == np.float32 and m.shape == (3, 1, 16, 16)
    assert m[2, 0, 0, 5] < -0.99 and m[2, 0, 15, 5] > 0.99
    np.testing.assert_allclose(m[:2, 0, 8, 3], [-0.9394131, 0.9394131], rtol=0, atol=1e-6)
    np.testing.assert_array_equal(config.two_domain((16, 8, 1), cell, (0, 0, -1), (1, 1, 0), (0, 0, 1)),
                                  config.sample((16, 8, 1), cell,
                                                config.two_domain_fn(cell, (0, 0, -1), (1, 1, 0), (0, 0, 1))))
