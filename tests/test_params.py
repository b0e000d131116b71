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
