"""SaveAs(m) / m.LoadFile through OVF 2.0 and the dump format on a GPU simulation."""
import numpy as np
import pytest

from tests import golden_pins as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt", ["binary 4", "text", "dump"])
def test_save_load_m(fmt, tmp_path):
    from umagnus_b200 import engine, fileio
    N, cell = (20, 12, 3), (3e-9, 3e-9, 2e-9)
    a = engine.Simulation(N, cell, 8e5, 1.3e-11, 0.1)
    a.set_m(G.random_unit(N, 4))
    a.steps(3)
    p = tmp_path / "m.ovf"
    if fmt == "dump":
        m = a.get_m().cpu().numpy()
        fileio.write_dump(p, m, cell, name="m", time=a.state()["time"])
    else:
        fileio.save_m(a, p, format=fmt)
    ma = a.get_m().cpu().numpy()
    arr, meta = fileio.read(p)
    np.testing.assert_array_equal(arr, ma)  # the file holds m exactly
    assert meta["time"] == pytest.approx(a.state()["time"], rel=1e-15)
    b = engine.Simulation(N, cell, 8e5, 1.3e-11, 0.1)
    fileio.load_m(b, p)  # SetArray renormalises (engine/magnetization.go:55), a 1-ulp change at most
    np.testing.assert_allclose(b.get_m().cpu().numpy(), ma, rtol=0, atol=2.5e-7)
    a.free()
    b.free()
