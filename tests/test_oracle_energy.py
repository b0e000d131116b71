"""The oracle's energy restatement (engine/energy.go terms) against closed
forms, and its Relax() restatement on a small film (CPU only)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G

MU0 = 4e-7 * np.pi


def _uniform(N, v):
    m = np.empty((3, N[2], N[1], N[0]), np.float32)
    for c in range(3):
        m[c] = v[c]
    return m


def test_energy_closed_forms():
    """Uniform state of a box: exchange 0; Zeeman -V N Ms m.B; uniaxial
    -V N (K1 cos^2 + K2 cos^4 / ... ) in the reference's convention
    (B_K1.M = 2 K1 cos^2, B_K2.M = 4 K2 cos^4); demag 1/2 mu0 Ms^2 V_tot m.N.m
    with the Aharoni prism factors."""
    N, cell = (12, 10, 6), (3e-9, 2.5e-9, 2e-9)
    Ms, K1, K2 = 8e5, 4e4, 1.5e4
    u = (0.0, 0.6, 0.8)
    b = (0.02, -0.01, 0.03)
    m = np.array([0.36, 0.48, 0.8])
    sim = O.Simulation(N, cell, Ms, 1.3e-11, 0.1, dtype=np.float64, Ku1=K1, Ku2=K2, anisU=u, B_ext=b)
    E = O.energies(sim, _uniform(N, m))
    n = N[0] * N[1] * N[2]
    V = cell[0] * cell[1] * cell[2]
    cos = float(np.dot(m, u))
    assert abs(E["exchange"]) < 1e-12 * abs(E["zeeman"])
    assert E["zeeman"] == pytest.approx(-V * n * Ms * float(np.dot(m, b)), rel=1e-12)
    want_anis = V * n * (-0.5 * 2 * K1 * cos ** 2 - 0.25 * 4 * K2 * cos ** 4)
    assert E["anisotropy"] == pytest.approx(want_anis, rel=1e-12)
    Nf = G.prism_factors(N, cell)
    want_demag = 0.5 * MU0 * Ms ** 2 * V * n * sum(Nf[i] * m[i] ** 2 for i in range(3))
    assert E["demag"] == pytest.approx(want_demag, rel=1e-9)
    assert E["total"] == pytest.approx(E["anisotropy"] + E["demag"] + E["exchange"] + E["zeeman"], rel=1e-15)


def test_relax_lowers_energy_and_torque():
    """Relax() from a tilted uniform state of a small film: total energy goes
    down, the torque ends far below its start, time is unchanged."""
    N, cell = (16, 8, 1), (4e-9, 4e-9, 3e-9)
    sim = O.Simulation(N, cell, 8e5, 1.3e-11, 0.02, Ku1=1e4, anisU=(1, 0, 0))
    sim.set_m(_uniform(N, (1.0, 1.0, 0.2)))
    E0 = O.energies(sim)["total"]
    tau0 = O.max_vec_norm(sim.torque().reshape(3, -1))
    t0 = sim.solver.time
    O.relax(sim)
    E1 = O.energies(sim)["total"]
    tau1 = O.max_vec_norm(sim.torque().reshape(3, -1))
    assert E1 < E0
    assert tau1 < 1e-3 * tau0
    assert sim.solver.time == t0
    assert sim.solver.solver == 5 and sim.sys.precess == 1


def test_relax_twice_from_exact_equilibrium():
    """test/regression017.mx3 on the oracle: with m exactly along the easy
    axis the torque is exactly zero, so every relax step is accepted with
    err = 0 and dt doubles (87 steps per relax).  After the second relax the
    float32 step dt*GammaLL would overflow; dt is capped so that it stays
    finite (2^120) and m stays put instead of turning into NaN."""
    N = (5, 1, 1)
    o = O.Simulation(N, (1e-9, 1e-9, 1e-9), 1000e3, 10e-12, 0.02, Ku1=1.3e6, anisU=(0, 0, 1))
    for mz, steps in ((1.0, 87), (-1.0, 174)):
        m = np.zeros((3, 1, 1, 5), np.float32)
        m[2] = mz
        o.set_m(m)
        O.relax(o)
        assert o.solver.status == 0 and o.solver.nsteps == steps
        assert np.array_equal(o.m[2], np.full((1, 1, 5), mz, np.float32))
    assert o.solver.dt * o.solver.gamma_ll == pytest.approx(2.0 ** 120, rel=1e-12)


def test_no_demag_spins_restatement():
    """engine/demag.go:67-98 on the oracle: with NoDemagSpins in region 1 the
    demag field equals that of a geometry without region 1, and is zero in
    region 1 itself (uniform m: no exchange field, no other terms)."""
    N, cell = (12, 10, 2), (2e-9, 2e-9, 2e-9)
    regions = np.zeros((2, 10, 12), np.uint8)
    regions[:, :, 7:] = 1
    m = np.zeros((3, 2, 10, 12), np.float32)
    m[0], m[1], m[2] = 0.6, 0.0, 0.8
    a = O.Simulation(N, cell, 8e5, 0.0, 0.1, regions=regions, NoDemagSpins=[0, 1])
    a.set_m(m)
    _, Ba = a.torque(beff=True)
    b = O.Simulation(N, cell, 8e5, 0.0, 0.1, regions=regions, vol=(regions == 0).astype(np.float32))
    b.set_m(m)
    _, Bb = b.torque(beff=True)
    r0 = np.broadcast_to(regions == 0, Ba.shape)
    assert np.array_equal(Ba[r0], Bb[r0]) and np.abs(Ba[r0]).max() > 1e-3
    assert np.all(Ba[~r0] == 0)


def _exchange_inhomo_case():
    """test/exchange_inhomo.mx3: 4x4x1 cells of 1 m, the random m of
    testdata/randommag4x4x1.ovf (tests/golden/randommag4x4x1.npy), regions
    1-4 the quadrants (rect(2,2) translated by (+-1, +-1)), Aex 1.2, 1.6, 4.3,
    4.3 (harmonic mean between regions); E_exch from OOMMF 154.4891365 J."""
    import os
    from umagnus_b200 import config
    N, cell = (4, 4, 1), (1.0, 1.0, 1.0)
    m = np.load(os.path.join(os.path.dirname(__file__), "golden", "randommag4x4x1.npy"))
    regions = np.zeros((1, 4, 4), np.uint8)
    for r, (dx, dy) in zip((1, 2, 3, 4), ((1, 1), (-1, 1), (-1, -1), (1, -1))):
        regions[config.rect(N, cell, 2, 2, transl=(dx, dy, 0)) > 0] = r
    aex = np.ones(256)
    aex[1:5] = (1.2, 1.6, 4.3, 4.3)
    return N, cell, m, regions, aex


@pytest.mark.parametrize("ms", [(3.2, 4.6, 3.9, 7.8), (1.1, 1.1, 1.1, 1.1)])
def test_exchange_inhomo_against_oommf(ms):
    """The oracle's exchange energy with per-region Aex and Msat equals
    OOMMF's within the script's 1e-5 J, whatever the Msat values."""
    N, cell, m, regions, aex = _exchange_inhomo_case()
    assert sorted(np.unique(regions)) == [1, 2, 3, 4]
    Ms = np.asarray((0.0,) + tuple(ms))[regions]
    o = O.Simulation(N, cell, Ms, 1.0, 0.1, regions=regions, Aex_regions=aex, demag=False)
    o.set_m(m)
    assert abs(O.energies(o)["exchange"] - 154.4891365) <= 1e-5
