"""The thermal-noise generator's restatement (oracle.thermal_normals):
Philox4x32-10 against the known-answer vectors published with the algorithm
(Salmon et al., SC'11, Random123 kat_vectors), and the distribution of the
normals it yields.  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O

KAT = [
    # counter (4 words), key (2 words) -> output (4 words)
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    out = O.philox4x32_10(*[np.array([c]) for c in ctr], *key)
    assert tuple(int(o[0]) for o in out) == want


def test_normals_distribution():
    n = 400000
    z = O.thermal_normals(0x1234567890ABCDEF, 7, n).astype(np.float64)
    assert z.shape == (3, n)
    for c in range(3):
        assert abs(z[c].mean()) < 5 / np.sqrt(n)
        assert abs(z[c].var() - 1) < 8 * np.sqrt(2 / n)
        assert abs(np.mean(z[c] ** 4) - 3) < 0.05
    assert abs(np.corrcoef(z)[0, 1]) < 5 / np.sqrt(n) and abs(np.corrcoef(z)[0, 2]) < 5 / np.sqrt(n)
    # different steps and seeds give independent numbers
    z2 = O.thermal_normals(0x1234567890ABCDEF, 8, n).astype(np.float64)
    z3 = O.thermal_normals(0x1234567890ABCDEE, 7, n).astype(np.float64)
    assert abs(np.corrcoef(z[0], z2[0])[0, 1]) < 5 / np.sqrt(n)
    assert abs(np.corrcoef(z[0], z3[0])[0, 1]) < 5 / np.sqrt(n)
