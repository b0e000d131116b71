"""Regenerates the small fixtures in this folder from the reference's own
test data (run where the reference tree is present; the GPU tests read only
the fixtures).

- randommag4x4x1.npy: the magnetisation of test/testdata/randommag4x4x1.ovf
  (the input of test/exchange_inhomo.mx3), float32 (3, 1, 4, 4), read with
  this package's OVF reader.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import build_ref  # noqa: E402
from umagnus_b200 import fileio  # noqa: E402


def main():
    ref = build_ref.reference_root()
    if ref is None:
        raise SystemExit("reference checkout not found: set UMAG_REFERENCE to its root")
    arr, _ = fileio.read(os.path.join(ref, "test", "testdata", "randommag4x4x1.ovf"))
    np.save(os.path.join(HERE, "randommag4x4x1.npy"), np.asarray(arr, np.float32))


if __name__ == "__main__":
    main()
