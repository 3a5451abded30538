"""Copies the NACA section tables of the reference's own tests into a fixture.

    python tests/golden/make_naca_tables.py

test/naca4digit_test.cpp and test/naca00XX_test.cpp of xeno14/UVLM check the
generators against two published tables in test/wing/data/: NACA62XX.dat
(mean camber y_c against x, chord 100) and NACA0012.dat (half thickness z
against x, chord 1).  This script reads them as text from the reference tree
and stores them as tests/golden/naca_tables.npz, so that the known-answer
tests run where the reference tree is absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"


def read_table(path):
    # the tests read pairs with `ifs >> x >> y` until EOF
    vals = open(path).read().split()
    return np.array([float(v) for v in vals]).reshape(-1, 2)


def main():
    data = os.path.join(REF, "test", "wing", "data")
    out = dict(naca62xx=read_table(os.path.join(data, "NACA62XX.dat")),
               naca0012=read_table(os.path.join(data, "NACA0012.dat")))
    np.savez_compressed(os.path.join(HERE, "naca_tables.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
