"""Generate the golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The reference ships no stored outputs for this path, and its Fortran cannot
be built here, so the fixtures are outputs of the oracle (oracle/sht_oracle.c,
a statement-by-statement restatement of the reference routines), whose own
correctness is pinned in tests/test_oracle.py against independent known
answers (scipy Legendre functions, numpy FFTs and Gauss-Legendre nodes).
Inputs are seeded power-law coefficients (S(l) = (l+1)^-2).

Each .npz holds the input coefficients, the option set, and the grid and the
re-expanded coefficients produced by the oracle.
"""
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def cases():
    for L in (7, 15):
        for norm, cs, samp, ext, lcsel in itertools.product(
                (1, 2, 3, 4), (1, -1), (1, 2), (0, 1), (0, 1)):
            yield ("dh", L, norm, cs, samp, ext, L if lcsel == 0 else L // 2)
        for norm, cs, ext, lcsel in itertools.product((1, 2, 3, 4), (1, -1),
                                                      (0, 1), (0, 1)):
            yield ("glq", L, norm, cs, 1, ext, L if lcsel == 0 else L // 2)
    for kind in ("dh", "glq"):
        for norm in (1, 4):
            yield (kind, 64, norm, 1, 2 if kind == "dh" else 1, 0, 64)


def main():
    out = {}
    for i, (kind, L, norm, cs, samp, ext, lc) in enumerate(cases()):
        c = O.power_law_cilm(L, 7000 + i)
        if kind == "dh":
            g = O.makegrid_dh(c, norm=norm, sampling=samp, csphase=cs,
                              lmax_calc=lc, extend=ext)
            n = 2 * L + 2
            back = O.shexpand_dh(g[:n, :samp * n], norm=norm, sampling=samp,
                                 csphase=cs, lmax_calc=lc)
            zero = w = np.zeros(0)
        else:
            zero, w = O.shglq(L)
            g = O.makegrid_glq(c, zero=zero, norm=norm, csphase=cs,
                               lmax_calc=lc, extend=ext)
            back = O.shexpand_glq(g[:, :2 * L + 1], w=w, zero=zero, norm=norm,
                                  csphase=cs, lmax_calc=lc)
        key = "%s_L%d_n%d_c%d_s%d_e%d_lc%d" % (kind, L, norm, cs, samp, ext, lc)
        out[key + "__cilm"] = c
        out[key + "__grid"] = g
        out[key + "__back"] = back
        if kind == "glq":
            out[key + "__zero"] = zero
            out[key + "__w"] = w
    path = os.path.join(HERE, "transforms_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    main()
