"""Regenerates the coefficients of fn_asin_poly (fibrenet_b200/csrc/fn_detmath.h).

R(z) = (asin(sqrt z) - sqrt z) / z^1.5 on [0, 1/4] (R(0) = 1/6), interpolated
at the 14 Chebyshev points of the first kind mapped to [0, 1/4]
(z_k = 1/8 + 1/8 cos((2k + 1) pi / 28)) in 60-digit arithmetic, written in
monomial form in z and rounded to the nearest double.

    python tests/detmath_fit.py      # prints the C initialiser
"""
from __future__ import annotations

import mpmath as mp

DEGREE = 13
DIGITS = 60


def coefficients() -> list[float]:
    with mp.workdps(DIGITS):
        def r(z):
            if z == 0:
                return mp.mpf(1) / 6
            s = mp.sqrt(z)
            return (mp.asin(s) - s) / (z * s)

        a, b = mp.mpf(0), mp.mpf(1) / 4
        n = DEGREE
        nodes = [(a + b) / 2 + (b - a) / 2 * mp.cos((2 * k + 1) * mp.pi / (2 * (n + 1)))
                 for k in range(n + 1)]
        vander = mp.matrix(n + 1, n + 1)
        rhs = mp.matrix(n + 1, 1)
        for i, z in enumerate(nodes):
            for j in range(n + 1):
                vander[i, j] = z ** j
            rhs[i] = r(z)
        c = mp.lu_solve(vander, rhs)
        return [float(c[j]) for j in range(n + 1)]


if __name__ == "__main__":
    print("const double c[14] = {\n" + ",\n".join(f"    {x!r}" for x in coefficients()) + "};")
