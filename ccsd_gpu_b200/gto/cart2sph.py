"""Cartesian -> real spherical transformation blocks (libcint convention).

For l >= 2 a spherical AO is r^l Y_lm(theta, phi) times the radial part,
with Y_lm the orthonormal real spherical harmonics without the
Condon-Shortley phase (m > 0: cos(m phi), m < 0: sin(|m| phi), ordered
m = -l .. l).  libcint's l >= 2 Cartesian functions are the bare monomials
x^a y^b z^c (times the radial part), so the block holds the monomial
coefficients of r^l Y_lm.  For l = 0, 1 libcint folds the angular constant
into the Cartesian functions themselves and orders p as (x, y, z), so those
blocks are identities.

Coefficients from the closed form of the real solid harmonics
(T. Helgaker, P. Jorgensen, J. Olsen, Molecular Electronic-Structure Theory,
Wiley 2000, eqs. 6.4.47-6.4.50), which gives S_lm = sqrt(4 pi/(2l+1)) r^l Y_lm.
"""
from fractions import Fraction
from functools import lru_cache
from math import comb, factorial, pi, sqrt

import numpy as np


def cart_components(l):
    return [(a, b, l - a - b) for a in range(l, -1, -1) for b in range(l - a, -1, -1)]


@lru_cache(maxsize=None)
def cart2sph_block(l):
    """(ncart, 2l+1) array C with sph_m = sum_c C[c, m] * cart_c."""
    if l < 2:
        return np.eye((l + 1) * (l + 2) // 2)
    comps = cart_components(l)
    index = {c: i for i, c in enumerate(comps)}
    C = np.zeros((len(comps), 2 * l + 1))
    for col, m in enumerate(range(-l, l + 1)):
        am = abs(m)
        nlm = sqrt(2.0 * factorial(l + am) * factorial(l - am) / (2.0 if m == 0 else 1.0)) \
            / (2 ** am * factorial(l))
        vm2 = 0 if m >= 0 else 1          # 2 v_m
        terms = {}
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                # v runs over v_m, v_m + 1, ..., floor(|m|/2 - v_m) + v_m ; use 2v
                v2 = vm2
                while v2 <= 2 * ((am - vm2) // 2) + vm2 and v2 <= am:
                    sign = (-1) ** (t + (v2 - vm2) // 2)
                    c = Fraction(sign, 4 ** t) * comb(l, t) * comb(l - t, am + t) \
                        * comb(t, u) * comb(am, v2)
                    px = 2 * t + am - 2 * u - v2
                    py = 2 * u + v2
                    pz = l - 2 * t - am
                    key = (px, py, pz)
                    terms[key] = terms.get(key, 0) + c
                    v2 += 2
        norm = nlm * sqrt((2 * l + 1) / (4 * pi))
        for key, c in terms.items():
            if c != 0:
                C[index[key], col] = float(c) * norm
    return C
