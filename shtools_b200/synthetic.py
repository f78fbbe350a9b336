"""Seeded synthetic spherical-harmonic fields.

The recipe of the reference's timing and accuracy examples
(examples/python/TimingAccuracy/TimingAccuracyDH.py:16-74) with a numpy
Generator in place of the global seed: Gaussian coefficients whose degree
power is S(l) = (l+1)^-beta, each with standard deviation sqrt(S(l)/(2l+1)).
"""
import numpy as np


def power_law_cilm(lmax, seed, beta=2.0):
    """Real coefficients (2, lmax+1, lmax+1); m > l and the m = 0 sine terms
    are zero."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((2, lmax + 1, lmax + 1))
    l = np.arange(lmax + 1)
    c *= np.sqrt((l + 1.0) ** (-beta) / (2 * l + 1.0))[None, :, None]
    mask = l[None, :, None] >= l[None, None, :]
    c = np.where(mask, c, 0.0)
    c[1, :, 0] = 0.0
    return c


def power_law_cilm_complex(lmax, seed, beta=2.0):
    """Complex coefficients (2, lmax+1, lmax+1) of the same per-degree power
    (orders +m and -m); cilm[1, :, 0] is zero."""
    rng = np.random.default_rng(seed)
    shape = (2, lmax + 1, lmax + 1)
    c = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    l = np.arange(lmax + 1)
    c *= np.sqrt((l + 1.0) ** -beta / (2 * (2 * l + 1.0)))[None, :, None]
    c = np.where(l[:, None] >= l[None, :], c, 0.0)
    c[1, :, 0] = 0.0
    return c
