"""Mixture-of-Gaussians profiles: the MixtureOfGaussians container
(tractor/mixture_profiles.py:47-172), the exp / deV tables and the Sersic
mixtures (tractor/sersic.py:25-342).

The numeric tables are in data/profile_tables.json (regenerated from the
reference by data/make_profile_tables.py).  Sersic amplitudes and
log-variances are cubic (or linear) interpolating splines in the Sersic
index; the tables store each spline's knots and B-spline coefficients, which
this module evaluates with de Boor's recursion (no scipy at run time).
"""
import functools
import json
import os

import numpy as np

_TABLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data', 'profile_tables.json')


@functools.lru_cache(maxsize=1)
def tables():
    with open(_TABLES) as f:
        return json.load(f)


class MixtureOfGaussians(object):
    """amp (K,), mean (K, 2), var (K, 2, 2) (mixture_profiles.py:47-129)."""

    def __init__(self, amp, mean, var, quick=False):
        if quick:
            self.amp, self.mean, self.var = amp, mean, var
            self.K, self.D = self.mean.shape
            return
        self.amp = np.atleast_1d(amp).astype(float)
        self.mean = np.atleast_2d(np.array(mean)).astype(float)
        self.K, self.D = self.mean.shape
        var = np.asarray(var)
        if var.size == self.K:
            self.var = np.zeros((self.K, self.D, self.D))
            for d in range(self.D):
                self.var[:, d, d] = var
        else:
            self.var = np.array(var).astype(float)
        for i in range(self.D):
            for j in range(i):
                t = 0.5 * (self.var[:, i, j] + self.var[:, j, i])
                self.var[:, i, j] = t
                self.var[:, j, i] = t

    def copy(self):
        return MixtureOfGaussians(self.amp, self.mean, self.var, quick=True)

    def normalize(self):
        self.amp /= np.sum(self.amp)

    def __add__(self, other):
        """Concatenation, renormalised (mixture_profiles.py:114-129)."""
        s = MixtureOfGaussians(np.append(self.amp, other.amp),
                               np.append(self.mean, other.mean, axis=0),
                               np.append(self.var, other.var, axis=0), quick=True)
        s.normalize()
        return s

    def apply_affine(self, shift, scale):
        """mean + shift, var -> T V T^T (mixture_profiles.py:131-144)."""
        return MixtureOfGaussians(self.amp, self.mean + shift, scale @ self.var @ scale.T, quick=True)

    def apply_shear(self, scale):
        """var -> T V T^T (mixture_profiles.py:146-155)."""
        return MixtureOfGaussians(self.amp, self.mean, scale @ self.var @ scale.T, quick=True)

    def convolve(self, other):
        """All pairs, PSF component outermost (mixture_profiles.py:158-172)."""
        K, P = self.K, other.K
        amp = (self.amp[np.newaxis, :] * other.amp[:, np.newaxis]).ravel()
        mean = (self.mean[np.newaxis, :, :] + other.mean[:, np.newaxis, :]).reshape(K * P, 2)
        var = (self.var[np.newaxis] + other.var[:, np.newaxis]).reshape(K * P, 2, 2)
        return MixtureOfGaussians(amp, mean, var, quick=True)


def _mog(amp, var):
    return MixtureOfGaussians(np.array(amp), np.zeros((len(amp), 2)), np.array(var))


@functools.lru_cache(maxsize=1)
def exp_mixture():
    t = tables()['exp']
    m = _mog(t['amp'], t['var'])
    m.normalize()
    return m


@functools.lru_cache(maxsize=1)
def dev_mixture():
    t = tables()['dev']
    m = _mog(t['amp'], t['var'])
    m.normalize()
    return m


def get_exp_mixture():
    """A new copy of the exp profile's mixture (mixture_profiles.py:41-42)."""
    m = exp_mixture()
    return MixtureOfGaussians(m.amp.copy(), m.mean.copy(), m.var.copy())


def get_dev_mixture():
    """A new copy of the deV profile's mixture (mixture_profiles.py:44-45)."""
    m = dev_mixture()
    return MixtureOfGaussians(m.amp.copy(), m.mean.copy(), m.var.copy())


def gaussian_mixture():
    m = MixtureOfGaussians(np.array([1.]), np.zeros((1, 2)), np.array([[[1., 0.], [0., 1.]]]))
    m.normalize()
    return m


# ---------------------------------------------------------------------------
# B-spline evaluation (knots t, coefficients c, degree k), de Boor recursion.
# ---------------------------------------------------------------------------

def bspline_eval(t, c, k, x):
    """Value of the spline sum_i c_i B_{i,k}(x) for x inside its base
    interval [t[k], t[n]] (n = len(t) - k - 1); the right end is closed."""
    t = np.asarray(t, np.float64)
    c = np.asarray(c, np.float64)
    n = len(t) - k - 1
    x = float(x)
    # knot span l with t[l] <= x < t[l+1], k <= l < n
    l = int(np.searchsorted(t, x, side='right')) - 1
    l = min(max(l, k), n - 1)
    d = [c[j + l - k] for j in range(k + 1)]
    for r in range(1, k + 1):
        for j in range(k, r - 1, -1):
            i = j + l - k
            den = t[i + k + 1 - r] - t[i]
            alpha = 0.0 if den == 0 else (x - t[i]) / den
            d[j] = (1.0 - alpha) * d[j - 1] + alpha * d[j]
    return d[k]


class SersicMixture(object):
    """The Sersic-index-dependent mixture (tractor/sersic.py:25-342): pick the
    index range, interpolate amplitudes and log-variances, normalise, add the
    delta core for n > 1 and sort by variance."""

    def __init__(self):
        S = tables()['sersic']
        self.ranges = S['ranges']
        self.core = S['core_spline']
        self.lowest = S['lowest']
        self.highest = S['highest']

    @functools.lru_cache(maxsize=4096)
    def profile(self, sindex):
        """(amp (K,), var (K,)) for Sersic index `sindex`."""
        n = float(sindex)
        if n <= self.lowest:
            r = self.ranges[0]
            n = self.lowest
        elif n >= self.highest:
            r = self.ranges[-1]
            n = self.highest
        else:
            r = [g for g in self.ranges if g['lo'] <= n < g['hi']]
            assert len(r) == 1
            r = r[0]
        amps = np.array([bspline_eval(s['t'], s['c'], s['k'], n) for s in r['amp_splines']])
        amps /= amps.sum()
        varr = np.exp(np.array([bspline_eval(s['t'], s['c'], s['k'], n)
                                for s in r['logvar_splines']]))
        if n > 1.:
            core = bspline_eval(self.core['t'], self.core['c'], self.core['k'], n)
            amps *= (1. - core) / amps.sum()
            amps = np.append(amps, core)
            varr = np.append(varr, 0.)
        I = np.argsort(varr)
        return amps[I], varr[I]

    def getProfile(self, sindex):
        amp, var = self.profile(float(sindex))
        return MixtureOfGaussians(amp.copy(), np.zeros((len(amp), 2)), var.copy())


_sersic = None


def sersic_mixture():
    global _sersic
    if _sersic is None:
        _sersic = SersicMixture()
    return _sersic
