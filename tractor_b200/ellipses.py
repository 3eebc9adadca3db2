"""Galaxy shape parameterisations (tractor/galaxy.py:37-89,
tractor/ellipses.py:1-263): each gives getRaDecBasis(), the matrix taking
unit vectors in r_e to (RA, Dec) degrees."""
import math

import numpy as np

from .params import ParamList


class GalaxyShape(ParamList):
    """(re [arcsec], ab, phi [deg]) (tractor/galaxy.py:37-89)."""

    @staticmethod
    def getName():
        return 'Galaxy Shape'

    @staticmethod
    def getNamedParams():
        return dict(re=0, ab=1, phi=2)

    def __repr__(self):
        return 're=%g, ab=%g, phi=%g' % (self.re, self.ab, self.phi)

    def __str__(self):
        return '%s: re=%.2f, ab=%.2f, phi=%.1f' % (self.getName(), self.re, self.ab, self.phi)

    def getRaDecBasis(self):
        phi = np.deg2rad(90 - self.phi)
        re_deg = max(1. / 30, self.re) / 3600.
        cp, sp = np.cos(phi), np.sin(phi)
        return re_deg * np.array([[cp, sp * self.ab], [-sp, cp * self.ab]])

    def getTensor(self, cd):
        return np.dot(np.linalg.inv(self.getRaDecBasis()), cd)


class EllipseE(ParamList):
    """(re, e1, e2) (tractor/ellipses.py:13-155): step 0.01 with the sign of
    the e1 / e2 steps chosen away from the |e| = 1 boundary; bounds re >= 0,
    |e_i| <= 1; max steps (1, 0.1, 0.1)."""

    @staticmethod
    def getName():
        return 'EllipseE'

    @staticmethod
    def getNamedParams():
        return dict(re=0, e1=1, e2=2)

    def __init__(self, *args, **kwargs):
        super(EllipseE, self).__init__(*args, **kwargs)
        self.stepsizes = [0.01] * 3
        self.lowers = [0., -1., -1.]
        self.uppers = [None, 1., 1.]
        self.maxstep = [1., 0.1, 0.1]

    @staticmethod
    def fromEllipseESoft(esoft, maxe=0.999999):
        e = min(maxe, esoft.e)
        theta = esoft.theta
        return EllipseE(esoft.re, e * math.cos(2. * theta), e * math.sin(2. * theta))

    @staticmethod
    def fromRAbPhi(r, ba, phi):
        ab = 1. / ba
        e = (ab - 1) / (ab + 1)
        angle = math.radians(2. * (-phi))
        return EllipseE(r, e * math.cos(angle), e * math.sin(angle))

    @staticmethod
    def fromCovariance(cov):
        u, s, v = np.linalg.svd(cov)
        r = math.sqrt(s[0])
        ab = math.sqrt(s[1] / s[0])
        theta = math.degrees(math.atan2(u[0, 0], u[0, 1]))
        return EllipseE.fromRAbPhi(r, ab, -theta)

    @property
    def e(self):
        return math.hypot(self.e1, self.e2)

    @property
    def theta(self):
        return math.atan2(self.e2, self.e1) / 2.

    @property
    def ab(self):
        e = self.e
        return (1. - e) / (1. + e)

    def __repr__(self):
        return 're=%g, e1=%g, e2=%g' % (self.re, self.e1, self.e2)

    def __str__(self):
        return self.getName() + ': ' + repr(self)

    def getAllStepSizes(self, *args, **kwargs):
        # Note: getStepSizes() returns the stored `stepsizes` ([0.01] * 3) and
        # never reaches this sign-flipping variant, as in the reference.
        return [0.01, 0.01 if self.e1 <= 0 else -0.01, 0.01 if self.e2 <= 0 else -0.01]

    def isLegal(self):
        return (self.e1 ** 2 + self.e2 ** 2) < 1. and self.re >= 0.

    def toEllipseE(self, **kwargs):
        return self.copy()

    def getCovariance(self):
        G = self.getRaDecBasis() * 3600.
        return G @ G.T

    def getRaDecBasis(self):
        theta = self.theta
        ct, st = math.cos(theta), math.sin(theta)
        e = self.e
        maxab = 1000.
        ab = maxab if e >= 1. else min(maxab, (1. + e) / (1. - e))
        r_deg = self.re / 3600.
        return r_deg * np.array([[ct / ab, st], [-st / ab, ct]])

    def getTensor(self, cd):
        return np.dot(np.linalg.inv(self.getRaDecBasis()), cd)


class EllipseESoft(EllipseE):
    """(log re, ee1, ee2) with e = 1 - exp(-|ee|) (tractor/ellipses.py:165-263)."""

    @staticmethod
    def getName():
        return 'EllipseESoft'

    @staticmethod
    def getNamedParams():
        return dict(logre=0, ee1=1, ee2=2)

    def __init__(self, *args, **kwargs):
        super(EllipseESoft, self).__init__(*args, **kwargs)
        self.lowers = [None, None, None]
        self.uppers = [None, None, None]

    @staticmethod
    def fromEllipseE(ell, maxe=0.999999):
        e = min(ell.e, maxe)
        esoft = -math.log(1. - e)
        return EllipseESoft(math.log(ell.re), ell.e1 / e * esoft, ell.e2 / e * esoft)

    @staticmethod
    def fromRAbPhi(r, ba, phi):
        return EllipseESoft(*EllipseESoft.rAbPhiToESoft(r, ba, phi))

    @staticmethod
    def rAbPhiToESoft(r, ba, phi):
        ab = 1. / ba
        e = (ab - 1) / (ab + 1)
        ee = -math.log(1 - e)
        angle = math.radians(2. * (-phi))
        return (math.log(r), ee * math.cos(angle), ee * math.sin(angle))

    def __repr__(self):
        return 'log r_e=%.3f, ee1=%.3f, ee2=%.3f' % (self.logre, self.ee1, self.ee2)

    @property
    def re(self):
        return math.exp(self.logre)

    @property
    def e(self):
        return 1. - math.exp(-math.hypot(self.ee1, self.ee2))

    @property
    def softe(self):
        return math.hypot(self.ee1, self.ee2)

    @property
    def theta(self):
        return math.atan2(self.ee2, self.ee1) / 2.

    def getAllStepSizes(self, *args, **kwargs):
        # The reference inherits EllipseE's version, which reads e1 / e2 and
        # raises AttributeError here; the stored step sizes are returned instead.
        return list(self.stepsizes)

    def isLegal(self):
        return True

    def toEllipseE(self, maxe=0.999999):
        return EllipseE.fromEllipseESoft(self, maxe=maxe)

    def getRaDecBasis(self):
        return self.toEllipseE().getRaDecBasis()
