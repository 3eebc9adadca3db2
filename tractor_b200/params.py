"""Parameter containers with the semantics of the reference Tractor's Params
duck type (tractor/utils.py:195-1270): thawed ("liquid") / frozen parameters,
flat getParams / setParams over thawed values, step sizes, bounds, maximum
steps, Gaussian priors and their least-squares rows.

Only the behaviour the forward-model path relies on is provided, with the same
names and argument meanings, so code written against the reference's
ParamList / MultiParams runs unchanged.
"""
import numpy as np


def _class_name(obj):
    name = getattr(obj.__class__, 'classname', None)
    return name if name is not None else obj.__class__.__name__


def _isint(i):
    try:
        return int(i) == i
    except Exception:
        return False


class BaseParams(object):
    """tractor/utils.py:195-330."""

    def __repr__(self):
        return _class_name(self) + repr(self.getParams())

    def __str__(self):
        return _class_name(self) + ': ' + str(self.getParams())

    def copy(self):
        return self.__class__(*self.getAllParams())

    def hashkey(self):
        return (_class_name(self),) + tuple(self.getAllParams())

    @classmethod
    def fromFitsHeader(clazz, hdr, prefix=''):
        """ImageCalibration.fromFitsHeader (ducks.py:170-178): the
        constructor's arguments from cards <prefix>A0, A1, ...; where a header
        has none, from the <prefix>P0, P1, ... cards that the default
        toFitsHeader (ducks.py:163-168) writes, so that images written by
        Image.toFits read back."""
        for key in ('A', 'P'):
            args = []
            for i in range(100):
                k = prefix + key + '%i' % i
                if k not in hdr:
                    break
                args.append(hdr.get(k))
            if args:
                return clazz(*args)
        return clazz()

    def getParamNames(self):
        return []

    def numberOfParams(self):
        return len(self.getParams())

    def getParams(self):
        return []

    def getAllParams(self):
        return self.getParams()

    def getAllStepSizes(self, *args, **kwargs):
        return self.getStepSizes(*args, **kwargs)

    def getStepSizes(self, *args, **kwargs):
        ss = getattr(self, 'stepsizes', None)
        if ss is not None:
            return ss
        return [1.] * self.numberOfParams()

    def setStepSizes(self, ss):
        self.stepsizes = ss

    def setAllStepSizes(self, ss):
        self.setStepSizes(ss)

    def setParams(self, p):
        assert len(p) == self.numberOfParams()
        for i, v in enumerate(p):
            self.setParam(i, v)

    def setAllParams(self, p):
        return self.setParams(p)

    def setParam(self, i, p):
        P = self.getParams()
        old = P[i]
        P[i] = p
        return old

    def getLogPrior(self):
        return 0.

    def getLogPriorDerivatives(self):
        return None

    def getLowerBounds(self):
        return []

    def getUpperBounds(self):
        return []

    def getMaxStep(self):
        return []

    def getGaussianPriors(self):
        return []

    def isLegal(self):
        return True


class ScalarParam(BaseParams):
    """A single float parameter in self.val (tractor/utils.py:332-420)."""
    stepsize = 1.
    strformat = '%g'

    def __init__(self, val=0):
        self.val = val
        self.lower = None
        self.upper = None
        self.maxstep = None

    def __str__(self):
        return _class_name(self) + ': ' + self.strformat % self.val

    def __repr__(self):
        return _class_name(self) + '(' + repr(self.val) + ')'

    def __eq__(self, other):
        return self.getValue() == other.getValue()

    def __lt__(self, other):
        return self.getValue() < other.getValue()

    __hash__ = object.__hash__

    def copy(self):
        return self.__class__(self.val)

    def getParamNames(self):
        return [_class_name(self)]

    def numberOfParams(self):
        return 1

    def getStepSizes(self, *args, **kwargs):
        return [self.stepsize]

    def setStepSizes(self, ss):
        self.stepsize = ss[0]

    def getParams(self):
        return [self.val]

    def getAllParams(self):
        return [self.val]

    def setParams(self, p):
        assert len(p) == 1
        self._set(p[0])

    def setAllParams(self, p):
        self.setParams(p)

    def setParam(self, i, p):
        assert i == 0
        old = self.val
        self._set(p)
        return old

    def _set(self, val):
        self.val = val

    def getValue(self):
        return self.val

    def setValue(self, v):
        self._set(v)

    def getLowerBounds(self):
        return [self.lower]

    def getUpperBounds(self):
        return [self.upper]

    def getMaxStep(self):
        return [self.maxstep]


class NamedParams(object):
    """Named, freezable parameters (tractor/utils.py:429-706)."""

    @staticmethod
    def getNamedParams():
        return {}

    def __new__(cls, *args, **kwargs):
        self = super(NamedParams, cls).__new__(cls)
        self.namedparams = {}
        self.paramnames = {}
        self.addNamedParams(**self.getNamedParams())
        return self

    def __init__(self):
        super(NamedParams, self).__init__()
        self.liquid = [True] * self._numberOfThings()

    def addNamedParams(self, **d):
        self._addNamedParams(False, **d)

    def addParamAliases(self, **d):
        self._addNamedParams(True, **d)

    def _addNamedParams(self, alias, **d):
        self.namedparams.update(d)
        if not alias:
            self.paramnames.update(dict((v, k) for k, v in d.items()))
        for n in self.namedparams:
            if hasattr(self.__class__, n):
                continue

            def getter(x, nm=n):
                return x._getThing(x.namedparams[nm])

            def setter(x, v, nm=n):
                return x._setThing(x.namedparams[nm], v)
            setattr(self.__class__, n, property(getter, setter, None, 'named param %s' % n))

    def getNamedParamIndex(self, name):
        return self.namedparams.get(name, None)

    def getNamedParamName(self, i):
        return self.paramnames.get(i, None)

    def _iterNamesAndVals(self):
        for i, val in enumerate(self._getThings()):
            yield (self.paramnames.get(i, None), val)

    def getStepSizes(self, *args, **kwargs):
        ss = getattr(self, 'stepsizes', None)
        if ss is None:
            ss = self.getAllStepSizes(*args, **kwargs)
        return list(self._getLiquidArray(ss))

    def getAllStepSizes(self, *args, **kwargs):
        ss = getattr(self, 'stepsizes', None)
        if ss is not None:
            return ss
        return [1.] * len(self.getAllParams())

    def setStepSizes(self, ss):
        if getattr(self, 'stepsizes', None) is None:
            it = iter(ss)
            self.stepsizes = [next(it) if l else 1. for l in self.liquid]
        else:
            for (i, _), s in zip(self._enumerateLiquidArray(self.stepsizes), ss):
                self.stepsizes[i] = s

    def setAllStepSizes(self, ss):
        self.stepsizes = ss

    # freeze / thaw
    def _index(self, name):
        if _isint(name):
            return name
        i = self.getNamedParamIndex(name)
        assert i is not None, name
        return i

    def freezeParam(self, name):
        self.liquid[self._index(name)] = False

    def freezeParams(self, *names):
        for n in names:
            self.freezeParam(n)

    def thawParam(self, name):
        if not _isint(name) and not isinstance(name, str):
            self.liquid[self._getThings().index(name)] = True
            return
        self.liquid[self._index(name)] = True

    def thawParams(self, *names):
        for n in names:
            self.thawParam(n)

    unfreezeParam = thawParam
    unfreezeParams = thawParams

    def freezeAllParams(self):
        self.liquid[:] = [False] * len(self.liquid)

    def thawAllParams(self):
        self.liquid[:] = [True] * len(self.liquid)

    unfreezeAllParams = thawAllParams

    def freezeAllBut(self, *names):
        self.freezeAllParams()
        self.thawParams(*names)

    def freezeParamsRecursive(self, *names):
        for nm in names:
            i = self.getNamedParamIndex(nm)
            if i is not None:
                self.liquid[i] = False
        if '*' in names:
            self.freezeAllParams()

    def thawParamsRecursive(self, *names):
        for nm in names:
            i = self.getNamedParamIndex(nm)
            if i is not None:
                self.liquid[i] = True
        if '*' in names:
            self.thawAllParams()

    def thawPathsTo(self, *names):
        thawed = False
        for nm in names:
            i = self.getNamedParamIndex(nm)
            if i is not None:
                self.liquid[i] = True
                thawed = True
        return thawed

    def isParamFrozen(self, name):
        return not self.liquid[self._index(name)]

    def isParamThawed(self, name):
        return self.liquid[self._index(name)]

    def getFrozenParamIndices(self):
        return (i for i, v in enumerate(self.liquid) if not v)

    def getThawedParamIndices(self):
        return (i for i, v in enumerate(self.liquid) if v)

    def getThawedParamIndicesAndNames(self):
        return ((i, self.getNamedParamName(i)) for i, v in enumerate(self.liquid) if v)

    def getFrozenParams(self):
        return [self.getNamedParamName(i) for i in self.getFrozenParamIndices()]

    def getThawedParams(self):
        return [self.getNamedParamName(i) for i in self.getThawedParamIndices()]

    def getLiquidIndexOfIndex(self, i):
        if not self.liquid[i]:
            return -1
        return sum(self.liquid[:i])

    def getLiquidIndex(self, name):
        i = self.getNamedParamIndex(name)
        if i is None:
            raise KeyError('No such parameter "%s"' % name)
        return self.getLiquidIndexOfIndex(i)

    def _enumerateLiquidArray(self, array):
        return ((i, array[i]) for i, v in enumerate(self.liquid) if v)

    def _getLiquidArray(self, array):
        return (a for v, a in zip(self.liquid, array) if v)

    def _getFrozenArray(self, array):
        return (a for v, a in zip(self.liquid, array) if not v)

    def _countLiquid(self):
        return sum(self.liquid)

    def _indexLiquid(self, j):
        for i, v in enumerate(self.liquid):
            if v:
                if j == 0:
                    return i
                j -= 1
        raise IndexError(j)

    def _indexBoth(self):
        i = 0
        for j, v in enumerate(self.liquid):
            if v:
                yield (i, j)
                i += 1


class GaussianPriors(object):
    """Gaussian prior terms on named parameters (tractor/utils.py:65-133)."""

    def __init__(self, param):
        self.terms = []
        self.param = param

    def add(self, name, mu, sigma, param=None):
        param = param if param is not None else self.param
        i = param.getNamedParamIndex(name)
        if i is None:
            raise KeyError('GaussianPriors.add: parameter not found: "%s"' % name)
        self.terms.append((name, i, mu, sigma))

    def getLogPrior(self, param=None):
        param = param if param is not None else self.param
        p = param.getAllParams()
        return -0.5 * sum((p[i] - mu) ** 2 / sigma ** 2 for _, i, mu, sigma in self.terms)

    def getGaussianPriors(self):
        return [(i, mu, sigma) for _, i, mu, sigma in self.terms]

    def getDerivs(self, param=None):
        """Least-squares rows (rows, cols, vals, b, mu) of the priors on the
        thawed parameters (tractor/utils.py:104-133)."""
        param = param if param is not None else self.param
        rows, cols, vals, bs, mus = [], [], [], [], []
        p = param.getParams()
        r0 = 0
        for _, j, mu, sigma in self.terms:
            i = param.getLiquidIndexOfIndex(j)
            if i == -1:
                continue
            cols.append(i)
            vals.append([1. / sigma])
            rows.append([r0])
            bs.append([-(p[i] - mu) / sigma])
            mus.append([mu])
            r0 += 1
        return rows, cols, vals, bs, mus


class GaussianPriorsMixin(object):
    """tractor/utils.py:136-192."""

    def __init__(self, *args, **kwargs):
        super(GaussianPriorsMixin, self).__init__(*args, **kwargs)
        self.gpriors = GaussianPriors(self)

    def addGaussianPrior(self, name, mu, sigma):
        self.gpriors.add(name, mu, sigma, param=self)

    def getLogPriorDerivatives(self):
        return self.gpriors.getDerivs(param=self)

    def getGaussianPriors(self):
        return self.gpriors.getGaussianPriors()

    def isLegal(self):
        return True

    def getLogPrior(self):
        if not self.isLegal():
            return -np.inf
        return self.gpriors.getLogPrior(param=self)


class ParamList(GaussianPriorsMixin, NamedParams, BaseParams):
    """Parameters held in a list (tractor/utils.py:708-830)."""

    def __init__(self, *args):
        self.vals = list(args)
        self.lowers = [None] * len(self.vals)
        self.uppers = [None] * len(self.vals)
        self.maxstep = [None] * len(self.vals)
        super(ParamList, self).__init__()

    def copy(self):
        c = self.__class__(*self.getAllParams())
        c.liquid = list(self.liquid)
        return c

    def getFormatString(self, i):
        return '%g'

    def __str__(self):
        ss = []
        for i, (name, val) in enumerate(self._iterNamesAndVals()):
            fmt = self.getFormatString(i)
            ss.append(('%s=' + fmt) % (name, val) if name is not None else fmt % val)
        return _class_name(self) + ': ' + ', '.join(ss)

    def getParamNames(self):
        return [self.getNamedParamName(j) or 'param%i' % i for i, j in self._indexBoth()]

    def _setThing(self, i, val):
        self.vals[i] = val

    def _getThing(self, i):
        return self.vals[i]

    def _getThings(self):
        return self.vals

    def _numberOfThings(self):
        return len(self.vals)

    def setParam(self, i, val):
        ii = self._indexLiquid(i)
        old = self._getThing(ii)
        self._setThing(ii, val)
        return old

    def setParams(self, p):
        for i, j in self._indexBoth():
            self._setThing(j, p[i])

    def numberOfParams(self):
        return self._countLiquid()

    def getParams(self):
        return list(self._getLiquidArray(self._getThings()))

    def getAllParams(self):
        return list(self._getThings())

    def getParam(self, i):
        return self._getThing(self._indexLiquid(i))

    def setAllParams(self, p):
        for i, v in enumerate(p):
            self._setThing(i, v)

    def getLowerBounds(self):
        return list(self._getLiquidArray(self.lowers))

    def getUpperBounds(self):
        return list(self._getLiquidArray(self.uppers))

    def getMaxStep(self):
        return list(self._getLiquidArray(self.maxstep))

    def __len__(self):
        return self.numberOfParams()

    def __getitem__(self, i):
        return self.getParam(i)

    def __iter__(self):
        return iter(self.getParams())


def _listmax(X, default=0):
    mx = [np.max(x) for x in X if len(x)]
    return np.max(mx) if len(mx) else default


class MultiParams(BaseParams, NamedParams):
    """A container of sub-Params (tractor/utils.py:990-1270)."""

    def __init__(self, *args):
        self.subs = list(args)
        super(MultiParams, self).__init__()

    def copy(self):
        x = self.__class__(*[s.copy() for s in self.subs])
        x.liquid = list(self.liquid)
        return x

    def append(self, x):
        self.subs.append(x)
        self.liquid.append(True)

    def extend(self, xs):
        self.subs.extend(xs)
        self.liquid.extend([True] * len(xs))

    def remove(self, x):
        i = self.subs.index(x)
        del self.subs[i]
        del self.liquid[i]

    def index(self, x):
        return self.subs.index(x)

    def __len__(self):
        return len(self.subs)

    def __getitem__(self, k):
        return self.subs[k]

    def __setitem__(self, k, v):
        self.subs[k] = v

    def __iter__(self):
        return iter(self.subs)

    def hashkey(self):
        return tuple([_class_name(self)] + [None if s is None else s.hashkey() for s in self.subs])

    def __str__(self):
        s = []
        for n, v in self._iterNamesAndVals():
            s.append(str(v) if n is None else '%s: %s' % (n, v))
        return _class_name(self) + ': ' + ', '.join(s)

    def _setThing(self, i, val):
        self.subs[i] = val

    def _getThing(self, i):
        return self.subs[i]

    def _getThings(self):
        return self.subs

    def _numberOfThings(self):
        return len(self.subs)

    def _getActiveSubs(self):
        return (s for s in self._getLiquidArray(self.subs) if s is not None)

    def _enumerateActiveSubs(self):
        return ((i, s) for i, s in self._enumerateLiquidArray(self.subs) if s is not None)

    def freezeParamsRecursive(self, *names):
        for name, sub in self._iterNamesAndVals():
            if hasattr(sub, 'freezeParamsRecursive'):
                sub.freezeParamsRecursive(*names)
            if name in names:
                self.freezeParam(name)
        if '*' in names:
            self.freezeAllParams()

    def freezeAllRecursive(self):
        self.freezeParamsRecursive('*')

    def thawParamsRecursive(self, *names):
        for name, sub in self._iterNamesAndVals():
            if hasattr(sub, 'thawParamsRecursive'):
                sub.thawParamsRecursive(*names)
            if name in names:
                self.thawParam(name)
        if '*' in names:
            self.thawAllParams()

    def thawAllRecursive(self):
        self.thawParamsRecursive('*')

    def thawPathsTo(self, *names):
        thawed = False
        for i, (name, sub) in enumerate(self._iterNamesAndVals()):
            if hasattr(sub, 'thawPathsTo') and sub.thawPathsTo(*names):
                self.thawParam(i)
                thawed = True
            if name in names:
                self.thawParam(i)
                thawed = True
        return thawed

    def printThawedParams(self):
        for nm, val in zip(self.getParamNames(), self.getParams()):
            print('  ', nm, '=', val)

    def getParamNames(self):
        n = []
        for i, s in self._enumerateLiquidArray(self.subs):
            if s is None:
                continue
            pre = self.getNamedParamName(i) or 'param%i' % i
            sn = s.getParamNames()
            if sn is not None and len(sn) == s.numberOfParams():
                n.extend('%s.%s' % (pre, p) for p in sn)
            else:
                n.extend('%s.param%i' % (pre, k) for k in range(s.numberOfParams()))
        return n

    def numberOfParams(self):
        return sum(s.numberOfParams() for s in self._getActiveSubs())

    def getParams(self):
        p = []
        for s in self._getActiveSubs():
            pp = s.getParams()
            if pp is not None:
                p.extend(pp)
        return p

    def getAllParams(self):
        p = []
        for s in self.subs:
            if s is not None:
                p.extend(s.getAllParams())
        return p

    def setAllParams(self, p):
        i = 0
        for s in self.subs:
            if s is None:
                continue
            n = len(s.getAllParams())
            s.setAllParams(p[i:i + n])
            i += n

    def setParams(self, p):
        i = 0
        for s in self._getActiveSubs():
            n = s.numberOfParams()
            s.setParams(p[i:i + n])
            i += n

    def setParam(self, i, p):
        off = 0
        for s in self._getActiveSubs():
            n = s.numberOfParams()
            if i < off + n:
                return s.setParam(i - off, p)
            off += n
        raise RuntimeError('setParam(%i,...) for a %s that only has %i elements' %
                           (i, _class_name(self), self.numberOfParams()))

    def getLowerBounds(self):
        return [b for s in self._getActiveSubs() for b in s.getLowerBounds()]

    def getUpperBounds(self):
        return [b for s in self._getActiveSubs() for b in s.getUpperBounds()]

    def getMaxStep(self):
        return [b for s in self._getActiveSubs() for b in s.getMaxStep()]

    def getGaussianPriors(self):
        p = []
        off = 0
        for s in self._getActiveSubs():
            p.extend((off + i, mu, sig) for i, mu, sig in s.getGaussianPriors())
            off += s.numberOfParams()
        return p

    def getStepSizes(self, *args, **kwargs):
        return [x for s in self._getActiveSubs() for x in s.getStepSizes(*args, **kwargs)]

    def getAllStepSizes(self, *args, **kwargs):
        return [x for s in self.subs for x in s.getAllStepSizes(*args, **kwargs)]

    def setStepSizes(self, ss):
        off = 0
        for s in self._getActiveSubs():
            n = s.numberOfParams()
            s.setStepSizes(ss[off:off + n])
            off += n

    def getLogPrior(self):
        return sum(s.getLogPrior() for s in self._getActiveSubs())

    def isLegal(self):
        return all(s.isLegal() for s in self._getActiveSubs())

    def getLogPriorDerivatives(self):
        """Prior rows for least squares, stacked over active subs
        (tractor/utils.py:1243-1270)."""
        rA, cA, vA, pb, mub = [], [], [], [], []
        r0 = c0 = 0
        for s in self._getActiveSubs():
            X = s.getLogPriorDerivatives()
            if X is None:
                c0 += s.numberOfParams()
                continue
            r, c, v, b, m = X
            rA.extend([[rij + r0 for rij in ri] for ri in r])
            cA.extend([ci + c0 for ci in c])
            vA.extend(v)
            pb.extend(b)
            mub.extend(m)
            c0 += s.numberOfParams()
            r0 += _listmax(r, -1) + 1
        if rA == []:
            return None
        return rA, cA, vA, pb, mub
