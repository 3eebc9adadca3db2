"""Regenerate profile_tables.json from the reference Tractor's source tree.

The galaxy profiles are fixed mixture-of-Gaussians tables that any
implementation must share to render the same galaxies: the exp (6 component)
and deV (8 component + delta core) amplitudes and variances in
tractor/mixture_profiles.py:20-38, and the Sersic fit grid and core-flux table
in tractor/sersic.py:40-243.  This script reads those literals with `ast`
(nothing is executed), applies the same normalisations the reference applies at
import time, and also stores, for every Sersic spline, the knots and B-spline
coefficients that scipy's InterpolatedUnivariateSpline builds from the grid
(tractor/sersic.py:242-282), so that the profile kernel can evaluate the same
splines without scipy.

Usage: python tractor_b200/data/make_profile_tables.py [REFERENCE_ROOT]
"""
import ast
import json
import os
import sys

import numpy as np


def _find_assign(tree, target_src):
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            if ast.unparse(node.targets[0]) == target_src:
                return ast.literal_eval(node.value)
    raise KeyError(target_src)


def main(ref_root):
    mp_src = open(os.path.join(ref_root, 'tractor', 'mixture_profiles.py')).read()
    se_src = open(os.path.join(ref_root, 'tractor', 'sersic.py')).read()
    mp_tree = ast.parse(mp_src)
    se_tree = ast.parse(se_src)

    def arr(name):
        for node in ast.walk(mp_tree):
            if isinstance(node, ast.Assign) and ast.unparse(node.targets[0]) == name:
                call = node.value
                if isinstance(call, ast.Call):
                    return np.array(ast.literal_eval(call.args[0]), np.float64)
        raise KeyError(name)

    exp_amp = arr('exp_amp')
    exp_var = arr('exp_var')
    dev_amp = arr('dev_amp')
    dev_var = arr('dev_var')
    dev_core = _find_assign(mp_tree, 'dev_core')
    # Normalisations done at import time in mixture_profiles.py:24,33-38 and
    # again by galaxy.py:727-763 (profile.normalize()).
    exp_amp = exp_amp / np.sum(exp_amp)
    dev_amp = dev_amp * ((1. - dev_core) / np.sum(dev_amp))
    dev_amp = np.append(dev_core, dev_amp)
    dev_var = np.append(0., dev_var)
    dev_amp = dev_amp / np.sum(dev_amp)

    fits = _find_assign(se_tree, 'fits')
    cores = _find_assign(se_tree, 'self.cores')

    from scipy.interpolate import InterpolatedUnivariateSpline

    def spline_rep(x, y, k):
        s = InterpolatedUnivariateSpline(x, y, k=k)
        t, c, kk = s._eval_args
        return dict(t=[float(v) for v in t], c=[float(v) for v in c], k=int(kk))

    ranges = []
    for lo, hi, grid in fits:
        K = len(grid[0][1])
        spline_k = 3 if len(grid) > 3 else 1
        ns = [g[0] for g in grid]
        ranges.append(dict(
            lo=lo, hi=hi, K=K, spline_k=spline_k,
            grid=[[g[0], list(g[1]), list(g[2])] for g in grid],
            amp_splines=[spline_rep(ns, [g[1][i] for g in grid], spline_k) for i in range(K)],
            logvar_splines=[spline_rep(ns, [np.log(g[2][i]) for g in grid], spline_k)
                            for i in range(K)],
        ))
    core_spline = spline_rep([s for s, c in cores], [c for s, c in cores], 3)
    out = dict(
        source='tractor/mixture_profiles.py:20-45, tractor/sersic.py:40-282',
        exp=dict(amp=list(exp_amp), var=list(exp_var)),
        dev=dict(amp=list(dev_amp), var=list(dev_var)),
        sersic=dict(ranges=ranges, cores=[list(c) for c in cores], core_spline=core_spline,
                    lowest=ranges[0]['lo'], highest=ranges[-1]['hi']),
    )
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'profile_tables.json')
    with open(dst, 'w') as f:
        json.dump(out, f, indent=1)
    print('wrote', dst)


if __name__ == '__main__':
    if len(sys.argv) < 2:
        sys.exit('usage: make_profile_tables.py REFERENCE_ROOT')
    main(sys.argv[1])
