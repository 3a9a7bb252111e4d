"""Shared helpers of the test-suite (the oracle is the checker)."""
import os
import tempfile

import numpy as np

from cudaprotoplanetarydisksfloat_b200 import configs, read_params, read_planets

SEED = 20261203


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def make(params, planets, name="t"):
    d = tempfile.mkdtemp(prefix="fargo_%s_" % name)
    par, cfg, out = configs.materialise(params, planets, d, name)
    P = read_params(par)
    L = read_planets(cfg, P)
    return P, L, d


def small(kind, nrad=32, nsec=96, **over):
    p, pl = configs.small(kind, nrad, nsec)
    p = dict(p, **over)
    return make(p, pl, kind)
