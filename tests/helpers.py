"""Shared test helpers: parameter construction and error norms."""
import numpy as np

from so3_b200 import SO3Parameters


def params(L, N, L0=0, reality=0, sampling=0, order=1, storage=0, mode=0, method=0, steerable=0):
    return SO3Parameters(L=L, N=N, L0=L0, reality=reality, sampling_scheme=sampling, n_order=order,
                         storage=storage, n_mode=mode, dl_method=method, steerable=steerable)


def oparams(O, p):
    """Same configuration as an oracle Params struct."""
    return O.params(p.L, p.N, L0=p.L0, reality=p.reality, sampling=p.sampling_scheme, order=p.n_order,
                    storage=p.storage, mode=p.n_mode, method=p.dl_method, steerable=p.steerable)


def rel_err(x, y):
    """max_i |x - y| / max_i |y| (normwise, well posed near zero samples)."""
    x = np.asarray(x)
    y = np.asarray(y)
    den = np.abs(y).max()
    return float(np.abs(x - y).max() / (den if den > 0 else 1.0))
