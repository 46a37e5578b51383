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


# Floor of the elementwise relative error, as a fraction of max |y|: entries
# smaller than this are compared against the floor instead of themselves
# (a relative error is ill-posed at samples that cross zero).
ELEM_FLOOR = 1e-3


def rel_err_elem(x, y, floor=ELEM_FLOOR):
    """max_i |x_i - y_i| / max(|y_i|, floor * max_j |y_j|): the elementwise
    relative error with a stated floor for near-zero entries."""
    x = np.asarray(x)
    y = np.asarray(y)
    ay = np.abs(y)
    if ay.size == 0:
        return 0.0
    den = np.maximum(ay, floor * ay.max())
    den = np.where(den > 0, den, 1.0)
    return float((np.abs(x - y) / den).max())
