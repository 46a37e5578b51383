"""Split-precision batch path: int8 tensor-core contractions (tcgen05, 7-digit
Ozaki split) against the FP64 path on the same inputs.  Tolerance: normwise
relative error 1e-10 (the split path's contract); measured values sit near
1e-12.  The FP64 path itself is pinned to the oracle by test_gpu_parity."""
import numpy as np
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import params, rel_err

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-10


@pytest.fixture(autouse=True)
def _no_kernel_timeouts(monkeypatch):
    # resident tables on first use, so every case runs the table-fed tensor-core kernels
    # (the default builds them on a geometry's second call; see test_tables_on_second_call)
    monkeypatch.setenv("SO3GPU_DIGIT_TABLE", "1")
    yield
    assert so3.take_kernel_error() == 0  # no bounded wait of the tensor-core kernels gave up


def _run(p, nsig, seed, dist="uniform"):
    import torch
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, seed + i, dist)).cuda() for i in range(nsig)]
    f64 = ctx.inverse_batch(fls, p, "fp64")
    fmx = ctx.inverse_batch(fls, p, "mixed")
    # forward from the same (FP64) samples
    b64 = ctx.forward_batch(f64, p, "fp64")
    bmx = ctx.forward_batch(f64, p, "mixed")
    torch.cuda.synchronize()
    return ([x.cpu().numpy() for x in fls], [x.cpu().numpy() for x in f64], [x.cpu().numpy() for x in fmx],
            [x.cpu().numpy() for x in b64], [x.cpu().numpy() for x in bmx])


CASES = [
    dict(L=32, N=8, nsig=3),
    dict(L=24, N=5, nsig=9, order=0, storage=1, L0=2),  # compact, zero-first, L0 > 0
    dict(L=70, N=3, nsig=18),                           # two groups of 16 signals, L past a 64-row tile
    dict(L=20, N=6, nsig=4, mode=1),                    # even n only
    dict(L=20, N=6, nsig=2, mode=3),                    # |n| = N-1 only
    dict(L=20, N=6, nsig=2, mode=4),                    # l = |n| only
    dict(L=33, N=4, nsig=5, sampling=1, method=1),      # MWSS, Trapani, L not a multiple of 32
    dict(L=1, N=1, nsig=2),
    dict(L=8, N=8, nsig=1),
]


@pytest.mark.parametrize("kw", CASES, ids=[str(i) for i in range(len(CASES))])
def test_mixed_batch_matches_fp64(kw):
    kw = dict(kw)
    nsig = kw.pop("nsig")
    L, N = kw.pop("L"), kw.pop("N")
    p = params(L, N, **kw)
    fls, f64, fmx, b64, bmx = _run(p, nsig, 100)
    for i in range(nsig):
        assert rel_err(fmx[i], f64[i]) < TOL_MIXED, (i, rel_err(fmx[i], f64[i]))
        assert rel_err(bmx[i], b64[i]) < TOL_MIXED, (i, rel_err(bmx[i], b64[i]))
        if p.n_mode == 0:
            assert rel_err(bmx[i], fls[i]) < 1e-10  # round trip


def test_mixed_fp64_batch_equals_single_transforms():
    """precision "fp64" of the batch API is the single-signal path."""
    import torch
    p = params(24, 6)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 7 + i)).cuda() for i in range(3)]
    outs = ctx.inverse_batch(fls, p, "fp64")
    for x, o in zip(fls, outs):
        ref = ctx.inverse(x, p)
        torch.cuda.synchronize()
        assert np.array_equal(o.cpu().numpy(), ref.cpu().numpy())


REAL_CASES = [
    dict(L=32, N=8, nsig=3),
    dict(L=24, N=5, nsig=9, order=0, storage=1, L0=2),  # compact, zero-first, L0 > 0
    dict(L=40, N=3, nsig=18),                           # two groups of 16 signals
    dict(L=20, N=6, nsig=4, mode=1),                    # even n only
    dict(L=33, N=4, nsig=5, sampling=1, method=1),      # MWSS, Trapani
]


@pytest.mark.parametrize("kw", REAL_CASES, ids=[str(i) for i in range(len(REAL_CASES))])
def test_mixed_real_batch_matches_fp64(kw):
    """Real signals: split contractions over the planes n >= 0 (the columns of
    the n = -nu combinations stay empty), FP64 DFT stages with r2c / c2r over
    gamma; every result against the FP64 path, and the round trip."""
    kw = dict(kw)
    nsig = kw.pop("nsig")
    L, N = kw.pop("L"), kw.pop("N")
    p = params(L, N, reality=1, **kw)
    fls, f64, fmx, b64, bmx = _run(p, nsig, 41)
    for i in range(nsig):
        assert rel_err(fmx[i], f64[i]) < TOL_MIXED, (i, rel_err(fmx[i], f64[i]))
        assert rel_err(bmx[i], b64[i]) < TOL_MIXED, (i, rel_err(bmx[i], b64[i]))
        if p.n_mode == 0:
            assert rel_err(bmx[i], fls[i]) < 1e-10  # round trip


def test_mixed_real_single_plane_uses_fp64():
    """N = 1 real signals stay on the FP64 path (its inverse symmetrises the
    single plane): results bit-identical to precision "fp64"."""
    import torch
    p = params(24, 1, reality=1)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 3 + i)).cuda() for i in range(2)]
    a = ctx.inverse_batch(fls, p, "fp64")
    b = ctx.inverse_batch(fls, p, "mixed")
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert np.array_equal(x.cpu().numpy(), y.cpu().numpy())


def test_mixed_batched_config_L128_N16_gauss():
    """The batched configuration's shape (L=128, N=16, MW, padded, Risbo,
    complex Gaussian with variance ~ (l+1)^-2, dynamic range ~1e4), 8 signals."""
    p = params(128, 16)
    fls, f64, fmx, b64, bmx = _run(p, 8, 500, "gauss")
    errs = [rel_err(fmx[i], f64[i]) for i in range(8)] + [rel_err(bmx[i], b64[i]) for i in range(8)]
    assert max(errs) < TOL_MIXED, errs


def test_mixed_metric_size_L512():
    """L=512 (the metric's band limit) with a few n-planes, 2 signals."""
    p = params(512, 3)
    fls, f64, fmx, b64, bmx = _run(p, 2, 900)
    for i in range(2):
        assert rel_err(fmx[i], f64[i]) < TOL_MIXED
        assert rel_err(bmx[i], b64[i]) < TOL_MIXED


def test_mixed_forward_leaves_skipped_blocks():
    import torch
    p = params(20, 6, mode=1)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 1)).cuda()]
    f = ctx.inverse_batch(fls, p, "fp64")
    out = [torch.full((so3.flmn_size(p),), 7.0 + 1j, dtype=torch.complex128, device="cuda")]
    ctx.forward_batch(f, p, "mixed", outs=out)
    ref = [torch.full((so3.flmn_size(p),), 7.0 + 1j, dtype=torch.complex128, device="cuda")]
    ctx.forward_batch(f, p, "fp64", outs=ref)
    torch.cuda.synchronize()
    assert rel_err(out[0].cpu().numpy(), ref[0].cpu().numpy()) < TOL_MIXED


@pytest.mark.parametrize("L,N,nsig,kw", [(70, 3, 5, {}), (130, 4, 3, dict(L0=5, storage=1)), (64, 64, 2, {})])
def test_resident_digits_equal_generated_digits(L, N, nsig, kw, monkeypatch):
    """The resident digit table (read as a K-major operand by the inverse and
    as an MN-major operand by the forward) and the on-the-fly generation from
    Delta hold the same digits, and the int32 accumulation is exact: the two
    paths give bit-identical results."""
    import torch
    p = params(L, N, **kw)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 40 + i)).cuda() for i in range(nsig)]
    f64 = ctx.inverse_batch(fls, p, "fp64")
    outs = {}
    for mode in ("1", "0"):  # "1" first: the forward beta table then exists for both runs
        monkeypatch.setenv("SO3GPU_DIGIT_TABLE", mode)
        inv = ctx.inverse_batch(fls, p, "mixed")
        fwd = ctx.forward_batch(f64, p, "mixed")
        torch.cuda.synchronize()
        outs[mode] = ([x.cpu().numpy() for x in inv], [x.cpu().numpy() for x in fwd])
    for a, b in zip(outs["0"][0] + outs["0"][1], outs["1"][0] + outs["1"][1]):
        assert np.array_equal(a, b)


def test_tables_on_second_call(monkeypatch):
    """Default policy: the first split-precision call of a geometry generates
    the digits from Delta and runs the FP64 forward beta stage; later calls
    use the resident tables (tensor-core forward beta stage).  Every call is
    within the split-precision tolerance of the FP64 path."""
    import torch
    monkeypatch.delenv("SO3GPU_DIGIT_TABLE", raising=False)
    p = params(77, 5)  # a geometry no other test uses
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 60 + i)).cuda() for i in range(3)]
    f64 = ctx.inverse_batch(fls, p, "fp64")
    b64 = [x.cpu().numpy() for x in ctx.forward_batch(f64, p, "fp64")]
    runs = []
    for _ in range(3):
        inv = ctx.inverse_batch(fls, p, "mixed")
        fwd = ctx.forward_batch(f64, p, "mixed")
        torch.cuda.synchronize()
        runs.append(([x.cpu().numpy() for x in inv], [x.cpu().numpy() for x in fwd]))
    f64n = [x.cpu().numpy() for x in f64]
    for inv, fwd in runs:
        for i in range(3):
            assert rel_err(inv[i], f64n[i]) < TOL_MIXED
            assert rel_err(fwd[i], b64[i]) < TOL_MIXED
    for i in range(3):  # second and third calls: same (table) path
        assert np.array_equal(runs[1][1][i], runs[2][1][i])


SLICE_CASES = [
    dict(L=32, N=8, nsig=3),
    dict(L=24, N=5, nsig=9, order=0, storage=1, L0=2),  # compact, zero-first, L0 > 0
    dict(L=70, N=3, nsig=18),                           # two groups, L past a 64-entry chunk
    dict(L=20, N=6, nsig=4, mode=1),                    # skipped planes
    dict(L=20, N=6, nsig=2, mode=3),
    dict(L=33, N=4, nsig=5, sampling=1, method=1),      # MWSS (FP64 forward beta stage)
    dict(L=130, N=2, nsig=2),                           # L not a multiple of 64 (zero rows in the last chunk)
    dict(L=520, N=2, nsig=2),                           # > 512 beta rows (per-pair beta slicing), 1039 columns
    dict(L=40, N=5, nsig=3, reality=1),                 # real signals: planes n >= 0
]


@pytest.mark.parametrize("kw", SLICE_CASES, ids=[str(i) for i in range(len(SLICE_CASES))])
def test_single_read_slicing_is_bit_identical(kw, monkeypatch):
    """The single-read slicing kernels (streaming inverse slicing in storage
    order, shared-memory staged beta slicing) cut the same digits with the same
    column scales as the per-pair kernels: the split results are equal bit for
    bit."""
    import torch
    kw = dict(kw)
    nsig = kw.pop("nsig")
    L, N = kw.pop("L"), kw.pop("N")
    p = params(L, N, **kw)
    ctx = so3.Context(0)
    fls = [torch.from_numpy(synth.gen_flmn(p, 300 + i)).cuda() for i in range(nsig)]
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("SO3GPU_STREAM_SLICE", mode)
        f = ctx.inverse_batch(fls, p, "mixed")
        b = ctx.forward_batch(f, p, "mixed")
        torch.cuda.synchronize()
        out[mode] = ([x.cpu().numpy() for x in f], [x.cpu().numpy() for x in b])
    for i in range(nsig):
        assert np.array_equal(out["0"][0][i], out["1"][0][i]), i
        assert np.array_equal(out["0"][1][i], out["1"][1][i]), i
