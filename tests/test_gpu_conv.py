"""Directional convolution then inverse transform (config C4 shape: one S^2
signal flm, complex Gaussian with variance (l+1)^-2, convolved with kernels
glm that are complex Gaussian for |m| < N = 8 and zero otherwise,
so3_conv_s2toso3_harmonic_convolution of src/c/so3_conv.c:186-215, then the
inverse transform to MW samples), through so3gpu_s2toso3_inverse_batch.

* FP64 against the oracle (s2toso3 then inverse) at 1e-12 normwise;
* split precision (h computed inside the contraction's operand load, never
  stored) against FP64 at <= 1e-10 normwise, the split path's contract."""
import pytest

import so3_b200 as so3
from so3_b200 import synth
from tests.helpers import oparams, params, rel_err, rel_err_elem

pytestmark = pytest.mark.gpu


def _inputs(L, N, nker, seed):
    import torch
    flm = torch.from_numpy(synth.gen_flm(L, seed, "gauss")).cuda()
    glms = [torch.from_numpy(synth.gen_flm(L, seed + 1 + k, "gauss", mmax=N - 1)).cuda() for k in range(nker)]
    return flm, glms


@pytest.mark.parametrize("L,N,mode,nker", [(32, 8, 0, 2), (64, 5, 2, 2), (1024, 8, 3, 1)])
def test_conv_inverse_fp64_against_oracle(O, L, N, mode, nker):
    """L=1024 with n_mode=MAXIMUM (planes n = +-7) keeps the oracle's run short."""
    import torch
    hp = params(L, N, mode=mode)
    ctx = so3.Context(0)
    flm, glms = _inputs(L, N, nker, 300 + L)
    fs = ctx.s2toso3_inverse_batch(hp, flm, glms, "fp64")
    torch.cuda.synchronize()
    op = oparams(O, hp)
    for k in range(len(glms)):
        h = O.s2toso3(op, flm.cpu().numpy(), glms[k].cpu().numpy())
        f_ref = O.inverse(h, op)
        assert rel_err(fs[k].cpu().numpy(), f_ref) < 1e-12
    # same as the two public calls in sequence
    h0 = ctx.s2toso3(hp, flm, glms[0])
    f0 = ctx.inverse(h0, hp)
    torch.cuda.synchronize()
    assert rel_err(fs[0].cpu().numpy(), f0.cpu().numpy()) < 1e-15


@pytest.mark.parametrize("L,N,nker", [(32, 8, 3), (70, 4, 17), (1024, 8, 3)])
def test_conv_inverse_split_against_fp64(L, N, nker):
    import torch
    hp = params(L, N)
    ctx = so3.Context(0)
    flm, glms = _inputs(L, N, nker, 500 + L)
    f64 = ctx.s2toso3_inverse_batch(hp, flm, glms, "fp64")
    fmx = ctx.s2toso3_inverse_batch(hp, flm, glms, "mixed")
    torch.cuda.synchronize()
    assert so3.take_kernel_error() == 0
    for a, b in zip(fmx, f64):
        x, y = a.cpu().numpy(), b.cpu().numpy()
        assert rel_err(x, y) <= 1e-10
        assert rel_err_elem(x, y) <= 1e-7
    del f64, fmx
    ctx.close()
    torch.cuda.empty_cache()


def test_conv_inverse_rejects_real():
    import torch
    hp = params(8, 4, reality=1)
    ctx = so3.Context(0)
    flm, glms = _inputs(8, 4, 1, 1)
    out = [torch.zeros(so3.f_size(hp), dtype=torch.complex128, device="cuda")]
    with pytest.raises(so3.SO3Error, match="status 3"):
        ctx.s2toso3_inverse_batch(hp, flm, glms, "fp64", outs=out)
