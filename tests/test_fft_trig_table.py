"""The butterfly constants of the DFT engine (so3_b200/csrc/fft_trig.h) are
generated by gen_fft_trig.py; the committed header must be that script's
output, and every literal must be cos / sin (2 pi k / R): within 1e-15 of the
libm values at the rounded angle (the literals are the correctly rounded values
at the exact angle, so they differ from those by argument rounding only)."""
import importlib.util
import math
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "so3_b200", "csrc")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_fft_trig", os.path.join(CSRC, "gen_fft_trig.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_header_is_generator_output():
    with open(os.path.join(CSRC, "fft_trig.h")) as fh:
        assert fh.read() == _gen().render()


def test_literals_are_cos_sin():
    gen = _gen()
    text = gen.render()

    def table(name):
        body = re.search(name + r"\[\d+\] = \{(.*?)\};", text, re.S).group(1)
        return [float.fromhex(v) for v in re.findall(r"-?0x[0-9a-f.]+p[+-]\d+", body)]

    cs, sn = table("kTrigCos"), table("kTrigSin")
    off = 0
    for R in gen.RADICES:
        H = (R - 1) // 2
        assert re.search(r"struct TrigOff<%d> \{\s*static constexpr int v = %d;" % (R, off), text)
        for k in range(H + 1):
            a = 2 * math.pi * k / R
            assert abs(cs[off + k] - math.cos(a)) <= 1e-15
            assert abs(sn[off + k] - math.sin(a)) <= 1e-15
        off += H + 1
    assert off == len(cs) == len(sn)
