"""The C ABI library loads and exports every function the public headers
declare; host-side error handling works without a GPU."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import so3_b200 as so3

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b((?:so3|so3gpu)_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_reference_entry_points():
    names = set(declared_functions())
    for ref in ("so3_core_inverse_via_ssht", "so3_core_forward_via_ssht", "so3_core_inverse_via_ssht_real",
                "so3_core_forward_via_ssht_real", "so3_conv_harmonic_convolution",
                "so3_conv_s2toso3_harmonic_convolution", "so3_conv_get_parameters_of_convolved_lmn",
                "so3_sampling_elmn2ind", "so3_sampling_flmn_size", "so3_sampling_f_size"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    lib = so3._lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", so3._lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)


def test_params_struct_layout():
    """so3_parameters_t is eleven 4-byte fields in the reference's order."""
    assert ctypes.sizeof(so3._lib.Params) == 44
    names = [f[0] for f in so3._lib.Params._fields_]
    assert names == ["verbosity", "reality", "L0", "L", "N", "sampling_scheme", "n_order", "storage", "n_mode",
                     "dl_method", "steerable"]


def test_no_gpu_fails_loudly_without_fallback():
    """Without a usable GPU the transform reports a CUDA error (status 2);
    it never computes on the CPU."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    p = so3.SO3Parameters(L=4, N=2)
    with pytest.raises(so3.SO3Error, match="status 2"):
        so3.inverse(np.zeros(so3.flmn_size(p), complex), p)


def test_invalid_parameters_rejected_before_device_work():
    p = so3.SO3Parameters(L=4, N=2, n_mode=9)
    with pytest.raises(so3.SO3Error, match="status 1"):
        so3.inverse(np.zeros(so3.flmn_size(so3.SO3Parameters(L=4, N=2)), complex), p)


def test_reference_exit_semantics_in_default_mode(tmp_path):
    """In the default error mode an invalid parameter prints the reference's
    'ERROR: ...' message and exits with status 1 (so3_error.h)."""
    code = (
        "import ctypes, so3_b200._lib as L\n"
        "lib = ctypes.CDLL(L.LIB_PATH)\n"
        "p = L.Params(0,0,0,4,2,5,1,0,0,0,0)\n"
        "lib.so3_sampling_nalpha(ctypes.byref(p))\n"
    )
    r = subprocess.run(["python", "-c", code], cwd=ROOT, capture_output=True, text=True)
    assert r.returncode == 1
    assert "ERROR: Invalid sampling scheme." in r.stdout


def test_stage_variant_pinning_round_trip(lib):
    """Pinned DFT-stage variants are stored per device and geometry (host
    state only; no GPU needed)."""
    import ctypes
    from tests.helpers import params
    p = params(40, 3, sampling=1).to_struct()
    got = (ctypes.c_int * 8)()
    assert lib.so3gpu_get_stage_variants(5, ctypes.byref(p), got) == 0
    want = (ctypes.c_int * 8)(0, 1, 2, 0, 0, 1, 1, 0)
    assert lib.so3gpu_set_stage_variants(5, ctypes.byref(p), want) == 0
    assert lib.so3gpu_get_stage_variants(5, ctypes.byref(p), got) == 1
    assert list(got) == list(want)
    bad = (ctypes.c_int * 8)(0, 9, 0, 0, 0, 0, 0, 0)
    assert lib.so3gpu_set_stage_variants(5, ctypes.byref(p), bad) == 1
