"""Host-side pieces of bench.py that feed its JSON line: the per-launch
int8 multiply-add counts of the split-precision kernels (against a direct
count over work items), the compulsory bytes of the stages, and the DRAM
traffic read from the committed ncu summary."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _items_chunks(L, N, fwd):
    """Reduction chunks of 64 summed over the work items (pair, 64-row tile),
    restated from the kernels' item decoding (mixed.cu decode_item)."""
    T, tot = 64, 0
    MT = (L + T - 1) // T
    for mu in range(L):
        for nu in range(N):
            lmin = max(mu, nu)
            for t in range(MT):
                r0 = t * T
                if fwd:
                    tot += (min(L, r0 + T) + T - 1) // T if (r0 + T > lmin and r0 < L) else 0
                else:
                    ks = (max(lmin, r0) // T) * T
                    tot += (L - ks + T - 1) // T if ks < L else 0
    return tot


def test_mixed_tc_macs_counts_items():
    for L, N in [(8, 3), (70, 5), (130, 2)]:
        for fwd in (False, True):
            assert bench.mixed_tc_macs(L, N, fwd) == _items_chunks(L, N, fwd) * 2 * 28 * 128 * 64 * 32


def test_beta_tc_macs():
    L, N = 512, 64
    nc = 8
    assert bench.beta_tc_macs(L, N) == (2 * N - 1) * 2 * nc * nc * nc * 2 * 28 * 128 * 64 * 32


def test_stage_bytes_metric_geometry():
    sb = bench.stage_bytes(512, 64)
    part = 127 * 512 * 1023 * 16
    assert sb["inv_beta"] == 2 * part == 2128625664
    assert sb["inv_contract"] == 127 * 512 * 512 * 16 + part


def test_traffic_from_committed_profile():
    assert bench.traffic_from_profiles("mixed_fwd_beta", 512, 64) == 62189000000.0
    assert bench.traffic_from_profiles("mixed_fwd_contract", 512, 64) == 92604000000.0
    assert bench.traffic_from_profiles("mixed_inv_contract", 512, 64) == 71686000000.0
    assert bench.traffic_from_profiles("mixed_fwd_beta", 256, 64) is None


def test_split_stage_rooflines():
    L, N, B, peak = 512, 64, 16, 4550.0
    per = {"mixed_fwd_beta": 26.8, "mixed_inv_contract": 21.6, "mixed_fwd_contract": 26.9, "inv_beta": 0.9}
    r = bench.split_stage_rooflines(per, L, N, B, peak)
    assert set(r) == {"mixed_fwd_beta", "mixed_inv_contract", "mixed_fwd_contract"}
    b = r["mixed_fwd_beta"]
    assert b["int8_macs_per_launch"] == bench.beta_tc_macs(L, N) * B
    assert abs(b["achieved_tops"] - 2.0 * b["int8_macs_per_launch"] / 26.8e-3 / 1e12) < 0.1
    assert abs(b["frac_int8_peak"] - b["achieved_tops"] / peak) < 1e-3
    assert bench.split_stage_rooflines({}, L, N, B, peak) == {}
