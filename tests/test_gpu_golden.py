"""Parity of the CUDA executor with the reference's golden vectors.

Every case in tests/golden (random programs covering every DSL form,
per-operator known answers incl. carry chains across many tiles, and the
bits->=N corner cases) runs through the C ABI and must match the reference
interpreter's outputs bit for bit (streams masked to the bitlength as the
reference harness compares them, ints exactly) and its op count.  Cases on
which the reference raises must raise.
"""

import pytest

from conftest import expected_masked, load_golden, run_golden_case
import bitstreamzoo_b200 as bz

GROUPS = ["random_programs", "kat_ops", "tail_corners"]
MODES = [bz.MODE_PLAIN, bz.MODE_FUSED, bz.MODE_VM, bz.MODE_AUTO]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("group", GROUPS)
def test_golden_group(ctx, group, mode):
    fails = []
    n = 0
    for rec in load_golden(group):
        if "error" in rec:
            with pytest.raises(bz.BszError):
                run_golden_case(ctx, rec, mode)
            continue
        got, ops, _ = run_golden_case(ctx, rec, mode)
        if got != expected_masked(rec) or ops != rec["op_count"]:
            fails.append(rec["name"])
        n += 1
    assert not fails, f"{len(fails)} of {n} mismatched: {fails[:10]}"
