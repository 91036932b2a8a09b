"""The device deletion rules against the oracle's restatement on every
neighbourhood of a foreground centre: 2^8 per 2D direction, 2^26 per 3D
direction (the oracle's rules are in turn checked against the reference's
own rule functions in test_oracle.py)."""
import numpy as np
import pytest

from oracle import pyoracle as po


@pytest.mark.gpu
@pytest.mark.parametrize("dims,direction", [(2, d) for d in range(4)] + [(3, d) for d in range(6)])
def test_device_rule_table_equals_oracle(ctx, dims, direction):
    import torch
    from begputhinning_b200._lib import check, lib
    n = 8 if dims == 2 else 1 << 21
    dev = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    check(lib().bgt_rule_table(dims, direction, dev.data_ptr(), None))
    got = dev.cpu().numpy().view(np.uint32)
    want = po.rule_table(dims, direction)
    bad = np.bitwise_xor(got, want)
    nbad = int(np.unpackbits(bad.view(np.uint8)).sum())
    assert nbad == 0, f"{nbad} neighbourhoods differ (dims {dims}, direction {direction})"


def test_oracle_rule_table_2d_matches_rule_function():
    """Layout check of the oracle table on the CPU: bit n of the 2D table is
    the rule evaluated on neighbourhood n."""
    for d in range(4):
        t = po.rule_table(2, d)
        for n in range(256):
            x = np.array([(n >> i) & 1 for i in range(8)], np.uint64)
            assert ((int(t[n >> 5]) >> (n & 31)) & 1) == (int(po.rule2d(d, x)) & 1), (d, n)
