"""The batched form's size draw (host code of the C ABI) against the oracle's
generator stream: n_i = 128 * (2 + floor((v_i + 0.5) * 31)), v_i = value i of
the stream seeded with the size seed."""
import math

import pytest


def test_batch_sizes_follow_the_generator(mxp, orc):
    count, seed = 64, 3
    got = mxp.batch_sizes(count, seed)
    want = []
    for i in range(count):
        v = orc.lib().orc_elem(1, seed, i, 0)
        want.append(128 * min(32, max(2, 2 + math.floor((v + 0.5) * 31))))
    assert got == want
    assert all(256 <= n <= 4096 and n % 128 == 0 for n in mxp.batch_sizes(2048, 3))


def test_batch_sizes_reject_bad_count(mxp):
    with pytest.raises(mxp.MxpError):
        mxp.batch_sizes(0, 3)


@pytest.mark.parametrize("nparts", [1, 2, 3, 8])
def test_batch_partition_balances_lu_work(mxp, nparts):
    """mxp_batch_partition: largest system first, each to the part with the least
    n^3 so far (ties to the lower part), restated here in Python."""
    sizes = mxp.batch_sizes(2048, 3)
    got = mxp.batch_partition(sizes, nparts)
    load = [0.0] * nparts
    want = [0] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        p = min(range(nparts), key=lambda k: (load[k], k))
        load[p] += float(sizes[i]) ** 3
        want[i] = p
    assert got == want
    assert max(load) / (sum(load) / nparts) < 1.01


def test_batch_partition_rejects_bad_arguments(mxp):
    with pytest.raises(mxp.MxpError):
        mxp.batch_partition([256, 512], 0)
    with pytest.raises(mxp.MxpError):
        mxp.batch_partition([256, -1], 2)
