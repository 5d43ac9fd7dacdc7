"""A CPU model of the persistent kernels' grid barrier (grid_barrier in common.cuh), run
under random arrival and polling orders over many episodes.

The barrier is one 32-bit counter: block 0 adds 2^31 - (n - 1), every other block adds 1,
so one episode adds exactly 2^31. Bit 31 flips when the last block arrives and the low 31
bits return to where they started; a block leaves when bit 31 differs from its own
pre-add value. The model checks that no block leaves an episode before every block has
arrived at it, that every block leaves, and that a block running ahead into the next
episode cannot release or trap a slow block still polling the previous one. It also
shows why the host zeroes the control block before every launch: a counter whose low
bits are left over from an aborted launch releases blocks early."""
import numpy as np
import pytest

MASK = 0xFFFFFFFF


def _simulate(n, episodes, rng, start=0):
    """Returns the list of (block, episode, arrived_count_when_left) for every leave."""
    bar = start
    ep = [0] * n            # episode each block is in
    before = [None] * n     # pre-add value while waiting, None when running
    arrived = [0] * episodes
    leaves = []
    steps = 0
    while any(e < episodes for e in ep):
        steps += 1
        assert steps < 100000, "no progress"
        b = int(rng.integers(0, n))
        if ep[b] >= episodes:
            continue
        if before[b] is None:  # arrive: atomicAdd
            inc = (0x80000000 - (n - 1)) & MASK if b == 0 else 1
            before[b] = bar
            bar = (bar + inc) & MASK
            arrived[ep[b]] += 1
        else:  # poll: ld.acquire of the counter
            if ((bar ^ before[b]) & 0x80000000) != 0:
                leaves.append((b, ep[b], arrived[ep[b]]))
                before[b] = None
                ep[b] += 1
    return leaves


@pytest.mark.parametrize("n", [1, 2, 3, 7, 148, 592])
def test_no_block_leaves_before_all_arrive(n):
    rng = np.random.default_rng(n)
    episodes = 6 if n > 100 else 25
    leaves = _simulate(n, episodes, rng)
    assert len(leaves) == n * episodes  # every block left every episode
    assert all(count == n for _, _, count in leaves)


def test_leftover_low_bits_release_blocks_early():
    """Planted mistake: start from a counter whose low bits are not zero (a launch that
    ended early, reused without the host's reset)."""
    n = 8
    early = 0
    for seed in range(20):
        rng = np.random.default_rng(seed)
        try:
            leaves = _simulate(n, 4, rng, start=n - 1)
        except AssertionError:
            early += 1  # blocks stuck instead
            continue
        early += int(any(count < n for _, _, count in leaves))
    assert early > 0
