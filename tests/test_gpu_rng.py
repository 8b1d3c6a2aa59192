"""The lcg32 throughput kernel (swb_lcg32_benchmark, the counterpart of TestRNG --target)
against the oracle's restatement of LCG32<CPU>::NextReal: the reported stream's last 64
numbers bit for bit, and the XOR of every number of every stream."""
import numpy as np
import pytest

from computational_physics_b200 import rng_bench


@pytest.mark.gpu
@pytest.mark.parametrize("W", [8, 16, 32])
def test_lcg32_kernel_matches_oracle(gpu, oracle, W):
    n_streams, per = 37, 64 // W
    updates = 45 * per          # crosses many parameter rotations (every 15th update)
    r = rng_bench.generate(n_streams, updates, lcg_width=W, seed_base=1, report_id=5)
    want_x = 0
    for s in range(n_streams):
        nums = oracle.next_real(W, 1 + s, [64] * (updates * W // 64))
        want_x ^= int(np.bitwise_xor.reduce(nums.view(np.uint32)))
        if s == 5:
            np.testing.assert_array_equal(r["report"].view(np.uint32), nums[-64:].view(np.uint32))
    assert r["checksum"] == want_x
    assert r["numbers"] == n_streams * updates * W and r["ms"] > 0


@pytest.mark.gpu
def test_lcg32_argument_errors(gpu):
    with pytest.raises(gpu.NativeError):
        rng_bench.generate(4, 3, lcg_width=16)        # not a multiple of 64 / 16
    with pytest.raises(gpu.NativeError):
        rng_bench.generate(4, 4, lcg_width=12)
    with pytest.raises(gpu.NativeError):
        rng_bench.generate(4, 4, lcg_width=16, report_id=4)
