"""swb_sweep_static: sweeps of caller-owned device buffers with the scratch in a static device
array, checked against swb_sweep on the same state (bit-exact: spins and lcg32 streams) over two
calls in a row, so the second call runs on the scratch the first one left behind."""
import ctypes

import numpy as np
import pytest

from computational_physics_b200._native import lib

T_C = 2.2691853
PAIRS = [(1372383749, 1289706101), (2891336453, 1640531513), (2024337845, 797082193),
         (32310901, 626627237), (29943829, 1013904223)]   # random/src/lcg32.cpp:17-24


def _sel(a, c):
    sel = np.full(a.shape, 255, np.uint8)
    for k, (pa, pc) in enumerate(PAIRS):
        sel[(a == pa) & (c == pc)] = k
    assert (sel != 255).all()
    return sel


def _call(stream, shape, tile, w, T, n, spins, state, sel, it):
    return lib().swb_sweep_static(stream, shape[0], shape[1], tile[0], tile[1], w, T, n, spins.data_ptr(),
                                  state.data_ptr(), sel.data_ptr(), it.data_ptr(), 1)


def test_rejects_before_any_cuda_call():
    """Argument and size errors come back before the first CUDA call (runs without a GPU)."""
    L = lib()
    p = 4096  # aligned dummy address, never dereferenced
    assert L.swb_sweep_static(None, 4096, 2048, 16, 8, 16, T_C, 1, p, p, p, p, 1) == 4   # 2^23 sites
    assert "static scratch limit" in L.swb_last_error().decode()
    assert L.swb_sweep_static(None, 64, 64, 16, 8, 16, T_C, 1, None, p, p, p, 1) == 1
    assert L.swb_sweep_static(None, 64, 64, 16, 8, 16, T_C, 1, p + 4, p, p, p, 1) == 1  # spins alignment
    assert L.swb_sweep_static(None, 63, 64, 16, 8, 16, T_C, 1, p, p, p, p, 1) == 1
    assert L.swb_sweep_static(None, 64, 64, 12, 8, 16, T_C, 1, p, p, p, p, 1) == 1
    assert L.swb_sweep_static(None, 64, 64, 16, 8, 16, -1.0, 1, p, p, p, p, 1) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("shape,tile,w", [((256, 128), (16, 8), 16), ((2048, 2048), (16, 8), 16),
                                          ((96, 64), (8, 4), 8), ((160, 96), (32, 6), 32)])
def test_static_sweep_matches_sweep(gpu, shape, tile, w):
    import torch
    cp = gpu
    with cp.SwendsenWang2D(shape[0], shape[1], tile, w, seed_base=11) as ref:
        ref.hot_start(5)
        st, a, c, it = ref.get_rng()
        dev = torch.device("cuda", 0)
        spins = torch.from_numpy(ref.get_spins().reshape(-1).copy()).to(dev)
        state = torch.from_numpy(st.view(np.int32).reshape(-1).copy()).to(dev)
        sel = torch.from_numpy(_sel(a, c).reshape(-1)).to(dev)
        itd = torch.from_numpy(it.view(np.int32).copy()).to(dev)
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize(dev)
        for call, (T, n) in enumerate([(T_C, 3), (2.0, 2)]):
            ref.update(T, n)
            ref.synchronize()
            free0 = torch.cuda.mem_get_info(dev)[0]
            rc = _call(stream, shape, tile, w, T, n, spins, state, sel, itd)
            assert rc == 0, lib().swb_last_error().decode()
            if call == 1:  # after the first call's set-up: device free memory unchanged
                assert torch.cuda.mem_get_info(dev)[0] == free0
            torch.cuda.synchronize(dev)
            np.testing.assert_array_equal(spins.cpu().numpy(), ref.get_spins().reshape(-1))
            st, a, c, it = ref.get_rng()
            np.testing.assert_array_equal(state.cpu().numpy().view(np.uint32), st.reshape(-1))
            np.testing.assert_array_equal(sel.cpu().numpy(), _sel(a, c).reshape(-1))
            np.testing.assert_array_equal(itd.cpu().numpy().view(np.uint32), it)
