"""CPU: the ragged plan is host-only and validates its input."""

from __future__ import annotations

import ctypes

from gpumode_cholesky_b200 import _lib, inputs


def _plan(orders, offsets=None, mode=0, tc_min_n=0):
    lib = _lib.load()
    offsets = offsets if offsets is not None else inputs.pack_offsets(orders)[:-1]
    offs = (ctypes.c_int64 * max(len(orders), 1))(*offsets)
    ns = (ctypes.c_int32 * max(len(orders), 1))(*orders)
    h = ctypes.c_void_p()
    st = lib.b2p_ragged_plan_create(offs, ns, len(orders), mode, tc_min_n, ctypes.byref(h))
    return st, h


def _padded_elems(orders, min_n=129):
    return sum(((n + 63) // 64 * 64) ** 2 for n in orders if n > 128 and n >= min_n)


def test_plan_sizes_and_destroy():
    lib = _lib.load()
    orders = [1, 16, 32, 33, 100, 128, 129, 300, 1000]
    st, h = _plan(orders)
    assert st == _lib.B2P_OK
    # FP32: three blocked matrices -> one 64x64 inverse slot each (+ alignment slack)
    assert lib.b2p_ragged_plan_workspace_bytes(h) == 3 * 64 * 64 * 4 + 1024
    assert lib.b2p_ragged_plan_table_bytes(h) > 8 * len(orders)
    lib.b2p_ragged_plan_destroy(h)


def test_plan_tensor_mode_pads_into_dense_groups():
    """Tensor modes: n > 128 matrices are padded to multiples of 64 (A and L copies)."""
    lib = _lib.load()
    orders = [1, 16, 100, 129, 130, 192, 300, 1000, 1500]
    st, h = _plan(orders, mode=_lib.MODE_BF16X3)
    assert st == _lib.B2P_OK
    ws = lib.b2p_ragged_plan_workspace_bytes(h)
    assert ws >= 2 * 4 * _padded_elems(orders)
    tb_dense = lib.b2p_ragged_plan_table_bytes(h)
    lib.b2p_ragged_plan_destroy(h)
    # dense_min_n above every order: all big matrices take the blocked schedule
    st, h = _plan(orders, mode=_lib.MODE_BF16X3, tc_min_n=1 << 16)
    assert st == _lib.B2P_OK
    assert lib.b2p_ragged_plan_workspace_bytes(h) == 6 * 64 * 64 * 4 + 1024
    assert lib.b2p_ragged_plan_table_bytes(h) != tb_dense
    lib.b2p_ragged_plan_destroy(h)
    # a threshold in between splits them
    st, h = _plan(orders, mode=_lib.MODE_BF16X3, tc_min_n=300)
    assert st == _lib.B2P_OK
    assert lib.b2p_ragged_plan_workspace_bytes(h) >= 2 * 4 * _padded_elems(orders, 300) + 3 * 64 * 64 * 4
    lib.b2p_ragged_plan_destroy(h)


def test_plan_empty_and_small_only():
    lib = _lib.load()
    st, h = _plan([])
    assert st == _lib.B2P_OK
    assert lib.b2p_ragged_plan_workspace_bytes(h) == 0
    lib.b2p_ragged_plan_destroy(h)
    st, h = _plan([3, 7, 32, 64, 128])
    assert st == _lib.B2P_OK and lib.b2p_ragged_plan_workspace_bytes(h) == 0
    lib.b2p_ragged_plan_destroy(h)


def test_plan_rejects_bad_input():
    lib = _lib.load()
    st, h = _plan([8, 8], offsets=[0, 66])  # not a multiple of 4
    assert st == _lib.B2P_ERR_INVALID_ARG and not h.value
    assert b"multiples of 4" in lib.b2p_last_error()
    st, h = _plan([8, -1])
    assert st == _lib.B2P_ERR_INVALID_ARG
    st, h = _plan([8], mode=_lib.MODE_FP8)
    assert st == _lib.B2P_ERR_UNSUPPORTED


def test_config4_orders_plan():
    """The 3000-matrix log-uniform [16, 2048] draw plans without a device."""
    lib = _lib.load()
    orders = inputs.ragged_orders(3000, seed=4)
    assert min(orders) >= 16 and max(orders) <= 2048
    big = sum(1 for n in orders if n > 128)
    st, h = _plan(orders, mode=0)
    assert st == _lib.B2P_OK
    assert lib.b2p_ragged_plan_workspace_bytes(h) == big * 64 * 64 * 4 + 1024
    lib.b2p_ragged_plan_destroy(h)
    st, h = _plan(orders, mode=_lib.MODE_BF16X3)
    assert st == _lib.B2P_OK
    assert lib.b2p_ragged_plan_workspace_bytes(h) >= 2 * 4 * _padded_elems(orders)
    lib.b2p_ragged_plan_destroy(h)


def _plan_ex(orders, mode, **kw):
    lib = _lib.load()
    offsets = inputs.pack_offsets(orders)[:-1]
    offs = (ctypes.c_int64 * max(len(orders), 1))(*offsets)
    ns = (ctypes.c_int32 * max(len(orders), 1))(*orders)
    opt = _lib.RaggedOptions(
        kw.get("dense_min_n", 0),
        kw.get("pad_step", 0),
        kw.get("pad_step_large", 0),
        kw.get("large_path", 0),
        kw.get("streams", 0),
    )
    h = ctypes.c_void_p()
    st = lib.b2p_ragged_plan_create_ex(offs, ns, len(orders), mode, ctypes.byref(opt), ctypes.byref(h))
    return st, h


def test_plan_options():
    lib = _lib.load()
    orders = [130, 200, 250, 1030, 1500, 2048]
    st, h = _plan_ex(orders, _lib.MODE_BF16X3, pad_step=256, pad_step_large=256, large_path=_lib.PATHS["fused_ws"])
    assert st == _lib.B2P_OK
    padded = 256**2 * 3 + 1280**2 + 1536**2 + 2048**2
    assert lib.b2p_ragged_plan_workspace_bytes(h) >= 2 * 4 * padded
    lib.b2p_ragged_plan_destroy(h)
    st, h = _plan_ex(orders, _lib.MODE_BF16X3, streams=8)
    assert st == _lib.B2P_OK
    lib.b2p_ragged_plan_destroy(h)
    for bad in (
        {"pad_step": 96},
        {"pad_step_large": 32},
        {"large_path": _lib.PATHS["blocked"]},
        {"dense_min_n": -1},
        {"streams": 9},
        {"streams": -1},
    ):
        st, h = _plan_ex(orders, _lib.MODE_BF16X3, **bad)
        assert st == _lib.B2P_ERR_INVALID_ARG and not h.value, bad
    # null options = defaults
    offs = (ctypes.c_int64 * 2)(*inputs.pack_offsets([300, 40])[:-1])
    ns = (ctypes.c_int32 * 2)(300, 40)
    h = ctypes.c_void_p()
    assert lib.b2p_ragged_plan_create_ex(offs, ns, 2, _lib.MODE_BF16X3, None, ctypes.byref(h)) == _lib.B2P_OK
    assert lib.b2p_ragged_plan_workspace_bytes(h) >= 2 * 4 * 320**2
    lib.b2p_ragged_plan_destroy(h)


def test_split_runs_cover_the_list_in_order():
    import random

    from gpumode_cholesky_b200.ragged import split_runs

    rng = random.Random(5)
    for _ in range(300):
        orders = [rng.choice([1, 3, 16, 64, 200, 1000, 2048]) for _ in range(rng.randint(1, 60))]
        offs = inputs.pack_offsets(orders)[:-1]
        parts = rng.randint(1, 70)
        runs = split_runs(orders, offs, parts)
        assert runs[0][0] == 0 and runs[-1][1] == len(orders)
        assert all(a < b for a, b in runs)
        assert all(runs[i][1] == runs[i + 1][0] for i in range(len(runs) - 1))
        assert len(runs) <= min(parts, len(orders))
    # equal orders split evenly
    assert split_runs([10] * 8, inputs.pack_offsets([10] * 8)[:-1], 4) == [(0, 2), (2, 4), (4, 6), (6, 8)]
    assert split_runs([], [], 3) == []


def test_host_plan_rejects_overlapping_offsets():
    import pytest

    from gpumode_cholesky_b200.ragged import RaggedHostPlan

    with pytest.raises(ValueError):
        RaggedHostPlan([4, 4], [0, 8])  # the second matrix starts inside the first
    with pytest.raises(ValueError):
        RaggedHostPlan([4], [0, 16])
    with pytest.raises(ValueError):
        RaggedHostPlan([4, 4], parts=-1)
