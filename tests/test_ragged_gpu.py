"""GPU: ragged batches against the oracle and the dense entry point.

FP32 mode runs the same kernels as the dense path with per-matrix
addressing, so results must be bitwise identical to the dense path; tensor
modes are checked by relative residual (<= 1e-5 for BF16x3).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from gpumode_cholesky_b200 import cholesky, inputs
from gpumode_cholesky_b200.ragged import RaggedPlan, cholesky_ragged, pack, unpack

pytestmark = pytest.mark.gpu

ORDERS = [1, 2, 5, 16, 17, 31, 32, 33, 48, 64, 65, 100, 127, 128, 129, 130, 200, 256, 300, 512, 513]


def _mats(orders, seed):
    return [inputs.generate_input(1, n, 2, seed + n, "dense", device="cpu")[0] for n in orders]


def test_ragged_fp32_bitwise_equals_dense():
    mats = _mats(ORDERS, 100)
    buf, orders, offs = pack(mats, device="cuda")
    info = torch.full((len(orders),), -5, dtype=torch.int32, device="cuda")
    plan = RaggedPlan(orders, offs, mode="fp32")
    out = plan.factor(buf, info=info)
    torch.cuda.synchronize()
    assert (info == 0).all()
    for m, l in zip(mats, unpack(out, orders, offs)):
        dense = cholesky(m.unsqueeze(0).cuda(), mode="fp32")[0]
        assert torch.equal(l, dense), m.shape
    for m, l in zip(mats, unpack(out, orders, offs)):
        ok, msg = oracle.check_implementation(m.unsqueeze(0).numpy(), l.unsqueeze(0).cpu().numpy())
        assert ok, (m.shape, msg)


@pytest.mark.parametrize("mode", ["bf16x3", "tf32"])
def test_ragged_tensor_modes_residual(mode):
    orders = ORDERS + [640, 1000]
    mats = [inputs.well_conditioned(1, n, seed=n, device="cpu")[0] for n in orders]
    buf, orders, offs = pack(mats, device="cuda")
    out = RaggedPlan(orders, offs, mode=mode, tc_min_n=200).factor(buf)
    tol = 1e-5 if mode == "bf16x3" else 1e-3
    for m, l in zip(mats, unpack(out, orders, offs)):
        ld, ad = l.double(), m.cuda().double()
        r = torch.linalg.norm(ld @ ld.T - ad) / torch.linalg.norm(ad)
        assert r.item() <= tol, (m.shape, r.item())
        assert (torch.triu(l, 1) == 0).all()


def test_ragged_graph_replay():
    orders = [8, 40, 150, 333]
    mats = _mats(orders, 7)
    buf, orders, offs = pack(mats, device="cuda")
    plan = RaggedPlan(orders, offs, mode="bf16x3")
    out = torch.zeros_like(buf)
    g = plan.capture(buf, out)
    out.zero_()
    g.replay()
    torch.cuda.synchronize()
    first = out.clone()
    mats2 = _mats(orders, 9)
    buf2, _, _ = pack(mats2, device="cuda")
    buf.copy_(buf2)
    g.replay()
    torch.cuda.synchronize()
    for m, l in zip(mats2, unpack(out, orders, offs)):
        ok, msg = oracle.check_implementation(m.unsqueeze(0).numpy(), l.unsqueeze(0).cpu().numpy())
        assert ok, msg
    assert not torch.equal(first, out)


def test_ragged_nonspd_info():
    orders = [20, 70, 190]
    mats = _mats(orders, 3)
    mats[2][100, 100] = -3.0
    buf, orders, offs = pack(mats, device="cuda")
    info = torch.zeros(3, dtype=torch.int32, device="cuda")
    RaggedPlan(orders, offs).factor(buf, info=info)
    want = [int(oracle.potrf_f64(m.unsqueeze(0).numpy())[1][0]) for m in mats]
    assert info.cpu().tolist() == want


def _identity_padded(m: torch.Tensor, p: int) -> torch.Tensor:
    n = m.shape[-1]
    out = torch.eye(p, dtype=torch.float32)
    out[:n, :n] = m
    return out


def test_ragged_dense_groups_bitwise_equal_padded_dense():
    """Tensor modes: a matrix of order n > 128 is factored as its identity-padded
    copy (order rounded up to 64) in a dense batch of all matrices sharing that
    padded order, so its factor equals the dense entry point's factor of the
    padded batch, bit for bit.  The workspace is filled with NaN first: the
    padded copies must not read anything the gather did not write."""
    orders = [200, 150, 256, 300, 1000, 1100, 1090, 40]
    mats = [inputs.generate_input(1, n, 2, 17 + n, "dense", device="cpu")[0] for n in orders]
    buf, orders, offs = pack(mats, device="cuda")
    # Pad steps of 64 and the split path above 1024: the groups are exactly
    # the batches the dense dispatcher would see.
    plan = RaggedPlan(orders, offs, mode="bf16x3", pad_step=64, pad_step_large=64, large_path="split")
    plan.workspace.fill_(0xFF)
    info = torch.full((len(orders),), -5, dtype=torch.int32, device="cuda")
    out = plan.factor(buf, info=info)
    torch.cuda.synchronize()
    assert (info == 0).all()
    groups: dict[int, list[int]] = {}
    for i, n in enumerate(orders):
        if n > 128:
            groups.setdefault((n + 63) // 64 * 64, []).append(i)
    ls = unpack(out, orders, offs)
    for p, idx in groups.items():
        batch = torch.stack([_identity_padded(mats[i], p) for i in idx]).cuda()
        dense = cholesky(batch, mode="bf16x3")
        for j, i in enumerate(idx):
            n = orders[i]
            assert torch.equal(ls[i], dense[j, :n, :n]), (n, p)
            assert torch.equal(dense[j, n:, n:], torch.eye(p - n, device="cuda")), (n, p)


def test_ragged_options_same_factors():
    """Stream count and the large-group path change the schedule, not the
    arithmetic of a group: factors are bitwise those of the one-stream plan
    with the same pad steps; graph capture works with several streams."""
    orders = [150, 150, 200, 300, 520, 640, 1000, 1100, 1300, 60, 20]
    mats = [inputs.well_conditioned(1, n, seed=3 * n, device="cpu")[0] for n in orders]
    buf, orders, offs = pack(mats, device="cuda")
    base = RaggedPlan(orders, offs, mode="bf16x3", large_path="fused_ws", streams=1).factor(buf)
    plan = RaggedPlan(orders, offs, mode="bf16x3", large_path="fused_ws", streams=4)
    out = torch.zeros_like(buf)
    g = plan.capture(buf, out)
    out.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, base)
    split = RaggedPlan(
        orders, offs, mode="bf16x3", pad_step=128, pad_step_large=256, large_path="split", streams=3
    ).factor(buf)
    for m, l in zip(mats, unpack(split, orders, offs)):
        ld, ad = l.double(), m.cuda().double()
        assert (torch.linalg.norm(ld @ ld.T - ad) / torch.linalg.norm(ad)).item() <= 1e-5


@pytest.mark.parametrize("mode", ["bf16x3", "tf32", "fp32"])
def test_ragged_nonspd_info_all_buckets(mode):
    orders = [20, 70, 190, 300, 640, 1090]
    mats = [inputs.well_conditioned(1, n, seed=n, device="cpu")[0] for n in orders]
    bad = {0: 7, 1: 33, 2: 100, 3: 299, 5: 1088}
    for i, j in bad.items():
        mats[i][j, j] = -3.0
    buf, orders, offs = pack(mats, device="cuda")
    info = torch.full((len(orders),), -5, dtype=torch.int32, device="cuda")
    RaggedPlan(orders, offs, mode=mode).factor(buf, info=info)
    want = [int(oracle.potrf_f64(m.unsqueeze(0).double().numpy())[1][0]) for m in mats]
    assert want[4] == 0 and all(want[i] == j + 1 for i, j in bad.items())
    assert info.cpu().tolist() == want


def test_config4_full_size():
    """3000 matrices, n log-uniform in [16, 2048]: every factor reconstructs its matrix."""
    orders = inputs.ragged_orders(3000, seed=4)
    buf, offs = inputs.ragged_batch(orders, seed=5, device="cuda")
    out = cholesky_ragged(buf, orders, offs[:-1], mode="bf16x3")
    worst = 0.0
    for n, o in zip(orders, offs[:-1]):
        l = out[o : o + n * n].view(n, n).double()
        a = buf[o : o + n * n].view(n, n).double()
        worst = max(worst, (torch.linalg.norm(l @ l.T - a) / torch.linalg.norm(a)).item())
    assert worst <= 1e-5


def test_autotune_picks_a_working_plan():
    """autotune times each candidate and returns the fastest plan, which
    factors the buffer like any other plan."""
    from gpumode_cholesky_b200.ragged import autotune

    orders = [20, 90, 150, 260, 300, 700, 1100]
    mats = [inputs.well_conditioned(1, n, seed=5 * n, device="cpu")[0] for n in orders]
    buf, orders, offs = pack(mats, device="cuda")
    cands = [
        {"pad_step": 64, "pad_step_large": 128, "large_path": "split", "streams": 1},
        {"pad_step": 128, "pad_step_large": 128, "large_path": "fused_ws", "streams": 2},
    ]
    plan, results = autotune(buf, orders, offs, mode="bf16x3", candidates=cands, reps=1)
    assert len(results) == 2 and all(us > 0 for _, us in results)
    best = min(results, key=lambda r: r[1])[0]
    assert plan.options.pad_step == best["pad_step"] and plan.options.streams == best["streams"]
    out = plan.factor(buf)
    for m, l in zip(mats, unpack(out, orders, offs)):
        ld, ad = l.double(), m.cuda().double()
        assert (torch.linalg.norm(ld @ ld.T - ad) / torch.linalg.norm(ad)).item() <= 1e-5


def test_host_plan_runs_match_device_plans():
    """RaggedHostPlan: host in, host out; each run equals its own device plan bit for bit."""
    from gpumode_cholesky_b200.ragged import RaggedHostPlan

    rng = np.random.default_rng(11)
    orders = [int(x) for x in np.exp(rng.uniform(np.log(16), np.log(700), 120)).astype(int)]
    mats = [inputs.well_conditioned(1, n, seed=n + 3 * i, device="cpu")[0] for i, n in enumerate(orders)]
    bad = 57
    mats[bad] = -mats[bad]  # not SPD
    host, orders, offs = pack(mats, device="cpu")
    host = host.pin_memory()
    plan = RaggedHostPlan(orders, offs, mode="bf16x3", parts=5)
    assert len(plan.runs) == 5
    info = torch.full((len(orders),), -4, dtype=torch.int32, device="cuda")
    out = torch.zeros_like(host).pin_memory()
    plan.factor(host, out, info=info, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    want = [int(oracle.potrf_f64(m.unsqueeze(0).numpy())[1][0]) for m in mats]
    assert info.cpu().tolist() == want
    dev = host.cuda()
    for i0, i1, e0, e1, p in plan.runs:
        ref = p.factor(dev[e0:e1]).cpu()
        for n, o in zip(orders[i0:i1], offs[i0:i1]):
            torch.testing.assert_close(out[o : o + n * n], ref[o - e0 : o - e0 + n * n], rtol=0, atol=0, equal_nan=True)
    for i, (m, l) in enumerate(zip(mats, unpack(out, orders, offs))):
        if i == bad:
            continue
        ld, ad = l.double(), m.double()
        assert (torch.linalg.norm(ld @ ld.T - ad) / torch.linalg.norm(ad)).item() <= 1e-5, m.shape
    # a blocking second call on pageable buffers gives the same factors
    again = plan.factor(host.clone())
    for x, y in zip(unpack(again, orders, offs), unpack(out, orders, offs)):
        torch.testing.assert_close(x, y, rtol=0, atol=0, equal_nan=True)
