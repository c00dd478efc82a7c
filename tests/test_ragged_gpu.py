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
