"""Generates the golden fixtures in this directory from the reference itself.

Run where a checkout of the reference exists, naming its root:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_golden.py

For every case it calls the reference's own ``generate_input`` and
``check_implementation`` (reference/reference.py:37-188) and its entry point
``custom_kernel`` (submission.py:4101-4268), which on a CPU-only host routes to
``torch.linalg.cholesky_ex`` -- the same values as ``ref_kernel``
(reference/reference.py:129-130).  It stores the input, the reference's L,
the LAPACK info vector and the checker's verdict and message in
``cases.npz``.  ``backward.npz`` holds FP64 torch-autograd gradients of the
Cholesky factor for the adjoint tests (the reference has no backward).
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
if "REFERENCE_ROOT" not in os.environ:
    sys.exit("set REFERENCE_ROOT to the root of the reference checkout")
REF = Path(os.environ["REFERENCE_ROOT"])

# (batch, n, cond, seed, case): the reference's own test specs
# (scripts/_gpu_runner.py:40-109) at reduced batch, plus edge orders.
CASES = [
    (16, 32, 2, 53124, "dense"),
    (8, 64, 2, 53125, "dense"),
    (4, 128, 2, 3321, "dense"),
    (1, 256, 2, 94010, "dense"),
    (4, 128, 5, 1200, "spectrum"),
    (4, 128, 5, 1201, "diagonal"),
    (1, 256, 4, 32524, "lowrank"),
    (1, 160, 4, 32525, "rowscale"),
    (1, 160, 1, 32526, "tridiagonal"),
    (16, 32, 5, 90001, "spectrum"),
    (16, 32, 5, 90002, "diagonal"),
    (16, 32, 4, 90003, "lowrank"),
    (16, 32, 4, 90004, "rowscale"),
    (16, 32, 1, 90005, "tridiagonal"),
    (8, 64, 5, 95129, "spectrum"),
    (8, 64, 4, 95131, "lowrank"),
    (8, 64, 4, 95132, "rowscale"),
    (8, 64, 1, 95133, "tridiagonal"),
    # edge orders: 1, tiny, odd, warp/CTA/blocked boundaries
    (3, 1, 2, 11, "dense"),
    (3, 2, 2, 12, "dense"),
    (5, 3, 2, 13, "dense"),
    (4, 17, 2, 14, "dense"),
    (4, 31, 2, 15, "dense"),
    (4, 33, 2, 16, "dense"),
    (3, 65, 2, 17, "dense"),
    (2, 100, 2, 18, "dense"),
    (2, 127, 2, 19, "dense"),
    (2, 129, 2, 20, "dense"),
    (1, 193, 2, 21, "dense"),
    (1, 300, 2, 22, "dense"),
]


def main() -> None:
    sys.path.insert(0, str(REF / "reference"))
    sys.path.insert(0, str(REF))
    from reference import check_implementation, generate_input  # noqa: E402
    from submission import custom_kernel  # noqa: E402

    torch.set_num_threads(max(1, os.cpu_count() or 1))
    arrays: dict[str, np.ndarray] = {}
    meta = []
    for idx, (batch, n, cond, seed, case) in enumerate(CASES):
        a = generate_input(batch=batch, n=n, cond=cond, seed=seed, case=case)
        l = custom_kernel(a.clone())
        ex = torch.linalg.cholesky_ex(a, check_errors=False)
        assert torch.equal(l, ex.L), "reference custom_kernel on CPU must equal ref_kernel"
        ok, msg = check_implementation(a, l)
        arrays[f"a{idx}"] = a.numpy()
        arrays[f"l{idx}"] = l.numpy()
        arrays[f"info{idx}"] = ex.info.numpy().astype(np.int32)
        meta.append({"batch": batch, "n": n, "cond": cond, "seed": seed, "case": case, "ok": bool(ok), "message": msg})
        print(idx, batch, n, case, ok, msg)
    # One non-SPD case: LAPACK stops at the first bad pivot and reports info.
    a = generate_input(batch=2, n=32, cond=2, seed=77, case="dense")
    a[1, 5, 5] = -1.0
    ex = torch.linalg.cholesky_ex(a, check_errors=False)
    arrays["nonspd_a"] = a.numpy()
    arrays["nonspd_info"] = ex.info.numpy().astype(np.int32)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "cases.npz", **arrays)

    # Backward: FP64 torch autograd of L = cholesky(A) against random Lbar.
    bw: dict[str, np.ndarray] = {}
    gen = torch.Generator().manual_seed(1234)
    for idx, n in enumerate([1, 5, 32, 48, 96, 130]):
        m = torch.randn((2, n, n), dtype=torch.float64, generator=gen)
        a = (m @ m.transpose(-1, -2)) / n + torch.eye(n, dtype=torch.float64)
        a = (0.5 * (a + a.transpose(-1, -2))).requires_grad_(True)
        lbar = torch.randn((2, n, n), dtype=torch.float64, generator=gen).tril()
        lfac = torch.linalg.cholesky(a)
        (g,) = torch.autograd.grad(lfac, a, lbar)
        bw[f"a{idx}"] = a.detach().numpy()
        bw[f"l{idx}"] = lfac.detach().numpy()
        bw[f"lbar{idx}"] = lbar.numpy()
        bw[f"abar{idx}"] = g.numpy()
    np.savez_compressed(HERE / "backward.npz", **bw)


if __name__ == "__main__":
    main()
