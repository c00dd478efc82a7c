"""Output checker on the tensors' own device (GPU at full size).

Restates the reference's gate for ``custom_kernel`` outputs
(reference/reference.py:132-188) with torch on the device the data lives on,
so a 1 x 32768 factor is checked in seconds instead of minutes of CPU time:

  * the output has the input's shape, FP32 dtype and device, and is finite;
  * ||triu(L, 1)||_1 <= 8 * n * eps * ||A||_1 (lower triangular);
  * every diagonal entry is > 0;
  * ||L L^T - A||_1 <= 20 * n * eps * ||A||_1 (reconstruction),

with eps the FP32 machine epsilon and ||.||_1 the matrix 1-norm (largest
column absolute sum), per matrix.  Verdicts and messages have the reference
checker's form, so they compare with its own.

``precision="fp32"`` forms L L^T in FP32 with TF32 off, as the reference
does.  ``precision="fp64"`` forms it in FP64, where the products of FP32
entries are exact, so the residual is the factor's own and not the check's
rounding.  The batch is processed in slices of about ``slice_bytes`` of
input, which bounds the FP64 temporaries at large orders.
"""

from __future__ import annotations

import torch

TRIANGULAR_FACTOR = 8.0
RECONSTRUCTION_FACTOR = 20.0
_EPS32 = float(torch.finfo(torch.float32).eps)
_TINY32 = float(torch.finfo(torch.float32).tiny)


def _col_abs_max(x: torch.Tensor) -> torch.Tensor:
    """Matrix 1-norm per matrix: the largest column absolute sum."""
    return x.abs().sum(dim=-2).amax(dim=-1)


def residual_norms(
    data: torch.Tensor, output: torch.Tensor, precision: str = "fp32", slice_bytes: int = 1 << 30
) -> dict[str, torch.Tensor]:
    """Per-matrix norms the checker gates on, on the data's device (FP64 results).

    Keys: ``a_l1`` (||A||_1), ``upper_l1`` (||triu(L,1)||_1), ``resid_l1``
    (||L L^T - A||_1), ``rel_fro`` (||L L^T - A||_F / ||A||_F), ``min_diag``
    and ``finite`` (1.0 when every entry of L is finite).
    """
    if precision not in ("fp32", "fp64"):
        raise ValueError(f"precision must be fp32 or fp64, not {precision!r}")
    if data.dim() != 3 or data.shape != output.shape:
        raise ValueError("data and output must both be (batch, n, n)")
    batch, n, _ = data.shape
    step = max(1, int(slice_bytes // max(1, n * n * 4)))
    keys = ("a_l1", "upper_l1", "resid_l1", "rel_fro", "min_diag", "finite")
    out = {k: torch.empty(batch, dtype=torch.float64, device=data.device) for k in keys}
    saved = torch.backends.cuda.matmul.allow_tf32
    try:
        torch.backends.cuda.matmul.allow_tf32 = False
        for b0 in range(0, batch, step):
            a = data[b0 : b0 + step]
            l = output[b0 : b0 + step]
            sl = slice(b0, b0 + a.shape[0])
            out["finite"][sl] = torch.isfinite(l).flatten(1).all(dim=1).double()
            out["a_l1"][sl] = _col_abs_max(a).double()
            out["upper_l1"][sl] = _col_abs_max(torch.triu(l, diagonal=1)).double()
            out["min_diag"][sl] = torch.diagonal(l, dim1=-2, dim2=-1).amin(dim=-1).double()
            if precision == "fp64":
                ld = l.double()
                r = torch.matmul(ld, ld.transpose(-1, -2))
                del ld
                r -= a.double()
            else:
                r = torch.matmul(l, l.transpose(-1, -2))
                r -= a
            out["resid_l1"][sl] = _col_abs_max(r).double()
            fro_r = torch.linalg.matrix_norm(r).double()
            del r
            out["rel_fro"][sl] = fro_r / torch.linalg.matrix_norm(a.double()).clamp_min(_TINY32)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = saved
    return out


def check(data: torch.Tensor, output, precision: str = "fp32") -> tuple[bool, str]:
    """The reference's verdict for ``output`` as the factor of ``data``: (ok, message)."""
    if not isinstance(output, torch.Tensor):
        return False, "output must be a torch.Tensor"
    if output.shape != data.shape:
        return False, f"output shape must be {tuple(data.shape)}, got {tuple(output.shape)}"
    if output.dtype != torch.float32:
        return False, f"output dtype must be torch.float32, got {output.dtype}"
    if output.device != data.device:
        return False, f"output must be on {data.device}, got {output.device}"
    batch, n, _ = data.shape
    nrm = residual_norms(data, output, precision)
    if not bool((nrm["finite"] > 0).all()):
        return False, "output contains NaN or Inf"
    scale = nrm["a_l1"].float().clamp_min(_TINY32).double()
    nn = max(n, 1)
    tri = nrm["upper_l1"]
    if bool((tri > TRIANGULAR_FACTOR * nn * _EPS32 * scale).any()):
        return False, f"output is not lower triangular enough: relative_residual={float((tri / scale).max()):.3g}"
    if bool((nrm["min_diag"] <= 0).any()):
        return False, "output diagonal must be strictly positive"
    res = nrm["resid_l1"]
    if bool((res > RECONSTRUCTION_FACTOR * nn * _EPS32 * scale).any()):
        return False, f"L @ L.T does not reconstruct A: relative_residual={float((res / scale).max()):.3g}"
    scaled = float((res / (_EPS32 * nn * scale)).max())
    return True, f"scaled_reconstruction_residual={scaled:.3g}; batch={batch}; n={n}"
