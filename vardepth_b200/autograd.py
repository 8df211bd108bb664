"""Differentiable PairHMM log-likelihood: a torch.autograd.Function over the C ABI.

The reference scores reads with fixed penalties only (gap 0.001 / ext 0.1 in
caller/native/caller/batch_hmm.cpp:42-97, the caller's Q45/Q10 settings); this
module adds what the fixed drop-in does not have: the gradient of ln L with
respect to the indel and base-error model, so the model can be fitted to a
sample's own reads.  The parameters are six Phred-scale scalars

    theta = (Qg, Qx, o0, o1, o2, o3)
    gap-open g = 10^(-Qg/10), gap-continuation x = 10^(-Qx/10),
    base error 10^(-max(0, min(q,60) + o_bin(q))/10), bins q<15, q<25, q<35, q>=35.

``PairHMMLogLik.apply(theta, batch)`` returns ln L of every output of the
batch (float64, the output order of vd_forward).  When theta requires a
gradient the forward pass runs vd_forward_backward, which returns ln L and the
per-pair Jacobian d ln L / d theta in one reverse-wavefront sweep (sqrt-L
checkpointing by default); the backward pass is grad_output @ Jacobian.
Without a gradient it runs the plain forward (vd_forward).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import native

THETA_NAMES = ("gap_open_phred", "gap_continuation_phred", "offset_q_lt15", "offset_q_lt25", "offset_q_lt35",
               "offset_q_ge35")


def params_from_theta(theta: np.ndarray, precision: int = native.VD_PRECISION_MIXED, anchored: bool = False):
    """vd_params for theta = (Qg, Qx, o0..o3)."""
    t = np.asarray(theta, np.float64)
    if t.shape != (6,):
        raise ValueError("theta must hold 6 values (Qg, Qx, o0, o1, o2, o3)")
    return native.make_params(10.0 ** (-t[0] / 10.0), 10.0 ** (-t[1] / 10.0), anchored, precision,
                              quality_offsets=t[2:6])


class Batch:
    """A packed region or pair batch bound to an engine, for repeated likelihood calls."""

    def __init__(self, engine: native.Engine, packed: native.Packed, precision: int = native.VD_PRECISION_MIXED,
                 checkpoint: int = native.VD_CHECKPOINT_SQRT, anchored: bool = False):
        self.engine = engine
        self.packed = packed
        self.precision = precision
        self.checkpoint = checkpoint
        self.anchored = anchored
        self.last_stats = None

    def loglik(self, theta: np.ndarray) -> np.ndarray:
        params, _keep = params_from_theta(theta, self.precision, self.anchored)
        out, st = self.engine.forward(self.packed, params)
        self.last_stats = st
        return out

    def loglik_and_jacobian(self, theta: np.ndarray):
        params, _keep = params_from_theta(theta, self.precision, self.anchored)
        ln, jac, st = self.engine.forward_backward(self.packed, params, self.checkpoint)
        self.last_stats = st
        return ln, jac


class PairHMMLogLik(torch.autograd.Function):
    """ln L per pair as a differentiable function of theta (a 6-element tensor)."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, batch: Batch) -> torch.Tensor:
        th = theta.detach().to("cpu", torch.float64).numpy()
        ctx.theta_dtype = theta.dtype
        if ctx.needs_input_grad[0]:
            ln, jac = batch.loglik_and_jacobian(th)
            ctx.save_for_backward(torch.from_numpy(jac).to(theta.device),
                                  torch.from_numpy(np.isfinite(ln)).to(theta.device))
        else:
            ln = batch.loglik(th)
        return torch.from_numpy(ln).to(theta.device)

    @staticmethod
    def backward(ctx, grad_ln: torch.Tensor):
        jac, finite = ctx.saved_tensors
        # empty reads or haplotypes give -inf with a zero Jacobian row: their
        # upstream gradient (often NaN after -inf arithmetic) is dropped
        g = torch.where(finite, grad_ln.to(jac.dtype), torch.zeros((), dtype=jac.dtype, device=jac.device))
        return (g @ jac).to(ctx.theta_dtype), None


def loglik(theta: torch.Tensor, batch: Batch) -> torch.Tensor:
    """ln L of every output of the batch, differentiable in theta."""
    return PairHMMLogLik.apply(theta, batch)


def region_mixture_loglik(ln: torch.Tensor, region_read_off: np.ndarray, region_hap_off: np.ndarray) -> torch.Tensor:
    """sum over reads of ln(mean over the region's haplotypes of L): each read comes from one
    haplotype of its region, which is not known, with a uniform prior."""
    rr = np.diff(np.asarray(region_read_off, np.int64))
    hh = np.diff(np.asarray(region_hap_off, np.int64))
    total = ln.new_zeros(())
    o = 0
    # regions with the same haplotype count are reduced together
    groups: dict[int, list[tuple[int, int]]] = {}
    for g in range(len(rr)):
        k = int(rr[g] * hh[g])
        if k:
            groups.setdefault(int(hh[g]), []).append((o, k))
        o += k
    for H, spans in groups.items():
        idx = torch.from_numpy(np.concatenate([np.arange(a, a + k) for a, k in spans])).to(ln.device)
        rows = ln.index_select(0, idx).view(-1, H)
        total = total + (torch.logsumexp(rows, dim=1) - math.log(H)).sum()
    return total


def fit_error_model(batch: Batch, region_read_off, region_hap_off, theta0, max_iter: int = 60,
                    tolerance: float = 1e-7, history: list | None = None) -> torch.Tensor:
    """Maximise the region mixture log-likelihood over theta with L-BFGS (float32 parameters)."""
    theta = torch.tensor(np.asarray(theta0, np.float32), requires_grad=True)
    opt = torch.optim.LBFGS([theta], lr=1.0, max_iter=max_iter, tolerance_grad=tolerance,
                            tolerance_change=1e-9, history_size=20, line_search_fn="strong_wolfe")
    scale = 1.0 / max(1, int(np.sum(np.diff(np.asarray(region_read_off)))))

    def closure():
        opt.zero_grad()
        ln = loglik(theta, batch)
        loss = -region_mixture_loglik(ln, region_read_off, region_hap_off) * scale
        loss.backward()
        if history is not None:
            history.append((float(loss.detach()), theta.detach().clone().numpy()))
        return loss

    opt.step(closure)
    return theta.detach()
