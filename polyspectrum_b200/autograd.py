"""torch.autograd binding of the estimator (test / analysis helper).

``polyspectrum(field, ctx, cfg, method, use_only_phase)`` returns B of one
configuration as a 0-d float64 tensor; its backward calls ps_gpu_grad, which
evaluates dB/d(delta) = V^(n-1) N^(-3n) / sum_I * sum_i IFFT[F_i FFT[prod_{j!=i} D_j]]
on the GPU (through the transpose of d(z/|z|) per mode for phase-only fields).
The field is the real input grid (what get_FT_field transforms, DENS slot).
"""
from __future__ import annotations

import torch

from . import PS_FIELD_DENS, PS_FP64_PLAIN, Context


class _Polyspectrum(torch.autograd.Function):
    @staticmethod
    def forward(fctx, field: torch.Tensor, ctx: Context, cfg, method: int, use_only_phase: int):
        f = field.detach().contiguous()
        if use_only_phase:
            ctx.keep_modulus(True)
        ctx.get_FT_field(PS_FIELD_DENS, f, use_only_phase=use_only_phase)
        B, _, _, _ = ctx.batch([cfg], method)
        fctx.ctx = ctx
        fctx.cfg = cfg
        fctx.method = method
        fctx.phase = use_only_phase
        fctx.save_for_backward(f)
        return torch.tensor(float(B[0]), dtype=torch.float64, device=field.device)

    @staticmethod
    def backward(fctx, gout: torch.Tensor):
        (f,) = fctx.saved_tensors
        ctx, cfg = fctx.ctx, fctx.cfg
        ctx.get_FT_field(PS_FIELD_DENS, f, use_only_phase=fctx.phase)  # the field this B was taken on
        g = torch.empty_like(f)
        n = cfg.n
        ctx.grad(n, [cfg.k[i] for i in range(n)], [cfg.kmin[i] for i in range(n)],
                 [cfg.kmax[i] for i in range(n)], cfg.kbinwidth, cfg.kbinningCase,
                 method=fctx.method, out=g)
        return gout.to(g.dtype) * g, None, None, None, None


def polyspectrum(field: torch.Tensor, ctx: Context, cfg, method: int = PS_FP64_PLAIN,
                 use_only_phase: int = 0) -> torch.Tensor:
    """B of configuration `cfg` (a ps_cfg) on `field`, differentiable in `field`."""
    return _Polyspectrum.apply(field, ctx, cfg, method, use_only_phase)
