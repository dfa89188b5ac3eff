"""A-posteriori training of the SGS MLP closure through the hand-written adjoint.

The LES advances u_{n+1} = Step(u_n, F(u_n; theta)) where F are the six
'tensor'-slot stresses of the MLP closure (sfsmodel_mlp), evaluated once per
step from the step's input like the reference's tensor SFS models
(src/data/domain.py:353-355).  The loss of a window of ``steps`` steps is the
mean squared error of the LES velocity against the filtered DNS at every step.
Its gradient runs backwards through

  * the time step: pyflow_b200.adjoint.ForwardStep (stage-exact RK4 adjoint,
    one checkpoint per step, RK stages recomputed), which also returns dL/dF;
  * the closure: MLPClosure below -- forward on the tensor cores
    (pf_mlp_closure), backward by recomputing the closure in torch with the
    kernel's BF16 roundings applied as straight-through estimators, then
    differentiating to the FP32 master weights and to the velocity.

Targets: a DNS on a grid ``factor`` times finer (same spectrum, its own seed),
advanced with ``factor`` substeps per LES step and reduced to the LES grid by
the staggered box restriction below.

The reference trains a different, 'source'-type network with an L1 objective
and RMSprop (src/sfsmodel/sfsmodel_ML.py:284-349, src/core/PyFlow.py:518-520);
this trainer uses the MSE objective and RMSprop on the MLP's FP32 weights.
"""
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import adjoint as A
from . import initial
from . import ops
from . import sfsmodel_mlp as M

PARAM_NAMES = ("W1", "b1", "W2", "b2", "W3", "b3")


def grad9(u, v, w, spacing):
    """The nine cell-centred velocity gradients (ux, uy, uz, vx, ..., wz) as
    differentiable torch ops, the same formulas as pf_sgs_closure's
    'gradients' model (metric_uniform.grad_vel_center,
    src/metric/metric_staggered.py:215-268) with periodic wrap."""
    dxi, dyi, dzi = (1.0 / h for h in spacing)

    def fwd(a, d):
        return torch.roll(a, -1, d)

    def bwd(a, d):
        return torch.roll(a, 1, d)

    def transverse(c, d, hi):
        return (0.5 * (fwd(c, d) + c) - 0.5 * (c + bwd(c, d))) * hi

    cu = 0.5 * (fwd(u, 0) + u)
    cv = 0.5 * (fwd(v, 1) + v)
    cw = 0.5 * (fwd(w, 2) + w)
    return torch.stack([
        (fwd(u, 0) - u) * dxi, transverse(cu, 1, dyi), transverse(cu, 2, dzi),
        transverse(cv, 0, dxi), (fwd(v, 1) - v) * dyi, transverse(cv, 2, dzi),
        transverse(cw, 0, dxi), transverse(cw, 1, dyi), (fwd(w, 2) - w) * dzi])


def box_restrict(u, v, w, factor):
    """Staggered box restriction of a fine periodic field to a grid ``factor``
    times coarser: a coarse face value is the mean of the fine face values
    covering that coarse face (factor x factor in the two transverse
    directions, at the coincident fine face).  The coarse field's discrete
    divergence is the mean of the fine divergence over each coarse cell, so a
    divergence-free field stays divergence free."""
    f = int(factor)
    nx, ny, nz = u.shape
    assert nx % f == 0 and ny % f == 0 and nz % f == 0
    X, Y, Z = nx // f, ny // f, nz // f
    uc = u[::f].reshape(X, Y, f, Z, f).mean(dim=(2, 4))
    vc = v[:, ::f].reshape(X, f, Y, Z, f).mean(dim=(1, 4))
    wc = w[:, :, ::f].reshape(X, f, Y, f, Z).mean(dim=(1, 3))
    return uc.contiguous(), vc.contiguous(), wc.contiguous()


def _ste_bf16(x):
    """BF16 rounding in the forward pass, identity in the backward pass."""
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


def _ste_bf16_trunc(x):
    """BF16 truncation (the kernel's pre-activations) in the forward pass,
    identity in the backward pass."""
    return x + (M._bf16_trunc(x).to(x.dtype) - x).detach()


def closure_torch(u, v, w, spacing, delta, W1, b1, W2, b2, W3, b3, rounding=True):
    """Torch restatement of the tensor-core closure: BF16 inputs, weights and
    hidden activations as straight-through roundings, FP32 accumulation.
    With rounding=False the same map is evaluated in FP64 without roundings
    (a smooth function of the weights, for finite-difference checks)."""
    g9 = grad9(u, v, w, spacing)
    g2 = torch.mean(g9 * g9)
    g_rms = torch.sqrt(g2)
    shape = u.shape
    x = g9.reshape(9, -1).T / g_rms
    if rounding:
        rnd, trn, dt = _ste_bf16, _ste_bf16_trunc, torch.float32
    else:
        rnd, trn, dt = (lambda t: t), (lambda t: t), torch.float64
    W1, b1, W2, b2, W3, b3 = (t.to(dt) for t in (W1, b1, W2, b2, W3, b3))
    x = rnd(x.to(dt))
    h1 = rnd(torch.tanh(trn(x @ rnd(W1).T + b1)))
    h2 = rnd(torch.tanh(trn(h1 @ rnd(W2).T + b2)))
    y = h2 @ rnd(W3).T + b3
    F = y.to(torch.float64) * ((delta * delta) * g2)
    return F.T.reshape((6,) + tuple(shape)).contiguous()


class MLPClosure(torch.autograd.Function):
    """F(u, v, w; W1..b3): forward on the tensor cores, backward through
    closure_torch."""

    @staticmethod
    def forward(ctx, u, v, w, W1, b1, W2, b2, W3, b3, spacing, delta):
        params = {k: t.detach().float().cpu().numpy()
                  for k, t in zip(PARAM_NAMES, (W1, b1, W2, b2, W3, b3))}
        wpack = torch.as_tensor(M.pack(params)).to(u.device)
        out, _, _, err = M.closure(u.detach().contiguous(), v.detach().contiguous(),
                                   w.detach().contiguous(), spacing, wpack, delta)
        if int(err.item()) != 0:
            raise RuntimeError("pf_mlp_closure: a tensor-core wait timed out")
        ctx.save_for_backward(u, v, w, W1, b1, W2, b2, W3, b3)
        ctx.cfg = (tuple(spacing), float(delta))
        return out

    @staticmethod
    def backward(ctx, gout):
        saved = ctx.saved_tensors
        spacing, delta = ctx.cfg
        with torch.enable_grad():
            leaves = [t.detach().requires_grad_(True) for t in saved]
            F = closure_torch(leaves[0], leaves[1], leaves[2], spacing, delta, *leaves[3:])
            grads = torch.autograd.grad(F, leaves, gout.contiguous())
        return tuple(grads) + (None, None)


def mse(a, b):
    return sum(torch.mean((x - y) ** 2) for x, y in zip(a, b)) / 3.0


@dataclass
class LESConfig:
    """LES with the ML closure trained against filtered DNS (64^3, nu = 0.001,
    dt = 0.005, 20-step window; DNS 256^3, seed 2)."""
    n: int = 64
    factor: int = 4
    nu: float = 0.001
    dt: float = 0.005
    steps: int = 20
    k0: float = 4.0
    urms: float = 1.0
    dns_seed: int = 2
    mlp_seed: int = 1
    # RMSprop's first steps move every weight by about 10 lr: 1e-4 keeps the
    # closure's stresses (scaled by Delta^2 <|grad u|^2>) small against the
    # viscous terms at nu = 0.001
    lr: float = 1e-4
    tol: float = 1e-12
    dns_prec: str = "fp64"


def dns_targets(cfg, device="cuda"):
    """Filtered DNS velocity at the start and after every LES step
    (steps + 1 snapshots on the LES grid)."""
    nf = cfg.n * cfg.factor
    sp = (2 * math.pi / nf,) * 3
    u, v, w = (t.contiguous() for t in initial.spectral_velocity_device(
        (nf, nf, nf), k0=cfg.k0, urms=cfg.urms, seed=cfg.dns_seed, device=device))
    p = torch.zeros_like(u)
    DP = torch.zeros_like(u)
    out = [box_restrict(u, v, w, cfg.factor)]
    sub = cfg.dt / cfg.factor
    for _ in range(cfg.steps):
        for _ in range(cfg.factor):
            info = ops.forward_step(u, v, w, p, DP, sp, cfg.nu, 1.0, sub, min_res=1e-10,
                                    max_it=20000, prec=cfg.dns_prec)
            if info.status != 0:
                raise RuntimeError("DNS pressure solve failed (status %d)" % info.status)
        out.append(box_restrict(u, v, w, cfg.factor))
    del u, v, w, p, DP
    return out


class Trainer:
    """RMSprop on the closure's FP32 weights; one call to ``step`` runs the
    LES window forward, the adjoint backward and one optimizer update."""

    def __init__(self, cfg, targets, params=None, device="cuda", closure="kernel",
                 dtype=torch.float32):
        """closure: 'kernel' (tensor-core forward) or 'fp64' (the closure's
        torch restatement in FP64 without BF16 roundings); dtype: type of the
        master weights."""
        self.cfg = cfg
        self.closure = closure
        self.targets = targets
        self.spacing = (2 * math.pi / cfg.n,) * 3
        self.delta = self.spacing[0]
        p0 = params if params is not None else M.xavier_init(cfg.mlp_seed)
        self.params = [torch.tensor(np.asarray(p0[k]), dtype=dtype, device=device,
                                    requires_grad=True) for k in PARAM_NAMES]
        self.opt = torch.optim.RMSprop(self.params, lr=cfg.lr)
        self.history = []
        self.skipped = 0   # windows whose gradient was not finite (no update)

    def loss(self):
        cfg = self.cfg
        u, v, w = (t.clone() for t in self.targets[0])
        total = 0.0
        for n in range(cfg.steps):
            if self.closure == "kernel":
                F = MLPClosure.apply(u, v, w, *self.params, self.spacing, self.delta)
            else:
                F = closure_torch(u, v, w, self.spacing, self.delta, *self.params,
                                  rounding=False)
            u, v, w = A.forward_step(u, v, w, self.spacing, cfg.nu, 1.0, cfg.dt, sfs=F,
                                     rk4=True, tol=cfg.tol)
            total = total + mse((u, v, w), self.targets[n + 1])
        return total / cfg.steps

    def step(self):
        """One window: forward, backward, update.  A window whose loss or
        gradient is not finite updates nothing (counted in ``skipped``) and
        reports its loss."""
        self.opt.zero_grad(set_to_none=True)
        L = self.loss()
        val = float(L.detach())
        if math.isfinite(val):
            try:
                L.backward()
                finite = all(bool(torch.isfinite(p.grad).all())
                             for p in self.params if p.grad is not None)
            except RuntimeError:
                finite = False   # a non-finite adjoint field stopped the backward pass
            if finite:
                self.opt.step()
            else:
                self.skipped += 1
        self.history.append(val)
        return val

    def state_dict(self):
        return {k: t.detach().cpu().numpy() for k, t in zip(PARAM_NAMES, self.params)}
