"""SGS MLP closure in the reference's 'tensor' SFS slot.

The model has no reference code: the reference's ML closure
(src/sfsmodel/sfsmodel_ML.py) is a 'source'-type network.  This one maps the
nine cell-centred velocity gradients (normalised by their RMS, g_rms) through
9 -> 128 (tanh) -> 128 (tanh) -> 6 to the stresses FXX, FYY, FZZ, FXY, FXZ,
FYZ, scaled by Delta^2 g_rms^2 like the gradient model's Delta^2/12 du du
(src/sfsmodel/sfsmodel_gradient.py:70-148), and plugs into the velocity RHS
exactly where the gradient model does (src/solver/velocity.py:262-267,...).
BF16 weights, FP32 accumulation, Xavier-uniform weights and zero biases from
seed 1.  The forward pass runs on the tensor cores (pf_mlp_closure).
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import ops

HIDDEN = 128
N_IN, N_OUT = 9, 6


def xavier_init(seed=1):
    """Xavier-uniform weights (torch.nn.init.xavier_uniform_ convention,
    bound sqrt(6/(fan_in+fan_out))) and zero biases, from numpy seed ``seed``."""
    rng = np.random.default_rng(seed)

    def xav(o, i):
        b = np.sqrt(6.0 / (i + o))
        return rng.uniform(-b, b, size=(o, i)).astype(np.float32)

    return dict(W1=xav(HIDDEN, N_IN), b1=np.zeros(HIDDEN, np.float32),
                W2=xav(HIDDEN, HIDDEN), b2=np.zeros(HIDDEN, np.float32),
                W3=xav(N_OUT, HIDDEN), b3=np.zeros(N_OUT, np.float32))


def _bf16_bits(a):
    t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16)
    return t.view(torch.int16).numpy().view(np.uint16)


def _kmajor_offsets(rows, cols, slice_bytes):
    r = np.arange(rows)[:, None]
    k = np.arange(cols)[None, :]
    return ((k >> 4) * slice_bytes + (r >> 3) * 256 + ((k >> 3) & 1) * 128 +
            (r & 7) * 16 + (k & 7) * 2)


def pack(params):
    """The packed device image read by pf_mlp_closure: W1 (128x16, inputs
    padded 9 -> 16), W2 (128x128), W3 (16x128, outputs padded 6 -> 16) as BF16
    in the K-major no-swizzle UMMA layout, then b1, b2, b3 (padded to 16) as
    float32."""
    size = L.lib().pf_mlp_pack_bytes()
    buf = np.zeros(size, np.uint8)
    W1 = np.zeros((HIDDEN, 16), np.float32); W1[:, :N_IN] = params["W1"]
    W3 = np.zeros((16, HIDDEN), np.float32); W3[:N_OUT] = params["W3"]
    base = 0
    for W, rows, cols, sl in ((W1, 128, 16, 4096), (params["W2"], 128, 128, 4096),
                              (W3, 16, 128, 512)):
        off = _kmajor_offsets(rows, cols, sl) + base
        bits = _bf16_bits(W)
        buf[off] = (bits & 0xFF).astype(np.uint8)
        buf[off + 1] = (bits >> 8).astype(np.uint8)
        base += rows * cols * 2
    b3 = np.zeros(16, np.float32); b3[:N_OUT] = params["b3"]
    bias = np.concatenate([params["b1"], params["b2"], b3]).astype(np.float32)
    buf[base:base + bias.nbytes] = bias.view(np.uint8)
    assert base + bias.nbytes == size
    return buf


def _bf16(x):
    return x.to(torch.bfloat16).to(torch.float32)


def _bf16_trunc(x):
    """FP32 -> BF16 by truncation (the kernel keeps the high half of each
    pre-activation), back to FP32."""
    return torch.bitwise_and(x.float().contiguous().view(torch.int32), -65536).view(torch.float32)


def reference_forward(grads, params, in_scale, out_scale):
    """Torch model of the tensor-core forward pass: BF16 inputs and weights,
    FP32 accumulation, pre-activations truncated to BF16 before tanh, BF16
    hidden activations.  grads: (9, n) float64 tensor."""
    dev = grads.device
    x = _bf16((grads.T.to(torch.float32) * in_scale))
    W1 = _bf16(torch.as_tensor(params["W1"], device=dev))
    W2 = _bf16(torch.as_tensor(params["W2"], device=dev))
    W3 = _bf16(torch.as_tensor(params["W3"], device=dev))
    b1, b2, b3 = (torch.as_tensor(params[k], device=dev) for k in ("b1", "b2", "b3"))
    h1 = _bf16(torch.tanh(_bf16_trunc(x @ W1.T + b1)))
    h2 = _bf16(torch.tanh(_bf16_trunc(h1 @ W2.T + b2)))
    y = h2 @ W3.T + b3
    return (y.to(torch.float64) * out_scale).T.contiguous()


_scales_ws = {}


def closure(u, v, w, spacing, wpack, delta, out=None, err=None, grads=False):
    """Run the tensor-core closure; returns (stresses (6,nx,ny,nz) float64,
    the nine gradients (9,nx,ny,nz) when ``grads`` else None, scales, err).
    The input normalisation uses the RMS of the nine gradients: scales =
    [1/g_rms, delta^2 g_rms^2] from pf_mlp_scales (FP64 mean square in a
    fixed order, rounded once to float), the same kernel a step plan with
    this closure runs."""
    g = ops.grid(u.shape, spacing)
    dev = u.device
    ws = _scales_ws.get(dev)
    if ws is None:
        ws = torch.empty(L.lib().pf_mlp_scales_workspace_bytes(), dtype=torch.uint8, device=dev)
        _scales_ws[dev] = ws
    scales = torch.empty(2, dtype=torch.float32, device=dev)
    L.check("pf_mlp_scales", L.lib().pf_mlp_scales(
        ctypes.byref(g), ops._p(u), ops._p(v), ops._p(w), float(delta) * float(delta),
        ops._p(scales), ops._p(ws), ws.numel(), ops._stream(u)))
    shape = (6,) + tuple(u.shape)
    if out is None or tuple(out.shape) != shape:
        out = torch.empty(shape, dtype=torch.float64, device=dev)
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=dev)
    L.check("pf_mlp_closure", L.lib().pf_mlp_closure(
        ctypes.byref(g), ops._p(u), ops._p(v), ops._p(w), ops._p(wpack),
        ops._p(scales), ops._p(out), ops._p(err), ops._stream(u)))
    g9 = ops.sgs_closure("gradients", u, v, w, spacing) if grads else None
    return out, g9, scales, err


class residual_stress:
    """'tensor'-type SFS model object (same interface as
    sfsmodel_gradient.residual_stress)."""

    def __init__(self, inputConfig, decomp, geo, params=None):
        self.modelType = "tensor"
        self.spacing = (geo.dx, geo.dy, geo.dz)
        self.Delta = geo.dx * getattr(inputConfig, "expFilterFac", 1.0)
        self.params = params if params is not None else xavier_init(
            getattr(inputConfig, "mlpSeed", 1))
        self.set_params(self.params)
        self.stacked = None
        self.err = torch.zeros(1, dtype=torch.int32, device=decomp.device)
        self.epoch = 0

    def set_params(self, params):
        self.params = params
        self.wpack = torch.as_tensor(pack(params)).cuda()

    def update(self, state_u, state_v, state_w, metric=None):
        out, g9, scales, _ = closure(state_u.interior(), state_v.interior(),
                                     state_w.interior(), self.spacing, self.wpack,
                                     self.Delta, out=self.stacked, err=self.err)
        self.stacked = out
        (self.FXX, self.FYY, self.FZZ, self.FXY, self.FXZ, self.FYZ) = out.unbind(0)

    def check(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("pf_mlp_closure: a tensor-core wait timed out")

    def save(self, path="mlp_closure.pt"):
        torch.save({k: torch.as_tensor(v) for k, v in self.params.items()}, path)

    def finalize(self, comms=None):
        pass
