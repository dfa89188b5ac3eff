"""The tensor-core SGS MLP closure (pf_mlp_closure) against two torch models:

* a model of the same arithmetic (BF16 inputs and weights, FP32 accumulation,
  BF16 pre-activations and activations).  Tolerance: 3e-2 of the output range
  at any cell and 1e-2 at 90 % of the cells -- the kernel's hardware tanh
  (tanh.approx.bf16x2) and the tensor core's FP32 summation order can flip
  the BF16 rounding of a hidden activation, which moves an output by a few
  BF16 ulps of its inputs;
* the FP64 model (the network with the same BF16-valued weights evaluated in
  FP64 without roundings): the closure's error against exact arithmetic.
  Tolerance: 5e-2 of the output range at any cell, 1.5e-2 in RMS.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 20, 36), (5, 7, 9)])
def test_mlp_closure_matches_bf16_model(shape):
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    import pyflow_b200.sfsmodel_mlp as M
    sp = tuple(2 * np.pi / n for n in shape)
    u, v, w = (torch.tensor(a, device="cuda") for a in
               ic.spectral_velocity(shape, k0=3.0, seed=4))
    params = M.xavier_init(1)
    rng = np.random.default_rng(7)
    for k in ("b1", "b2", "b3"):
        params[k] = (0.1 * rng.standard_normal(params[k].shape)).astype(np.float32)
    wpack = torch.as_tensor(M.pack(params)).cuda()
    out, g9, scales, err = M.closure(u, v, w, sp, wpack, delta=sp[0], grads=True)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = M.reference_forward(g9.reshape(9, -1), params, float(scales[0]),
                              float(scales[1])).reshape(out.shape)
    got = out
    scale = ref.abs().max().item()
    assert scale > 0
    err_max = (got - ref).abs().max().item()
    assert err_max <= 3e-2 * scale, (err_max, scale)
    # most cells agree to about one BF16 ulp of the hidden activations: the
    # hardware's packed BF16 tanh and torch's tanh rounded to BF16 differ by
    # one ulp on a fraction of the activations
    close = ((got - ref).abs() <= 1e-2 * scale).double().mean().item()
    assert close > 0.9, close


@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 20, 36)])
def test_mlp_closure_vs_fp64_model(shape):
    import pyflow_b200.initial as ic
    import pyflow_b200.sfsmodel_mlp as M
    sp = tuple(2 * np.pi / n for n in shape)
    u, v, w = (torch.tensor(a, device="cuda") for a in
               ic.spectral_velocity(shape, k0=3.0, seed=5))
    params = M.xavier_init(1)
    rng = np.random.default_rng(8)
    for k in ("b1", "b2", "b3"):
        params[k] = (0.1 * rng.standard_normal(params[k].shape)).astype(np.float32)
    wpack = torch.as_tensor(M.pack(params)).cuda()
    out, g9, scales, err = M.closure(u, v, w, sp, wpack, delta=sp[0], grads=True)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    g2 = torch.mean(g9 * g9)
    x = g9.reshape(9, -1).T / torch.sqrt(g2)
    W = {k: M._bf16(torch.as_tensor(params[k], device="cuda")).double()
         for k in ("W1", "W2", "W3")}
    b = {k: torch.as_tensor(params[k], device="cuda").double() for k in ("b1", "b2", "b3")}
    h1 = torch.tanh(x @ W["W1"].T + b["b1"])
    h2 = torch.tanh(h1 @ W["W2"].T + b["b2"])
    y = (h2 @ W["W3"].T + b["b3"]) * ((sp[0] * sp[0]) * g2)
    ref = y.T.reshape(out.shape)
    scale = ref.abs().max().item()
    d = (out - ref).abs()
    assert d.max().item() <= 5e-2 * scale, (d.max().item(), scale)
    rms = torch.sqrt(torch.mean((out - ref) ** 2) / torch.mean(ref ** 2)).item()
    assert rms <= 1.5e-2, rms


def test_mlp_in_rhs_slot_runs():
    """The closure feeds the 'tensor' slot of the RHS like the gradient model."""
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    import pyflow_b200.sfsmodel_mlp as M
    n = 16
    sp = (2 * np.pi / n,) * 3
    u, v, w = (torch.tensor(a, device="cuda") for a in
               ic.spectral_velocity((n, n, n), k0=3.0, seed=2))
    wpack = torch.as_tensor(M.pack(M.xavier_init(1))).cuda()
    F, _, _, err = M.closure(u, v, w, sp, wpack, delta=sp[0])
    r0 = ops.rhs_ns(u, v, w, sp, 0.001, 1.0)
    r1 = ops.rhs_ns(u, v, w, sp, 0.001, 1.0, sfs=F)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    d = max((a - b).abs().max().item() for a, b in zip(r0, r1))
    assert 0 < d < 1e3


@pytest.mark.parametrize("shape", [(32, 32, 32), (12, 20, 9)])
def test_mlp_scales_match_torch_mean(shape):
    """pf_mlp_scales (FP64 mean square of the nine gradients in a fixed
    order) against torch.mean of the gradient fields: the float scales agree
    to one float rounding."""
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    import pyflow_b200.sfsmodel_mlp as M
    sp = tuple(2 * np.pi / n for n in shape)
    u, v, w = (torch.tensor(a, device="cuda") for a in
               ic.spectral_velocity(shape, k0=3.0, seed=6))
    wpack = torch.as_tensor(M.pack(M.xavier_init(1))).cuda()
    _, _, scales, _ = M.closure(u, v, w, sp, wpack, delta=sp[0])
    g9 = ops.sgs_closure("gradients", u, v, w, sp)
    g2 = torch.mean(g9 * g9)
    want = torch.stack([1.0 / torch.sqrt(g2), (sp[0] * sp[0]) * g2]).to(torch.float32)
    rel = ((scales.double() - want.double()).abs() / want.double().abs()).max().item()
    assert rel <= 1.2e-7, rel
