"""The reference's 'source'-type ML closure (sfsmodel_ML.residual_stress,
src/sfsmodel/sfsmodel_ML.py:122-593) evaluated on the GPU, so SFS models
trained with the reference load and run unchanged.

Per RHS evaluation (every RK stage, src/solver/velocity.py:360-383):
  * the staggered velocity is interpolated to cell centres (interp_u_xm /
    interp_v_ym / interp_w_zm, src/metric/metric_staggered.py:148-166) and
    cast to FP32;
  * 21 features per cell: u, v, w, their central first derivatives and their
    second derivatives (Finite_Difference_ConCat, :392-460; every direction
    uses the x spacing, as in the reference);
  * the network input of a cell is its own 21 features and those of its
    12 neighbours at offsets +-1, +-2 along each axis, each divided by the
    reference's normalisation constants (ML_Closure, :467-510): 273 inputs;
  * the gated network NeuralNetworkModel2 (:77-116) maps them to 18 outputs;
  * the closure terms are central differences of outputs 0-8
    (GX = d0/dx + d1/dy + d2/dz, GY from 3-5, GZ from 6-8, :513-590);
  * GX, GY, GZ are interpolated to the faces and SUBTRACTED from the RHS
    (src/solver/velocity.py:374-383).

Boundary semantics: the reference evaluates all of this on its ghost-padded
arrays and wraps its shifts around the padded array, so its closure at the
three cells nearest each periodic boundary also depends on ghost-layer
contents.  Here every shift wraps periodically on the interior; the two agree
on all cells at least three cells away from a periodic boundary (the tests
check exactly those cells).

The network is torch modules with the reference's parameter names and
shapes (a reference checkpoint's 'model_state_dict' loads as is).  On a CUDA
device in FP32 without gradients (every forward RK stage) the whole closure
runs as the library's kernels (pf_mlsrc_closure: features, the network on
the tensor cores as three TF32 products per FP32 product, closure terms and
face sources), with the weights repacked whenever a parameter changed.
With gradients (training), in FP64 (config key mlDtype) or on the CPU it
runs as the torch ops below.
"""
import numpy as np
import torch
import torch.nn as nn

from . import ops

H = 200
N_FEATURES = 21
N_INPUTS = N_FEATURES + 12 * N_FEATURES
N_OUTPUTS = 18

# normalisation of the 21 features (src/sfsmodel/sfsmodel_ML.py:268-274)
NORM = 10.0 * np.array([1.0233662e+00, 1.0241578e+00, 1.0196122e+00,
                        5.0992206e+02, 5.2713013e+02, 5.2689368e+02, 5.2550342e+02,
                        5.1325964e+02, 5.2564642e+02, 5.3132422e+02, 5.2574353e+02,
                        5.1027972e+02, 9.5621462e+05, 1.2852805e+06, 1.2698791e+06,
                        1.2744681e+06, 9.6111162e+05, 1.2722050e+06, 1.2891108e+06,
                        1.2891108e+06, 9.6587112e+05])


class GatedClosureNet(nn.Module):
    """The reference's NeuralNetworkModel2 (src/sfsmodel/sfsmodel_ML.py:77-116):
    H1 = tanh(fc1 x); H2 = tanh(fc2 H1) * tanh(fcG x);
    H4 = tanh(fc3 H2) * tanh(fcG2 x); out = fc4 H4."""

    def __init__(self):
        super().__init__()
        self.fc1 = nn.Linear(N_INPUTS, H)
        self.fcG = nn.Linear(N_INPUTS, H)
        self.fcG2 = nn.Linear(N_INPUTS, H)
        self.fc2 = nn.Linear(H, H)
        self.fc3 = nn.Linear(H, H)
        self.fc4 = nn.Linear(H, N_OUTPUTS)

    def forward(self, x):
        h2 = torch.tanh(self.fc2(torch.tanh(self.fc1(x)))) * torch.tanh(self.fcG(x))
        h4 = torch.tanh(self.fc3(h2)) * torch.tanh(self.fcG2(x))
        return self.fc4(h4)


def _centred(u, v, w):
    """Cell-centre interpolants of the staggered velocity (periodic)."""
    return (0.5 * (torch.roll(u, -1, 0) + u), 0.5 * (torch.roll(v, -1, 1) + v),
            0.5 * (torch.roll(w, -1, 2) + w))


def _derivatives(a, dx):
    """First and second central differences of a centred FP32 field along
    x, y, z (all with spacing dx, as the reference)."""
    d1, d2 = [], []
    for ax in range(3):
        p, m = torch.roll(a, -1, ax), torch.roll(a, 1, ax)
        d1.append((p - m) / (2 * dx))
    for ax in range(3):
        p, m = torch.roll(a, -1, ax), torch.roll(a, 1, ax)
        d2.append((p - 2 * a + m) / (dx * dx))
    return d1, d2


def features(u, v, w, dx, dtype=torch.float32):
    """The 21 cell-centred features (FP32 like the reference), shape
    (nx, ny, nz, 21), in the reference's order: u, v, w, u_x, u_y, u_z, v_x,
    ..., w_z, u_xx, u_yy, u_zz, v_xx, ..., w_zz."""
    uc, vc, wc = (t.to(dtype) for t in _centred(u, v, w))
    first, second = [], []
    for a in (uc, vc, wc):
        d1, d2 = _derivatives(a, dx)
        first += d1
        second += d2
    return torch.stack([uc, vc, wc] + first + second, dim=3)


def network_input(F, norm):
    """273 normalised inputs per cell: own features, then the features at
    x+1, x-1, y+1, y-1, z+1, z-1, x+2, x-2, y+2, y-2, z+2, z-2."""
    parts = [F / norm]
    for sh in (1, 2):
        for ax in range(3):
            parts.append(torch.roll(F, -sh, ax) / norm)
            parts.append(torch.roll(F, sh, ax) / norm)
    return torch.cat(parts, dim=3)


def closure_terms(p, dx):
    """GX, GY, GZ (centred, FP32) from the network outputs p (..., 18)."""
    def cd(ch, ax):
        a = p[..., ch]
        return (torch.roll(a, -1, ax) - torch.roll(a, 1, ax)) / (2 * dx)
    gx = cd(0, 0) + cd(1, 1) + cd(2, 2)
    gy = cd(3, 0) + cd(4, 1) + cd(5, 2)
    gz = cd(6, 0) + cd(7, 1) + cd(8, 2)
    return gx, gy, gz


class residual_stress:
    """'source'-type SFS model object with the reference's interface
    (src/sfsmodel/sfsmodel_ML.py:122-279): ``update`` fills GX, GY, GZ;
    ``face_sources`` gives what the RHS subtracts."""

    def __init__(self, inputConfig, decomp, geo, model=None):
        self.modelType = "source"
        self.device = decomp.device
        self.simDt = getattr(inputConfig, "simDt", 0.0)
        if getattr(geo, "type", "uniform") != "uniform":
            raise Exception("sfsmodel_ML: geometry type not implemented")
        self.dx = geo.dx
        self.const = geo.dx * geo.dx / 12.0
        self.model = (model if model is not None else GatedClosureNet()).to(self.device)
        self.epoch = 0
        self.LR = 0.01
        self.optimizer = torch.optim.RMSprop(self.model.parameters(), lr=self.LR)
        self.outParamsList, self.sumParamsList = [], []
        if getattr(inputConfig, "loadModel", False):
            ck = torch.load(inputConfig.modelDictName, map_location=self.device)
            self.epoch = ck.get("epoch", 0)
            self.model.load_state_dict(ck["model_state_dict"])
            if "optimizer_state_dict" in ck:
                self.optimizer.load_state_dict(ck["optimizer_state_dict"])
            self.LR = ck.get("LR", self.LR)
            self.outParamsList = list(ck.get("outParamsList", []))
            self.sumParamsList = list(ck.get("sumParamsList", []))
        if hasattr(inputConfig, "LR"):
            # the reference records the override but leaves the optimizer's
            # learning rate as created (src/sfsmodel/sfsmodel_ML.py:214-216);
            # the halving schedule then acts on both values separately
            self.LR = inputConfig.LR
        # training settings (src/sfsmodel/sfsmodel_ML.py:219-243)
        self.saveModel = hasattr(inputConfig, "modelDictSave")
        self.modelDictSave = getattr(inputConfig, "modelDictSave", None)
        self.LR_decay = int(getattr(inputConfig, "LR_decay", 2500))
        self.numSumDistr = int(getattr(inputConfig, "numSumDistr", 8))
        self.optimizer.zero_grad()
        # evaluation precision: FP32 like the reference; 'float64' (config key
        # mlDtype) evaluates features and network in FP64
        self.dtype = torch.float64 if getattr(inputConfig, "mlDtype", "float32") == "float64" \
            else torch.float32
        self.model.to(self.dtype)
        self.norm = torch.tensor(NORM, dtype=self.dtype, device=self.device)
        self.GX = self.GY = self.GZ = None
        self._faces = None          # face sources written by the kernel path
        self._pack = None
        self._pack_key = None

    def _kernel_path(self, u, requires_grad):
        return (not requires_grad and u.is_cuda and self.dtype == torch.float32
                and all(p.dtype == torch.float32 and p.is_cuda for p in self.model.parameters())
                and min(u.shape) >= 5)

    def _packed(self):
        """The packed network, rebuilt when a parameter changed (optimizer
        steps and load_state_dict modify the parameters in place)."""
        params = [self.model.fc1.weight, self.model.fc1.bias, self.model.fcG.weight,
                  self.model.fcG.bias, self.model.fcG2.weight, self.model.fcG2.bias,
                  self.model.fc2.weight, self.model.fc2.bias, self.model.fc3.weight,
                  self.model.fc3.bias, self.model.fc4.weight, self.model.fc4.bias]
        key = tuple((p.data_ptr(), p._version) for p in params)
        if self._pack is None or key != self._pack_key:
            self._pack = ops.mlsrc_pack(params, self.norm, self._pack)
            self._pack_key = key
        return self._pack

    def update(self, u, v, w, requires_grad=False):
        """Closure terms at cell centres from the staggered velocity (FP64
        interiors); stored as FP64 like the reference (:370-380)."""
        self._faces = None
        if self._kernel_path(u, requires_grad):
            G, S, self._err = ops.mlsrc_closure(u.contiguous(), v.contiguous(), w.contiguous(),
                                                self.dx, self._packed())
            self.GX, self.GY, self.GZ = G[0], G[1], G[2]
            self._faces = (S[0], S[1], S[2])
            return
        with torch.set_grad_enabled(requires_grad):
            F = features(u, v, w, self.dx, self.dtype)
            x = network_input(F, self.norm)
            p = self.model(x)
            gx, gy, gz = closure_terms(p, self.dx)
        self.GX, self.GY, self.GZ = (g.to(torch.float64) for g in (gx, gy, gz))
        if not requires_grad:
            self.GX, self.GY, self.GZ = (g.detach() for g in (self.GX, self.GY, self.GZ))

    def face_sources(self):
        """interp_sc_x/y/z of GX, GY, GZ (src/metric/metric_staggered.py:112-124,
        interp factor 1/2 on a uniform grid): face i gets (G[i] + G[i-1]) / 2."""
        if self._faces is not None:
            return self._faces
        return (0.5 * (self.GX + torch.roll(self.GX, 1, 0)),
                0.5 * (self.GY + torch.roll(self.GY, 1, 1)),
                0.5 * (self.GZ + torch.roll(self.GZ, 1, 2)))

    def save(self, path=None):
        """Checkpoint in the reference's format (src/sfsmodel/sfsmodel_ML.py:280-291)."""
        path = path or self.modelDictSave
        torch.save({"epoch": self.epoch, "LR": self.LR,
                    "model_state_dict": self.model.state_dict(),
                    "optimizer_state_dict": self.optimizer.state_dict(),
                    "outParamsList": self.outParamsList,
                    "sumParamsList": self.sumParamsList}, path)

    def finalize(self, comms=None):
        """One training update after an adjoint window, with the reference's
        schedule (src/sfsmodel/sfsmodel_ML.py:296-349): the parameter
        gradients are accumulated over numSumDistr windows and their average
        (summed over ranks) is applied at every window until the next
        average exists; RMSprop step; the learning rate halves every LR_decay
        windows once 4/5 of LR_decay have passed.  The gradients held by the
        parameters are already dL/dtheta (the reference's accumulation needs
        a factor -dt to become that; the hand-written adjoint here does not)."""
        params = list(self.model.parameters())
        grads = [p.grad.detach().clone() if p.grad is not None else torch.zeros_like(p)
                 for p in params]
        if self.epoch == 0 or not self.sumParamsList:
            self.outParamsList = [torch.zeros_like(g) for g in grads]
            self.sumParamsList = [torch.zeros_like(g) for g in grads]
        for s, g in zip(self.sumParamsList, grads):
            s.add_(g)
        if (self.epoch + 1) % self.numSumDistr == 0:
            size = getattr(comms, "size", 1) if comms is not None else 1
            for i, s in enumerate(self.sumParamsList):
                tot = s
                if comms is not None and size > 1:
                    tot = torch.as_tensor(comms.parallel_sum(s.cpu().numpy()), device=s.device)
                self.outParamsList[i] = tot / float(self.numSumDistr * size)
                self.sumParamsList[i] = torch.zeros_like(s)
        for p, a in zip(params, self.outParamsList):
            p.grad = a.clone().to(p.dtype)
        self.optimizer.step()
        self.optimizer.zero_grad()
        self.epoch += 1
        if self.epoch >= 4 * self.LR_decay // 5 and self.epoch % self.LR_decay == 0:
            self.LR *= 0.5
            for g in self.optimizer.param_groups:
                g["lr"] = 0.5 * g["lr"]
