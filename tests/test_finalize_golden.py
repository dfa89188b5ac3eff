"""The 'source' closure's training update against the reference's own
(tests/golden/finalize_8.npz, made by running sfsmodel_ML.residual_stress.finalize,
src/sfsmodel/sfsmodel_ML.py:284-349, over seven windows with seeded gradients).

Every operation of the update (gradient accumulation and averaging over
numSumDistr windows, RMSprop, the learning-rate schedule) is elementwise, so
the fixture holds the first K elements of every parameter; the rest of each
parameter is zero here and in no way affects those K.  The reference's
accumulated gradients become dL/dtheta after its factor -dt; this build's
finalize takes dL/dtheta, so it is fed -dt times the reference's gradients
(the same FP32 multiply).  Parameters must agree bit for bit after every
window, and both learning-rate values (the attribute and the optimizer's)
must follow the reference's schedule.
"""
import types

import numpy as np
import torch


def test_finalize_matches_reference(golden):
    import pyflow_b200.sfsmodel_ML as M
    g = golden("finalize_8.npz")
    K = int(g["K"])
    IC = types.SimpleNamespace(simDt=float(g["simDt"]), LR=float(g["LR_config"]),
                               LR_decay=int(g["LR_decay"]), numSumDistr=int(g["numSumDistr"]),
                               modelDictSave="unused.dict")
    decomp = types.SimpleNamespace(device=torch.device("cpu"))
    geo = types.SimpleNamespace(type="uniform", dx=0.1)
    ml = M.residual_stress(IC, decomp, geo)
    params = dict(ml.model.named_parameters())
    assert sorted(params) == sorted(str(n) for n in g["names"])
    with torch.no_grad():
        for k, prm in params.items():
            prm.zero_()
            prm.view(-1)[:K] = torch.from_numpy(g["w0_" + k])
    for e in range(int(g["epochs"])):
        for k, prm in params.items():
            gr = torch.zeros_like(prm)
            gr.view(-1)[:K] = torch.from_numpy(g["g%d_%s" % (e, k)])
            prm.grad = gr * -float(g["simDt"])
        ml.finalize(None)
        for k, prm in params.items():
            got = prm.detach().view(-1)[:K].numpy()
            assert np.array_equal(got, g["w%d_%s" % (e + 1, k)]), (e, k)
        lr_attr, lr_opt = g["lr%d" % (e + 1)]
        assert ml.LR == lr_attr and ml.optimizer.param_groups[0]["lr"] == lr_opt, e
