"""Error of a mixed-precision form against the FP64 form over a run.

``compare_forms`` advances the same initial field with two captured step
plans (``plan.StepPlan``), one in the FP64 form (the reference's algorithm:
unpreconditioned BiCGStab to the reference's relative residual) and one in a
mixed form, and records after every step the monitor statistics of
PyFlow.run (src/core/PyFlow.py:379-395) plus the dissipation rate
eps = 2 nu <S_ij S_ij> (``ops.flow_stats``).  It returns the error report of
the mixed form: relative L2 and max-norm velocity errors after the last step,
and the largest relative errors of KE(t) and eps(t) over the run, next to
max|div u| of both forms.  Everything runs on the device; the host reads the
per-step records once at the end.
"""
import numpy as np
import torch

from . import ops
from .plan import StepPlan


def _run(u0, v0, w0, spacing, nu, rho, dt, steps, prec, min_res, max_it, device):
    f = [torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)
         for a in (u0, v0, w0)]
    f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
    plan = StepPlan(*f, spacing, nu * rho, rho, dt, min_res=min_res, max_it=max_it, prec=prec)
    rec = torch.zeros((steps, 6), dtype=torch.float64, device=device)
    st = torch.cuda.current_stream(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for s in range(steps):
        plan.launch(1, stream=st)
        ops.flow_stats(f[0], f[1], f[2], spacing, nu, out=rec[s])
    e1.record(st)
    torch.cuda.synchronize(device)
    info = plan.stats()
    plan.close()
    return f, rec.cpu().numpy(), e0.elapsed_time(e1), info


def compare_forms(u0, v0, w0, spacing, nu, dt, steps, prec="mixed_mg", rho=1.0,
                  min_res=1e-10, max_it=20000, device="cuda", keep_fields=False):
    """Run ``steps`` steps in FP64 and in ``prec`` from (u0, v0, w0) and
    return the error report of ``prec`` against FP64 (a dict).  Times include
    the per-step statistics."""
    dev = torch.device(device)
    ref, rref, ms_ref, inf_ref = _run(u0, v0, w0, spacing, nu, rho, dt, steps, "fp64",
                                      min_res, max_it, dev)
    mix, rmix, ms_mix, inf_mix = _run(u0, v0, w0, spacing, nu, rho, dt, steps, prec,
                                      min_res, max_it, dev)
    num = sum(float(torch.sum((a - b) ** 2)) for a, b in zip(mix[:3], ref[:3]))
    den = sum(float(torch.sum(b ** 2)) for b in ref[:3])
    linf = max(float((a - b).abs().max()) for a, b in zip(mix[:3], ref[:3]))
    vmax = max(float(b.abs().max()) for b in ref[:3])
    ke_err = np.abs(rmix[:, 3] - rref[:, 3]) / np.abs(rref[:, 3])
    eps_err = np.abs(rmix[:, 5] - rref[:, 5]) / np.abs(rref[:, 5])
    out = {
        "steps": steps, "prec": prec,
        "u_rel_l2": float(np.sqrt(num / den)),
        "u_rel_linf": linf / vmax,
        "ke_rel_err_max": float(ke_err.max()),
        "dissipation_rel_err_max": float(eps_err.max()),
        "max_div_fp64": float(rref[:, 4].max()),
        "max_div_mixed": float(rmix[:, 4].max()),
        "ke_final": float(rref[-1, 3]), "dissipation_final": float(rref[-1, 5]),
        "ke_decay": float(rref[-1, 3] / rref[0, 3]),
        "fp64_ms_per_step": ms_ref / steps, "mixed_ms_per_step": ms_mix / steps,
        "fp64_iterations_per_step": inf_ref["total_iterations"] / steps,
        "mixed_iterations_per_step": inf_mix["total_iterations"] / steps,
        "fp64_status": int(inf_ref["status"]), "mixed_status": int(inf_mix["status"]),
        "per_step": {"fp64": rref.tolist(), "mixed": rmix.tolist()},
    }
    if keep_fields:
        out["fields"] = (mix, ref)
    return out
