"""Time advancers with the reference's interface (src/solver/advancer.py).

With this package's ForwardRHS, ``step`` is one fused C-ABI call
(pf_predictor_step: four stage kernels for RK4, one for Euler) that is bit for
bit the reference's sequence, including its stage-4 state u + dt/2 k3
(src/solver/advancer.py:93-96).  With any other RHS object the reference's
stage sequence is composed from ``evaluate`` calls.
"""
from . import ops
from .velocity import ForwardRHS, sfs_args, visc_args


def _fused_args(rhsClass):
    if not isinstance(rhsClass, ForwardRHS):
        return None
    r = rhsClass.rhs1
    if getattr(r.sfsmodel, "modelType", None) == "source":
        return None  # per-stage source closure: compose the stages
    mu, visc = visc_args(r.VISC)
    return dict(spacing=r.metric.spacing, mu=mu, rho=r.rho, visc=visc,
                sfs=sfs_args(r.sfsmodel))


class Euler:
    """src/solver/advancer.py:41-57"""

    def __init__(self, state_u, state_v, state_w, rhsClass):
        self.state_u, self.state_v, self.state_w = state_u, state_v, state_w
        self.rhsClass = rhsClass

    def step(self, simDt):
        a = _fused_args(self.rhsClass)
        if a is not None:
            ops.predictor_step(self.state_u.interior(), self.state_v.interior(),
                               self.state_w.interior(), a["spacing"], a["mu"],
                               a["rho"], simDt, rk4=False, visc=a["visc"],
                               sfs=a["sfs"])
            return
        r = self.rhsClass.rhs1
        r.evaluate(self.state_u, self.state_v, self.state_w)
        self.state_u.update(self.state_u.interior() + r.rhs_u * simDt)
        self.state_v.update(self.state_v.interior() + r.rhs_v * simDt)
        self.state_w.update(self.state_w.interior() + r.rhs_w * simDt)


class RK4:
    """src/solver/advancer.py:63-113"""

    def __init__(self, state_u, state_uTmp, state_v, state_vTmp, state_w,
                 state_wTmp, rhsClass, prec="fp64"):
        self.state_u, self.state_v, self.state_w = state_u, state_v, state_w
        self.state_uTmp, self.state_vTmp, self.state_wTmp = state_uTmp, state_vTmp, state_wTmp
        self.rhsClass = rhsClass
        self.prec = prec

    def step(self, simDt):
        a = _fused_args(self.rhsClass)
        if a is not None:
            visc, sfs = a["visc"], a["sfs"]
            if self.prec != "fp64":
                # the mixed forms' stages read the closure fields in FP32
                visc = None if visc is None else visc.float()
                sfs = None if sfs is None else sfs.float()
            ops.predictor_step(self.state_u.interior(), self.state_v.interior(),
                               self.state_w.interior(), a["spacing"], a["mu"],
                               a["rho"], simDt, rk4=True, prec=self.prec,
                               visc=visc, sfs=sfs)
            return
        rc = self.rhsClass
        u, v, w = self.state_u, self.state_v, self.state_w
        ut, vt, wt = self.state_uTmp, self.state_vTmp, self.state_wTmp
        rc.rhs1.evaluate(u, v, w)
        for prev, cur in ((rc.rhs1, rc.rhs2), (rc.rhs2, rc.rhs3), (rc.rhs3, rc.rhs4)):
            ut.ZAXPY(0.5 * simDt, prev.rhs_u, u.interior())
            vt.ZAXPY(0.5 * simDt, prev.rhs_v, v.interior())
            wt.ZAXPY(0.5 * simDt, prev.rhs_w, w.interior())
            cur.evaluate(ut, vt, wt)
        for st, c in ((u, "u"), (v, "v"), (w, "w")):
            k = [getattr(r, "rhs_" + c) for r in (rc.rhs1, rc.rhs2, rc.rhs3, rc.rhs4)]
            st.update(st.interior() + simDt / 6.0 * (k[0] + 2.0 * k[1] + 2.0 * k[2] + k[3]))
