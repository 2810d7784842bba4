"""Dense PyTorch reference of unrolled synchronous causal BP (float64,
autograd), for checking the adjoint kernels' gradients on small graphs
without clamps. It restates the sweep in log-odds on the reference's
factor-major arrays: every slot's f->v message from the closed forms of the
AND/OR factor (OR = AND on negated log-odds; singletons send logit(p)),
then S_v = sum of a variable's incoming messages and v->f = S_v - own
message; beliefs are sigmoid(S_v) after the last sweep. Test code only."""

import numpy as np
import torch


def unrolled(arrays, p, sweeps):
    off = torch.as_tensor(np.asarray(arrays["factor_offsets"]), dtype=torch.long)
    sv = torch.as_tensor(np.asarray(arrays["slot_var"]), dtype=torch.long)
    head = torch.as_tensor(np.asarray(arrays["factor_head"]), dtype=torch.long)
    typ = torch.as_tensor(np.asarray(arrays["factor_type"]), dtype=torch.long)
    q = torch.as_tensor(np.asarray(arrays["factor_q"]), dtype=torch.float64)
    V, F, E = int(arrays["n_vars"]), off.numel() - 1, int(off[-1])
    fac = torch.repeat_interleave(torch.arange(F), off[1:] - off[:-1])
    is_head = torch.zeros(E, dtype=torch.bool)
    is_head[head] = True
    body = ~is_head
    single = typ == 0
    sgn = torch.where(typ == 2, -1.0, 1.0).to(torch.float64)
    ps = torch.where(single, p, torch.full_like(p, 0.5))  # logit only where it is used (no 0 * inf)
    logit = torch.log(ps) - torch.log1p(-ps)
    vf = torch.zeros(E, dtype=torch.float64)
    S = None
    for _ in range(sweeps):
        s_slot = sgn[fac]
        y = s_slot * vf
        ls = torch.where(body, torch.nn.functional.logsigmoid(y), torch.zeros_like(y))
        L = torch.zeros(F, dtype=torch.float64).index_add(0, fac, ls)
        P, R = torch.exp(L), -torch.expm1(L)
        # log(pP + qR), taken as log p + L when q == 0 so that an underflowing P stays exact
        q0 = q == 0
        lA = torch.where(q0, torch.log(torch.where(q0, p, torch.ones_like(p))) + L,
                         torch.log(torch.where(q0, torch.ones_like(p), p * P + q * R)))
        f_head = lA - torch.log((1 - p) * P + (1 - q) * R)
        lh = s_slot[head] * vf[head]
        sh, th = torch.sigmoid(lh), torch.sigmoid(-lh)
        lo = L[fac] - ls
        Po, Ro = torch.exp(lo), -torch.expm1(lo)
        pf, qf = p[fac], q[fac]
        a = pf * Po + qf * Ro
        m1 = sh[fac] * a + th[fac] * (1 - a)
        m0 = sh[fac] * qf + th[fac] * (1 - qf)
        one = torch.ones_like(m1)
        f_body = torch.log(torch.where(body, m1, one)) - torch.log(torch.where(body, m0, one))
        fv = torch.where(is_head, (sgn * f_head)[fac], s_slot * f_body)
        fv = torch.where(single[fac], logit[fac], fv)
        S = torch.zeros(V, dtype=torch.float64).index_add(0, sv, fv)
        vf = S[sv] - fv
    return torch.sigmoid(S)
