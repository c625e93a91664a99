"""CPU oracle of lmie_solution_adjoint (test infrastructure).

The reference cannot express a binned distribution in one call, so the
oracle composes it from per-radius SIZE_DIST_MONO solves of the CPU oracle
(the reference's algorithm restated in oracle/, pinned to the reference), with
accuracy 0 (no truncation of the expansion, so pf at the user angles is the
exact phase matrix) and the forward-mode (tangent-linear) derivatives w.r.t.
mr and mi.  The per-radius results are combined with the bin weights
W_r = weight[b] q_r exactly:
    Cext = sum W Cext_r / sum W,   Csca likewise,
    g    = sum W Csca_r g_r / sum W Csca_r,
    P    = sum W Csca_r P_r(theta) / sum W Csca_r   (P11 = pf[0], P12 = pf[4]),
and the loss and its derivatives follow by the chain rule: mr, mi through the
forward-mode outputs of each radius, the bin weights analytically.
"""
from __future__ import annotations

import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import numpy as np

import libs
from lmie_b200 import abi


def gauss_leg(n: int, a: float, b: float):
    x = np.zeros(n)
    w = np.zeros(n)
    p = lambda v: v.ctypes.data_as(C.POINTER(C.c_double))
    orc = libs.oracle()
    orc.oracle_gauss_leg.argtypes = [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    orc.oracle_gauss_leg(n, a, b, p(x), p(w))
    return x, w


def radii(p):
    rs, qs, bs = [], [], []
    for b in range(p.n_bins):
        x, w = gauss_leg(p.n_quad, p.edges[b], p.edges[b + 1])
        rs.append(x)
        qs.append(w)
        bs.append(np.full(p.n_quad, b))
    return np.concatenate(rs), np.concatenate(qs), np.concatenate(bs)


def per_radius(p, k: int, r: float):
    """Cext, Csca, g, P11[n_angles], P12[n_angles] of one radius and their
    derivatives w.r.t. (mr, mi) (leading axis 2)."""
    case = abi.Case(dist="mono", lam=float(p.lam[k]), mr=float(p.mr[k]), mi=float(p.mi[k]), a1=float(r),
                    r1=float(r), r2=float(r), n_angles=p.n_angles, accuracy=0.0, calc_gc=1,
                    derivs=abi.deriv_unit("mr", "mi"))
    res = abi.solve(libs.oracle(), case, kind="oracle")
    if res.rc != 0:
        raise RuntimeError("oracle MONO solve failed")
    v = (res.scalars["cext"], res.scalars["csca"], res.scalars["g"], res.pf[0], res.pf[4])
    d = (res.scalars_l["cext"], res.scalars_l["csca"], res.scalars_l["g"], res.pf_l[:, 0], res.pf_l[:, 4])
    return v, d


def solve(p, threads: int = 1) -> dict:
    """Loss, gradients and per-wavelength outputs by forward mode; the
    per-radius solves run on `threads` host threads (the oracle keeps no
    state between calls)."""
    rad, q, binof = radii(p)
    W = p.weight[binof] * q
    N = W.sum()
    L, na, nb = p.n_lambda, p.n_angles, p.n_bins
    out = {"loss": 0.0, "grad_mr": np.zeros(L), "grad_mi": np.zeros(L), "grad_weight": np.zeros(nb),
           "cext": np.zeros(L), "csca": np.zeros(L), "g": np.zeros(L),
           "p11": np.zeros((L, na)), "p12": np.zeros((L, na))}
    pool = ThreadPoolExecutor(threads) if threads > 1 else None
    for k in range(L):
        if pool is None:
            vs = [per_radius(p, k, r) for r in rad]
        else:
            vs = list(pool.map(lambda r: per_radius(p, k, r), rad))
        ce = np.array([v[0][0] for v in vs]); cs = np.array([v[0][1] for v in vs])
        gg = np.array([v[0][2] for v in vs])
        p11 = np.array([v[0][3] for v in vs]); p12 = np.array([v[0][4] for v in vs])
        dce = np.array([v[1][0] for v in vs]); dcs = np.array([v[1][1] for v in vs])
        dgg = np.array([v[1][2] for v in vs])
        dp11 = np.array([v[1][3] for v in vs]); dp12 = np.array([v[1][4] for v in vs])
        Sw = (W * cs).sum()
        Cext = (W * ce).sum() / N
        Csca = (W * cs).sum() / N
        g = (W * cs * gg).sum() / Sw
        P11 = (W * cs) @ p11 / Sw
        P12 = (W * cs) @ p12 / Sw
        c = p.c[k]
        loss = c[0] * Cext + c[1] * Csca + c[2] * g + p.d11[k] @ P11 + p.d12[k] @ P12
        # mr, mi (axis 1 of the d* arrays)
        dSw = W @ dcs
        dCext = W @ dce / N
        dCsca = W @ dcs / N
        dg = (W @ (dcs * gg[:, None] + cs[:, None] * dgg) - g * dSw) / Sw
        dP11 = (np.einsum("r,rdi->di", W, dcs[:, :, None] * p11[:, None, :] + cs[:, None, None] * dp11)
                - dSw[:, None] * P11[None, :]) / Sw
        dP12 = (np.einsum("r,rdi->di", W, dcs[:, :, None] * p12[:, None, :] + cs[:, None, None] * dp12)
                - dSw[:, None] * P12[None, :]) / Sw
        dL = c[0] * dCext + c[1] * dCsca + c[2] * dg + dP11 @ p.d11[k] + dP12 @ p.d12[k]
        out["grad_mr"][k], out["grad_mi"][k] = dL[0], dL[1]
        # bin weights: dW_r / dweight_b = q_r for r in bin b
        dL_dW = (c[0] * (ce - Cext) / N + c[1] * (cs - Csca) / N + c[2] * cs * (gg - g) / Sw
                 + cs * ((p11 - P11) @ p.d11[k] + (p12 - P12) @ p.d12[k]) / Sw)
        out["grad_weight"] += np.bincount(binof, weights=q * dL_dW, minlength=nb)
        out["loss"] += loss
        out["cext"][k], out["csca"][k], out["g"][k] = Cext, Csca, g
        out["p11"][k], out["p12"][k] = P11, P12
    if pool is not None:
        pool.shutdown()
    return out
