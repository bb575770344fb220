"""numpy restatement of the MMA update PyTO's density-based optimiser calls
(TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the device MMA
update, never by the product package).

PyTO's ``topopt_mma`` (src/topopt_mma.py:246-373) drives ``runMMA``
(src/mmaWrapper.py:18-128), which calls ``mmasub`` and ``kktcheck`` of the
third-party package mmapy (GCMMA-MMA-Python, a port of K. Svanberg's MATLAB
code; the reference's requirements.txt pins no version, and the package is not
installed here).  This file restates the published algorithm: Svanberg's
2007 "MMA and GCMMA - two methods for nonlinear optimization" report,
mmasub (moving asymptotes, bounds alfa/beta, the convex approximation p0, q0,
P, Q, b) and subsolv (the primal-dual interior-point Newton method for the
subproblem, epsi from 1 down to 1e-7, backtracking on the residual norm), and
kktcheck (the KKT residual of the original problem), with mmapy's defaults
for the parameters runMMA leaves at their defaults (asyinit 0.5, asydecr 0.7,
asyincr 1.2, asymin 0.01, asymax 10, raa0 1e-5, albefa 0.1).

PARITY UNPINNED: with mmapy absent, no output of the reference's own MMA can be
produced here; the restatement follows the published algorithm, not a run.
"""
from __future__ import annotations

import numpy as np

ASYINIT, ASYDECR, ASYINCR, ASYMIN, ASYMAX = 0.5, 0.7, 1.2, 0.01, 10.0
RAA0, ALBEFA, EPSIMIN = 1e-5, 0.1, 1e-7


def mmasub(m, n, it, xval, xmin, xmax, xold1, xold2, f0val, df0dx, fval, dfdx, low, upp, a0, a, c, d, move):
    """One MMA subproblem (vectors as 1-D arrays, dfdx (m, n)).  Returns
    (xmma, ymma, zmma, lam, xsi, eta, mu, zet, s, low, upp)."""
    xval, xmin, xmax = (np.asarray(v, dtype=float).ravel() for v in (xval, xmin, xmax))
    xold1, xold2, df0dx = (np.asarray(v, dtype=float).ravel() for v in (xold1, xold2, df0dx))
    fval = np.asarray(fval, dtype=float).ravel()
    dfdx = np.asarray(dfdx, dtype=float).reshape(m, n)
    a, c, d = (np.asarray(v, dtype=float).ravel() for v in (a, c, d))
    span = xmax - xmin
    if it <= 2:
        low = xval - ASYINIT * span
        upp = xval + ASYINIT * span
    else:
        zzz = (xval - xold1) * (xold1 - xold2)
        factor = np.ones(n)
        factor[zzz > 0] = ASYINCR
        factor[zzz < 0] = ASYDECR
        low = xval - factor * (xold1 - np.asarray(low, dtype=float).ravel())
        upp = xval + factor * (np.asarray(upp, dtype=float).ravel() - xold1)
        low = np.minimum(np.maximum(low, xval - ASYMAX * span), xval - ASYMIN * span)
        upp = np.maximum(np.minimum(upp, xval + ASYMAX * span), xval + ASYMIN * span)
    alfa = np.maximum(np.maximum(low + ALBEFA * (xval - low), xval - move * span), xmin)
    beta = np.minimum(np.minimum(upp - ALBEFA * (upp - xval), xval + move * span), xmax)
    xmamiinv = 1.0 / np.maximum(span, 1e-5)
    ux1, xl1 = upp - xval, xval - low
    ux2, xl2 = ux1 * ux1, xl1 * xl1
    p0, q0 = np.maximum(df0dx, 0.0), np.maximum(-df0dx, 0.0)
    pq0 = 0.001 * (p0 + q0) + RAA0 * xmamiinv
    p0 = (p0 + pq0) * ux2
    q0 = (q0 + pq0) * xl2
    P, Q = np.maximum(dfdx, 0.0), np.maximum(-dfdx, 0.0)
    PQ = 0.001 * (P + Q) + RAA0 * xmamiinv[None, :]
    P = (P + PQ) * ux2[None, :]
    Q = (Q + PQ) * xl2[None, :]
    b = P @ (1.0 / ux1) + Q @ (1.0 / xl1) - fval
    out = subsolv(m, n, EPSIMIN, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d)
    return (*out, low, upp)


def _residual(m, x, y, z, lam, xsi, eta, mu, zet, s, epsi, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d):
    ux1, xl1 = upp - x, x - low
    plam = p0 + P.T @ lam
    qlam = q0 + Q.T @ lam
    gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
    dpsidx = plam / (ux1 * ux1) - qlam / (xl1 * xl1)
    res = np.concatenate([dpsidx - xsi + eta, c + d * y - mu - lam, [a0 - zet - a @ lam],
                          gvec - a * z - y + s - b, xsi * (x - alfa) - epsi, eta * (beta - x) - epsi,
                          mu * y - epsi, [zet * z - epsi], lam * s - epsi])
    return np.sqrt(res @ res), np.max(np.abs(res))


def subsolv(m, n, epsimin, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d):
    """Primal-dual Newton method for the MMA subproblem (Svanberg 2007, m < n form)."""
    x = 0.5 * (alfa + beta)
    y = np.ones(m)
    z = 1.0
    lam = np.ones(m)
    xsi = np.maximum(1.0 / (x - alfa), 1.0)
    eta = np.maximum(1.0 / (beta - x), 1.0)
    mu = np.maximum(np.ones(m), 0.5 * c)
    zet = 1.0
    s = np.ones(m)
    epsi = 1.0
    args = (low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d)
    while epsi > epsimin:
        resnorm, resmax = _residual(m, x, y, z, lam, xsi, eta, mu, zet, s, epsi, *args)
        ittt = 0
        while resmax > 0.9 * epsi and ittt < 200:
            ittt += 1
            ux1, xl1 = upp - x, x - low
            ux2, xl2 = ux1 * ux1, xl1 * xl1
            ux3, xl3 = ux1 * ux2, xl1 * xl2
            plam = p0 + P.T @ lam
            qlam = q0 + Q.T @ lam
            gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
            GG = P / ux2[None, :] - Q / xl2[None, :]
            dpsidx = plam / ux2 - qlam / xl2
            delx = dpsidx - epsi / (x - alfa) + epsi / (beta - x)
            dely = c + d * y - lam - epsi / y
            delz = a0 - a @ lam - epsi / z
            dellam = gvec - a * z - y - b + epsi / lam
            diagx = 2.0 * (plam / ux3 + qlam / xl3) + xsi / (x - alfa) + eta / (beta - x)
            diagy = d + mu / y
            diaglamyi = s / lam + 1.0 / diagy
            blam = dellam + dely / diagy - GG @ (delx / diagx)
            Alam = np.diag(diaglamyi) + (GG / diagx[None, :]) @ GG.T
            AA = np.zeros((m + 1, m + 1))
            AA[:m, :m] = Alam
            AA[:m, m] = a
            AA[m, :m] = a
            AA[m, m] = -zet / z
            sol = np.linalg.solve(AA, np.concatenate([blam, [delz]]))
            dlam, dz = sol[:m], sol[m]
            dx = -delx / diagx - (GG.T @ dlam) / diagx
            dy = -dely / diagy + dlam / diagy
            dxsi = -xsi + epsi / (x - alfa) - (xsi * dx) / (x - alfa)
            deta = -eta + epsi / (beta - x) + (eta * dx) / (beta - x)
            dmu = -mu + epsi / y - (mu * dy) / y
            dzet = -zet + epsi / z - zet * dz / z
            ds = -s + epsi / lam - (s * dlam) / lam
            xx = np.concatenate([y, [z], lam, xsi, eta, mu, [zet], s])
            dxx = np.concatenate([dy, [dz], dlam, dxsi, deta, dmu, [dzet], ds])
            stmxx = np.max(-1.01 * dxx / xx)
            stmalfa = np.max(-1.01 * dx / (x - alfa))
            stmbeta = np.max(1.01 * dx / (beta - x))
            steg = 1.0 / max(stmalfa, stmbeta, stmxx, 1.0)
            old = (x, y, z, lam, xsi, eta, mu, zet, s)
            itto = 0
            resinew = 2.0 * resnorm
            while resinew > resnorm and itto < 50:
                itto += 1
                x, y, z, lam, xsi, eta, mu, zet, s = (o + steg * dv for o, dv in zip(
                    old, (dx, dy, dz, dlam, dxsi, deta, dmu, dzet, ds)))
                resinew, resmax = _residual(m, x, y, z, lam, xsi, eta, mu, zet, s, epsi, *args)
                steg /= 2.0
            resnorm = resinew
        epsi *= 0.1
    return x, y, z, lam, xsi, eta, mu, zet, s


def kktcheck(m, n, x, y, z, lam, xsi, eta, mu, zet, s, xmin, xmax, df0dx, fval, dfdx, a0, a, c, d):
    """KKT residual of the original problem: (residual, norm, max |.|)."""
    dfdx = np.asarray(dfdx, dtype=float).reshape(m, n)
    rex = df0dx + dfdx.T @ lam - xsi + eta
    res = np.concatenate([rex, c + d * y - mu - lam, [a0 - zet - a @ lam], fval - a * z - y + s,
                          xsi * (x - xmin), eta * (xmax - x), mu * y, [zet * z], lam * s])
    return res, np.sqrt(res @ res), np.max(np.abs(res))
