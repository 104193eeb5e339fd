"""LBFGS minimiser of the oracle (test infrastructure only, like maf_oracle).

Restates magnumaf/src/solvers/lbfgs_minimizer.cpp: the m = 5 two-loop
recursion on the normalised magnetisation with the gradient m x (m x H)
(:33-42, :55-198), the More-Thuente line search cvsrch (:213-360) and its
step-interval update cstep (:362-505), with the reference's constants and
stopping tests.  Returns the final energy and the number of iterations.
"""
import math

import numpy as np

import maf_oracle as O


def energy_and_gradient(state, terms):
    """EnergyAndGradient (lbfgs_minimizer.cpp:38-42): sum of per-term energies
    and g = m x (m x Heff)."""
    h = None
    E = 0.0
    for t in terms:
        ht = t.H_in_Apm(state)
        E += t.Energy_in_J(state, ht) if not isinstance(t, O.ExchangeField) else t.Energy_in_J(state)
        h = ht if h is None else h + ht
    return E, O.cross4(state.m, O.cross4(state.m, h))


def mydot(a, b):
    return float(np.sum(a * b))


def cstep(stx, fx, dx, sty, fy, dy, stp, fp, dp, brackt, stpmin, stpmax):
    """lbfgs_minimizer.cpp:362-505; returns the updated tuple and info."""
    info = 0
    bound = False
    if (brackt and (stp <= min(stx, sty) or stp >= max(stx, sty))) or dx * (stp - stx) >= 0.0 or stpmax < stpmin:
        return stx, fx, dx, sty, fy, dy, stp, brackt, info
    sgnd = dp * (dx / abs(dx))
    if fp > fx:
        info = 1
        bound = True
        theta = 3. * (fx - fp) / (stp - stx) + dx + dp
        s = max(theta, max(dx, dp))
        gamma = s * math.sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s))
        if stp < stx:
            gamma = -gamma
        p = (gamma - dx) + theta
        q = ((gamma - dx) + gamma) + dp
        r = p / q
        stpc = stx + r * (stp - stx)
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.) * (stp - stx)
        stpf = stpc if abs(stpc - stx) < abs(stpq - stx) else stpc + (stpq - stpc) / 2
        brackt = True
    elif sgnd < 0.0:
        info = 2
        bound = False
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(theta, max(dx, dp))
        gamma = s * math.sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = ((gamma - dp) + gamma) + dx
        r = p / q
        stpc = stp + r * (stx - stp)
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
        brackt = True
    elif abs(dp) < abs(dx):
        info = 3
        bound = True
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(theta, max(dx, dp))
        gamma = s * math.sqrt(max(0., (theta / s) * (theta / s) - (dx / s) * (dp / s)))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = (gamma + (dx - dp)) + gamma
        r = p / q
        if r < 0.0 and gamma != 0.0:
            stpc = stp + r * (stx - stp)
        elif stp > stx:
            stpc = stpmax
        else:
            stpc = stpmin
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        if brackt:
            stpf = stpc if abs(stp - stpc) < abs(stp - stpq) else stpq
        else:
            stpf = stpc if abs(stp - stpc) > abs(stp - stpq) else stpq
    else:
        info = 4
        bound = False
        if brackt:
            theta = 3 * (fp - fy) / (sty - stp) + dy + dp
            s = max(theta, max(dy, dp))
            gamma = s * math.sqrt((theta / s) * (theta / s) - (dy / s) * (dp / s))
            if stp > sty:
                gamma = -gamma
            p = (gamma - dp) + theta
            q = ((gamma - dp) + gamma) + dy
            r = p / q
            stpc = stp + r * (sty - stp)
            stpf = stpc
        elif stp > stx:
            stpf = stpmax
        else:
            stpf = stpmin
    if fp > fx:
        sty, fy, dy = stp, fp, dp
    else:
        if sgnd < 0.0:
            sty, fy, dy = stx, fx, dx
        stx, fx, dx = stp, fp, dp
    stpf = min(stpmax, stpf)
    stpf = max(stpmin, stpf)
    stp = stpf
    if brackt and bound:
        if sty > stx:
            stp = min(stx + 0.66 * (sty - stx), stp)
        else:
            stp = max(stx + 0.66 * (sty - stx), stp)
    return stx, fx, dx, sty, fy, dy, stp, brackt, info


def cvsrch(state, terms, wa, f, g, stp, s, tolf):
    """lbfgs_minimizer.cpp:213-360; returns (f, g, stp, nfev)."""
    infoc = 1
    xtol, ftol, gtol = 1e-15, 1.0e-4, 0.9
    eps = tolf
    stpmin, stpmax, xtrapf, maxfev = 1e-15, 1e15, 4, 20
    nfev = 0
    dginit = mydot(g, s)
    if dginit >= 0.0:
        return f, g, stp, nfev
    brackt = False
    stage1 = True
    finit = f
    dgtest = ftol * dginit
    width = stpmax - stpmin
    width1 = 2 * width
    stx, fx, dgx = 0.0, finit, dginit
    sty, fy, dgy = 0.0, finit, dginit
    while True:
        if brackt:
            stmin, stmax = min(stx, sty), max(stx, sty)
        else:
            stmin, stmax = stx, stp + xtrapf * (stp - stx)
        stp = max(stp, stpmin)
        stp = min(stp, stpmax)
        if (brackt and (stp <= stmin or stp >= stmax)) or nfev >= maxfev - 1 or infoc == 0 or \
                (brackt and stmax - stmin <= xtol * stmax):
            stp = stx
        state.m = O.normalize(wa + stp * s)
        f, g = energy_and_gradient(state, terms)
        nfev += 1
        dg = mydot(g, s)
        ftest1 = finit + stp * dgtest
        ftest2 = finit + eps * abs(finit)
        ft = 2 * ftol - 1
        info = 0
        if (brackt and (stp <= stmin or stp >= stmax)) or infoc == 0:
            info = 6
        if stp == stpmax and f <= ftest2 and dg <= dgtest:
            info = 5
        if stp == stpmin and (f > ftest2 or dg >= dgtest):
            info = 4
        if nfev >= maxfev:
            info = 3
        if brackt and stmax - stmin <= xtol * stmax:
            info = 2
        if f <= ftest1 and abs(dg) <= gtol * (-dginit):
            info = 1
        if (f <= ftest2 and ft * dginit >= dg) and abs(dg) <= gtol * (-dginit):
            info = 1
        if info != 0:
            return f, g, stp, nfev
        if stage1 and (f <= ftest2 and ft * dginit >= dg) and dg >= min(ftol, gtol) * dginit:
            stage1 = False
        if stage1 and f <= fx and not (f <= ftest2 and ft * dginit >= dg):
            fm = f - stp * dgtest
            fxm = fx - stx * dgtest
            fym = fy - sty * dgtest
            dgm = dg - dgtest
            dgxm = dgx - dgtest
            dgym = dgy - dgtest
            stx, fxm, dgxm, sty, fym, dgym, stp, brackt, infoc = cstep(stx, fxm, dgxm, sty, fym, dgym, stp, fm, dgm,
                                                                       brackt, stmin, stmax)
            fx = fxm + stx * dgtest
            fy = fym + sty * dgtest
            dgx = dgxm + dgtest
            dgy = dgym + dgtest
        else:
            stx, fx, dgx, sty, fy, dgy, stp, brackt, infoc = cstep(stx, fx, dgx, sty, fy, dgy, stp, f, dg, brackt,
                                                                   stmin, stmax)
        if brackt:
            if abs(sty - stx) >= 0.66 * width1:
                stp = stx + 0.5 * (sty - stx)
            width1 = width
            width = abs(sty - stx)


def minimize(state, terms, tolerance=1e-6, maxIter=230):
    """LBFGS_Minimizer::Minimize (lbfgs_minimizer.cpp:55-198); returns (f, iterations)."""
    eps = 2.22e-16
    eps2 = math.sqrt(eps)
    epsr = eps ** 0.9
    tolf2 = math.sqrt(tolerance)
    tolf3 = tolerance ** 0.3333333333333333333333333
    f, grad = energy_and_gradient(state, terms)
    gradNorm = float(np.max(np.abs(grad)))
    if gradNorm < epsr * (1 + abs(f)):
        return f, 0
    m = 5
    sV = [np.zeros_like(grad) for _ in range(m)]
    yV = [np.zeros_like(grad) for _ in range(m)]
    alpha = [0.0] * m
    it = 0
    glob = 0
    H0k = 1.0
    while True:
        f_old = f
        x_old = state.m.copy()
        grad_old = grad
        q = grad.copy()
        k = min(m, it)
        for i in range(k - 1, -1, -1):
            rho = 1.0 / mydot(sV[i], yV[i])
            alpha[i] = rho * mydot(sV[i], q)
            q = q - alpha[i] * yV[i]
        q = H0k * q
        for i in range(k):
            rho = 1.0 / mydot(sV[i], yV[i])
            beta = rho * mydot(yV[i], q)
            q = q + sV[i] * (alpha[i] - beta)
        phiPrime0 = -mydot(grad, q)
        if phiPrime0 > 0:
            q = grad
            it = 0
        f, grad, rate, _ = cvsrch(state, terms, x_old, f, grad, 1.0, -q, tolerance)
        f1 = 1 + abs(f)
        gradNorm = float(np.max(np.abs(grad)))
        if gradNorm < epsr * f1:
            return f, glob
        s = state.m - x_old
        if (f_old - f) < tolerance * f1 and float(np.max(np.abs(s))) < tolf2 * (1 + float(np.max(np.abs(state.m)))) \
                and gradNorm <= tolf3 * f1:
            break
        y = grad - grad_old
        ys = mydot(y, s)
        if ys <= eps2 * math.sqrt(mydot(y, y)) * math.sqrt(mydot(s, s)):
            pass
        else:
            if it < m:
                sV[it] = s
                yV[it] = y
            else:
                sV = sV[1:] + [s]
                yV = yV[1:] + [y]
            H0k = ys / mydot(y, y)
            it += 1
        glob += 1
        if glob >= maxIter:
            break
    return f, glob
