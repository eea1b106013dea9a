"""Fitting drivers: the callers of the objective, over the batched evaluator.

The reference runs its optimizers one objective call at a time.  Here the
independent evaluations of each driver go to the GPU in one launch:

* powell_fit   -- Powell least squares (opt_powell.cpp:96-315) with the
                  reference's constants and steps.  gamma_init's P forward
                  differences (opt_powell.cpp:348-389) are ONE batched launch
                  whose residual vectors stay on the device; the Jacobian,
                  its column norms and the normal equations gamma^T gamma,
                  -gamma^T e (opt_powell.cpp:441-493) are formed there in FP64.
                  The line search is the reference's golden bracket + Brent
                  (line_min.cpp:83-151, line_min_brent.cpp:37-126).
* lbfgs_fit    -- L-BFGS on the hand-written adjoint (no reference
                  counterpart).
* anneal_chains -- simulated annealing (opt_simann.cpp:89-264) run as
                  independent Metropolis chains evaluated together.
* genetic_fit  -- the genetic algorithm's breeding (opt_genalg.cpp:105-309),
                  each generation's children evaluated together.
"""
from __future__ import annotations

import math
import time
from typing import Callable, Optional

import numpy as np

from .potential import MZ_FP64, MZ_MIXED, Evaluator

# OptPowell constants (opt_powell.h:43-47), LineMin (line_min.h:45-46),
# LineMinBrent (line_min_brent.h:29-31), OptSimAnn (opt_simann.h:41-46),
# OptGenAlg (opt_genalg.h:48-49).
EPS = 1.0e-4
PRECISION = 1.0e-7
NOTHING = 1.0e-12
INNERLOOPS = 801
TOOBIG = 1.0e4
CGOLD = 0.381966012
MAX_BRACKET = 100
ITMAX = 100
TOL = 1.0e-1
ZEPS = 1.0e-9
SA_EPS, SA_NEPS, SA_NSTEP, SA_STEPVAR, SA_TEMPVAR = 0.1, 4, 20, 2.0, 0.85
GA_EPS, GA_NEPS = 0.001, 10


class FitError(RuntimeError):
    pass


# ---------------------------------------------------------------- line search

def _bracket(f: Callable[[float], float]):
    """Golden-section bracketing of a minimum, LineMin::get_bracket."""
    xl, xr = 0.0, 0.1
    Fl, Fr = f(xl), f(xr)
    if Fr >= Fl:
        xm, Fm = xl, Fl
        xl = -(xr - xm) / CGOLD + xr
        Fl = f(xl)
    else:
        xm, Fm = xr, Fr
        xr = (xm - xl) / CGOLD + xl
        Fr = f(xr)
    for _ in range(MAX_BRACKET):
        if Fm < Fl:
            if Fm < Fr:
                return xl, xm, xr, Fl, Fm, Fr
            elif Fm > Fr:
                xl, Fl, xm, Fm = xm, Fm, xr, Fr
                xr = (xm - xl) / CGOLD + xl
                Fr = f(xr)
            else:
                xr = (xr - xl) * CGOLD + xr
                Fr = f(xr)
        elif Fm > Fl:
            xr, Fr, xm, Fm = xm, Fm, xl, Fl
            xl = -(xr - xm) / CGOLD + xr
            Fl = f(xl)
        else:
            xl = -(xr - xl) * CGOLD + xl
            Fl = f(xl)
    raise FitError("ERROR: problems with bracketing of minimum - ")


def _brent(f, xa, xb, xc, Fb):
    """Brent's minimisation inside a bracket, LineMinBrent::find_minima.
    Returns (xmin1, xmin2, Fmin1, Fmin2)."""
    a, b = min(xa, xc), max(xa, xc)
    v = w = x = xb
    d = e = 0.0
    Fx = Fv = Fw = Fb
    for _ in range(ITMAX):
        xm = 0.5 * (a + b)
        tol1 = TOL * abs(x) + ZEPS
        tol2 = 2.0 * tol1
        if abs(x - xm) <= (tol2 - 0.5 * (b - a)):
            return x, w, Fx, Fw
        if abs(e) > tol1:
            r = (x - w) * (Fx - Fv)
            q = (x - v) * (Fx - Fw)
            p = (x - v) * q - (x - w) * r
            q = 2.0 * (q - r)
            if q > 0.0:
                p = -p
            else:
                q = -q
            etemp = e
            e = d
            if abs(p) >= abs(0.5 * q * etemp) or p <= q * (a - x) or p >= q * (b - x):
                e = (b - x) if x < xm else -(x - a)
                d = CGOLD * e
            else:
                d = p / q
                u = x + d
                if (u - a) < tol2 or (b - u) < tol2:
                    d = tol1 if x < xm else -tol1
        else:
            e = (b - x) if x < xm else -(x - a)
            d = CGOLD * e
        u = x + d if abs(d) >= tol1 else x + (tol1 if d > 0 else -tol1)
        Fu = f(u)
        if Fu <= Fx:
            if u >= x:
                a = x
            else:
                b = x
            v, Fv, w, Fw, x, Fx = w, Fw, x, Fx, u, Fu
        else:
            if u < x:
                a = u
            else:
                b = u
            if Fu <= Fw or w == x:
                v, Fv, w, Fw = w, Fw, u, Fu
            elif Fu <= Fv or v == x or v == w:
                v, Fv = u, Fu
    raise FitError("ERROR: too many iterations in Brent minimization - ")


# ------------------------------------------------------------------- Powell

class _DeviceResiduals:
    """Residual vectors of many candidates evaluated into device memory."""

    def __init__(self, ev: Evaluator, precision=MZ_FP64):
        import torch
        self.torch = torch
        self.ev = ev
        self.precision = precision
        self.dev = torch.device("cuda", torch.cuda.current_device())

    def __call__(self, X: np.ndarray):
        torch = self.torch
        X = np.atleast_2d(X)
        n = X.shape[0]
        Xd = torch.tensor(X, dtype=torch.float64, device=self.dev)
        obj = torch.empty(n, dtype=torch.float64, device=self.dev)
        E = torch.empty((n, self.ev.esize), dtype=torch.float64, device=self.dev)
        self.ev.objective_device(Xd, obj, self.precision, errvec=E)
        self.ev.sync()
        return obj, E


def _gram(ev, A, B):
    """A @ B.T in FP64 (A: na x n, B: nb x n).  Device residuals go through
    the evaluator's hand-written kernel (mz_gram_device); host tensors, which
    only a host evaluator's residuals produce, are multiplied on the host."""
    import torch
    if not A.is_cuda:
        return A @ B.T
    out = torch.empty((A.shape[0], B.shape[0]), dtype=torch.float64, device=A.device)
    ev.gram_device(A, B, out)
    ev.sync()
    return out


def device_rescaler(precision=MZ_FP64):
    """Rescale hook of powell_fit on the GPU: Potential::rescale(flag) from
    the evaluator's densities; (evaluator, coefficients, residuals) of the
    rescaled potential, or None when nothing changed."""
    def rescaler(ev, x, flag):
        from .potential import Potential
        pt = Potential(ev, x, precision)
        if not pt.rescale(flag):
            return None
        return pt.ev, np.array(pt.x, dtype=np.float64), _DeviceResiduals(pt.ev, precision)
    return rescaler


def powell_fit(ev: Evaluator, x0, max_steps: int = 1000, d_eps: float = 0.0, precision=MZ_FP64,
               log: Optional[Callable[[str], None]] = None, max_evals: Optional[int] = None,
               residuals: Optional[Callable] = None, rescale: int = 0, rescaler: Optional[Callable] = None):
    """Powell least-squares fit of the coefficient vector x0.

    `residuals(X) -> (obj[n], errvec[n, esize])` as torch tensors evaluates
    many candidates at once; by default the evaluator's device residuals.
    `rescale` is the parameter file's value (PotList::get_rescale): non-zero
    turns on the optimizer's two rescale hooks -- Potential::rescale(1) when F
    does not depend on a coefficient, then one more try
    (opt_powell.cpp:138-146), and a trial Potential::rescale(0) every 4th
    outer step, kept when it does not raise F (opt_powell.cpp:262-292).
    `rescaler(ev, x, flag)` does the rescale: None when nothing changed, else
    (evaluator, coefficients, residuals) of the rescaled potential -- a new
    evaluator, since a rescale may move U's knots; device_rescaler() by
    default.  Returns (x, F, info) with info = {outer, evals, seconds,
    history, outer_history, rescales, evaluator}: history holds (seconds, F)
    after each inner step, outer_history (F, x) after each outer step, and
    evaluator is the evaluator of x."""
    import torch
    t0 = time.time()
    res = _DeviceResiduals(ev, precision) if residuals is None else residuals
    if rescaler is None:
        rescaler = device_rescaler(precision)
    rescales = []
    outer_history = []
    P = ev.ncoeff
    x = np.array(x0, dtype=np.float64)
    evals = [0]
    history = []

    def resid(X):
        evals[0] += np.atleast_2d(X).shape[0]
        return res(X)

    def f_line(base, delta):
        def f(a):
            evals[0] += 1
            return float(ev.objective((base + a * delta)[None, :], precision)[0])
        return f

    o, E = resid(x)
    F = float(o[0])
    e = E[0].clone()
    history.append((time.time() - t0, F))
    if F < NOTHING or max_steps == 0:
        return x, F, dict(outer=0, evals=evals[0], seconds=time.time() - t0, history=history,
                          outer_history=outer_history, rescales=rescales,
                          evaluator=ev)

    def gamma_init(x, e):
        """P forward differences in one launch; normalised columns
        (OptPowell::gamma_init, opt_powell.cpp:348-389).  Column j of the
        reference's gamma is row j here (P x esize, as the residual vectors
        come out of the evaluator)."""
        X = np.repeat(x[None, :], P, axis=0) + EPS * np.eye(P)
        _, Ep = resid(X)
        gam = (Ep - e[None, :]) / EPS
        mag = torch.sqrt((gam * gam).sum(dim=1))
        bad = torch.nonzero(mag < NOTHING)
        if bad.numel():
            return int(bad[0, 0]) + 1, None, None
        gam /= mag[:, None]
        d = np.diag(1.0 / mag.cpu().numpy())
        return 0, gam, d

    n_out = 0
    while True:
        code, gam, d = gamma_init(x, e)
        if code and rescale:
            if log:
                log("F does not depend on coefficient %d, trying to rescale if it is an option!" % (code - 1))
            r = rescaler(ev, x, 1)
            if r is not None:
                ev, x, res = r
                rescales.append((n_out, "flag 1"))
            o, E = resid(x)
            F = float(o[0])
            e = E[0].clone()
            code, gam, d = gamma_init(x, e)
        if code:
            if log:
                log("F does not depend on coefficient %d, fit impossible!" % (code - 1))
            break
        F_older = F
        # lineqsys_init (opt_powell.cpp:438-472): gamma^T gamma, -gamma^T e
        lin = _gram(ev, gam, gam).cpu().numpy()
        p = -_gram(ev, gam, e[None, :])[:, 0].cpu().numpy()
        m = 0
        while True:
            F_old = F
            from scipy.linalg import lapack
            _, _, _, _, q, rcond, ferr, berr, info = lapack.dsysvx(lin, p[:, None], lower=0)
            if 0 < info <= P:
                if log:
                    log("Linear equation system singular after step %d i=%d" % (m, info))
                break
            q = q[:, 0]
            delta = d @ q
            delta_mag = float(delta @ delta)
            a, b_, c, Fa, Fb, Fc = _bracket(f_line(x, delta))
            xmin1, xmin2, F, F2 = _brent(f_line(x, delta), a, b_, c, Fb)
            x = x + xmin1 * delta
            o, E = resid(x)
            e = E[0].clone()
            F = float(o[0])
            if float(ferr[0] + berr[0]) > 1.0 and m > 5:
                break
            max_col = int(np.argmax(np.abs(p * q)))
            # gamma_update (opt_powell.cpp:397-434): secant column from the
            # two best line points; the displaced potential is evaluated
            _, E2 = resid((x + (xmin2 - xmin1) * delta)[None, :])
            f2 = E2[0]
            col = (e - f2) / (xmin1 - xmin2)
            mu = float((col * e).sum()) / F
            col = col - mu * e
            mag = float(torch.sqrt((col * col).sum()))
            if mag < NOTHING:
                if log:
                    log("Matrix gamma singular after step %d, restarting inner loop" % m)
                break
            gam[max_col] = col / mag
            delta = delta / mag
            d[:, max_col] = delta
            # lineqsys_update (opt_powell.cpp:476-493): -gamma^T e and
            # gamma^T gamma[:, max_col] in one pass over gamma
            pr = _gram(ev, gam, torch.stack((e, gam[max_col]))).cpu().numpy()
            p = -pr[:, 0]
            row = pr[:, 1]
            lin[max_col, :] = row
            lin[:, max_col] = row
            dF = F_old - F
            m += 1
            history.append((time.time() - t0, F))
            if max_evals and evals[0] >= max_evals:
                break
            if not ((m < P or (m <= INNERLOOPS and dF > PRECISION)) and dF < TOOBIG and delta_mag < TOOBIG):
                break
        if log:
            log("powell outer %d: F = %.10e (%d evaluations)" % (n_out + 1, F, evals[0]))
        # every 4th outer step, a trial rescale kept when F does not rise
        if (n_out + 1) % 4 == 0 and rescale:
            r = rescaler(ev, x, 0)
            if r is not None:
                F2 = float(r[0].objective(r[1][None, :], precision)[0])
                evals[0] += 1
                if log:
                    log("F before rescale = %f, after = %f" % (F, F2))
                if F2 <= F:
                    ev, x, res = r
                    o, E = resid(x)
                    F = float(o[0])
                    e = E[0].clone()
                    rescales.append((n_out, "flag 0"))
        n_out += 1
        outer_history.append((F, x.copy()))
        if max_evals and evals[0] >= max_evals:
            break
        if not (((F_older - F > PRECISION / 10.0) or (F_older - F < 0)) and (F_older - F > d_eps) and n_out < max_steps):
            break
    return x, F, dict(outer=n_out, evals=evals[0], seconds=time.time() - t0, history=history,
                      outer_history=outer_history, rescales=rescales, evaluator=ev)


# -------------------------------------------------------------------- L-BFGS

def lbfgs_fit(ev: Evaluator, x0, precision=MZ_FP64, maxiter: int = 1000, gtol: float = 1e-10,
              ftol: float = 1e-15, target: Optional[float] = None):
    """L-BFGS on the adjoint gradient.  With `target`, stops as soon as the
    objective reaches it.  Returns (x, F, info)."""
    from scipy.optimize import minimize
    t0 = time.time()
    history = []
    evals = [0]

    class Reached(Exception):
        pass

    best = [None, math.inf]

    def fg(x):
        o, g = ev.objective_grad(x[None, :], precision)
        evals[0] += 1
        F = float(o[0])
        if F < best[1]:
            best[0], best[1] = x.copy(), F
        history.append((time.time() - t0, F))
        if target is not None and F <= target:
            raise Reached()
        return F, g[0]

    try:
        r = minimize(fg, np.array(x0, dtype=np.float64), jac=True, method="L-BFGS-B",
                     options=dict(maxiter=maxiter, gtol=gtol, ftol=ftol, maxcor=30))
        x, F = r.x, float(r.fun)
    except Reached:
        x, F = best[0], best[1]
    if best[1] < F:
        x, F = best[0], best[1]
    return x, F, dict(evals=evals[0], seconds=time.time() - t0, history=history)


# ------------------------------------------------------- simulated annealing

def _bump(pot_layout, x, c, height, width):
    """Spline::modify_coeff (spline.cpp:120-149): a Gaussian bump of knot
    values around coefficient c, or a shift of an end slope."""
    kind, spline_coeffs = pot_layout[c]
    if kind == "grad":
        x[c] += height
        return
    # spline_coeffs: list of (knot index, coefficient index) of free knots of this spline
    knots = {k: ci for k, ci in spline_coeffs}
    kk = next(k for k, ci in spline_coeffs if ci == c)
    w = int(4 * width)
    for i in range(-w, w + 1):
        k = kk + i
        if k in knots:
            x[knots[k]] += 0.3989422804014326779 * math.exp(-i * i * 0.5 / (width * width)) * height


def coefficient_layout(pot):
    """For every coefficient: ('knot', free knots of its spline) or ('grad', None)."""
    out = []
    ci = 0
    for s in range(pot.nsplines):
        sp = pot.spline(s)
        free = []
        for k in range(sp["nknots"]):
            if not sp["y_fixed"][k]:
                free.append((k, ci))
                ci += 1
        for _ in free:
            out.append(("knot", free))
        for e in range(2):
            if not sp["grad_fixed"][e] and not sp["nat"][e]:
                out.append(("grad", None))
                ci += 1
    return out


def anneal_chains(ev: Evaluator, x0, nchains: int, temp: float, max_temps: int = 10, seed: int = 0,
                  precision=MZ_FP64, sweeps: Optional[int] = None):
    """Independent simulated-annealing chains (opt_simann.cpp:89-206), all
    chains' trial potentials evaluated in one launch per step.  Each chain
    sweeps the coefficients with Gaussian bumps (height N(0,1) v_c, width
    |N(0,1)|), accepts by Metropolis (opt_simann.cpp:239-264), adapts v_c
    every NSTEP sweeps and cools by TEMPVAR.  Returns (best x, best F, info)."""
    rng = np.random.default_rng(seed)
    layout = coefficient_layout(ev.pot)
    P = ev.ncoeff
    X = np.repeat(np.asarray(x0, dtype=np.float64)[None, :], nchains, axis=0)
    F = ev.objective(X, precision)
    best_x, best_F = X[np.argmin(F)].copy(), float(F.min())
    v = np.ones((nchains, P))
    T = temp
    sweeps = sweeps if sweeps is not None else 3 * P
    evals = nchains
    t0 = time.time()
    for k in range(max_temps):
        for m in range(sweeps):
            naccept = np.zeros((nchains, P), dtype=np.int64)
            for j in range(SA_NSTEP):
                for c in range(P):
                    trial = X.copy()
                    heights = rng.normal(size=nchains) * v[:, c]
                    widths = np.abs(rng.normal(size=nchains))
                    for ch in range(nchains):
                        _bump(layout, trial[ch], c, heights[ch], widths[ch])
                    F2 = ev.objective(trial, precision)
                    evals += nchains
                    u = rng.random(nchains)
                    with np.errstate(over="ignore"):
                        acc = (F2 <= F) | (u < np.exp(np.minimum((F - F2) / T, 0.0)))
                    X[acc] = trial[acc]
                    F[acc] = F2[acc]
                    naccept[acc, c] += 1
                    i = int(np.argmin(F))
                    if F[i] < best_F:
                        best_F, best_x = float(F[i]), X[i].copy()
            hi = naccept > 0.6 * SA_NSTEP
            lo = naccept < 0.4 * SA_NSTEP
            v[hi] *= 1 + SA_STEPVAR * (naccept[hi] / SA_NSTEP - 0.6) / 0.4
            v[lo] /= 1 + SA_STEPVAR * (0.4 - naccept[lo] / SA_NSTEP) / 0.4
        T *= SA_TEMPVAR
    return best_x, best_F, dict(evals=evals, seconds=time.time() - t0)


# ---------------------------------------------------------- genetic algorithm

def genetic_fit(ev: Evaluator, x0, pop_size: int = 32, generations: int = 10, cross_rate: float = 0.5,
                mut_rate: float = 0.02, fit_rate: float = 0.5, init_scale: float = 0.1, seed: int = 0,
                precision=MZ_FP64):
    """Genetic algorithm (opt_genalg.cpp:105-309): population seeded by
    Gaussian bumps of x0 scaled by init_scale, the two best kept, children
    bred by uniform crossover (at least one switch) and mutation from random
    members; every generation's children are evaluated in one launch."""
    rng = np.random.default_rng(seed)
    layout = coefficient_layout(ev.pot)
    P = ev.ncoeff
    x0 = np.asarray(x0, dtype=np.float64)
    pop = np.repeat(x0[None, :], pop_size, axis=0)
    for i in range(1, pop_size):
        for c in range(P):
            _bump(layout, pop[i], c, rng.normal() * pop[i, c] * init_scale, abs(rng.normal()))
    F = ev.objective(pop, precision)
    evals = pop_size
    order = np.argsort(F)
    pop, F = pop[order], F[order]
    t0 = time.time()
    history = [float(F[0])]
    for g in range(generations):
        children = pop.copy()
        parent = 0
        pool = list(range(1, pop_size - 1))
        for i in range(2, pop_size):
            if i > 2 and rng.random() < fit_rate:
                parent += 1
            while True:
                t = int(rng.random() * len(pool))
                parent2 = pool[t]
                if len(pool) == 1 and parent2 == parent:
                    parent += 1
                if parent2 != parent:
                    break
            pool.pop(t)
            switch = int(rng.random() * 2)
            success = False
            for c in range(P):
                if rng.random() < cross_rate:
                    switch = (switch + 1) % 2
                    success = True
                if c == P - 1 and not success:
                    switch = (switch + 1) % 2
                children[i, c] = pop[parent if switch == 0 else parent2, c]
                if rng.random() < mut_rate:
                    while True:
                        r = int(rng.random() * pop_size)
                        if r != parent and r != parent2:
                            break
                    children[i, c] = pop[r, c]
        Fc = ev.objective(children[2:], precision)
        evals += pop_size - 2
        F = np.concatenate([F[:2], Fc])
        pop = children
        order = np.argsort(F)
        pop, F = pop[order], F[order]
        history.append(float(F[0]))
    return pop[0].copy(), float(F[0]), dict(evals=evals, seconds=time.time() - t0, history=history)
