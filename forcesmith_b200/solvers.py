"""Step consumers driven by a GpuSession — the reference's CSolver family
(include/forcesmith/optimization/solver.hpp:13-150, src/optimization/solver.cpp).

Each solver has the reference's knobs and defaults, `honors_bounds()` and
`one_shot()`, and `minimize(sess, x, lower, upper, w_e, w_s)` returning
`(status, x, info)`.  The residual vector, the Jacobian and the normal
equations stay on the device: a step reads back D-sized vectors (and, for the
dogleg, the D×D JᵀJ), never J.

  LMSolver              EigenLMSolver       solver.cpp:67-85
  HybridSolver          EigenHybridSolver   solver.cpp:87-111
  DESolver              BoostDESolver       solver.cpp:113-155
  SurrogateDESolver     (none: DE with a learned pre-screen of trial vectors)
  NormalEquationsSolver NormalEquationsSolver solver.cpp:242-266

The reference's LM is MINPACK lmder (QR with column pivoting) and its hybrid
solver is Powell's dogleg on a finite-difference gradient; here LM is a
damped FP64 Cholesky on JᵀJ (device) with batched λ trials, and the dogleg is
a trust region on the Gauss–Newton model (F, J).  They minimise the same
objective ‖F‖²; their trajectories are not the reference's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Eigen::LevenbergMarquardtSpace::Status values the reference returns
LM_IMPROPER_INPUT = 0
LM_RELATIVE_REDUCTION_TOO_SMALL = 1
LM_RELATIVE_ERROR_TOO_SMALL = 2
LM_RELATIVE_ERROR_AND_REDUCTION_TOO_SMALL = 3
LM_TOO_MANY_FUNCTION_EVALUATION = 5
# Eigen::HybridNonLinearSolverSpace::Status
HY_RELATIVE_ERROR_TOO_SMALL = 1
HY_TOO_MANY_FUNCTION_EVALUATION = 2
HY_NOT_MAKING_PROGRESS_ITERATIONS = 5


def de_box(x, lower=None, upper=None):
    """The DE search box of BoostDESolver::minimize (solver.cpp:118-124): a
    finite bound is kept, an infinite one becomes x ∓ max(2|x|, 5e-4)."""
    x = np.asarray(x, np.float64)
    lo = np.full(x.size, -np.inf) if lower is None else np.asarray(lower, np.float64)
    hi = np.full(x.size, np.inf) if upper is None else np.asarray(upper, np.float64)
    half = np.maximum(2.0 * np.abs(x), 5e-4)
    lb = np.where(np.isfinite(lo), lo, x - half)
    ub = np.where(np.isfinite(hi), hi, x + half)
    return lb, ub


def _objectives(sess, xs, w_e, w_s):
    return sess.eval_population(np.atleast_2d(xs), w_e, w_s)


@dataclass
class LMSolver:
    """Levenberg–Marquardt with FP64 damped Cholesky steps on the device.

    Per iteration: one residual+Jacobian evaluation (normal equations formed
    on the device), then damping values λ·trial_factors solved by device
    Cholesky and their objectives evaluated together in one population
    launch.  The trial with the lowest objective among those with a
    positive gain ratio ρ is taken and λ is updated from it by Nielsen's
    rule λ·max(1/3, 1 − (2ρ − 1)³); when no trial decreases the objective, λ
    grows ×`reject_factor` and the trials repeat without a new Jacobian.

    Damping is Levenberg's λ·I (mode 0) starting from λ₀ = τ·max diag(JᵀJ)
    (Madsen–Nielsen).  Marquardt's λ·diag(JᵀJ) (mode 1, τ used as λ₀) is
    available but leaves knots that the data barely constrains almost
    undamped, and on spline fits those steps run away.

    Termination follows MINPACK's tests: `ftol` on the actual and predicted
    relative reduction (status 1), `xtol` on the relative step (status 2),
    both (3); still running after `max_iter` returns 2, as the reference does
    (solver.cpp:83-84); more than `maxfev` = 100·max_iter+100 objective
    evaluations returns 5.
    """
    max_iter: int = 500
    xtol: float = 1e-7
    ftol: float = 1e-7
    tau: float = 1e-3
    mode: int = 0
    trial_factors: tuple = (0.25, 1.0, 4.0)
    reject_factor: float = 16.0

    def honors_bounds(self):
        return False

    def one_shot(self):
        return False

    def minimize(self, sess, x, lower=None, upper=None, w_e=1.0, w_s=0.0, callback=None):
        x = np.array(x, np.float64)
        D = x.size
        info = dict(obj=[], lam=[], njev=0, nfev=0, iterations=0)
        if D == 0:
            return LM_IMPROPER_INPUT, x, info
        maxfev = max(self.max_iter, 1) * 100 + 100
        lam = None
        sess.set_params(x)
        status = None
        for it in range(self.max_iter):
            sess.jacobian_async(w_e, w_s)
            JtJ, g, obj = sess.normal_equations()
            info["njev"] += 1
            info["nfev"] += 1
            if it == 0:
                info["obj"].append(obj)
            diag = np.diag(JtJ).copy()
            if lam is None:
                lam = self.tau * (max(float(diag.max()), 1e-300) if self.mode == 0 else 1.0)
            if self.mode == 1:
                diag[diag <= 0.0] = 1.0
            else:
                diag[:] = 1.0
            accepted = False
            while not accepted:
                lams = [lam * f for f in self.trial_factors]
                steps = [sess.lm_step(l, self.mode) for l in lams]
                objs = _objectives(sess, np.stack([x + s for s in steps]), w_e, w_s)
                info["nfev"] += len(lams)
                best, best_rho = -1, 0.0
                for k, (l, s, o) in enumerate(zip(lams, steps, objs)):
                    pred = -float(g @ s) + l * float(s @ (diag * s))
                    rho = (obj - o) / pred if pred > 0.0 else -1.0
                    if np.isfinite(o) and rho > 0.0 and (best < 0 or o < objs[best]):
                        best, best_rho = k, rho
                if best >= 0:
                    accepted = True
                    s, o, l = steps[best], objs[best], lams[best]
                    pred = -float(g @ s) + l * float(s @ (diag * s))
                    x_new = x + s
                    act_rel = (obj - o) / obj if obj > 0 else 0.0
                    pred_rel = pred / obj if obj > 0 else 0.0
                    dnorm = math.sqrt(float(s @ s))
                    xnorm = math.sqrt(float(x_new @ x_new))
                    x, obj = x_new, o
                    lam = l * max(1.0 / 3.0, 1.0 - (2.0 * best_rho - 1.0) ** 3)
                    info["obj"].append(obj)
                    info["lam"].append(l)
                    f_conv = abs(act_rel) <= self.ftol and pred_rel <= self.ftol and best_rho <= 2.0
                    x_conv = dnorm <= self.xtol * xnorm
                    if f_conv and x_conv:
                        status = LM_RELATIVE_ERROR_AND_REDUCTION_TOO_SMALL
                    elif f_conv:
                        status = LM_RELATIVE_REDUCTION_TOO_SMALL
                    elif x_conv:
                        status = LM_RELATIVE_ERROR_TOO_SMALL
                else:
                    lam *= self.reject_factor
                    if lam > 1e16:
                        status = LM_RELATIVE_ERROR_TOO_SMALL  # no decrease along any damped step
                        break
                if info["nfev"] >= maxfev and status is None:
                    status = LM_TOO_MANY_FUNCTION_EVALUATION
                    break
            info["iterations"] = it + 1
            sess.set_params(x)
            if callback is not None:
                callback(it, x, obj)
            if status is not None:
                break
        if status is None:
            status = LM_RELATIVE_ERROR_TOO_SMALL  # the reference returns 2 while still running
        return status, x, info


@dataclass
class HybridSolver:
    """Trust-region dogleg on the Gauss–Newton model of ‖F‖².

    Each accepted point costs one residual+Jacobian evaluation.  The
    Gauss–Newton point is the device Cholesky solve of (JᵀJ + μI) p = −Jᵀr
    with a small Levenberg regulariser μ (from τ·max diag JᵀJ, ÷3 after a
    very successful step, ×2 after a poor or rejected one) so that knots the
    data barely constrain do not dominate it; the Cauchy point uses g = Jᵀr
    and JᵀJ read back (D×D).  The dogleg path is cut at the trust radius
    (initially radius0·max(‖x‖, 1)), which grows ×2 when a step at the
    boundary has gain ratio > 0.75 and shrinks to ¼ of the step below 0.25;
    a rejected step retries without a new Jacobian.  maxfev = max_iter·D as
    in the reference (solver.cpp:108); ten accepted steps in a row that each
    reduce the objective by less than 0.1 % stop it (status 5).
    """
    max_iter: int = 500
    xtol: float = 1e-7
    tau: float = 1e-3
    radius0: float = 0.1

    def honors_bounds(self):
        return False

    def one_shot(self):
        return False

    def minimize(self, sess, x, lower=None, upper=None, w_e=1.0, w_s=0.0):
        x = np.array(x, np.float64)
        D = x.size
        info = dict(obj=[], njev=0, nfev=0, iterations=0)
        if D == 0:
            return 0, x, info
        maxfev = self.max_iter * D
        sess.set_params(x)
        delta = None
        mu = None
        status = None
        stall = 0
        for it in range(self.max_iter):
            sess.jacobian_async(w_e, w_s)
            A, g, obj = sess.normal_equations()
            info["njev"] += 1
            info["nfev"] += 1
            if it == 0:
                info["obj"].append(obj)
            if mu is None:
                mu = self.tau * max(float(np.max(np.diag(A))), 1e-300)
            p_gn = sess.lm_step(mu, 0)
            gAg = float(g @ (A @ g))
            p_sd = -(float(g @ g) / gAg) * g if gAg > 0 else -g
            if delta is None:
                delta = self.radius0 * max(float(np.linalg.norm(x)), 1.0)
            while True:
                p = self._dogleg(p_gn, p_sd, delta)
                pred = -2.0 * float(g @ p) - float(p @ (A @ p))
                o = float(_objectives(sess, x + p, w_e, w_s)[0])
                info["nfev"] += 1
                rho = (obj - o) / pred if pred > 0 else -1.0
                pn = float(np.linalg.norm(p))
                if rho < 0.25:
                    delta = 0.25 * pn
                elif rho > 0.75 and pn >= 0.99 * delta:
                    delta = 2.0 * delta
                if rho > 0.0 and np.isfinite(o):
                    mu *= 1.0 / 3.0 if rho > 0.75 else (2.0 if rho < 0.25 else 1.0)
                    x = x + p
                    stall = 0 if (obj - o) > 1e-3 * obj else stall + 1
                    obj = o
                    info["obj"].append(obj)
                    break
                mu *= 2.0
                p_gn = sess.lm_step(mu, 0)
                if delta <= self.xtol * max(float(np.linalg.norm(x)), self.xtol):
                    status = HY_RELATIVE_ERROR_TOO_SMALL
                    break
                if info["nfev"] >= maxfev:
                    status = HY_TOO_MANY_FUNCTION_EVALUATION
                    break
            info["iterations"] = it + 1
            sess.set_params(x)
            if status is not None:
                break
            if delta <= self.xtol * max(float(np.linalg.norm(x)), self.xtol):
                status = HY_RELATIVE_ERROR_TOO_SMALL
                break
            if stall >= 10:
                status = HY_NOT_MAKING_PROGRESS_ITERATIONS
                break
        return (status if status is not None else HY_TOO_MANY_FUNCTION_EVALUATION), x, info

    @staticmethod
    def _dogleg(p_gn, p_sd, delta):
        if np.linalg.norm(p_gn) <= delta:
            return p_gn
        nsd = float(np.linalg.norm(p_sd))
        if nsd >= delta:
            return p_sd * (delta / nsd)
        d = p_gn - p_sd
        a = float(d @ d)
        b = 2.0 * float(p_sd @ d)
        c = nsd * nsd - delta * delta
        t = (-b + math.sqrt(max(b * b - 4 * a * c, 0.0))) / (2 * a)
        return p_sd + t * d


@dataclass
class DESolver:
    """Differential evolution on the device with BoostDESolver's knobs
    (solver.hpp:90-101): F = 0.65, CR = 0.5, NP = NP_factor·D, seeded; the
    search box is `de_box`; member 0 starts at clamp(x).  Generations run as
    a replayed CUDA graph."""
    mutation_factor: float = 0.65
    crossover_probability: float = 0.5
    NP_factor: int = 15
    max_generations: int = 1000
    seed: int = 42
    use_graph: bool = True

    def honors_bounds(self):
        return True

    def one_shot(self):
        return False

    def minimize(self, sess, x, lower=None, upper=None, w_e=1.0, w_s=0.0, history=False):
        x = np.array(x, np.float64)
        lb, ub = de_box(x, lower, upper)
        sess.de_init(lb, ub, x0=np.clip(x, lb, ub), NP=self.NP_factor * x.size,
                     mutation=self.mutation_factor, crossover=self.crossover_probability,
                     seed=self.seed, w_e=w_e, w_s=w_s)
        out = sess.de_run(self.max_generations, use_graph=self.use_graph, history=history)
        best, xb = out[0], out[1]
        sess.set_params(xb)
        info = dict(obj=best, generations=self.max_generations, lower=lb, upper=ub)
        if history:
            info["history"] = out[2]
        return 0, xb, info


@dataclass
class SurrogateDESolver(DESolver):
    """DESolver with learned pre-screening (no reference counterpart).

    A BF16 MLP D → 256 → 256 → 1 trained on the device (Adam, lr 1e-3) on
    the log objective of every exact evaluation ranks `screen` candidate
    trials per member; only the best-ranked one is evaluated exactly, and
    the exact objective alone decides acceptance.  The first
    `warm_generations` generations are plain DE, and a generation falls back
    to plain DE while the model's Spearman correlation on the held-out
    archive slice is below `gate`."""
    screen: int = 4
    warm_generations: int = 5
    batch: int = 512
    steps_per_generation: int = 32
    lr: float = 1e-3
    gate: float = 0.8
    holdout: float = 0.1

    def minimize(self, sess, x, lower=None, upper=None, w_e=1.0, w_s=0.0, history=False):
        x = np.array(x, np.float64)
        lb, ub = de_box(x, lower, upper)
        sess.de_init(lb, ub, x0=np.clip(x, lb, ub), NP=self.NP_factor * x.size,
                     mutation=self.mutation_factor, crossover=self.crossover_probability,
                     seed=self.seed, w_e=w_e, w_s=w_s)
        sess.surrogate_init(screen=self.screen, warm_generations=self.warm_generations,
                            batch=self.batch, steps_per_generation=self.steps_per_generation,
                            lr=self.lr, gate=self.gate, holdout=self.holdout, seed=self.seed)
        best, xb, info = sess.de_run_screened(self.max_generations)
        sess.set_params(xb)
        info.update(obj=best, generations=self.max_generations, lower=lb, upper=ub)
        return 0, xb, info


@dataclass
class NormalEquationsSolver:
    """One ridge-regularised Gauss–Newton step: x ← x − (JᵀJ + λI)⁻¹ Jᵀr,
    λ = ridge, or 1e-8·max(mean diag JᵀJ, 1) when ridge ≤ 0
    (solver.cpp:242-266).  Device Cholesky in place of LDLT."""
    ridge: float = 0.0

    def honors_bounds(self):
        return False

    def one_shot(self):
        return True

    def minimize(self, sess, x, lower=None, upper=None, w_e=1.0, w_s=0.0):
        x = np.array(x, np.float64)
        if x.size == 0:
            return 0, x, {}
        sess.set_params(x)
        sess.jacobian_async(w_e, w_s)
        x = x + sess.lsq_step(self.ridge)
        sess.set_params(x)
        return 0, x, {}


def make_default_solver(max_iter=500, xtol=1e-7, ftol=1e-7):
    """solver.cpp:268-271: the default solver is LM."""
    return LMSolver(max_iter=max_iter, xtol=xtol, ftol=ftol)
