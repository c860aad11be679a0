"""Joint pose refinement of assembled groups through the CUDA adjoint (sherd_adjoint).

A group is G fragments with world poses W_g (fragment frame -> world) and E edges (a, b):
pairs whose fracture surfaces meet. For an edge, T = W_a^-1 W_b maps B's frame into A's. The
library returns, per (group pose, edge):
  * the point-to-plane energy E = 1/2 sum r^2 (the ICP's residual);
  * the smoothed tight counts (T_B, F_B) of B's fracture samples against A's fracture faces;
  * the same counts (T_A, F_A) of A's samples against B's faces;
  * the exact twist gradients of all five, with the matches and faces held fixed.

`GroupObjectives` is a torch.autograd.Function over the world poses W (P, G, 4, 4). Its
backward maps the edge twists to world-pose gradients through the SE(3) adjoint. Any rigid
parametrisation of W therefore gets exact gradients by autograd, for instance
W = exp(xi^) W0 through torch.linalg.matrix_exp.

Memory: the forward keeps only the (P, E, 5, 6) twist gradients, never a correspondence.
Each call recomputes the matches on the device.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _abi as A
from .backend import Context


def hat(xi: torch.Tensor) -> torch.Tensor:
    """(..., 6) twists (w, v) -> (..., 4, 4) elements of se(3)."""
    z = torch.zeros_like(xi[..., 0])
    w0, w1, w2, v0, v1, v2 = xi.unbind(-1)
    rows = [torch.stack([z, -w2, w1, v0], -1), torch.stack([w2, z, -w0, v1], -1),
            torch.stack([-w1, w0, z, v2], -1), torch.stack([z, z, z, z], -1)]
    return torch.stack(rows, -2)


def exp_se3(xi: torch.Tensor) -> torch.Tensor:
    return torch.linalg.matrix_exp(hat(xi))


def _skew(w: torch.Tensor) -> torch.Tensor:
    return hat(torch.cat([w, torch.zeros_like(w)], -1))[..., :3, :3]


def adjoint_transpose(m: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
    """Ad_M^T g for rigid M = (R, t) and twist covectors g = (g_w, g_v):
    (R^T (g_w - t x g_v), R^T g_v), where Ad_M (w, v) = (R w, R v + t x R w)."""
    rt = m[..., :3, :3].transpose(-1, -2)
    t = m[..., :3, 3]
    gw, gv = g[..., :3], g[..., 3:]
    top = (rt @ (gw - torch.linalg.cross(t, gv)).unsqueeze(-1)).squeeze(-1)
    bot = (rt @ gv.unsqueeze(-1)).squeeze(-1)
    return torch.cat([top, bot], -1)


@dataclass
class Group:
    """The edges of an assembled group on one context."""

    ctx: Context
    edges: list          # backend.Pair per edge: A = fragment a, B = fragment b
    a: np.ndarray        # (E,) fragment index of each edge's A
    b: np.ndarray        # (E,) fragment index of each edge's B
    n_fragments: int
    n_source: np.ndarray  # (E,) B's fracture sample count (the plane term's points)
    t: np.ndarray         # (E,) the pair's t
    opts: A.AdjointOptions
    centroid: np.ndarray | None = None  # (G, 3) each fragment's fracture centroid, own frame
    rho: np.ndarray | None = None       # (G,) RMS radius of its fracture samples about it

    def relative(self, w: np.ndarray):
        """(P, G, 4, 4) world poses -> T = W_a^-1 W_b and T^-1, each (P, E, 4, 4)."""
        inv = np.linalg.inv(w)
        t = inv[:, self.a] @ w[:, self.b]
        return t, inv[:, self.b] @ w[:, self.a]

    def evaluate(self, w: np.ndarray):
        """values (P, E, 5) and twist gradients (P, E, 5, 6) at world poses w."""
        t, ti = self.relative(w)
        return self.ctx.adjoint(self.edges, t, ti, self.opts)


class GroupObjectives(torch.autograd.Function):
    """values (P, E, 5) = E, T_B, F_B, T_A, F_A of every edge at world poses W (P, G, 4, 4)."""

    @staticmethod
    def forward(ctx, w: torch.Tensor, group: Group):
        values, grads = group.evaluate(w.detach().cpu().numpy().astype(np.float64))
        ctx.save_for_backward(w)
        ctx.grads = torch.from_numpy(grads).to(w)
        ctx.group = group
        return torch.from_numpy(values).to(w)

    @staticmethod
    def backward(ctx, gv: torch.Tensor):
        (w,) = ctx.saved_tensors
        group = ctx.group
        a = torch.as_tensor(group.a, device=w.device)
        b = torch.as_tensor(group.b, device=w.device)
        g = ctx.grads
        g_t = (gv[..., :3, None] * g[..., :3, :]).sum(-2)    # twist of T, A's frame
        g_ti = (gv[..., 3:, None] * g[..., 3:, :]).sum(-2)   # twist of T^-1, B's frame
        winv = torch.linalg.inv(w)
        # A world perturbation exp(d^) of W_b turns T into exp((Ad_{W_a^-1} d)^) T, and one of
        # W_a turns T^-1 into exp((Ad_{W_b^-1} d)^) T^-1; the other fragment sees the negative.
        u_t = adjoint_transpose(winv[:, a], g_t)
        u_ti = adjoint_transpose(winv[:, b], g_ti)
        gamma = torch.zeros(w.shape[0], group.n_fragments, 6, dtype=w.dtype, device=w.device)
        gamma.index_add_(1, b, u_t - u_ti)
        gamma.index_add_(1, a, u_ti - u_t)
        # The Euclidean gradient with the same pairing on every tangent direction d^ W:
        # <N W^-T, d^ W> = <N, d^> = gamma . d for N = [[skew(gamma_w) / 2, gamma_v], [0, 0]].
        n = torch.zeros_like(w)
        n[..., :3, :3] = 0.5 * _skew(gamma[..., :3])
        n[..., :3, 3] = gamma[..., 3:]
        return n @ winv.transpose(-1, -2), None


def alignment_loss(values: torch.Tensor, group: Group, plane_weight=1.0, tight_weight=0.1,
                   min_facing=20.0) -> torch.Tensor:
    """(P,) loss per group pose, summed over the edges:
    plane_weight * E / (n t^2), the mean squared point-to-plane residual in units of t^2,
    minus tight_weight * the mean of the two smoothed tight fractions T / max(F, min_facing)
    (R 6 returns 0 below 20 facing points, verify.rs:338-349)."""
    n = torch.as_tensor(group.n_source, dtype=values.dtype, device=values.device)
    t = torch.as_tensor(group.t, dtype=values.dtype, device=values.device)
    plane = values[..., 0] / (n * t * t)
    tight_b = values[..., 1] / values[..., 2].clamp_min(min_facing)
    tight_a = values[..., 3] / values[..., 4].clamp_min(min_facing)
    return (plane_weight * plane - tight_weight * 0.5 * (tight_a + tight_b)).sum(-1)


class _BudgetSpent(Exception):
    pass


def refine(group: Group, w0: np.ndarray, steps=50, fixed=0, stages=((0.2, 0.0), (0.08, 1.0)),
           plane_weight=1.0):
    """Joint refinement of every group pose in w0 (P, G, 4, 4), one twist per fragment with
    fragment `fixed` held (the objective is invariant to a common motion).

    Each fragment turns about its own fracture centroid c (world frame, at w0), so that its
    rotation and translation do not mix through the distance to the world origin:
    W = C exp(xi^) C^-1 W0. The twist is scaled so that a unit step moves the fragment's
    samples by about t: xi = (u_w t / rho, u_v t), with rho the RMS radius of its fracture
    samples about c.

    `stages` are (correspondence radius_k, tight_weight) pairs. Each gets an equal share of
    the `steps` objective evaluations (one sherd_adjoint call each) under L-BFGS with a
    strong-Wolfe line search, and ends at the best poses it evaluated. The default first
    closes the gap with the point-to-plane term at the first rung's radius. It then
    tightens with the smoothed tight fraction, whose distances are to the true faces and
    not to sampled planes. Returns the refined poses and the mean loss at each evaluation
    (at most `steps`)."""
    w0 = np.ascontiguousarray(w0, np.float64)
    p, g = w0.shape[:2]
    t_scale = float(np.min(group.t))
    local = np.zeros((g, 3)) if group.centroid is None else np.asarray(group.centroid)
    rho = np.full(g, t_scale) if group.rho is None else np.asarray(group.rho)
    scale = torch.from_numpy(np.concatenate([np.repeat((t_scale / rho)[:, None], 3, 1),
                                             np.full((g, 3), t_scale)], 1))[None]
    keep = torch.ones(1, g, 1, dtype=torch.float64)
    keep[0, fixed] = 0.0
    history = []
    radius0 = group.opts.radius_k
    per_stage = [steps // len(stages) + (1 if k < steps % len(stages) else 0)
                 for k in range(len(stages))]
    try:
        w = w0
        for (radius_k, tight_weight), n_eval in zip(stages, per_stage):
            group.opts = A.AdjointOptions(radius_k, group.opts.width_k, group.opts.window_k)
            c = np.einsum("pgij,gj->pgi", w[..., :3, :3], local) + w[..., :3, 3]
            to_c = torch.from_numpy(np.tile(np.eye(4), (p, g, 1, 1)))
            to_c[..., :3, 3] = torch.from_numpy(c)
            from_c = torch.linalg.inv(to_c)
            base = torch.from_numpy(w)
            u = torch.zeros(p, g, 6, dtype=torch.float64, requires_grad=True)

            def poses():
                return to_c @ exp_se3(u * scale * keep) @ from_c @ base

            opt = torch.optim.LBFGS([u], lr=1.0, max_iter=n_eval, max_eval=n_eval,
                                    history_size=20, line_search_fn="strong_wolfe",
                                    tolerance_grad=1e-12, tolerance_change=1e-15)
            best = [float("inf"), None]
            used = [0]

            def closure():
                if used[0] == n_eval:  # the line search may ask for more than the budget
                    raise _BudgetSpent
                used[0] += 1
                opt.zero_grad()
                loss = alignment_loss(GroupObjectives.apply(poses(), group), group,
                                      plane_weight, tight_weight).sum()
                loss.backward()
                value = float(loss.detach())
                history.append(value / p)
                if value < best[0]:
                    best[0], best[1] = value, u.detach().clone()
                return loss

            try:
                opt.step(closure)
            except _BudgetSpent:
                pass
            with torch.no_grad():
                u.copy_(best[1])
                w = poses().numpy()
    finally:
        group.opts = A.AdjointOptions(radius0, group.opts.width_k, group.opts.window_k)
    return w, history


def edge_errors(w: np.ndarray, group: Group, truth: np.ndarray):
    """Per group pose and edge, the error of the relative pose T = W_a^-1 W_b against the
    truth's: (rotation in degrees, displacement of B's fracture centroid), each (P, E)."""
    te = np.linalg.inv(w[:, group.a]) @ w[:, group.b]
    tt = np.linalg.inv(truth[group.a]) @ truth[group.b]
    d = np.linalg.inv(tt)[None] @ te
    cos = np.clip((np.trace(d[..., :3, :3], axis1=-2, axis2=-1) - 1.0) / 2.0, -1.0, 1.0)
    cb = np.asarray(group.centroid)[group.b]
    moved = np.einsum("peij,ej->pei", te[..., :3, :3], cb) + te[..., :3, 3]
    true = np.einsum("eij,ej->ei", tt[..., :3, :3], cb) + tt[..., :3, 3]
    return np.degrees(np.arccos(cos)), np.linalg.norm(moved - true[None], axis=-1)


def pose_errors(w: np.ndarray, truth: np.ndarray, centroid: np.ndarray, fixed=0):
    """Per group pose and fragment, the error of its pose relative to fragment `fixed` against
    the truth: (rotation in degrees, displacement of its fracture centroid `centroid` (G, 3,
    own frame) in length units), each of shape (P, G)."""
    rel = np.linalg.inv(w[:, fixed:fixed + 1]) @ w
    rel_true = np.linalg.inv(truth[fixed]) @ truth
    d = np.linalg.inv(rel_true)[None] @ rel
    cos = np.clip((np.trace(d[..., :3, :3], axis1=-2, axis2=-1) - 1.0) / 2.0, -1.0, 1.0)
    c = np.asarray(centroid)
    moved = np.einsum("pgij,gj->pgi", rel[..., :3, :3], c) + rel[..., :3, 3]
    true = np.einsum("gij,gj->gi", rel_true[..., :3, :3], c) + rel_true[..., :3, 3]
    return np.degrees(np.arccos(cos)), np.linalg.norm(moved - true[None], axis=-1)
