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


def refine(group: Group, w0: np.ndarray, steps=50, fixed=0, lr_rot=1e-3, lr_trans=0.02,
           plane_weight=1.0, tight_weight=0.1):
    """Joint refinement of every group pose in w0 (P, G, 4, 4): W = exp(xi^) W0 with one twist
    per fragment, fragment `fixed` held (the objective is invariant to a common motion), Adam
    steps of lr_rot radians and lr_trans * t with a cosine decay. Returns the refined poses
    and the mean loss before each step."""
    w0t = torch.from_numpy(np.ascontiguousarray(w0, np.float64))
    p, g = w0t.shape[:2]
    t_scale = float(np.min(group.t))
    rot = torch.zeros(p, g, 3, dtype=torch.float64, requires_grad=True)
    trans = torch.zeros(p, g, 3, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([{"params": [rot], "lr": lr_rot},
                            {"params": [trans], "lr": lr_trans * t_scale}])
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    keep = torch.ones(1, g, 1, dtype=torch.float64)
    keep[0, fixed] = 0.0
    history = []
    for _ in range(steps):
        opt.zero_grad()
        w = exp_se3(torch.cat([rot * keep, trans * keep], -1)) @ w0t
        loss = alignment_loss(GroupObjectives.apply(w, group), group, plane_weight, tight_weight)
        loss.sum().backward()
        history.append(float(loss.mean()))
        opt.step()
        sched.step()
    with torch.no_grad():
        w = exp_se3(torch.cat([rot * keep, trans * keep], -1)) @ w0t
    return w.numpy(), history


def pose_errors(w: np.ndarray, truth: np.ndarray, fixed=0):
    """Per group pose and fragment, the error of the pose relative to fragment `fixed` against
    the truth: (rotation in degrees, translation) arrays of shape (P, G)."""
    rel = np.linalg.inv(w[:, fixed:fixed + 1]) @ w
    rel_true = np.linalg.inv(truth[fixed]) @ truth
    d = np.linalg.inv(rel_true)[None] @ rel
    cos = np.clip((np.trace(d[..., :3, :3], axis1=-2, axis2=-1) - 1.0) / 2.0, -1.0, 1.0)
    return np.degrees(np.arccos(cos)), np.linalg.norm(d[..., :3, 3], axis=-1)
