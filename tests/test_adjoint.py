"""The adjoint of the group-alignment objectives (sherd_adjoint) and its torch wrapper.

No reference function computes these gradients; they are checked against the mathematics:
  * FP64 central finite differences (h = 1e-6) of the oracle's own f64 objective with the
    matches and faces held fixed, per twist component;
  * the ICP's analytic Jacobian: the point-to-plane twist gradient is J^T r of the normal
    equations (matching/icp.rs:599-640) at the same pose;
  * the torch Function's world-pose gradient, through the SE(3) adjoint, against central
    differences of the whole group objective;
  * on the GPU, the CUDA adjoint against the oracle (values and gradients), and a 50-step
    joint refinement that shrinks the pose error of perturbed assembled groups.
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest
import scipy.linalg as sl

from _slab import oracle_pair

H = 1e-6
OPTS = dict(radius_k=0.04, width_k=0.01, window_k=30.0)


def _hat(x):
    w, v = x[:3], x[3:]
    return np.array([[0.0, -w[2], w[1], v[0]], [w[2], 0.0, -w[0], v[1]],
                     [-w[1], w[0], 0.0, v[2]], [0.0, 0.0, 0.0, 0.0]])


def _near_accepted_pose(slab, seed=1):
    k = int(np.argmax(slab["s2_accepted"]))
    rng = np.random.default_rng(seed)
    xi = np.r_[rng.normal(size=3) * 0.002, rng.normal(size=3) * 0.05]
    return sl.expm(_hat(xi)) @ slab["s2_T_frac2"][k]


@pytest.fixture(scope="module")
def cpu_pair(oracle, slab):
    return oracle_pair(oracle, slab)


def test_oracle_gradients_match_central_differences(oracle, slab, cpu_pair):
    opts = oracle.AdjointOptions(**OPTS)
    t = _near_accepted_pose(slab)
    ti = np.linalg.inv(t)
    values, grads, assign = oracle.adjoint(cpu_pair["pair"], t, ti, opts)
    assert values[0] > 0 and values[2] > 20 and values[4] > 20
    for k in range(5):
        fd = np.zeros(6)
        for j in range(6):
            e = np.zeros(6)
            e[j] = H
            if k < 3:   # T moves B's samples: perturb T in A's frame
                tp, tm = sl.expm(_hat(e)) @ t, sl.expm(_hat(-e)) @ t
                vp = oracle.adjoint(cpu_pair["pair"], tp, np.linalg.inv(tp), opts, assign)[0]
                vm = oracle.adjoint(cpu_pair["pair"], tm, np.linalg.inv(tm), opts, assign)[0]
            else:       # T^-1 moves A's samples: perturb T^-1 in B's frame
                ip, im = sl.expm(_hat(e)) @ ti, sl.expm(_hat(-e)) @ ti
                vp = oracle.adjoint(cpu_pair["pair"], np.linalg.inv(ip), ip, opts, assign)[0]
                vm = oracle.adjoint(cpu_pair["pair"], np.linalg.inv(im), im, opts, assign)[0]
            fd[j] = (vp[k] - vm[k]) / (2 * H)
        scale = np.max(np.abs(grads[k]))
        assert np.max(np.abs(fd - grads[k])) <= 1e-6 * scale, (k, fd, grads[k])


def test_plane_gradient_is_the_icp_normal_equations_jtr(oracle, slab, cpu_pair):
    opts = oracle.AdjointOptions(**OPTS)
    t = _near_accepted_pose(slab, seed=2)
    _, grads, _ = oracle.adjoint(cpu_pair["pair"], t, np.linalg.inv(t), opts)
    sc = cpu_pair["scales"]
    _, jtr = oracle.normal_equations(cpu_pair["b"]["arrays"]["frac_p"], cpu_pair["frac_t"], t,
                                     OPTS["radius_k"] * sc.t * sc.icp)
    assert np.max(np.abs(grads[0] - jtr)) <= 1e-12 * np.max(np.abs(jtr))


class _OracleContext:
    """Answers Context.adjoint with the oracle, assignments held at the first call's."""

    def __init__(self, oracle, pair):
        self.oracle, self.pair, self.assign = oracle, pair, None

    def adjoint(self, edges, poses, inverses, opts):
        o = self.oracle.AdjointOptions(opts.radius_k, opts.width_k, opts.window_k)
        poses = np.asarray(poses).reshape(-1, len(edges), 4, 4)
        inverses = np.asarray(inverses).reshape(poses.shape)
        vals = np.empty(poses.shape[:2] + (5,))
        grads = np.empty(poses.shape[:2] + (5, 6))
        for p in range(poses.shape[0]):
            v, g, a = self.oracle.adjoint(self.pair, poses[p, 0], inverses[p, 0], o, self.assign)
            self.assign = a
            vals[p, 0], grads[p, 0] = v, g
        return vals, grads


def test_group_function_gradient_matches_central_differences(oracle, slab, cpu_pair):
    """The autograd Function over world poses, with the edge twists mapped through the SE(3)
    adjoint, against central differences of the loss in the fragments' world twists."""
    import torch
    adj = importlib.import_module("sherd-refit_b200.adjoint")
    abi = importlib.import_module("sherd-refit_b200._abi")
    rng = np.random.default_rng(3)
    wa = sl.expm(_hat(np.r_[rng.normal(size=3) * 0.7, rng.normal(size=3) * 40.0]))
    w = np.stack([wa, wa @ _near_accepted_pose(slab, seed=4)])[None]
    sc = cpu_pair["scales"]
    group = adj.Group(ctx=_OracleContext(oracle, cpu_pair["pair"]), edges=[None],
                      a=np.array([0]), b=np.array([1]), n_fragments=2,
                      n_source=np.array([len(cpu_pair["b"]["arrays"]["frac_p"])]),
                      t=np.array([sc.t]), opts=abi.AdjointOptions(**OPTS))

    def loss_at(xi):
        wt = adj.exp_se3(xi) @ torch.from_numpy(w)
        return adj.alignment_loss(adj.GroupObjectives.apply(wt, group), group, 1.0, 0.5).sum()

    xi = torch.zeros(1, 2, 6, dtype=torch.float64, requires_grad=True)
    loss_at(xi).backward()
    got = xi.grad.numpy()[0]
    fd = np.zeros((2, 6))
    with torch.no_grad():
        for g in range(2):
            for j in range(6):
                e = torch.zeros(1, 2, 6, dtype=torch.float64)
                e[0, g, j] = H
                fd[g, j] = (float(loss_at(e)) - float(loss_at(-e))) / (2 * H)
    assert np.max(np.abs(got - fd)) <= 1e-6 * np.max(np.abs(fd)), (got, fd)
    # A common motion of both fragments changes nothing.
    assert np.max(np.abs(got[0] + got[1] - 0.0)) <= 1e-9 * np.max(np.abs(got))


# ---- on the device -------------------------------------------------------------------------------


@pytest.mark.gpu
def test_cuda_adjoint_matches_the_oracle(sherd, gpu_ctx, gpu_slab, oracle, slab, cpu_pair):
    """Same matches and faces (bit-exact searches), f64 sums in another order: values and
    gradients within 1e-10 of their scale."""
    poses = np.stack([_near_accepted_pose(slab, seed) for seed in (5, 6, 7)])
    inverses = np.linalg.inv(poses)
    got_v, got_g = gpu_ctx.adjoint([gpu_slab["pair"]], poses[:, None], inverses[:, None],
                                   sherd.AdjointOptions(**OPTS))
    o = oracle.AdjointOptions(**OPTS)
    for k in range(len(poses)):
        v, g, _ = oracle.adjoint(cpu_pair["pair"], poses[k], inverses[k], o)
        assert np.all(np.abs(got_v[k, 0] - v) <= 1e-10 * np.maximum(np.abs(v), 1.0)), (got_v[k], v)
        for j in range(5):
            assert np.max(np.abs(got_g[k, 0, j] - g[j])) <= 1e-9 * np.max(np.abs(g[j])), (j,)


@pytest.mark.gpu
def test_adjoint_refuses_bad_arguments(sherd, gpu_ctx, gpu_slab):
    t = np.tile(np.eye(4), (1, 1, 1, 1))
    with pytest.raises(sherd.SherdError):
        gpu_ctx.adjoint([gpu_slab["pair"]], t, t, sherd.AdjointOptions(0.0, 0.01, 30.0))
    bad = t.copy()
    bad[0, 0, 0, 3] = np.nan
    with pytest.raises(sherd.SherdError):
        gpu_ctx.adjoint([gpu_slab["pair"]], bad, t, sherd.AdjointOptions(0.04, 0.01, 30.0))


@pytest.mark.gpu
def test_group_refinement_shrinks_the_pose_error(sherd, gpu_ctx):
    """A perturbed assembled pot (8 fragments, 18 edges; 0.5 deg and 0.2 t per fragment):
    50 joint evaluations lower the loss, raise every edge's smoothed tight fraction towards
    the truth's and shrink the relative pose errors of the edges."""
    synth = importlib.import_module("sherd-refit_b200.synth")
    workload = importlib.import_module("sherd-refit_b200.workload")
    adj = importlib.import_module("sherd-refit_b200.adjoint")
    wl = synth.make("pot", 0)
    dev = workload.to_device(gpu_ctx, wl)
    group = workload.assembled_group(dev, wl)
    truth, w0 = workload.perturbed_group_poses(wl, 4, seed=1)
    w, history = adj.refine(group, w0, steps=50)
    assert len(history) == 50 and min(history[25:]) < history[25]
    rot0, disp0 = adj.edge_errors(w0, group, truth)
    rot1, disp1 = adj.edge_errors(w, group, truth)
    assert rot1.mean() < 0.8 * rot0.mean(), (rot0.mean(), rot1.mean())
    assert disp1.mean() < 0.5 * disp0.mean(), (disp0.mean(), disp1.mean())
    v0, _ = group.evaluate(w0)
    v1, _ = group.evaluate(w)
    assert (v1[..., 1] / v1[..., 2]).mean() > 4 * (v0[..., 1] / v0[..., 2]).mean()
