"""Learned opening-angle controller (no reference counterpart).

A small network (12 -> 64 -> 64 -> 1, SiLU, bfloat16 weights at inference,
float32 accumulation) predicts each bucket's opening angle in [0.2, 1.0]
from features of the bucket's subtree and three of its ancestors.  All of it
runs in libcnb (csrc/controller.cu): the fused feature + inference kernel,
and the training kernels (forward/backward, parameter gradients, Adam).

Training pairs come from the batched boxes (cnb.core.batched): for sampled
buckets the plain fixed-theta traversal is run at every theta of a grid and
compared with the float64 direct sum; the labels are the per-bucket angles
that minimise the interactions while the global error percentile stays at
plain theta = 0.5's (allocate()).  Plain fixed-theta Barnes-Hut remains
the fallback (no weights: theta_per_bucket = None) and the reference for the
error budget.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .core.batched import BatchedBoxes

N_IN, N_H = 12, 64
N_PARAMS = _lib.MLP_PARAMS
THETA_GRID = (0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.0)


def _st():
    return int(torch.cuda.current_stream().cuda_stream)


class ThetaController:
    def __init__(self, device="cuda", seed=0):
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        p = np.zeros(N_PARAMS, np.float32)
        o = 0
        for fan_in, fan_out in ((N_IN, N_H), (N_H, N_H), (N_H, 1)):
            lim = np.sqrt(6.0 / (fan_in + fan_out))
            p[o:o + fan_in * fan_out] = rng.uniform(-lim, lim, fan_in * fan_out)
            o += fan_in * fan_out + fan_out   # weights then zero biases
        self.params = torch.from_numpy(p).to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.t = 0
        self.mean = torch.zeros(N_IN, device=self.device)
        self.std = torch.ones(N_IN, device=self.device)
        self.weights_bf16 = None

    # -------------------------------------------------------------- training
    def set_normalisation(self, X):
        """Fold a feature standardisation into the first layer later (export)."""
        self.mean = X.mean(0)
        self.std = X.std(0).clamp_min(1e-6)

    def _norm(self, X):
        return ((X - self.mean) / self.std).contiguous()

    def _grad_fn(self, n, tensor_cores):
        """A (X, y, g, loss, over_weight) -> None gradient call for n samples:
        the tensor-core kernels (bfloat16 contractions, float32 accumulation)
        or the float32 ones."""
        if tensor_cores:
            nbytes = int(_lib.load().cnb_mlp_grad_mma_scratch_bytes(n))
            scratch = torch.empty((nbytes + 15) // 16, 4, dtype=torch.float32, device=self.device)

            def fn(X, y, g, loss, ow):
                _lib.call("cnb_mlp_grad_mma", X.data_ptr(), y.data_ptr(), n, self.params.data_ptr(),
                          float(ow), scratch.data_ptr(), nbytes, g.data_ptr(), loss.data_ptr(), _st())
        else:
            scratch = torch.empty(4 * N_H * n + n, dtype=torch.float32, device=self.device)

            def fn(X, y, g, loss, ow):
                _lib.call("cnb_mlp_grad", X.data_ptr(), y.data_ptr(), n, self.params.data_ptr(),
                          float(ow), scratch.data_ptr(), g.data_ptr(), loss.data_ptr(), _st())
        return fn

    def grad(self, X, y, over_weight=4.0, tensor_cores=False):
        """Loss and gradient on the GPU (libcnb kernels) for normalised features X."""
        n = X.shape[0]
        g = torch.empty(N_PARAMS, dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self._grad_fn(n, tensor_cores)(X, y, g, loss, over_weight)
        return loss, g

    def train(self, X, y, steps=1500, lr=3e-3, over_weight=4.0, log_every=0, tensor_cores=True):
        """Full-batch Adam on (features X [n,12], labels y [n]); returns the loss
        curve.  tensor_cores: gradients from cnb_mlp_grad_mma (else cnb_mlp_grad)."""
        X = X.to(self.device, torch.float32)
        y = y.to(self.device, torch.float32).contiguous()
        self.set_normalisation(X)
        Xn = self._norm(X)
        n = Xn.shape[0]
        grad_fn = self._grad_fn(n, tensor_cores)
        g = torch.empty(N_PARAMS, dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        curve = []
        for it in range(steps):
            grad_fn(Xn, y, g, loss, over_weight)
            self.t += 1
            _lib.call("cnb_adam_step", self.params.data_ptr(), g.data_ptr(), self.m.data_ptr(),
                      self.v.data_ptr(), N_PARAMS, float(lr), 0.9, 0.999, 1e-8, self.t, _st())
            if it % 50 == 0 or it == steps - 1:
                curve.append(float(loss.item()))
        self.export()
        return curve

    def predict(self, X):
        """theta for raw features X (float32 weights)."""
        Xn = self._norm(X.to(self.device, torch.float32))
        out = torch.empty(Xn.shape[0], dtype=torch.float32, device=self.device)
        _lib.call("cnb_mlp_predict", Xn.data_ptr(), Xn.shape[0], self.params.data_ptr(),
                  out.data_ptr(), _st())
        return out

    # -------------------------------------------------------------- inference
    def folded_params(self):
        """Parameters with the feature standardisation folded into layer 1."""
        p = self.params.clone()
        W1 = p[:N_H * N_IN].view(N_H, N_IN)
        b1 = p[N_H * N_IN:N_H * N_IN + N_H]
        b1 -= (W1 * (self.mean / self.std)).sum(1)
        W1 /= self.std
        return p

    def export(self):
        """bfloat16 weights for the fused inference kernel."""
        p = self.folded_params()
        self.weights_bf16 = torch.empty(N_PARAMS, dtype=torch.bfloat16, device=self.device)
        _lib.call("cnb_to_bf16", p.data_ptr(), self.weights_bf16.data_ptr(), N_PARAMS, _st())
        return self.weights_bf16

    def theta_for_buckets(self, node_table, parents, workspace, n, accel, perm=None, out=None,
                          scale=1.0):
        """theta per bucket slot of a built tree (fused features + network);
        accel: the previous step's accelerations [N, 3], perm: row of accel
        for each body of the sorted order (None: the same order)."""
        if self.weights_bf16 is None:
            self.export()
        max_b = (workspace.numel() - 4) // 4
        if out is None:
            out = torch.empty(max_b, dtype=torch.float32, device=self.device)
        _lib.call("cnb_controller_theta", node_table.data_ptr(), parents.data_ptr(),
                  workspace.data_ptr(), n, accel.data_ptr(), perm.data_ptr() if perm is not None else None,
                  self.weights_bf16.data_ptr(), out.data_ptr(), max_b, _st())
        if scale != 1.0:
            out.mul_(scale).clamp_(0.2, 1.0)
        return out

    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), mean=self.mean.cpu().numpy(),
                 std=self.std.cpu().numpy())

    def load(self, path):
        d = np.load(path)
        self.params = torch.from_numpy(d["params"]).to(self.device)
        self.mean = torch.from_numpy(d["mean"]).to(self.device)
        self.std = torch.from_numpy(d["std"]).to(self.device)
        self.export()
        return self


def bucket_features(node_table, parents, workspace, n, accel, perm=None):
    max_b = (workspace.numel() - 4) // 4
    out = torch.empty((max_b, N_IN), dtype=torch.float32, device=node_table.device)
    _lib.call("cnb_bucket_features", node_table.data_ptr(), parents.data_ptr(), workspace.data_ptr(),
              n, accel.data_ptr(), perm.data_ptr() if perm is not None else None, out.data_ptr(),
              max_b, _st())
    nb = int(workspace[0].item())
    return out[:nb]


def direct_sum(pos, mass, targets, G, soft, periodic=False):
    """float64 direct sum (libcnb) for `targets` of one box: the minimum-image
    force law, or with `periodic` the periodic (Ewald) law."""
    T = targets.to(torch.int64).contiguous()
    out = torch.empty((T.numel(), 3), dtype=torch.float64, device=pos[0].device)
    _lib.call("cnb_direct_sum_ewald_f64" if periodic else "cnb_direct_sum_f64",
              *(p.data_ptr() for p in pos), mass.data_ptr(), pos[0].numel(),
              T.data_ptr(), T.numel(), float(G), float(soft), out.data_ptr(), _st())
    return out


def allocate(errors, costs, owner, budget, allowed):
    """Per-bucket choice of theta minimising the total cost subject to at most
    `allowed` bodies with an error above `budget` (the global-quantile
    constraint of the metric, not a per-bucket one).

    errors [T, n_bodies] per theta of the grid, costs [T, n_buckets] (body
    interactions of each bucket at each theta), owner [n_bodies] the bucket
    of each body.  Lagrangian relaxation: for a price lam per violating body
    every bucket picks the theta minimising cost + lam * violations; lam is
    bisected to the smallest price whose choice meets `allowed`.  Returns
    (index of the chosen theta per bucket, total cost, violations)."""
    errors = np.asarray(errors, np.float64)
    costs = np.asarray(costs, np.float64)
    T, G = costs.shape
    viol = np.zeros((T, G))
    for k in range(T):
        np.add.at(viol[k], owner, errors[k] > budget)

    def pick(lam):
        idx = np.argmin(costs + lam * viol, axis=0)
        return idx, viol[idx, np.arange(G)].sum()

    # with an unbounded price every bucket minimises its violations first
    big = costs[np.isfinite(costs)].max() * (G + 1) + 1.0   # infinite cost: a theta never chosen
    idx_big, v_big = pick(big)
    if v_big > allowed:
        return idx_big, float(costs[idx_big, np.arange(G)].sum()), float(v_big)
    lo, hi = 0.0, big
    idx_lo, v_lo = pick(lo)
    if v_lo <= allowed:
        return idx_lo, float(costs[idx_lo, np.arange(G)].sum()), float(v_lo)
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        _, v = pick(mid)
        if v <= allowed:
            hi = mid
        else:
            lo = mid
    idx, v = pick(hi)
    return idx, float(costs[idx, np.arange(G)].sum()), float(v)


def _per_body_errors(got, ref, refn):
    return ((got.double() - ref).norm(dim=1) / refn).cpu().numpy()


def make_labels(bb: BatchedBoxes, theta_grid=THETA_GRID, budget=None, per_box=48, seed=0,
                error="relative", objective=None, quantile=99.0):
    """(features, labels, info) for sampled buckets of every box of `bb`.

    For every theta of the grid the traversal runs with that theta in every
    bucket (a body's force depends only on its own bucket's theta); each
    sampled bucket's bodies are compared with the float64 direct sum of
    their box (minimum image, or periodic for the "ewald" test), relative to
    the body's own acceleration (error="relative") or to the box's RMS
    acceleration (error="rms").  `budget` None: the `quantile`-th percentile
    error of plain theta = 0.5 over all sampled bodies.

    objective "lagrangian" (default under the periodic law, which reports
    per-bucket costs): the labels are the per-bucket angles that minimise the
    sampled buckets' total interactions while no more bodies exceed the
    budget than under plain theta = 0.5 -- the metric's own constraint (a
    global percentile), found by allocate(); info["bound"] is that
    allocation's cost ratio against plain theta = 0.5, an upper bound for any
    per-bucket policy on these buckets.  objective "worst": the largest theta
    whose worst body stays within the budget (a stricter, per-bucket rule).

    The features' acceleration input is the plain theta = 0.5 force of the
    same state (the previous step's force in a running simulation)."""
    rng = np.random.default_rng(seed)
    periodic = bb.mac == _lib.MAC_EWALD
    if objective is None:
        objective = "lagrangian" if periodic else "worst"
    if objective == "lagrangian" and not periodic:
        raise ValueError("per-bucket costs are recorded under the periodic (Ewald) law only")
    bb.sort_and_build()
    bk = bb.buckets().cpu().numpy()
    nb = bk.shape[0]
    tpb = torch.full((max(nb, 1),), 0.5, dtype=torch.float32, device=bb.device)
    bb.compute_forces(theta_per_bucket=tpb)
    accel = bb.force.clone()
    feats = bucket_features(bb.table, bb.parent, bb.workspace, bb.n, accel)
    box_of = np.searchsorted(bb.offsets, bk[:, 0], side="right") - 1
    chosen = []
    for b in range(bb.n_boxes):
        idx = np.nonzero(box_of == b)[0]
        chosen.extend(rng.choice(idx, min(per_box, idx.size), replace=False).tolist())
    chosen = np.array(sorted(chosen))
    # bodies of the chosen buckets and their float64 direct sums, box by box
    bodies, owner = [], []
    ref = []
    for b in range(bb.n_boxes):
        sel = chosen[box_of[chosen] == b]
        if sel.size == 0:
            continue
        t = np.concatenate([np.arange(bk[g, 0], bk[g, 0] + bk[g, 1]) for g in sel])
        o = np.concatenate([np.full(bk[g, 1], k) for k, g in zip(np.searchsorted(chosen, sel), sel)])
        sl = bb.box_slice(b)
        local = torch.from_numpy(t - sl.start).to(bb.device)
        soft = 0.5 / bb.boxes[b]["n_grid"]
        ref.append(direct_sum([p[sl] for p in bb.pos], bb.mass[sl], local, bb.G, soft,
                              periodic=periodic))
        bodies.append(t)
        owner.append(o)
    box_rms = [r.norm(dim=1).pow(2).mean().sqrt().expand(r.shape[0]) for r in ref]
    bodies = torch.from_numpy(np.concatenate(bodies)).to(bb.device)
    owner = np.concatenate(owner)
    ref = torch.cat(ref)
    refn = ref.norm(dim=1) if error == "relative" else torch.cat(box_rms)
    T = len(theta_grid)
    body_err = np.zeros((T, bodies.numel()))
    costs = np.zeros((T, chosen.size))
    counts = bk[chosen, 1].astype(np.float64)
    inter = torch.zeros(max(nb, 1), dtype=torch.int32, device=bb.device)
    cost = []
    for k, th in enumerate(theta_grid):
        tpb = torch.full((max(nb, 1),), float(th), dtype=torch.float32, device=bb.device)
        bb.stats.zero_()
        bb.compute_forces(theta_per_bucket=tpb, bucket_inter=inter if periodic else None)
        body_err[k] = _per_body_errors(bb.force[bodies], ref, refn)
        if periodic:
            costs[k] = inter[torch.from_numpy(chosen).to(bb.device)].cpu().numpy() * counts
        cost.append(float(bb.stats[0].item()) / bb.n)
    bb.check()
    k05 = theta_grid.index(0.5)
    if budget is None:
        budget = float(np.percentile(body_err[k05], quantile))
    info = dict(budget=budget, error=error, objective=objective, cost_per_theta=cost,
                n_samples=int(chosen.size), n_bodies=int(bodies.numel()))
    if objective == "lagrangian":
        allowed = int((body_err[k05] > budget).sum())
        idx, total, v = allocate(body_err, costs, owner, budget, allowed)
        labels = np.asarray(theta_grid, np.float32)[idx]
        plain_cost = costs[k05].sum()
        info.update(allowed_violations=allowed, violations=v, bound=float(plain_cost / total))
    else:
        errs = np.zeros((T, chosen.size))
        for k in range(T):
            np.maximum.at(errs[k], owner, body_err[k])
        ok = errs <= budget
        labels = np.full(chosen.size, theta_grid[0], np.float32)
        for k, th in enumerate(theta_grid):
            labels[ok[k]] = th      # ascending grid: the largest passing theta wins
        info["saturated"] = float(np.mean(~ok.any(axis=0)))
    info["label_hist"] = np.bincount(np.searchsorted(theta_grid, labels), minlength=T).tolist()
    return feats[torch.from_numpy(chosen).to(bb.device)], torch.from_numpy(labels).to(bb.device), info
