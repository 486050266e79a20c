"""Batched gradient fabric inversion: per-grain c-axis angles of several ice
disks fitted to their multi-azimuth pulse-echo traces by L-BFGS.

Each disk is one seeded specimen (pefdtd.workloads) observed at a set of
azimuths; azimuth ``a`` turns the disk about its axis by -a, geometry and
c-axes together, as the reference's sweeps do (sim/core/rotation_test.py:
60-137, the axes rotated by ``axes @ R``), so a grain with c-axis angles
(theta, phi) in the specimen frame has (theta, phi - a) in the solve. The
misfit is J = sum over disks and azimuths of 0.5 ||traces - d||^2 and its
gradient with respect to every grain's (theta, phi) comes from the
hand-written adjoint (pefdtd.adjoint.misfit_gradients: all solves of an
evaluation batched, in waves that fit the device memory) chained through the
differentiable table ``adjoint.ice_table21`` by torch autograd. L-BFGS runs
on the concatenated angle vector (SciPy's L-BFGS-B, no bounds).

With a torch.distributed process group the (disk, azimuth) solves are dealt
to the ranks by cost (pefdtd.shard.assign) and the misfit and the gradient
vector are summed over the ranks with one all_reduce per evaluation; every
rank then takes the same L-BFGS step.

The reference has no FDTD inversion: its fabric fits are a 2-parameter
Watson (alpha, kappa) Nelder-Mead on ray/Born observables
(sim/model/fit_fabric.py:224-274) and ringfwi's Levenberg-Marquardt with a
finite-difference Jacobian (vendor/ringfwi/cof.py:85-140). The comparison
this module offers is the same inversion run plain, one solve at a time
(``batched=False``), which takes the same steps.
"""
from __future__ import annotations

import time

import numpy as np

from . import adjoint, shard, workloads


def rotate_labels(lab, az_deg):
    """The label volume turned by -az_deg about the grid's z axis: every
    z-plane resampled at the nearest cell (np.rint) of the rotated sampling
    points, as the reference's rotated_grid resamples; -1 (fluid) where a
    sample falls outside the grid."""
    lab = np.asarray(lab)
    nz, ny, nx = lab.shape
    a = np.radians(az_deg)
    ca, sa = np.cos(a), np.sin(a)
    X, Y = np.meshgrid(np.arange(nx) - (nx - 1) / 2.0, np.arange(ny) - (ny - 1) / 2.0, indexing="xy")
    xs = np.rint(ca * X - sa * Y + (nx - 1) / 2.0).astype(int)
    ys = np.rint(sa * X + ca * Y + (ny - 1) / 2.0).astype(int)
    ok = (xs >= 0) & (xs < nx) & (ys >= 0) & (ys < ny)
    xs, ys = np.clip(xs, 0, nx - 1), np.clip(ys, 0, ny - 1)
    out = lab[:, ys, xs]
    out[:, ~ok] = -1
    return out.astype(lab.dtype)


class Disk:
    """One specimen observed at several azimuths: its per-azimuth solves
    (adjoint.Problem) and its true c-axes."""

    def __init__(self, spec, azimuths_deg, nt=None, dtype="float32", checkpoint_every=200,
                 use_gpu=None):
        p = workloads.make_problem(spec, nt=nt, use_gpu=use_gpu)
        self.base = p
        self.azimuths = [float(a) for a in azimuths_deg]
        self.n_grains = int(p["n_grains"])
        self.true_axes = np.asarray(p["axes"], float)
        self.problems = []
        for az in self.azimuths:
            lab = rotate_labels(p["lab"], az)
            pts = workloads.top_probe(lab, p["h"], p["spec"]["aperture"])
            w = 1.0 / len(pts)
            self.problems.append(adjoint.Problem(
                (lab + 1).astype(np.uint16), p["rho_t"], p["h"], p["dt"], p["coeffs"],
                [(q, w) for q in pts], [(pts, np.full(len(pts), w))], p["wavelet"], record="vz",
                sponge_width=p["sponge"], damped_record=True, dtype=dtype,
                checkpoint_every=checkpoint_every))

    def cost(self):
        return float(np.prod(self.base["lab"].shape)) * float(len(self.base["wavelet"]))


def tables21(theta, phi, az_deg):
    """(n_g + 1, 21) stiffness table of one azimuth from the specimen-frame
    angles (torch float64, differentiable)."""
    import torch
    return adjoint.ice_table21(theta, phi - torch.as_tensor(np.radians(az_deg), dtype=torch.float64))


def isotropic_angles(n, rng):
    """Per-grain (theta, phi) of an isotropic fabric: c-axes uniform on the
    upper hemisphere (c and -c are the same axis)."""
    theta = np.arccos(rng.uniform(0.0, 1.0, n))
    phi = rng.uniform(-np.pi, np.pi, n)
    return theta, phi


def axes_of(theta, phi):
    st = np.sin(theta)
    return np.stack([st * np.cos(phi), st * np.sin(phi), np.cos(theta)], axis=1)


def eigen_error(axes_a, axes_b):
    """Largest difference between the orientation tensors' eigenvalues."""
    from .specimen import orientation_tensor
    return float(np.abs(orientation_tensor(axes_a)[0] - orientation_tensor(axes_b)[0]).max())


def _plain(problems, c21s, dobs):
    """misfit_gradients one solve at a time (the plain loop)."""
    out = []
    for p, c, d in zip(problems, c21s, dobs):
        out.extend(adjoint.misfit_gradients([p], [c], [d]))
    return out


class FabricInversion:
    """J(x) and dJ/dx for the concatenated per-grain angles x = [theta_0,
    phi_0, theta_1, phi_1, ...] of the disks, and L-BFGS on it.

    ``misfit_fn(problems, c21s, dobs) -> [(J, dJ/dc21)]`` computes the solves
    of one rank: adjoint.misfit_gradients (batched) by default, the plain
    loop with ``batched=False``; tests pass a stand-in. ``group``: a
    torch.distributed process group, or None for the default group when one
    is initialised."""

    def __init__(self, disks, d_obs, misfit_fn=None, batched=True, group=None):
        self.disks = list(disks)
        self.d_obs = d_obs
        self.misfit_fn = misfit_fn or (adjoint.misfit_gradients if batched else _plain)
        self.group = group
        self.jobs = [(k, a) for k, d in enumerate(self.disks) for a in range(len(d.azimuths))]
        rank, world = shard._group_info(group)
        self.rank, self.world = rank, world
        costs = [self.disks[k].cost() for k, _ in self.jobs]
        self.mine = [self.jobs[i] for i in shard.assign(costs, world)[rank]]
        self.sizes = [d.n_grains for d in self.disks]
        self.offsets = np.concatenate([[0], np.cumsum([2 * n for n in self.sizes])]).astype(int)
        self.n_params = int(self.offsets[-1])
        # the misfit is normalised by the observed records' energy 0.5 sum ||d||^2,
        # so that L-BFGS works on an O(1) objective (raw trace misfits are ~1e-20,
        # where the line search breaks down)
        e = sum(0.5 * float(np.sum(np.asarray(d, float) ** 2)) for per in d_obs for d in per
                if d is not None)
        self.scale = 1.0 / e if e > 0 else 1.0

    def split(self, x):
        x = np.asarray(x, float)
        return [(x[o:o + n], x[o + n:o + 2 * n]) for o, n in zip(self.offsets[:-1], self.sizes)]

    def objective(self, x):
        """(J, dJ/dx) summed over all disks and azimuths (all ranks), J
        normalised by the observed records' energy."""
        import torch
        parts = self.split(x)
        leaves = {}
        tabs, probs, dobs = [], [], []
        for k, a in self.mine:
            if k not in leaves:
                th, ph = parts[k]
                leaves[k] = (torch.tensor(th, dtype=torch.float64, requires_grad=True),
                             torch.tensor(ph, dtype=torch.float64, requires_grad=True))
            th, ph = leaves[k]
            tabs.append(tables21(th, ph, self.disks[k].azimuths[a]))
            probs.append(self.disks[k].problems[a])
            dobs.append(self.d_obs[k][a])
        J = 0.0
        g = np.zeros(self.n_params)
        if probs:
            res = self.misfit_fn(probs, [t.detach().numpy() for t in tabs], dobs)
            loss = 0.0
            for t, (j, G) in zip(tabs, res):
                J += float(j)
                loss = loss + (t * torch.as_tensor(np.asarray(G)[:t.shape[0]], dtype=torch.float64)).sum()
            loss.backward()
            for k, (th, ph) in leaves.items():
                o, n = self.offsets[k], self.sizes[k]
                g[o:o + n] = th.grad.numpy()
                g[o + n:o + 2 * n] = ph.grad.numpy()
        if self.world > 1:
            import torch.distributed as dist
            buf = torch.from_numpy(np.concatenate([[J], g]))
            if dist.get_backend(self.group) == "nccl":
                buf = buf.to(torch.device("cuda", torch.cuda.current_device()))
            dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=self.group)
            buf = buf.cpu().numpy()
            J, g = float(buf[0]), buf[1:].copy()
        return J * self.scale, g * self.scale

    def run(self, x0, iterations=10):
        """L-BFGS from x0 for `iterations` iterations. Returns a dict: x, J at
        x0 and at the end, and per iteration the misfit, the wall time and
        the number of (batched) evaluations it took."""
        from scipy.optimize import minimize
        evals = []

        def fun(x):
            J, g = self.objective(x)
            evals.append(J)
            return J, g

        its = []
        mark = [0, time.perf_counter()]

        def cb(intermediate_result):
            now = time.perf_counter()
            its.append({"J": float(intermediate_result.fun), "s": now - mark[1],
                        "evals": len(evals) - mark[0]})
            mark[0], mark[1] = len(evals), now

        r = minimize(fun, np.asarray(x0, float), jac=True, method="L-BFGS-B", callback=cb,
                     options={"maxiter": int(iterations), "maxcor": 10, "gtol": 0.0, "ftol": 0.0})
        return {"x": r.x, "J0": float(evals[0]), "J": float(r.fun), "iterations": int(r.nit),
                "evaluations": len(evals), "per_iteration": its, "message": str(r.message)}


def observe(disks):
    """Traces of every disk at every azimuth for its true c-axes
    (the synthetic observed data)."""
    from .adjoint import angles_from_axes
    import torch
    d_obs = []
    for d in disks:
        th, ph = angles_from_axes(d.true_axes)
        th_t = torch.as_tensor(th, dtype=torch.float64)
        ph_t = torch.as_tensor(ph, dtype=torch.float64)
        per = []
        for az, prob in zip(d.azimuths, d.problems):
            per.append(prob.traces_numpy(tables21(th_t, ph_t, az).numpy()))
        d_obs.append(per)
    return d_obs
