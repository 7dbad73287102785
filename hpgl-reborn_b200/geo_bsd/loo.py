"""Leave-one-out cross-validation of ordinary kriging, differentiable.

No counterpart in HPGL (the reference has neither cross-validation nor
gradients). Each conditioning point is kriged from its neighbours among the
other conditioning points, with HPGL's ordinary-kriging system and search rules;
the mean squared error of those estimates is a smooth function of the variogram
(ranges, angles, sill, nugget) and of the data values. The estimates come from
the engine's FP64 LOO kernel and the gradient from its hand-written adjoint
kernel, behind a ``torch.autograd.Function``; PyTorch appears only in this layer.

Neighbour sets are chosen once per geometry (``LooGeometry``) by the engine's
exact search: the k + 1 neighbours of the point's own cell with every point
present, the point itself (covariance C(0), the unique maximum) removed. They
stay fixed while the variogram varies, so the loss is differentiated on the
piece where the selection does not change; rebuild the geometry to re-select.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import hpgl_wrap as W



def transform_matrix(ranges, angles):
    """M = diag(1/r0, 1/r1, 1/r2) X(a2) Y(a1) Z(a0): the anisotropy transform of
    cov_model.h:16-61 (angles in degrees, a0 the azimuth about z) divided by
    ranges[0], as a differentiable torch 3x3 (FP64)."""
    r = torch.as_tensor(ranges, dtype=torch.float64)
    a = torch.as_tensor(angles, dtype=torch.float64) * (math.pi / 180.0)
    one, zero = torch.ones((), dtype=torch.float64), torch.zeros((), dtype=torch.float64)
    c0, s0 = torch.cos(a[0]), torch.sin(a[0])
    c1, s1 = torch.cos(a[1]), torch.sin(a[1])
    c2, s2 = torch.cos(a[2]), torch.sin(a[2])
    Z = torch.stack([torch.stack([c0, s0, zero]), torch.stack([-s0, c0, zero]), torch.stack([zero, zero, one])])
    Y = torch.stack([torch.stack([c1, zero, -s1]), torch.stack([zero, one, zero]), torch.stack([s1, zero, c1])])
    X = torch.stack([torch.stack([one, zero, zero]), torch.stack([zero, c2, s2]), torch.stack([zero, -s2, c2])])
    return torch.diag(1.0 / r) @ (X @ Y @ Z)


@dataclass
class LooGeometry:
    """Conditioning points and their fixed leave-one-out neighbour sets, on the GPU."""
    pts_xyz: "object"   # torch int32 [n, 3]
    values: "object"    # torch float64 [n]
    targets: "object"   # torch int32 [t]: point ids
    nb_idx: "object"    # torch int32 [t, k]: neighbour point ids
    nb_cnt: "object"    # torch int32 [t]
    k: int
    cov_type: int
    nodes: np.ndarray   # grid node of every point


def loo_geometry(prop, grid, radiuses: Sequence[int], max_neighbours: int, cov_model,
                 device: Optional[str] = None) -> LooGeometry:
    """Select the leave-one-out neighbours of every informed cell of `prop`.

    The search is the engine's exact ordinary-kriging search
    (hpgl_b200_find_neighbours, analytic covariance) for max_neighbours + 1
    neighbours at each informed cell; the cell's own point is dropped."""
    if max_neighbours < 1 or max_neighbours > 32:
        raise ValueError("leave-one-out kriging supports 1 to 32 neighbours")
    dims = (grid.x, grid.y, grid.z)
    data = np.asarray(prop.data, dtype=np.float32).reshape(-1, order="F")
    mask = np.ascontiguousarray(np.asarray(prop.mask, dtype=np.uint8).reshape(-1, order="F"))
    nodes = np.flatnonzero(mask).astype(np.int32)
    n = len(nodes)
    k1 = max_neighbours + 1
    idx = np.full((n, k1), -1, np.int32)
    cnt = np.zeros(n, np.int32)
    path = np.zeros(n, np.uint8)
    p = W._HPGL_SK_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                          angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                          radiuses=tuple(int(round(r)) for r in radiuses), max_neighbours=k1,
                          automatic_mean=1, mean=0.0)
    if n:
        rc = W._hpgl_so.hpgl_b200_find_neighbours(0, (C.c_int * 3)(*dims), mask.ctypes.data, C.byref(p),
                                                   nodes.ctypes.data, n, idx.ctypes.data, cnt.ctypes.data,
                                                   path.ctypes.data)
        W.check(rc, "find_neighbours")
    # node -> point id; drop each point's own cell from its list
    pid = np.searchsorted(nodes, np.where(idx >= 0, idx, 0)).astype(np.int32)
    nb = np.full((n, max_neighbours), -1, np.int32)
    nc = np.zeros(n, np.int32)
    for i in range(n):
        row = [int(pid[i, j]) for j in range(cnt[i]) if idx[i, j] != nodes[i]]
        row = row[:max_neighbours]
        nb[i, :len(row)] = row
        nc[i] = len(row)
    nx, ny = dims[0], dims[1]
    xyz = np.stack([nodes % nx, (nodes // nx) % ny, nodes // (nx * ny)], axis=1).astype(np.int32)
    dev = torch.device(device or "cuda")
    return LooGeometry(pts_xyz=torch.from_numpy(xyz).to(dev), values=torch.from_numpy(data[nodes].astype(np.float64)).to(dev),
                       targets=torch.arange(n, dtype=torch.int32, device=dev), nb_idx=torch.from_numpy(nb).to(dev),
                       nb_cnt=torch.from_numpy(nc).to(dev), k=max_neighbours, cov_type=int(cov_model.type),
                       nodes=nodes)


def _loo_args(geom: LooGeometry, M, r0: float, sill: float, nugget: float, values):
    m9 = (C.c_double * 9)(*[float(v) for v in M.detach().reshape(-1).cpu().tolist()])
    return (geom.pts_xyz.data_ptr(), values.data_ptr(), int(values.numel()), geom.targets.data_ptr(),
            geom.nb_idx.data_ptr(), geom.nb_cnt.data_ptr(), int(geom.targets.numel()), geom.k, geom.cov_type,
            m9, float(r0), float(sill), float(nugget))


class LooKriging(torch.autograd.Function):
    """zhat = LOO ordinary-kriging estimates of every target; differentiable in
    M (3x3), sill, nugget and the data values. The backward pass runs the
    adjoint kernel, which recomputes the factors."""

    @staticmethod
    def forward(ctx, M, sill, nugget, values, geom: LooGeometry, r0: float):
        values = values.detach().contiguous()
        zhat = torch.empty(geom.targets.numel(), dtype=torch.float64, device=values.device)
        status = torch.empty(geom.targets.numel(), dtype=torch.int8, device=values.device)
        stream = torch.cuda.current_stream(values.device).cuda_stream
        rc = W._hpgl_so.hpgl_b200_loo_ok(*_loo_args(geom, M, r0, float(sill), float(nugget), values),
                                         zhat.data_ptr(), status.data_ptr(), stream)
        W.check(rc, "hpgl_b200_loo_ok")
        ctx.save_for_backward(M.detach(), torch.as_tensor(sill).detach(), torch.as_tensor(nugget).detach(), values)
        ctx.geom, ctx.r0 = geom, r0
        ctx.mark_non_differentiable(status)
        return zhat, status

    @staticmethod
    def backward(ctx, g_zhat, g_status):
        M, sill, nugget, values = ctx.saved_tensors
        geom = ctx.geom
        g = g_zhat.detach().to(torch.float64).contiguous()
        grad_values = torch.zeros_like(values)
        grad_params = torch.zeros(11, dtype=torch.float64, device=values.device)
        stream = torch.cuda.current_stream(values.device).cuda_stream
        rc = W._hpgl_so.hpgl_b200_loo_ok_adjoint(*_loo_args(geom, M, ctx.r0, float(sill), float(nugget), values),
                                                 g.data_ptr(), grad_values.data_ptr(), grad_params.data_ptr(), stream)
        W.check(rc, "hpgl_b200_loo_ok_adjoint")
        gM = grad_params[:9].reshape(3, 3).to(M.device)
        return gM, grad_params[9], grad_params[10], grad_values, None, None


def loo_estimates(geom: LooGeometry, ranges, angles, sill, nugget, values=None):
    """LOO estimates (torch FP64) and per-target status; differentiable in every argument
    given as a tensor with requires_grad."""
    dev = geom.values.device
    ranges = torch.as_tensor(ranges, dtype=torch.float64)
    M = transform_matrix(ranges, angles).to(dev)
    sill = torch.as_tensor(sill, dtype=torch.float64, device=dev)
    nugget = torch.as_tensor(nugget, dtype=torch.float64, device=dev)
    vals = geom.values if values is None else values
    return LooKriging.apply(M, sill, nugget, vals, geom, float(ranges[0].detach()))


def loo_cv_mse(geom: LooGeometry, ranges, angles, sill, nugget, values=None):
    """Mean squared leave-one-out error over the targets that kriged."""
    vals = geom.values if values is None else values
    zhat, status = loo_estimates(geom, ranges, angles, sill, nugget, vals)
    ok = status == 0
    truth = vals[geom.targets.long()]
    err = torch.where(ok, zhat - truth, torch.zeros_like(zhat))
    return (err * err).sum() / ok.sum().clamp(min=1)


def fit_variogram_loo(prop, grid, radiuses, max_neighbours, cov_model, iters: int = 30, lr: float = 0.05,
                      fit_angles: bool = False):
    """Fit (ranges, sill, nugget[, azimuth]) of `cov_model` by minimising the LOO-CV
    MSE with Adam on log ranges, log sill and the nugget fraction. Neighbour sets
    are those of the starting model. Returns (fitted CovarianceModel, loss history)."""
    from .geo import CovarianceModel
    geom = loo_geometry(prop, grid, radiuses, max_neighbours, cov_model)
    log_r = torch.tensor(np.log(cov_model.ranges), dtype=torch.float64, requires_grad=True)
    log_s = torch.tensor(math.log(cov_model.sill), dtype=torch.float64, requires_grad=True)
    frac = cov_model.nugget / cov_model.sill
    logit_n = torch.tensor(math.log(max(frac, 1e-6) / max(1 - frac, 1e-6)), dtype=torch.float64, requires_grad=True)
    az = torch.tensor(float(cov_model.angles[0]), dtype=torch.float64, requires_grad=fit_angles)
    params = [log_r, log_s, logit_n] + ([az] if fit_angles else [])
    opt = torch.optim.Adam(params, lr=lr)
    history = []
    for _ in range(iters):
        opt.zero_grad()
        sill = torch.exp(log_s)
        nugget = sill * torch.sigmoid(logit_n)
        angles = torch.stack([az, torch.tensor(float(cov_model.angles[1]), dtype=torch.float64),
                              torch.tensor(float(cov_model.angles[2]), dtype=torch.float64)])
        loss = loo_cv_mse(geom, torch.exp(log_r), angles, sill, nugget)
        loss.backward()
        opt.step()
        history.append(float(loss))
    with torch.no_grad():
        sill = float(torch.exp(log_s))
        fitted = CovarianceModel(type=cov_model.type, ranges=tuple(float(v) for v in torch.exp(log_r)),
                                 angles=(float(az), float(cov_model.angles[1]), float(cov_model.angles[2])),
                                 sill=sill, nugget=sill * float(torch.sigmoid(logit_n)))
    return fitted, history
