"""Dense FP64 torch reference of leave-one-out ordinary kriging (test oracle only).

Builds every target's bordered OK system [A 1; 1^T 0] [lambda; mu] = [b; 1]
(my_kriging_weights.h:198-361) with the covariance of cov_model.h:146-183 written
in torch, solves it with torch.linalg.solve and lets torch autograd
differentiate the estimates: an independent check of the engine's LOO kernel
and of its hand-written adjoint.
"""
import torch

from geo_bsd.loo import transform_matrix


def covariance(cov_type, M, r0, sill, nugget, v):
    """C(v) for integer offsets v [..., 3] (double)."""
    w = v @ M.T
    u2 = (w * w).sum(-1)
    u = torch.sqrt(torch.clamp(u2, min=1e-30))
    at_zero = r0 * u < 1e-4
    if cov_type == 1:
        f = torch.exp(-3.0 * u)
    elif cov_type == 2:
        f = torch.exp(-3.0 * u * u)
    else:
        f = torch.where(u > 1.0, torch.zeros_like(u), 1.0 - 1.5 * u + 0.5 * u ** 3)
    return torch.where(at_zero, sill * torch.ones_like(u), (sill - nugget) * f)


def dense_loo(pts_xyz, values, targets, nb_idx, nb_cnt, cov_type, ranges, angles, sill, nugget):
    """Estimates [t] for CPU tensors; differentiable in ranges, angles, sill, nugget, values."""
    ranges = torch.as_tensor(ranges, dtype=torch.float64)
    M = transform_matrix(ranges, angles)
    r0 = float(ranges[0].detach())
    t, k = nb_idx.shape
    live = torch.arange(k)[None, :] < nb_cnt[:, None].long()
    idx = nb_idx.long().clamp(min=0)
    P = pts_xyz.double()[idx]                      # [t, k, 3]
    T = pts_xyz.double()[targets.long()]          # [t, 3]
    A = covariance(cov_type, M, r0, sill, nugget, P[:, :, None, :] - P[:, None, :, :])
    b = covariance(cov_type, M, r0, sill, nugget, P - T[:, None, :])
    pair = live[:, :, None] & live[:, None, :]
    eye = torch.eye(k, dtype=torch.float64).expand(t, k, k)
    A = torch.where(pair, A, eye)
    b = torch.where(live, b, torch.zeros_like(b))
    one = live.double()
    K = torch.zeros(t, k + 1, k + 1, dtype=torch.float64)
    K = torch.cat([torch.cat([A, one[:, :, None]], 2),
                   torch.cat([one[:, None, :], torch.zeros(t, 1, 1, dtype=torch.float64)], 2)], 1)
    rhs = torch.cat([b, torch.ones(t, 1, dtype=torch.float64)], 1)
    sol = torch.linalg.solve(K, rhs[:, :, None])[:, :k, 0]
    z = torch.where(live, values[idx], torch.zeros_like(b))
    return (sol * z).sum(1)
