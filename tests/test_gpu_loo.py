"""Leave-one-out kriging and its adjoint (the differentiated-OK configuration).

The engine's FP64 LOO kernel is checked against a dense FP64 torch solve of the
same bordered OK systems; its hand-written adjoint against torch autograd of
that dense reference and against FP64 central finite differences (step 1e-6)
of the engine's own forward pass. Neighbour sets come from the engine's exact
search and are shared by every side of each comparison.
"""
import numpy as np
import pytest
import torch

import geo_bsd
import loo_reference as R
from geo_bsd import loo as L
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu


def _setup(scale, cov_type=None, angles=None):
    wl = WL.gauss_cv(scale)
    grid = geo_bsd.SugarboxGrid(*wl.dims)
    prop = geo_bsd.ContProperty(wl.data.reshape(wl.dims, order="F"), wl.mask.reshape(wl.dims, order="F"))
    cm = geo_bsd.CovarianceModel(type=wl.cov.cov_type if cov_type is None else cov_type, ranges=wl.cov.ranges,
                                 angles=wl.cov.angles if angles is None else angles, sill=wl.cov.sill,
                                 nugget=wl.cov.nugget)
    geom = L.loo_geometry(prop, grid, wl.radiuses, wl.max_neighbours, cm)
    return wl, cm, geom


def _cpu(geom):
    return (geom.pts_xyz.cpu(), geom.values.cpu(), geom.targets.cpu(), geom.nb_idx.cpu(), geom.nb_cnt.cpu())


@pytest.mark.parametrize("cov_type,angles", [(2, (0.0, 0.0, 0.0)), (1, (30.0, 10.0, 5.0)), (0, (15.0, 0.0, 0.0))])
def test_loo_estimates_match_dense_fp64(cov_type, angles):
    wl, cm, geom = _setup(0.5, cov_type, angles)
    assert geom.targets.numel() > 100
    zhat, status = L.loo_estimates(geom, cm.ranges, cm.angles, cm.sill, cm.nugget)
    assert (status == 0).all()
    ref = R.dense_loo(*_cpu(geom), cov_type, cm.ranges, cm.angles, torch.tensor(cm.sill, dtype=torch.float64),
                      torch.tensor(cm.nugget, dtype=torch.float64))
    err = (zhat.cpu() - ref).abs().max() / ref.abs().max()
    assert float(err) <= 1e-10, float(err)


def _loss_and_grads_engine(geom, cm, angles):
    ranges = torch.tensor(cm.ranges, dtype=torch.float64, requires_grad=True)
    ang = torch.tensor(angles, dtype=torch.float64, requires_grad=True)
    sill = torch.tensor(cm.sill, dtype=torch.float64, requires_grad=True)
    nug = torch.tensor(cm.nugget, dtype=torch.float64, requires_grad=True)
    vals = geom.values.clone().requires_grad_(True)
    loss = L.loo_cv_mse(geom, ranges, ang, sill, nug, vals)
    loss.backward()
    return float(loss.detach()), ranges.grad, ang.grad, sill.grad, nug.grad, vals.grad.cpu()


@pytest.mark.parametrize("cov_type,angles", [(2, (0.0, 0.0, 0.0)), (1, (30.0, 10.0, 5.0)), (0, (15.0, 0.0, 0.0))])
def test_adjoint_matches_dense_torch_autograd(cov_type, angles):
    wl, cm, geom = _setup(0.5, cov_type, angles)
    loss, gr, ga, gs, gn, gv = _loss_and_grads_engine(geom, cm, angles)
    pts, vals, tg, nb, nc = _cpu(geom)
    ranges = torch.tensor(cm.ranges, dtype=torch.float64, requires_grad=True)
    ang = torch.tensor(angles, dtype=torch.float64, requires_grad=True)
    sill = torch.tensor(cm.sill, dtype=torch.float64, requires_grad=True)
    nug = torch.tensor(cm.nugget, dtype=torch.float64, requires_grad=True)
    v = vals.clone().requires_grad_(True)
    zh = R.dense_loo(pts, v, tg, nb, nc, cov_type, ranges, ang, sill, nug)
    ref_loss = ((zh - v[tg.long()]) ** 2).mean()
    ref_loss.backward()
    assert abs(loss - float(ref_loss)) <= 1e-12 * abs(float(ref_loss))

    def close(a, b, what):
        a, b = a.detach().cpu().double(), b.detach().cpu().double()
        err = float((a - b).abs().max() / b.abs().max().clamp(min=1e-300))
        assert err <= 1e-8, (what, err, a, b)

    close(gr, ranges.grad, "ranges")
    close(ga, ang.grad, "angles")
    close(gs, sill.grad, "sill")
    close(gn, nug.grad, "nugget")
    close(gv, v.grad, "values")


def test_adjoint_matches_central_finite_differences():
    """Config 4 (Gaussian (18, 18, 6), sill 1, nugget 0.05, k = 24) at full size, the model
    rotated by angles (30, 10, 5) so that no derivative vanishes by symmetry: the
    LOO-CV MSE gradient w.r.t. the three ranges, the three angles, sill, nugget and 32
    sampled data values against FP64 central differences of the engine's forward pass
    (step 1e-6), each within 1e-6 of the difference quotient plus 1e-9 for its rounding
    (about eps * loss / step)."""
    angles = (30.0, 10.0, 5.0)
    wl, cm, geom = _setup(1.0, angles=angles)
    loss, gr, ga, gs, gn, gv = _loss_and_grads_engine(geom, cm, angles)
    h = 1e-6

    def f(ranges=cm.ranges, ang=angles, sill=cm.sill, nug=cm.nugget, vals=None):
        with torch.no_grad():
            return float(L.loo_cv_mse(geom, torch.tensor(ranges, dtype=torch.float64),
                                      torch.tensor(ang, dtype=torch.float64), sill, nug, vals))

    def fd(**kw_pm):
        (plus, minus), = kw_pm.values()
        key = list(kw_pm)[0]
        return (f(**{key: plus}) - f(**{key: minus})) / (2 * h)

    checks = []
    for a in range(3):
        rp, rm = list(cm.ranges), list(cm.ranges)
        rp[a] += h
        rm[a] -= h
        checks.append((f"range{a}", float(gr[a]), fd(ranges=(tuple(rp), tuple(rm)))))
    for a in range(3):
        ap, am = list(angles), list(angles)
        ap[a] += h
        am[a] -= h
        checks.append((f"angle{a}", float(ga[a]), fd(ang=(tuple(ap), tuple(am)))))
    checks.append(("sill", float(gs), fd(sill=(cm.sill + h, cm.sill - h))))
    checks.append(("nugget", float(gn), fd(nug=(cm.nugget + h, cm.nugget - h))))
    rng = np.random.default_rng(7)
    for i in rng.choice(geom.values.numel(), 32, replace=False):
        vp, vm = geom.values.clone(), geom.values.clone()
        vp[i] += h
        vm[i] -= h
        checks.append((f"value{i}", float(gv[i]), fd(vals=(vp, vm))))
    assert all(abs(c[2]) > 0 for c in checks[:8]), checks[:8]
    for name, adj, num in checks:
        assert abs(adj - num) <= 1e-6 * abs(num) + 1e-9, (name, adj, num)


def test_loo_fitting_lowers_the_cv_error():
    wl = WL.gauss_cv(0.5)
    grid = geo_bsd.SugarboxGrid(*wl.dims)
    prop = geo_bsd.ContProperty(wl.data.reshape(wl.dims, order="F"), wl.mask.reshape(wl.dims, order="F"))
    start = geo_bsd.CovarianceModel(type=2, ranges=(10.0, 10.0, 3.0), angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.3)
    fitted, hist = L.fit_variogram_loo(prop, grid, wl.radiuses, wl.max_neighbours, start, iters=25, lr=0.05)
    assert hist[-1] < hist[0]
    assert all(np.isfinite(hist))
    assert fitted.ranges[0] > start.ranges[0]  # the field's true range is 18


def test_loo_argument_errors():
    import ctypes as C
    from geo_bsd import hpgl_wrap as W
    m9 = (C.c_double * 9)(*([1.0] * 9))
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    i = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = W._hpgl_so.hpgl_b200_loo_ok(i.data_ptr(), d.data_ptr(), 1, i.data_ptr(), i.data_ptr(), i.data_ptr(), 1, 33,
                                     2, m9, 1.0, 1.0, 0.0, d.data_ptr(), None, None)
    assert rc == W.ELIMIT and "32" in W.last_error()
    rc = W._hpgl_so.hpgl_b200_loo_ok(i.data_ptr(), d.data_ptr(), 1, i.data_ptr(), i.data_ptr(), i.data_ptr(), 1, 4,
                                     7, m9, 1.0, 1.0, 0.0, d.data_ptr(), None, None)
    assert rc == W.EINVAL
