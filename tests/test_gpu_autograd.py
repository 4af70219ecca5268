"""Differentiable cone-beam projector (torch.autograd.Function).

A scaled-down copy of the 256^3 / 360-angle / 384^2-detector autograd
workload (the same proportions at 1/16 size: 2 mm voxels, 1.6 mm pixels,
source and detector 31.25 mm from the axis), batch of 8 volumes.  Checks:
  * the dot-product test <Ax, y> = <x, A^T y> with FP64 accumulation,
    relative error <= 1e-5;
  * central finite differences of L(x) = 0.5 ||Ax - y||^2 on 32 random
    voxels against autograd's gradient (L is quadratic, so the central
    difference is exact up to FP32 rounding of the projections);
  * the backward pass against the reference's own back projector
    (cone_beam::b2D, Core/src/c2D.cpp:1052-1119): bit for bit;
  * a few Adam steps on the loss decrease it.
"""
import numpy as np
import pytest

import oracle as O
from conftest import max_rel

pytestmark = pytest.mark.gpu

S2O = O2D = 500.0 / 16


def geometry():
    return O.cone_geometry(16, 2.0, 36, 24, 1.6, S2O, O2D)


def plan_of(g):
    from ccpi.reconstruction.device import Plan
    return Plan("cone", g.angles, g.h_pixels, g.v_pixels, g.origin, g.size, g.shape,
                source=g.source, detector_x=g.detector_x)


def test_dot_product_batch(cuda):
    import torch
    from ccpi.reconstruction.autograd import project, backproject
    g = geometry()
    p = plan_of(g)
    gen = torch.Generator(device="cpu").manual_seed(5)
    x = torch.rand((8,) + g.shape, generator=gen).to(cuda)
    y = torch.rand((8,) + g.sino_shape, generator=gen).to(cuda)
    ax = project(x, p)
    aty = backproject(y, p)
    assert ax.shape == (8,) + g.sino_shape and aty.shape == (8,) + g.shape
    for i in range(8):
        lhs = float((ax[i].double() * y[i].double()).sum())
        rhs = float((x[i].double() * aty[i].double()).sum())
        assert abs(lhs - rhs) / abs(lhs) <= 1e-5, (i, lhs, rhs)


def test_gradient_finite_differences(cuda):
    import torch
    from ccpi.reconstruction.autograd import project
    g = geometry()
    p = plan_of(g)
    rng = np.random.default_rng(11)
    x_true = torch.from_numpy(rng.uniform(0, 1, g.shape).astype(np.float32)).to(cuda)
    y = project(x_true, p).detach()
    y += 0.05 * torch.from_numpy(rng.standard_normal(g.sino_shape).astype(np.float32)).to(cuda)
    x0 = torch.from_numpy(rng.uniform(0, 1, g.shape).astype(np.float32)).to(cuda)

    def loss64(x):
        r = project(x, p).double() - y.double()
        return 0.5 * float((r * r).sum())

    x = x0.clone().requires_grad_(True)
    r = project(x, p) - y
    (0.5 * (r * r).sum()).backward()
    grad = x.grad.detach().cpu().numpy()
    flat = rng.choice(np.prod(g.shape), 32, replace=False)
    h = 0.5
    worst = 0.0
    scale = np.abs(grad).max()
    for f in flat:
        idx = np.unravel_index(f, g.shape)
        xp = x0.clone()
        xm = x0.clone()
        xp[idx] += h
        xm[idx] -= h
        fd = (loss64(xp) - loss64(xm)) / (2 * h)
        worst = max(worst, abs(fd - grad[idx]) / scale)
    assert worst <= 1e-3, worst


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built")
def test_backward_matches_reference_backprojector(cuda):
    import torch
    from ccpi.reconstruction.autograd import project
    g = geometry()
    p = plan_of(g)
    rng = np.random.default_rng(3)
    w = rng.uniform(-1, 1, g.sino_shape).astype(np.float32)
    x = torch.zeros(g.shape, device=cuda, requires_grad=True)
    out = project(x, p)
    out.backward(torch.from_numpy(w).to(cuda))
    ref = O.ref_backward(g, w)
    assert np.array_equal(x.grad.cpu().numpy(), ref), max_rel(x.grad.cpu().numpy(), ref)


def test_adam_steps_reduce_loss(cuda):
    import torch
    from ccpi.reconstruction.autograd import Projector
    g = geometry()
    A = Projector(plan_of(g))
    gen = torch.Generator(device="cpu").manual_seed(2)
    xt = torch.rand((8,) + g.shape, generator=gen).to(cuda)
    y = A(xt).detach()
    x = torch.zeros_like(xt, requires_grad=True)
    opt = torch.optim.Adam([x], lr=0.05)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        r = A(x) - y
        loss = (r * r).sum()
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    assert min(losses[-5:]) < 0.3 * losses[0], losses


@pytest.mark.parametrize("kind", ["cone", "cone-tall", "parallel"])
def test_batch_projection_equals_per_item(kind, cuda):
    """ccpi_forward_batch / ccpi_backward_batch (one launch per direction
    for cone beam, sharing the walks and ray lists) give every item's
    single projection bit for bit; the tall cone case (columns over 1024
    voxels) takes the per-item atomic back projector, so only its forward
    batch is compared bit for bit."""
    import torch
    from ccpi.reconstruction.device import parallel_plan
    if kind == "cone":
        p = plan_of(geometry())
    elif kind == "cone-tall":
        p = plan_of(O.cone_geometry((8, 8, 1100), 1.0, 12, 16, 1.0, 600.0, 600.0, n_det_v=40))
    else:
        p = parallel_plan((24, 24, 8), 30, 36)
    g = torch.Generator(device=cuda).manual_seed(3)
    n = 5
    x = torch.rand((n,) + p.shape, device=cuda, generator=g)
    y = torch.rand((n,) + p.sino_shape, device=cuda, generator=g)
    fx = torch.empty((n,) + p.sino_shape, device=cuda)
    by = torch.empty((n,) + p.shape, device=cuda)
    p.forward_batch(x, fx)
    p.backward_batch(y, by)
    for b in range(n):
        assert torch.equal(fx[b], p.forward(x[b])), b
        if kind != "cone-tall":
            assert torch.equal(by[b], p.backward(y[b])), b
        else:
            assert max_rel(by[b].cpu().numpy(), p.backward(y[b]).cpu().numpy()) <= 1e-5
    if kind.startswith("cone"):
        # a plan set to the scatter back-projects a batch item by item with
        # it: equal to the gather's batch within the projector tolerance
        p.set_cone_backprojector(1)
        bs = torch.empty_like(by)
        p.backward_batch(y, bs)
        for b in range(n):
            assert max_rel(bs[b].cpu().numpy(), by[b].cpu().numpy()) <= 1e-5, b
