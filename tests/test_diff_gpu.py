"""Differentiable FLIP/PIC substeps: the adjoint gradient against central finite
differences of the structure-frozen forward (FP64), checkpoint invariance, the
FP32 gradient against the FP64 one, and the torch.autograd.Function binding.

The finite differences replay the base run's discrete structure (transfer
stencils, wall clamps, fluid SDF), the piece of the piecewise-smooth map whose
derivative the adjoint computes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod(gpu):
    import torch
    return torch


def _problem(n, steps, precision="f64", checkpoint_every=2, dt=1.0 / 120, ppc=8, **kw):
    from simcraft_b200.diff import DiffFlip, control_scene
    pos, param, target, h = control_scene(n, ppc=ppc)
    sim = DiffFlip((n, n, n), h, dt, steps, precision=precision, checkpoint_every=checkpoint_every,
                   flip_alpha=0.95, **kw)
    sim.set_particles(pos)
    sim.set_target(target)
    return sim, param


def _faces(torch, param):
    from simcraft_b200.diff import faces_from_cells
    return faces_from_cells(torch.from_numpy(param).cuda())


def _directional_check(torch, sim, param, ndir, eps, seed=8):
    from simcraft_b200.diff import faces_from_cells
    U = _faces(torch, param)
    loss = sim.forward(U, tape="record")
    grads = sim.backward()
    rng = np.random.default_rng(seed)
    errs = []
    for _ in range(ndir):
        d = rng.standard_normal(param.shape)
        D = faces_from_cells(torch.from_numpy(d).cuda())
        up = [u + eps * dd for u, dd in zip(U, D)]
        um = [u - eps * dd for u, dd in zip(U, D)]
        fd = (sim.forward(up, tape="replay") - sim.forward(um, tape="replay")) / (2 * eps)
        ad = sum(float((g * dd).sum()) for g, dd in zip(grads, D))
        errs.append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
    return loss, grads, errs


def test_gradient_matches_finite_differences_small(torch_mod):
    sim, param = _problem(16, steps=4)
    loss, grads, errs = _directional_check(torch_mod, sim, param, ndir=4, eps=1e-3)
    assert loss > 0 and max(float(g.abs().max()) for g in grads) > 0
    assert max(errs) < 1e-3, errs


def test_pic_gradient_matches_finite_differences(torch_mod):
    sim, param = _problem(12, steps=3, advection="pic", checkpoint_every=1)
    _, _, errs = _directional_check(torch_mod, sim, param, ndir=3, eps=1e-3)
    assert max(errs) < 1e-3, errs


def test_checkpointing_does_not_change_the_gradient(torch_mod):
    a, param = _problem(16, steps=6, checkpoint_every=1)
    b, _ = _problem(16, steps=6, checkpoint_every=6)
    c, _ = _problem(16, steps=6, checkpoint_every=4)
    U = _faces(torch_mod, param)
    la, lb, lc = a.forward(U), b.forward(U), c.forward(U)
    assert la == pytest.approx(lb, rel=1e-10) and la == pytest.approx(lc, rel=1e-10)
    ga, gb, gc = a.backward(), b.backward(), c.backward()
    for x, y, z in zip(ga, gb, gc):
        scale = float(x.abs().max())
        assert float((x - y).abs().max()) <= 1e-8 * scale
        assert float((x - z).abs().max()) <= 1e-8 * scale


def test_fp32_gradient_against_fp64(torch_mod):
    s64, param = _problem(16, steps=4)
    s32, _ = _problem(16, steps=4, precision="f32")
    U = _faces(torch_mod, param)
    l64, l32 = s64.forward(U), s32.forward(U)
    assert l32 == pytest.approx(l64, rel=1e-4)
    g64, g32 = s64.backward(), s32.backward()
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(g64, g32))
    den = sum(float((a ** 2).sum()) for a in g64)
    assert (num / den) ** 0.5 < 1e-3


def test_autograd_function(torch_mod):
    torch = torch_mod
    from simcraft_b200.diff import FlipLoss, cells_from_faces
    sim, param = _problem(12, steps=2)
    p = torch.from_numpy(param).cuda().requires_grad_(True)
    loss = FlipLoss.apply(p, sim)
    loss.backward()
    U = _faces(torch, param)
    sim.forward(U)
    g = cells_from_faces(sim.backward(), p.dtype)
    assert torch.allclose(p.grad, g, rtol=1e-4, atol=1e-12 * float(g.abs().max()))
    # one step of gradient descent lowers the loss
    with torch.no_grad():
        q = p - 1e-3 * p.grad / p.grad.norm() * p.norm()
    assert FlipLoss.apply(q, sim).item() < loss.item()


def test_control_problem_64(torch_mod):
    """The 64^3 differentiable control problem: fluid in the lower quarter
    (524,288 particles), 20 substeps of dt = 1/120, checkpoints every 5, FP64;
    central differences (eps = 1e-3) along 16 seeded directions, and the FP32
    gradient against the FP64 one."""
    sim, param = _problem(64, steps=20, checkpoint_every=5)
    assert sim.n == 64 * 16 * 64 * 8
    loss, g64, errs = _directional_check(torch_mod, sim, param, ndir=16, eps=1e-3)
    assert max(errs) < 1e-3, errs
    s32, _ = _problem(64, steps=20, precision="f32", checkpoint_every=5)
    s32.forward(_faces(torch_mod, param))
    g32 = s32.backward()
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(g64, g32))
    den = sum(float((a ** 2).sum()) for a in g64)
    assert (num / den) ** 0.5 < 1e-2


def _density_np(pos, dims, h):
    """rho_c = sum_p N(x_p - x_c) on the cell centres over the stencil
    nearest + {-1..2}, N the tensor-product cubic B-spline (the loss's density)."""
    def bs(r):
        r = np.abs(r)
        return np.where(r < 1.0, 2.0 / 3.0 - r * r + 0.5 * r ** 3, np.where(r < 2.0, (2.0 - r) ** 3 / 6.0, 0.0))
    rho = np.zeros(dims)
    base = np.floor(pos / h).astype(np.int64) - 1
    for a in range(4):
        for b in range(4):
            for c in range(4):
                idx = base + np.array([a, b, c])
                w = (bs(pos[:, 0] / h - (idx[:, 0] + 0.5)) * bs(pos[:, 1] / h - (idx[:, 1] + 0.5))
                     * bs(pos[:, 2] / h - (idx[:, 2] + 0.5)))
                ok = np.all((idx >= 0) & (idx < np.array(dims)), axis=1)
                np.add.at(rho, (idx[ok, 0], idx[ok, 1], idx[ok, 2]), w[ok])
    return rho


@pytest.mark.parametrize("n,advection", [(16, "flip"), (20, "pic")])
def test_forward_matches_oracle_simulator(oracle, torch_mod, n, advection):
    """The differentiable step's forward (FP64, no tape) is the simulator's
    substep with a fixed dt: against the oracle's simulator (fluid-simulator.cc:
    140-182) given the velocities the oracle samples from the same face field U
    (sampleVelocity, util.cc:40-85), with the same MIC(0) tau = 0 and relative
    1e-10 pressure solves: pressure within 1e-5 relative L2 and positions within
    1e-4 h after each of 4 substeps, and the density loss within 1e-10 relative."""
    torch = torch_mod
    from simcraft_b200.diff import DiffFlip, control_scene, faces_from_cells
    pos, param, target, h = control_scene(n)
    dims, dt = (n, n, n), 1.0 / 120
    U = faces_from_cells(torch.from_numpy(param).cuda())
    vel0 = oracle.sample_velocity(pos, dims, h, *[u.cpu().numpy() for u in U])
    flip = advection == "flip"
    cfg = oracle.default_config(n, n, n, h, flip=int(flip), flip_alpha=0.95, pcg_tol=1e-10, pcg_max_iter=2000,
                                pcg_criterion=1, mic_tau=0.0)
    ref = oracle.Sim(**cfg)
    ref.set_particles(pos, vel0)
    loss = None
    for k in range(1, 5):
        ref.substep(dt)
        sim = DiffFlip(dims, h, dt, k, flip_alpha=0.95, advection=advection, checkpoint_every=2)
        sim.set_particles(pos)
        sim.set_target(target)
        loss = sim.forward(U, tape="none")
        p_ref = ref.pressure()
        assert np.abs(p_ref).max() > 0
        perr = np.linalg.norm(sim.pressure() - p_ref) / np.linalg.norm(p_ref)
        x, v = sim.particles()
        x_ref, v_ref = ref.particles()
        xerr = np.abs(x - x_ref).max() / h
        assert perr <= 1e-5 and xerr <= 1e-4, (k, perr, xerr)
    rho_ref = _density_np(ref.particles()[0], dims, h)
    np.testing.assert_allclose(sim.density(), rho_ref, rtol=0, atol=1e-9)
    loss_ref = float(((rho_ref - target) ** 2).sum())
    assert abs(loss - loss_ref) <= 1e-10 * loss_ref, (loss, loss_ref)


def _oracle_loss(oracle, pos, U, target, dims, h, dt, steps, flip, sdfs=None):
    """The differentiable step's loss computed by the oracle's FP64 simulator
    (the reference's substep, fluid-simulator.cc:140-182) with MIC(0) tau = 0 and
    pressure solves to 1e-14 relative, from velocities sampleVelocity takes
    from U.  sdfs=None records the fluid SDF of every substep and returns
    (loss, sdfs); given sdfs, the substeps use them instead of reconstructing
    (the structure the adjoint holds fixed) and the loss is returned."""
    vel0 = oracle.sample_velocity(pos, dims, h, *U)
    cfg = oracle.default_config(*dims, h, flip=int(flip), flip_alpha=0.95, pcg_tol=1e-14, pcg_max_iter=4000,
                                pcg_criterion=1, mic_tau=0.0)
    sim = oracle.Sim(**cfg)
    sim.set_particles(pos, vel0)
    sim.sdf_tape(1, sdfs)
    for _ in range(steps):
        sim.substep(dt)
    rho = _density_np(sim.particles()[0], dims, h)
    loss = float(((rho - target) ** 2).sum())
    return (loss, sim.taped_sdfs()) if sdfs is None else loss


@pytest.mark.parametrize("n,steps,advection", [(8, 3, "flip"), (12, 2, "flip"), (10, 2, "pic")])
def test_adjoint_matches_oracle_central_differences(oracle, torch_mod, n, steps, advection):
    """An FP64 reference gradient independent of this repository's adjoint:
    central differences of the oracle's forward with the structure the adjoint
    holds fixed (the fluid SDF of each substep, taped from the oracle's own base
    run; at eps = 1e-5 no stencil base or wall clamp changes between the two
    evaluations) against the GPU adjoint: relative error below 1e-5."""
    torch = torch_mod
    from simcraft_b200.diff import DiffFlip, control_scene, faces_from_cells
    pos, param, target, h = control_scene(n)
    dims, dt, flip = (n, n, n), 1.0 / 120, advection == "flip"
    U = faces_from_cells(torch.from_numpy(param).cuda())
    sim = DiffFlip(dims, h, dt, steps, flip_alpha=0.95, advection=advection, checkpoint_every=1, pcg_tol=1e-13)
    sim.set_particles(pos)
    sim.set_target(target)
    loss = sim.forward(U, tape="none")
    grads = sim.backward()
    Uh = [u.cpu().numpy() for u in U]
    loss_ref, sdfs = _oracle_loss(oracle, pos, Uh, target, dims, h, dt, steps, flip)
    assert len(sdfs) == steps and abs(loss - loss_ref) <= 1e-10 * loss
    # replaying its own SDFs leaves the oracle's base loss unchanged
    assert _oracle_loss(oracle, pos, Uh, target, dims, h, dt, steps, flip, sdfs) == loss_ref
    rng = np.random.default_rng(8)
    eps = 1e-5
    errs = []
    for _ in range(6):
        d = faces_from_cells(torch.from_numpy(rng.standard_normal(param.shape)).cuda())
        dh = [x.cpu().numpy() for x in d]
        lp = _oracle_loss(oracle, pos, [u + eps * x for u, x in zip(Uh, dh)], target, dims, h, dt, steps, flip, sdfs)
        lm = _oracle_loss(oracle, pos, [u - eps * x for u, x in zip(Uh, dh)], target, dims, h, dt, steps, flip, sdfs)
        fd = (lp - lm) / (2 * eps)
        ad = sum(float((g * x).sum()) for g, x in zip(grads, d))
        errs.append(abs(fd - ad) / max(abs(fd), abs(ad)))
    assert max(errs) < 1e-5, errs
