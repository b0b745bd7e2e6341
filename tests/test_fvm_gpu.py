"""FvmSolver3D::buildSystem / ::project on the GPU against the oracle."""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _random_faces(rng, dims):
    nx, ny, nz = dims
    return (rng.uniform(-1, 1, (nx + 1, ny, nz)), rng.uniform(-1, 1, (nx, ny + 1, nz)),
            rng.uniform(-1, 1, (nx, ny, nz + 1)))


@pytest.mark.parametrize("dims,collider", [((16, 16, 16), False), ((24, 24, 24), True), ((20, 17, 13), False)])
def test_build_system_and_project_match_oracle(oracle, gpu, dims, collider):
    import torch
    from simcraft_b200 import _capi, scenes
    from simcraft_b200.solver import default_context
    nx, ny, nz = dims
    m = max(dims)
    h = 1.0 / m
    dt = 0.01
    rng = np.random.default_rng(11)
    sdf = np.ascontiguousarray(scenes.sphere_union_sdf(m, *scenes._spheres(3, 8, 0.1, 0.3))[:nx, :ny, :nz])
    col = None
    if collider:
        # a solid ball in one corner: exercises fractionInside and the SDF evaluation
        g = (np.arange(m) + 0.5) * h
        X, Y, Z = np.meshgrid(g[:nx], g[:ny], g[:nz], indexing="ij")
        col = np.ascontiguousarray(np.sqrt((X - 0.7) ** 2 + (Y - 0.3) ** 2 + (Z - 0.6) ** 2) - 0.22)
    u, v, w = _random_faces(rng, dims)
    ref = oracle.build_system(dims, h, dt, u, v, w, sdf, col)
    ctx = default_context()
    L = _capi.lib()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ud, vd, wd, sd = d(u), d(v), d(w), d(sdf)
    cd = d(col) if col is not None else None
    adiag = torch.zeros(dims, dtype=torch.float64, device="cuda")
    an = [torch.zeros_like(adiag) for _ in range(6)]
    rhs = torch.zeros_like(adiag)
    act = torch.zeros(dims, dtype=torch.uint8, device="cuda")
    uw, vw, ww = torch.zeros_like(ud), torch.zeros_like(vd), torch.zeros_like(wd)
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    torch.cuda.synchronize()
    rc = L.sc_fvm_build_system_device(ctx.handle, nx, ny, nz, h, dt, _capi.SC_REAL_F64, p(ud), p(vd), p(wd),
                                      p(sd), p(cd), p(adiag), _capi.ptr_array([p(a) for a in an]), p(rhs),
                                      p(act), p(uw), p(vw), p(ww))
    _capi.check("build", rc, ctx.handle)
    ctx.synchronize()
    assert np.array_equal(act.cpu().numpy(), ref["active"])
    for got, want in [(uw, ref["uwt"]), (vw, ref["vwt"]), (ww, ref["wwt"]), (adiag, ref["adiag"]), (rhs, ref["rhs"])]:
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-12, atol=1e-12)
    for k in range(6):
        np.testing.assert_allclose(an[k].cpu().numpy(), ref["an"][k], rtol=1e-12, atol=1e-12)
    # project with a random pressure
    pg = rng.uniform(-1, 1, dims) * ref["active"]
    ru, rv, rw = oracle.project(dims, h, dt, u, v, w, pg, sdf, ref["uwt"], ref["vwt"], ref["wwt"])
    rc = L.sc_fvm_project_device(ctx.handle, nx, ny, nz, h, dt, _capi.SC_REAL_F64, p(ud), p(vd), p(wd), p(d(pg)),
                                 p(sd), p(uw), p(vw), p(ww))
    _capi.check("project", rc, ctx.handle)
    ctx.synchronize()
    for got, want in [(ud, ru), (vd, rv), (wd, rw)]:
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-12, atol=1e-12)
