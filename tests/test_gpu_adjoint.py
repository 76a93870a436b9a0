"""
Tangent and discrete adjoint of the RK2 circumbinary-disk step.

  * the generic per-zone formulation behind the tangent reproduces the fused
    stage kernel bit for bit;
  * stage tangent versus central finite differences of the stage kernel;
  * dot-product tests <lambda, T delta> = <A lambda, delta> for a stage
    (state and the 12 point-mass / nu / sink-rate parameters) and for the
    objective;
  * the whole reverse sweep with checkpointing versus the forward-mode
    tangent of the run, and versus central finite differences of J.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sailfish_b200 import _capi  # noqa: E402
from sailfish_b200.adjoint import AdjointRun, Params, mass_jacobian, objective_function  # noqa: E402

P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _state(run, params, steps=3):
    """A developed state (a few steps from the seeded disk) and its solver."""
    prim = run.initial_state(seed=3)
    s = run._solver(params, prim)
    for _ in range(steps):
        s.advance(s.mesh.min_spacing() / s.maximum_wavespeed() * 0.3)
    return s


def _rand_like(t, seed, scale=1.0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return (torch.rand(t.shape, generator=g, dtype=torch.float64) * 2 - 1).to(t.device) * scale


@pytest.fixture(scope="module")
def stage_case():
    run = AdjointRun(resolution=48, steps=1)
    params = Params(0.5, 0.1, 1e-3, 10.0)
    s = _state(run, params)
    dt = 0.8 * s.mesh.min_spacing() / s.maximum_wavespeed() * 0.3
    dev, nb, times = run._records(s, s.time, dt)
    return run, params, s, dev, nb, times


def _stage(s, dev, off, a, p, pn):
    out = torch.empty_like(p)
    st = _capi.Stage()
    st.a = a
    _capi.check(s._lib.cbdiso_b200_advance_stage(ctypes.byref(s._grid), ctypes.byref(st),
                                                 ctypes.c_void_p(dev.data_ptr() + off), P(p),
                                                 P(pn) if pn is not None else None, P(out), None, P(s._scratch),
                                                 P(s._result), _stream()), "stage")
    return out


def _tangent(s, dev, off, p, dp, pn, dpn, dmass, dnu=0.0, drate=0.0):
    out, dout = torch.empty_like(p), torch.empty_like(p)
    d = (ctypes.c_double * 10)(*dmass)
    _capi.check(s._lib.cbdiso_b200_stage_tangent(ctypes.byref(s._grid), ctypes.c_void_p(dev.data_ptr() + off), d,
                                                 dnu, drate, P(p), P(dp), P(pn) if pn is not None else None,
                                                 P(dpn) if dpn is not None else None, P(out), P(dout), _stream()),
                "tangent")
    return out, dout


def _guarded(s, t):
    _capi.check(s._lib.cbdiso_b200_fill_guards(ctypes.byref(s._grid), P(t), _stream()), "guards")
    return t


@pytest.mark.parametrize("stage", [0, 1])
def test_generic_zone_update_matches_the_stage_kernel(stage_case, stage):
    run, params, s, dev, nb, _ = stage_case
    p = s._buf[0]
    pn = p if stage == 1 else None
    want = _stage(s, dev, stage * nb, 0.5 * stage, p, pn)
    got, _ = _tangent(s, dev, stage * nb, p, torch.zeros_like(p), pn, torch.zeros_like(p) if pn is not None else None,
                      [0.0] * 10)
    assert torch.equal(got[2:-2, 2:-2], want[2:-2, 2:-2])


@pytest.mark.parametrize("stage", [0, 1])
def test_stage_tangent_matches_finite_differences(stage_case, stage):
    run, params, s, dev, nb, _ = stage_case
    p = s._buf[0]
    dp = _guarded(s, _rand_like(p, 1) * p.abs().amax(dim=(0, 1)))
    pn = p.clone() if stage == 1 else None
    dpn = _guarded(s, _rand_like(p, 2) * p.abs().amax(dim=(0, 1))) if stage == 1 else None
    _, dout = _tangent(s, dev, stage * nb, p, dp, pn, dpn, [0.0] * 10)
    # The stage is piecewise smooth (limiter and HLLE branches): h is small
    # enough that the +-h states take the same branches in all but a zone or
    # so of this seeded state (larger h straddles near-ties of the limiter).
    h = 1e-8
    plus = _stage(s, dev, stage * nb, 0.5 * stage, p + h * dp, pn + h * dpn if pn is not None else None)
    minus = _stage(s, dev, stage * nb, 0.5 * stage, p - h * dp, pn - h * dpn if pn is not None else None)
    fd = ((plus - minus) / (2 * h))[2:-2, 2:-2]
    tan = dout[2:-2, 2:-2]
    for q in range(3):
        err = (fd[..., q] - tan[..., q]).abs().max() / tan[..., q].abs().max()
        assert err < 1e-6, (q, float(err))


@pytest.mark.parametrize("stage", [0, 1])
def test_stage_adjoint_dot_product(stage_case, stage):
    run, params, s, dev, nb, _ = stage_case
    lib = s._lib
    g = ctypes.byref(s._grid)
    p = s._buf[0]
    pn = p.clone() if stage == 1 else None
    out = _stage(s, dev, stage * nb, 0.5 * stage, p, pn)
    words = torch.zeros(p.shape[:2], dtype=torch.int32, device=p.device)
    rec = ctypes.c_void_p(dev.data_ptr() + stage * nb)
    _capi.check(lib.cbdiso_b200_stage_record_branches(g, rec, P(p), P(out), P(words), _stream()), "record")
    scale = p.abs().amax(dim=(0, 1))
    dp = _guarded(s, _rand_like(p, 11) * scale)
    dpn = _guarded(s, _rand_like(p, 12) * scale) if stage == 1 else None
    rng = np.random.default_rng(13)
    dmass = rng.uniform(-1, 1, 10) * 1e-2
    dnu, drate = 1e-4, 0.5
    _, dout = _tangent(s, dev, stage * nb, p, dp, pn, dpn, dmass, dnu, drate)
    lam = torch.zeros_like(p)
    lam[2:-2, 2:-2] = _rand_like(lam[2:-2, 2:-2], 14)
    lam_rd, lam_n = torch.zeros_like(p), torch.zeros_like(p)
    pars = torch.zeros(12, dtype=torch.float64, device=p.device)
    ws = torch.zeros(int(lib.cbdiso_b200_adjoint_workspace_bytes(g)) // 8 + 8, dtype=torch.float64, device=p.device)
    _capi.check(lib.cbdiso_b200_stage_adjoint(g, rec, P(p), P(pn) if pn is not None else None, P(out), P(words),
                                              P(lam), P(lam_rd), P(lam_n) if pn is not None else None, P(pars),
                                              P(ws), _stream()), "adjoint")
    I = (slice(2, -2), slice(2, -2))
    lhs = float((lam[I] * dout[I]).sum())
    rhs = float((lam_rd[I] * dp[I]).sum())
    if stage == 1:
        rhs += float((lam_n[I] * dpn[I]).sum())
    pv = pars.cpu().numpy()
    rhs += float(pv[:10] @ dmass) + pv[10] * dnu + pv[11] * drate
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


def test_objective_adjoint_dot_product(stage_case):
    run, params, s, dev, nb, _ = stage_case
    lib = s._lib
    g = ctypes.byref(s._grid)
    p = s._buf[0]
    rec = ctypes.c_void_p(dev.data_ptr() + nb)
    dp = _guarded(s, _rand_like(p, 21) * p.abs().amax(dim=(0, 1)))
    dmass = np.random.default_rng(22).uniform(-1, 1, 10) * 1e-2
    drate = 0.3
    parts = torch.zeros(64, dtype=torch.float64, device=p.device)
    d = (ctypes.c_double * 10)(*dmass)
    _capi.check(lib.cbdiso_b200_objective_tangent(g, rec, d, drate, P(p), P(dp), 0.7, 1.3, P(parts), 64, _stream()),
                "objective tangent")
    lhs = float(parts.sum())
    lam = torch.zeros_like(p)
    pars = torch.zeros(12, dtype=torch.float64, device=p.device)
    ws = torch.zeros(int(lib.cbdiso_b200_adjoint_workspace_bytes(g)) // 8 + 8, dtype=torch.float64, device=p.device)
    _capi.check(lib.cbdiso_b200_objective_adjoint(g, rec, P(p), 0.7, 1.3, P(lam), P(pars), P(ws), _stream()),
                "objective adjoint")
    I = (slice(2, -2), slice(2, -2))
    pv = pars.cpu().numpy()
    rhs = float((lam[I] * dp[I]).sum()) + float(pv[:10] @ dmass) + pv[11] * drate
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1e-300), (lhs, rhs)


def test_kepler_jacobian_matches_finite_differences():
    from sailfish_b200.kepler import OrbitalElements

    def state(q, e, t):
        a, b = OrbitalElements(1.0, 1.0, q, e).orbital_state(t)
        return np.array([a.position_x, a.position_y, a.velocity_x, a.velocity_y, a.mass,
                         b.position_x, b.position_y, b.velocity_x, b.velocity_y, b.mass])

    for t in (0.0, 0.7, 5.3):
        j = mass_jacobian(t, 0.5, 0.1)
        h = 1e-6
        fq = (state(0.5 + h, 0.1, t) - state(0.5 - h, 0.1, t)) / (2 * h)
        fe = (state(0.5, 0.1 + h, t) - state(0.5, 0.1 - h, t)) / (2 * h)
        np.testing.assert_allclose(j[:, 0], fq, rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(j[:, 1], fe, rtol=1e-6, atol=1e-9)


@pytest.fixture(scope="module")
def run_case():
    run = AdjointRun(resolution=48, steps=24, checkpoint_every=5)
    params = Params(0.5, 0.1, 1e-3, 10.0)
    prim = run.initial_state(seed=4)
    run.forward(prim, params, freeze=True, keep=True)
    return run, params, prim


@pytest.mark.parametrize("weights", [(1.0, 0.0), (0.0, 1.0)])
def test_run_gradient_matches_tangent(run_case, weights):
    run, params, prim = run_case
    run.forward(prim, params, keep=True)
    gs, gp = run.gradient(weights)
    rng = np.random.default_rng(31)
    for k in range(2):
        dprim = np.zeros_like(prim)
        dprim[..., 0] = rng.uniform(-1, 1, prim.shape[:2]) * 1e-2
        dpar = rng.uniform(-1, 1, 4) * np.array([0.1, 0.05, 1e-4, 1.0])
        tan = run.tangent(prim, params, dprim, dpar, weights)
        adj = float((gs * dprim).sum()) + float(gp @ dpar)
        assert abs(tan - adj) <= 1e-9 * max(abs(tan), 1e-300), (k, tan, adj)


@pytest.mark.parametrize("graph", [False, True])
def test_checkpointed_sweep_matches_the_stored_trajectory(run_case, graph):
    """Recomputing segments from checkpoints (K = 5: four full segments and
    a partial one; full ones replayed from a CUDA graph) reproduces the
    gradient of the stored-trajectory sweep bit for bit."""
    run, params, prim = run_case
    run.forward(prim, params, keep=True)
    gs, gp = run.gradient((0.7, 0.3))
    ck = AdjointRun(resolution=run.n, steps=run.steps, checkpoint_every=5, store_states=False)
    ck.dts = run.dts
    ck.forward(prim, params, keep=True)
    assert ck._fwd["trajectory"] is None
    for _ in range(2):  # the second call replays the cached graph
        cs, cp = ck.gradient((0.7, 0.3), graph=graph)
        np.testing.assert_array_equal(cs, gs)
        np.testing.assert_array_equal(cp, gp)


def _bump(run, rng):
    """A smooth surface-density perturbation: a Gaussian of width ~1 at a
    seeded position (smooth directions keep +-h runs on the same branches)."""
    x = -8.0 + (np.arange(run.n) + 0.5) * 16.0 / run.n
    cx, cy = rng.uniform(-1.0, 1.0, 2)  # near the binary, where the accretion rate is sensitive
    return np.exp(-((x[:, None] - cx) ** 2 + (x[None, :] - cy) ** 2) / 2.0)


def test_run_gradient_matches_central_differences(run_case):
    run, params, prim = run_case
    run.forward(prim, params, keep=True)
    gs, gp = run.gradient((1.0, 0.0))
    rng = np.random.default_rng(41)
    for k in range(3):
        dprim = np.zeros_like(prim)
        dprim[..., 0] = _bump(run, rng)
        adj = float((gs * dprim).sum())
        h = 1e-6
        jp = run.forward(prim + h * dprim, params)[0]
        jm = run.forward(prim - h * dprim, params)[0]
        fd = (jp - jm) / (2 * h)
        assert abs(fd - adj) <= 1e-5 * abs(adj) + 1e-10 * abs(jp), (k, fd, adj)
    for i, scale in enumerate([1.0, 1.0, 1e-3, 10.0]):
        h = 1e-6 * scale
        dp = np.zeros(4)
        dp[i] = h
        jp = run.forward(prim, Params(*(np.array(params) + dp)))[0]
        jm = run.forward(prim, Params(*(np.array(params) - dp)))[0]
        fd = (jp - jm) / (2 * h)
        assert abs(fd - gp[i]) <= 1e-4 * max(abs(gp[i]), 1e-12), (i, fd, gp[i])


def test_torch_autograd_function():
    run = AdjointRun(resolution=32, steps=6, checkpoint_every=4)
    prim = run.initial_state(seed=5)
    run.forward(prim, Params(), freeze=True)
    F = objective_function(run, (1.0, 0.5))
    sigma0 = torch.from_numpy(prim[..., 0].copy()).requires_grad_(True)
    params = torch.tensor([0.5, 0.1, 1e-3, 10.0], dtype=torch.float64, requires_grad=True)
    J = F.apply(sigma0, params)
    J.backward()
    assert sigma0.grad.shape == sigma0.shape and params.grad.shape == (4,)
    assert torch.isfinite(sigma0.grad).all() and torch.isfinite(params.grad).all()


@pytest.fixture(scope="module")
def full_run():
    """The full-size adjoint case: 512^2, config-0 physics with q = 0.5,
    e = 0.1, 400 RK2 steps at CFL 0.3, dt frozen, checkpoints every 20."""
    run = AdjointRun(resolution=512, steps=400, checkpoint_every=20)
    params = Params(0.5, 0.1, 1e-3, 10.0)
    prim = run.initial_state(seed=0)
    run.forward(prim, params, freeze=True, keep=True)
    return run, params, prim


def test_full_size_gradient_matches_central_differences(full_run):
    """Eight seeded directions, each a smooth surface-density bump plus a
    parameter direction, central differences with h = 1e-6."""
    run, params, prim = full_run
    run.forward(prim, params, keep=True)
    gs, gp = run.gradient((1.0, 0.0))
    rng = np.random.default_rng(8)
    scale = np.array([0.1, 0.05, 1e-3, 1.0])
    for k in range(8):
        dprim = np.zeros_like(prim)
        dprim[..., 0] = _bump(run, rng)
        dpar = rng.uniform(-1.0, 1.0, 4) * scale
        adj = float((gs * dprim).sum()) + float(gp @ dpar)
        h = 1e-6
        jp = run.forward(prim + h * dprim, Params(*(np.array(params) + h * dpar)))[0]
        jm = run.forward(prim - h * dprim, Params(*(np.array(params) - h * dpar)))[0]
        fd = (jp - jm) / (2 * h)
        assert abs(fd - adj) <= 1e-4 * abs(adj) + 1e-10 * abs(jp), (k, fd, adj)


def test_full_size_gradient_matches_tangent(full_run):
    """The dot-product test <lambda, du> = <grad J, d> against the
    forward-mode tangent at full size, for both objectives."""
    run, params, prim = full_run
    rng = np.random.default_rng(9)
    for weights in ((1.0, 0.0), (0.0, 1.0)):
        run.forward(prim, params, keep=True)
        gs, gp = run.gradient(weights)
        dprim = np.zeros_like(prim)
        dprim[..., 0] = rng.uniform(-1, 1, prim.shape[:2]) * 1e-2
        dpar = rng.uniform(-1, 1, 4) * np.array([0.1, 0.05, 1e-4, 1.0])
        tan = run.tangent(prim, params, dprim, dpar, weights)
        adj = float((gs * dprim).sum()) + float(gp @ dpar)
        assert abs(tan - adj) <= 1e-9 * abs(tan), (weights, tan, adj)


def test_batched_adjoint_matches_each_disk_alone():
    """Disks run concurrently on several streams and host threads give the
    J and gradients of each disk run alone with the batch's segment length,
    bit for bit; with the library's own segment choice the state gradient is
    the same bits and the parameter sums agree to rounding."""
    from sailfish_b200.adjoint import SHARED_SWEEP_ROWS, AdjointDisk, BatchedAdjoint

    disks = [AdjointDisk(32, Params(0.3, 0.2, 1e-3, 10.0)), AdjointDisk(48, Params(0.9, 0.0, 3e-4, 10.0), 20.0),
             AdjointDisk(40, Params(0.5, 0.4, 5e-3, 10.0)), AdjointDisk(32, Params(0.7, 0.1, 1e-4, 10.0), 15.0)]
    batch = BatchedAdjoint(disks, steps=12, checkpoint_every=5, streams=3)
    J = batch.forward(freeze=True, keep=True)
    grads = batch.gradient((1.0, 0.5))
    lib = _capi.lib()
    for i, d in enumerate(disks):
        run = AdjointRun(resolution=d.resolution, steps=12, checkpoint_every=5, mach=d.mach)
        j = run.forward(batch.prims[i], d.params, freeze=True, keep=True)
        _capi.check(lib.cbdiso_b200_set_adjoint_segment_rows(SHARED_SWEEP_ROWS), "segment_rows")
        try:
            gs, gp = run.gradient((1.0, 0.5))
        finally:
            lib.cbdiso_b200_set_adjoint_segment_rows(0)
        np.testing.assert_array_equal(j, J[i])
        np.testing.assert_array_equal(gs, grads[i][0])
        np.testing.assert_array_equal(gp, grads[i][1])
        own = AdjointRun(resolution=d.resolution, steps=12, checkpoint_every=5, mach=d.mach)
        own.forward(batch.prims[i], d.params, freeze=True, keep=True)
        gs_own, gp_own = own.gradient((1.0, 0.5))
        np.testing.assert_array_equal(gs_own, gs)
        np.testing.assert_allclose(gp_own, gp, rtol=1e-12, atol=1e-14 * np.abs(gp).max())


def test_captured_batch_matches_the_eager_batch():
    """The whole batch's forward and adjoint as one CUDA graph (one branch
    per disk) gives the eager batch's J and gradients bit for bit, on two
    replays in a row."""
    from sailfish_b200.adjoint import AdjointDisk, BatchedAdjoint

    disks = [AdjointDisk(32, Params(0.3, 0.2, 1e-3, 10.0)), AdjointDisk(48, Params(0.9, 0.0, 3e-4, 10.0), 20.0),
             AdjointDisk(40, Params(0.5, 0.4, 5e-3, 10.0))]
    batch = BatchedAdjoint(disks, steps=12, checkpoint_every=5, streams=3, store_states=True)
    J = batch.forward(freeze=True, keep=True)
    grads = batch.gradient((1.0, 0.5))
    batch.capture((1.0, 0.5))
    for _ in range(2):
        batch.replay()
        got = batch.results()
        for i in range(len(disks)):
            np.testing.assert_array_equal(got[i][0], J[i])
            np.testing.assert_array_equal(got[i][1], grads[i][0])
            np.testing.assert_array_equal(got[i][2], grads[i][1])


def _stage_adjoint(s, dev, nb, stage, p, pn, out, lam, variant, chained):
    lib = s._lib
    g = ctypes.byref(s._grid)
    _capi.check(lib.cbdiso_b200_set_adjoint_variant(variant), "variant")
    try:
        rec = ctypes.c_void_p(dev.data_ptr() + stage * nb)
        lam_rd, lam_n = torch.zeros_like(p), torch.zeros_like(p)
        ws = torch.zeros(int(lib.cbdiso_b200_adjoint_workspace_bytes(g)) // 8 + 8, dtype=torch.float64,
                         device=p.device)
        pnp = P(pn) if pn is not None else None
        lnp = P(lam_n) if pn is not None else None
        if chained:
            rows = int(lib.cbdiso_b200_adjoint_chain_blocks(g))
            chain = torch.zeros(rows * 4, dtype=torch.float64, device=p.device)
            jac = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, 20)).to(p.device)
            _capi.check(lib.cbdiso_b200_stage_adjoint_chained(g, rec, P(p), pnp, P(out), P(lam), P(lam_rd), lnp,
                                                              P(jac), P(chain), P(ws), _stream()), "chained")
            pars = torch.zeros(4, dtype=torch.float64, device=p.device)
            _capi.check(lib.cbdiso_b200_adjoint_chain_finish(P(chain), rows, P(pars), _stream()), "finish")
        else:
            words = torch.zeros(p.shape[:2], dtype=torch.int32, device=p.device)
            _capi.check(lib.cbdiso_b200_stage_record_branches(g, rec, P(p), P(out), P(words), _stream()), "rec")
            pars = torch.zeros(12, dtype=torch.float64, device=p.device)
            _capi.check(lib.cbdiso_b200_stage_adjoint(g, rec, P(p), pnp, P(out), P(words), P(lam), P(lam_rd), lnp,
                                                      P(pars), P(ws), _stream()), "adjoint")
        torch.cuda.synchronize()
        return lam_rd.cpu().numpy(), lam_n.cpu().numpy(), pars.cpu().numpy()
    finally:
        lib.cbdiso_b200_set_adjoint_variant(1)


@pytest.fixture(scope="module")
def wide_case():
    """256^2 (three column strips of the fused kernel, several row segments)."""
    run = AdjointRun(resolution=256, steps=1)
    params = Params(0.6, 0.2, 2e-3, 10.0)
    s = _state(run, params, steps=2)
    dt = 0.8 * s.mesh.min_spacing() / s.maximum_wavespeed() * 0.3
    dev, nb, _ = run._records(s, s.time, dt)
    return s, dev, nb


@pytest.mark.parametrize("chained", [False, True])
@pytest.mark.parametrize("stage", [0, 1])
@pytest.mark.parametrize("case", ["stage_case", "wide_case"])
def test_fused_stage_adjoint_matches_the_separate_passes(request, case, stage, chained):
    """The row-marching adjoint kernel gives the separate passes' lambda_rd and
    lambda_n bit for bit; the parameter sums (added in another order) to
    rounding."""
    c = request.getfixturevalue(case)
    s, dev, nb = (c[2], c[3], c[4]) if case == "stage_case" else c
    p = s._buf[0]
    pn = p.clone() if stage == 1 else None
    out = _stage(s, dev, stage * nb, 0.5 * stage, p, pn)
    lam = torch.zeros_like(p)
    lam[2:-2, 2:-2] = _rand_like(lam[2:-2, 2:-2], 31 + stage)
    a = _stage_adjoint(s, dev, nb, stage, p, pn, out, lam, 0, chained)
    b = _stage_adjoint(s, dev, nb, stage, p, pn, out, lam, 1, chained)
    np.testing.assert_array_equal(b[0], a[0])
    np.testing.assert_array_equal(b[1], a[1])
    np.testing.assert_allclose(b[2], a[2], rtol=1e-12, atol=1e-12 * np.abs(a[2]).max())
