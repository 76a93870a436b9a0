"""
Device-resident stepping (Solver.run): dt, stage times and the Kepler orbit
on the device, CUDA-graph replay. Checked against the host-driven driver loop
and against the reference fixtures.
"""

import numpy as np
import pytest

from cases import diagnostics, load
from test_gpu_parity import field_error, product_solver

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)


@pytest.mark.parametrize("name", ["cbd_t15_n64", "kitp_t18_n64_rk3_p2", "cbd_t18_48x40_ecc"])
@pytest.mark.parametrize("graph", [False, True])
def test_device_run_matches_reference_fixture(name, graph):
    d = load(name)
    meta = d["meta"]
    s = product_solver(d, "exact")
    rows = s.run(meta["steps"], cfl=0.3, graph=graph, steps_per_graph=4)
    assert len(rows) == meta["steps"]
    dts = np.array([r[-1] for r in rows])
    # device sin / cos may differ from the host libm by an ulp in the orbit
    np.testing.assert_allclose(dts, d["dts"], rtol=1e-12, atol=0)
    assert field_error(s.solution, d["last"]) <= 1e-12
    assert s.time == pytest.approx(float(d["time"]), rel=1e-13)


def test_device_run_matches_host_loop_with_reductions():
    d = load("cbd_t18_n64_p3")
    host = product_solver(d, "exact")
    dev = product_solver(d, "exact")
    want = []
    for _ in range(12):
        host.advance(host.mesh.min_spacing() / host.maximum_wavespeed() * 0.3)
        want.append(host.reductions())
    got = dev.run(12, cfl=0.3, graph=True, steps_per_graph=3)
    assert field_error(dev.solution, host.solution) <= 1e-13
    for a, b in zip(got, want):
        assert a[0] == pytest.approx(b[0], rel=1e-14)  # time
        np.testing.assert_allclose(np.array(a[1:-1], dtype=complex), np.array(b[1:], dtype=complex),
                                   rtol=1e-10, atol=1e-14)
    # the host API continues seamlessly after a device run
    assert dev.maximum_wavespeed() == pytest.approx(host.maximum_wavespeed(), rel=1e-13)


def test_device_run_rejects_arbitrary_point_mass_callbacks():
    from sailfish_b200 import make_solver
    from sailfish_b200.physics import PointMass
    from sailfish_b200.setups import CircumbinaryDisk

    setup = CircumbinaryDisk(domain_radius=8.0)
    physics = setup.physics
    physics["point_mass_function"] = lambda t: (PointMass(mass=1.0), PointMass())
    s = make_solver("cbdiso_2d", physics, {}, setup=setup, mesh=setup.mesh(32))
    with pytest.raises(ValueError, match="Kepler binary"):
        s.run(3)


@pytest.mark.parametrize("graph", [False, True])
def test_checkpoints_taken_inside_one_run(graph):
    """run(checkpoints=...) copies the state before every group of
    steps_per_graph steps on the device; the checkpoints, the time series and
    the final state equal those of the same steps run group by group with a
    host copy of the state before each group (the adjoint's former
    checkpointed forward)."""
    d = load("cbd_t15_n64")
    one, groups = product_solver(d, "exact"), product_solver(d, "exact")
    steps, k = 23, 5
    slots = [torch.empty_like(one._buf[0]) for _ in range(-(-steps // k))]
    rows = one.run(steps, cfl=0.3, graph=graph, steps_per_graph=k, checkpoints=slots)
    want_rows, want_states = [], []
    for start in range(0, steps, k):
        want_states.append(groups._buf[0].clone())
        want_rows += groups.run(min(k, steps - start), cfl=0.3, graph=graph, steps_per_graph=k)
    for got, want in zip(slots, want_states):
        assert torch.equal(got, want)
    assert np.array_equal(np.array(rows), np.array(want_rows))
    assert np.array_equal(one.solution, groups.solution)
    with pytest.raises(ValueError):
        one.run(steps, cfl=0.3, steps_per_graph=k, checkpoints=slots[:-1])
