"""
Pins the CPU oracle to the reference: the C restatement of the kernels and,
where built, the reference's own kernels (oracle/_ref) reproduce every golden
fixture bit for bit -- states, driver time steps, wavespeed and reductions.
"""

import os

import numpy as np
import pytest

from cases import diagnostics, golden_names, initial_state, load, long_names, oracle_config
from oracle import host as oh

NAMES = golden_names()


def _run(name, kind):
    d = load(name)
    meta = d["meta"]
    cfg = oracle_config(meta)
    prim = initial_state(d) if "first" in d else None
    if prim is None:
        x, y = oh.cell_centres(cfg)
        prim = oh.circumbinary_disk_primitive(x, y, 0.05, 1.0)
        assert np.array_equal(prim[::8, ::8], d["ic"])
        prim[..., 0] += oh.seeded_noise(cfg.ni, cfg.nj, meta["seed"])
    solver = oh.OracleSolver(cfg, prim, 0.0, oh.Kernels(kind, cfg.plm_theta, threads="omp"))
    dts, series = oh.run(solver, meta["steps"], 0.3, diagnostics(meta), meta["patches"])
    return d, solver, np.array(dts), np.array(series, dtype=complex)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_restatement_matches_reference_fixtures(name):
    d, solver, dts, series = _run(name, "oracle")
    assert np.array_equal(dts, d["dts"])
    assert np.array_equal(series, d["series"])
    if "last" in d:
        assert np.array_equal(solver.solution, d["last"])
    else:
        assert np.array_equal(solver.solution[::8, ::8], d["last_sub"])
        assert np.array_equal(np.array([solver.solution[..., q].sum() for q in range(3)]), d["last_sums"])
    assert solver.maximum_wavespeed() == d["max_wavespeed"]
    assert solver.time == d["time"]


REF_BUILT = os.path.exists(os.path.join(oh.HERE, "_ref", "libref_t18_omp.so"))


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("name", [n for n in NAMES if not n.startswith("config0")])
def test_reference_build_matches_fixtures(name):
    d, solver, dts, series = _run(name, "ref")
    assert np.array_equal(dts, d["dts"])
    assert np.array_equal(solver.solution, d["last"])


def test_oracle_theta_is_a_runtime_parameter():
    """Changing theta changes the result (the limiter is active on this data)."""
    d = load("cbd_t15_n64")
    cfg = oracle_config(d["meta"])
    prim = initial_state(d)
    out = []
    for theta in (1.5, 1.8):
        s = oh.OracleSolver(cfg._replace(plm_theta=theta), prim, 0.0, oh.Kernels("oracle", theta))
        oh.run(s, 3)
        out.append(s.solution)
    assert not np.array_equal(out[0], out[1])


def test_kepler_newton_rejects_nonconvergence():
    with pytest.raises(ValueError):
        oh.kepler_eccentric_anomaly(1.0, 1.0, 1.0, 1.5)  # e > 1: no bound orbit


@pytest.mark.parametrize("name", [n for n in long_names() if n.endswith("_n1024")])
def test_oracle_reproduces_first_step_of_long_fixture(name):
    """The 1000-step fixtures were written by the reference's solver in its
    OpenMP mode; the oracle reproduces their first step (state subsample,
    driver dt, wavespeed-derived time and reductions) bit for bit. (The
    larger fixtures hold the same data at 2048^2 and 4096^2; one CPU step of
    those takes too long for this suite.)"""
    d = load(name)
    meta = d["meta"]
    cfg = oracle_config(meta)
    x, y = oh.cell_centres(cfg)
    prim = oh.circumbinary_disk_primitive(x, y, 0.05, 1.0)
    assert np.array_equal(prim[::16, ::16], d["ic"])
    prim[..., 0] += oh.seeded_noise(cfg.ni, cfg.nj, meta["seed"])
    solver = oh.OracleSolver(cfg, prim, 0.0, oh.Kernels("oracle", cfg.plm_theta, threads="omp"))
    dts, series = oh.run(solver, 1, 0.3, diagnostics(meta))
    assert dts[0] == d["dts"][0]
    assert np.array_equal(np.array(series[0], dtype=complex), d["series"][0])
    assert np.array_equal(solver.solution[::16, ::16], d["first_sub"])
