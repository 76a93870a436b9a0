"""
The gamma-law oracle (oracle/cbdgam_2d_oracle.c through oracle/host_gam.py)
and the reference's own gamma-law kernels built in place (oracle/_ref)
against the fixtures the reference solver wrote (tests/golden/gam_*.npz):
bit for bit.
"""

import os

import numpy as np
import pytest

from cases import diagnostics, gam_initial_state, gam_names, gam_oracle_config, load
from oracle import host_gam as og

NAMES = gam_names()
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_gam_omp.so")


def _run(name, kind):
    d = load(name)
    meta = d["meta"]
    cfg = gam_oracle_config(meta)
    s = og.GamOracleSolver(cfg, gam_initial_state(d), 0.0, og.GamKernels(kind, cfg.plm_theta))
    dts, series, first = [], [], None
    for n in range(meta["steps"]):
        dt = min(cfg.dx, cfg.dy) / s.maximum_wavespeed() * meta["cfl"]
        s.advance(dt)
        dts.append(dt)
        series.append(s.reductions(diagnostics(meta), num_patches=meta["patches"]))
        if n == 0:
            first = s.solution
    return d, s, np.array(dts), np.array(series, dtype=complex), first


def _check(d, s, dts, series, first):
    np.testing.assert_array_equal(dts, d["dts"])
    np.testing.assert_array_equal(series, d["series"])
    assert s.time == float(d["time"])
    if "last" in d:
        np.testing.assert_array_equal(first, d["first"])
        np.testing.assert_array_equal(s.solution, d["last"])
    else:
        np.testing.assert_array_equal(first[::8, ::8], d["first_sub"])
        np.testing.assert_array_equal(s.solution[::8, ::8], d["last_sub"])


def test_there_are_gamma_law_fixtures():
    assert len(NAMES) >= 4


@pytest.mark.parametrize("name", NAMES)
def test_gamma_oracle_matches_reference_fixtures(name):
    _check(*_run(name, "oracle"))


@pytest.mark.skipif(not os.path.exists(REF), reason="reference tree not built here")
@pytest.mark.parametrize("name", NAMES)
def test_gamma_reference_build_matches_fixtures(name):
    _check(*_run(name, "ref"))


def test_gamma_initial_data_restatement():
    """oracle's gamma-law disk primitive equals the fixture's setup data."""
    d = load("gam_n64")
    x0, y0, x1, y1, ni, nj = d["meta"]["mesh"]
    dx, dy = (x1 - x0) / ni, (y1 - y0) / nj
    for i in (0, 17, 31, 32, 63):
        for j in (0, 5, 32, 63):
            got = og.gamma_disk_primitive(x0 + (i + 0.5) * dx, y0 + (j + 0.5) * dy)
            assert tuple(d["ic"][i, j]) == got
