"""
Test-side description of the golden cases (tests/golden/*.npz): turns a
fixture's recorded setup name and parameters into an oracle configuration,
with the physics each reference setup would hand to the solver
(sailfish/setups/circumbinary_disk.py, binary_bondi.py, simple2d.py).
"""

import glob
import json
import math
import os

import numpy as np

from oracle import host as oh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    """The isothermal solver-run fixtures (make_golden.py); the gamma-law ones
    (gam_*), the checkpoint fixtures (chkpt_*, make_checkpoint.py) and the
    1000-step throughput-configuration ones (config1_*, `long_names`) have
    their own tests."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("chkpt_", "gam_", "config1_")))


def long_names():
    """The 1000-step fixtures of the plain-solver throughput configuration
    (1024^2, 2048^2, 4096^2; make_golden.py LONG_CASES)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "config1_*.npz")))


def gam_names():
    """The gamma-law (cbdgam_2d) solver-run fixtures."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "gam_*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    data = {k: z[k] for k in z.files}
    data["meta"] = json.loads(str(data["meta"]))
    return data


CBD_DEFAULTS = dict(domain_radius=12.0, mach_number=10.0, eccentricity=0.0, mass_ratio=1.0, sink_rate=10.0,
                    sink_radius=0.05, softening_length=0.05, buffer_is_enabled=True, sink_model="torque_free",
                    nu=0.001, initial_sigma=1.0)
KITP_DEFAULTS = dict(mach_number=10.0, eccentricity=0.0, mass_ratio=1.0, sink_radius=0.05, softening_length=0.05,
                     nu=0.001, sink_model="acceleration_free", domain_radius=8.0, sink_rate=10.0,
                     buffer_is_enabled=True)
BONDI_DEFAULTS = dict(aspect=1, height=1.0, x_bin=0.0, sound_speed=1.0, wind_vel=1.0, bh_sep=0.25, bh_mass=1.0,
                      sink_radius=0.05, sink_model="acceleration_free", sink_rate=1e2, mass_ratio=1.0,
                      eccentricity=0.0, softening_length=0.05)


def kitp_sigma(r):
    """KitpCodeComparison.primitive surface density (circumbinary_disk.py:242-263)."""
    return 1.0 * (1e-5 + (1 - 1e-5) * math.exp(-((2.5 / r) ** 12)))


def oracle_config(meta):
    """Oracle configuration for one golden case."""
    x0, y0, x1, y1, ni, nj = meta["mesh"]
    common = dict(x0=x0, x1=x1, y0=y0, y1=y1, ni=int(ni), nj=int(nj), rk_order=meta["rk"],
                  plm_theta=meta["theta"])
    setup = meta["setup"]
    if setup == "circumbinary-disk":
        p = dict(CBD_DEFAULTS, **meta["params"])
        return oh.Config(
            **common, eos_type=2, mach_number=p["mach_number"], nu=p["nu"],
            buffer_is_enabled=p["buffer_is_enabled"], buffer_driving_rate=100.0, buffer_onset_width=1.0,
            buffer_surface_density=p["initial_sigma"],
            masses=oh.binary_masses(1.0, 1.0, p["mass_ratio"], p["eccentricity"], p["softening_length"],
                                    p["sink_model"], p["sink_rate"], p["sink_radius"]))
    if setup == "kitp-code-comparison":
        p = dict(KITP_DEFAULTS, **meta["params"])
        return oh.Config(
            **common, eos_type=2, mach_number=p["mach_number"], nu=p["nu"],
            buffer_is_enabled=p["buffer_is_enabled"], buffer_driving_rate=100.0, buffer_onset_width=1.0,
            buffer_surface_density=kitp_sigma(math.sqrt((x1 - 1.0) ** 2 + 0.0)),
            masses=oh.binary_masses(1.0, 1.0, p["mass_ratio"], p["eccentricity"], p["softening_length"],
                                    p["sink_model"], p["sink_rate"], p["sink_radius"]))
    if setup == "binary-bondi":
        p = dict(BONDI_DEFAULTS, **meta["params"])
        return oh.Config(
            **common, eos_type=1, sound_speed=p["sound_speed"], nu=0.0, reference_time_scale=1.0,
            masses=oh.binary_masses(p["bh_sep"], p["bh_mass"] * (1 + p["mass_ratio"]), p["mass_ratio"],
                                    p["eccentricity"], p["softening_length"], p["sink_model"], p["sink_rate"],
                                    p["sink_radius"], x_offset=p["x_bin"]))
    if setup == "cylindrical-explosion":
        return oh.Config(**common, eos_type=1, sound_speed=1.0, nu=0.0, reference_time_scale=1.0)
    raise ValueError(setup)


def initial_state(data):
    """The fixture's starting primitive state: setup data plus the seeded noise."""
    meta = data["meta"]
    prim = np.array(data["ic"], dtype=np.float64)
    if meta["seed"] is not None:
        ni, nj = prim.shape[:2]
        prim[..., 0] += oh.seeded_noise(ni, nj, meta["seed"])
    return prim


def diagnostics(meta):
    out = []
    for d in meta["diagnostics"]:
        d = dict(d)
        if d.get("radial_cut") is not None:
            d["radial_cut"] = tuple(d["radial_cut"])
        out.append(d)
    return out


GAM_DEFAULTS = dict(domain_radius=12.0, eccentricity=0.0, mass_ratio=1.0, sink_rate=10.0, sink_radius=0.05,
                    softening_length=0.05, buffer_is_enabled=True, sink_model="torque_free", initial_sigma=1.0,
                    initial_pressure=1e-2, cooling_coefficient=0.0, alpha=0.1, constant_softening=True,
                    gamma_law_index=5.0 / 3.0)


def gam_oracle_config(meta):
    """Gamma-law oracle configuration for one golden case: the physics the
    gamma-law CircumbinaryDisk hands to cbdgam_2d (circumbinary_disk.py:137-152)
    and the buffer state sampled at the onset radius (cbdgam_2d.py:291-303)."""
    from oracle import host_gam as og

    x0, y0, x1, y1, ni, nj = meta["mesh"]
    p = dict(GAM_DEFAULTS, **meta["params"])
    onset = 0.1
    bs, _, _, bp = og.gamma_disk_primitive(x1 - onset, 0.0, p["softening_length"], p["initial_sigma"],
                                           p["initial_pressure"])
    on = p["buffer_is_enabled"]
    return og.GamConfig(
        x0=x0, x1=x1, y0=y0, y1=y1, ni=int(ni), nj=int(nj), gamma_law_index=p["gamma_law_index"],
        alpha=p["alpha"], cooling_coefficient=p["cooling_coefficient"], constant_softening=p["constant_softening"],
        buffer_is_enabled=on, buffer_driving_rate=1000.0, buffer_onset_width=onset,
        buffer_surface_density=bs if on else 0.0, buffer_surface_pressure=bp if on else 0.0,
        masses=oh.binary_masses(1.0, 1.0, p["mass_ratio"], p["eccentricity"], p["softening_length"],
                                p["sink_model"], p["sink_rate"], p["sink_radius"]),
        plm_theta=meta["theta"])


def gam_initial_data(meta):
    """The gamma-law CircumbinaryDisk's initial data on the fixture's mesh,
    zone by zone through the oracle's restatement."""
    from oracle import host_gam as og

    x0, y0, x1, y1, ni, nj = meta["mesh"]
    ni, nj = int(ni), int(nj)
    p = dict(GAM_DEFAULTS, **meta["params"])
    dx, dy = (x1 - x0) / ni, (y1 - y0) / nj
    out = np.empty((ni, nj, 4))
    for i in range(ni):
        for j in range(nj):
            out[i, j] = og.gamma_disk_primitive(x0 + (i + 0.5) * dx, y0 + (j + 0.5) * dy, p["softening_length"],
                                                p["initial_sigma"], p["initial_pressure"])
    return out


def gam_initial_state(data):
    """A gamma-law fixture's starting state: setup data times (1 + seeded noise).
    Fixtures stored subsampled get their initial data rebuilt (and checked
    against the stored subsample)."""
    meta = data["meta"]
    prim = np.array(data["ic"], dtype=np.float64)
    if prim.shape[0] != int(meta["mesh"][4]):
        full = gam_initial_data(meta)
        assert np.array_equal(full[::8, ::8], prim)
        prim = full
    if meta["seed"] is not None:
        ni, nj = prim.shape[:2]
        prim[..., 0] *= 1.0 + oh.seeded_noise(ni, nj, meta["seed"])
    return prim
