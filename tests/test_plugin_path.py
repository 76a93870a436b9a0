"""
The solver-extension route of the repository's integration guide (its first
section) through the reference's own code: the one-line shims and the
`.sailfish` file are taken from the guide as written, the reference's
`load_user_config` reads the file (sailfish/driver.py:582-620) and registers the shims
(sailfish/solvers/__init__.py:13-15), and the reference's `make_solver`
(sailfish/solvers/__init__.py:18-46) is called the way its driver calls it
(sailfish/driver.py:439-449), with a reference setup's own physics dict and
mesh.

Without a CUDA device this package's Solver validates the physics and options
and then stops with its "needs a CUDA device" error. That error coming out of
the reference's make_solver shows that the shim's class was the one
constructed, with the reference's arguments. Each case runs in a fresh
interpreter with a copy of the reference package, so that its modules and
its extension registry do not leak into other tests.

Needs the reference tree (REFERENCE_ROOT); skipped where it is absent.
"""

import os
import re
import shutil
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("REFERENCE_ROOT", "/root/reference")
GUIDE = "INTEGRATION.md"  # the integration guide at the repository root

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "sailfish")),
                                reason="the reference tree is not present")


def _recipe_blocks():
    """The fenced python and ini blocks of the integration guide's first section."""
    text = open(os.path.join(ROOT, GUIDE)).read()
    section = text.split("## 1.")[1].split("## 2.")[0]
    py = re.findall(r"```python\n(.*?)```", section, re.S)
    ini = re.findall(r"```ini\n(.*?)```", section, re.S)
    return py, ini


SCRIPT = textwrap.dedent("""
    import os, sys
    sys.path[:0] = [{shims!r}, {ref!r}, {repo!r}]
    os.chdir({work!r})
    os.environ["CUDA_VISIBLE_DEVICES"] = ""
    from sailfish import driver
    from sailfish.solvers import make_solver, SolverInitializationError
    import sailfish.setups  # noqa: F401 (registers the setup classes)
    from sailfish.setup_base import SetupBase
    driver.load_user_config()
    for solver_name, setup_name, params in {cases!r}:
        setup = SetupBase.find_setup_class(setup_name)(**params)
        assert setup.solver == solver_name, (setup.solver, solver_name)
        mesh = setup.mesh(64)
        try:
            make_solver(setup.solver, setup.physics, dict(), setup=setup, mesh=mesh, time=0.0, solution=None,
                        num_patches=1, mode="gpu")
        except RuntimeError as e:
            assert "needs a CUDA device" in str(e), e
            mod = sys.modules[solver_name]
            assert mod.Solver.__module__ == "sailfish_b200." + solver_name, mod.Solver.__module__
            print("constructed", solver_name, "->", mod.Solver.__module__)
        else:
            raise AssertionError("the reference's own solver was constructed")
""")

CASES = [("cbdiso_2d", "kitp-code-comparison", dict(eccentricity=0.1, mass_ratio=0.5)),
         ("cbdgam_2d", "circumbinary-disk", dict(eos="gamma-law"))]


def _run(tmp_path, shims, ini, cases):
    ref_copy = tmp_path / "ref"
    shutil.copytree(os.path.join(REF, "sailfish"), ref_copy / "sailfish")
    shim_dir = tmp_path / "shims"
    shim_dir.mkdir()
    for name, code in shims.items():
        (shim_dir / f"{name}.py").write_text(code)
    work = tmp_path / "work"
    work.mkdir()
    (work / ".sailfish").write_text(ini)
    script = SCRIPT.format(shims=str(shim_dir), ref=str(ref_copy), repo=ROOT, work=str(work), cases=cases)
    return subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300)


def test_integration_recipe_swaps_both_solvers_in(tmp_path):
    py, ini = _recipe_blocks()
    assert len(py) == 2 and len(ini) == 2
    shims = {"cbdiso_2d": py[0], "cbdgam_2d": py[1]}
    r = _run(tmp_path, shims, ini[1], CASES)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "constructed cbdiso_2d -> sailfish_b200.cbdiso_2d" in r.stdout
    assert "constructed cbdgam_2d -> sailfish_b200.cbdgam_2d" in r.stdout


def test_single_solver_recipe(tmp_path):
    py, ini = _recipe_blocks()
    r = _run(tmp_path, {"cbdiso_2d": py[0]}, ini[0], CASES[:1])
    assert r.returncode == 0, r.stdout + r.stderr


def test_comma_separated_extension_list_fails_in_the_reference_driver(tmp_path):
    """Why the recipe separates names by whitespace: the driver splits the
    value with str.split(), so a comma stays in the module name."""
    py, _ = _recipe_blocks()
    r = _run(tmp_path, {"cbdiso_2d": py[0], "cbdgam_2d": py[1]}, "[extensions]\nsolvers = cbdiso_2d, cbdgam_2d\n",
             CASES)
    assert r.returncode != 0
    assert "cbdiso_2d," in r.stderr
