"""The reference's own test suite, run against this project's `_turboquant`.

The reference's Python package is a one-line front
(python/turboquant/__init__.py: `from ._turboquant import TurboQuantSpace`)
over its pybind11 extension.  Here that front is paired with this project's
`_turboquant` (turboquant-space_b200/bindings/tq_pybind.cpp, built over the C
ABI into turboquant-space_b200/python/refabi/), and the reference's
python/tests/test_turboquant.py runs unchanged on the GPU library.  Both
reference files travel as copies under oracle/_ref/refsuite (made by
`make -C oracle ref`, git-ignored); without them the test skips.
"""
import glob
import os
import shutil
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SUITE = os.path.join(ROOT, "oracle", "_ref", "refsuite")
MODULE_DIR = os.path.join(ROOT, "turboquant-space_b200", "python", "refabi")
LIB_DIR = os.path.join(ROOT, "turboquant-space_b200", "python", "turboquant")


@pytest.fixture(scope="module")
def dropin_pkg(tmp_path_factory, cuda_ok):
    front = os.path.join(SUITE, "turboquant", "__init__.py")
    if not os.path.exists(front):
        pytest.skip("the reference's package front and tests are not under oracle/_ref/refsuite")
    mods = glob.glob(os.path.join(MODULE_DIR, "_turboquant*.so"))
    assert mods, "the _turboquant module over the C ABI is not built (make -C turboquant-space_b200)"
    root = tmp_path_factory.mktemp("dropin")
    pkg = root / "turboquant"
    pkg.mkdir()
    shutil.copy(front, pkg / "__init__.py")
    shutil.copy(mods[0], pkg / os.path.basename(mods[0]))
    env = dict(os.environ)
    env["PYTHONPATH"] = str(root)
    env["LD_LIBRARY_PATH"] = LIB_DIR + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    return root, env


def test_the_front_loads_this_projects_module(dropin_pkg):
    root, env = dropin_pkg
    code = ("import turboquant, turboquant._turboquant as m; "
            "print(m.__file__); print(m.__doc__); "
            "s = turboquant.TurboQuantSpace(128); print(s.code_size_bytes())")
    out = subprocess.run([sys.executable, "-c", code], env=env, cwd=str(root), capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    assert lines[0].startswith(str(root)) and "B200" in lines[1] and lines[2] == "76"


def test_reference_suite_passes_on_the_gpu_library(dropin_pkg):
    root, env = dropin_pkg
    # run the suite from beside the package front, so that pytest's path
    # insertion finds this front and module only
    suite = root / "test_turboquant.py"
    shutil.copy(os.path.join(SUITE, "test_turboquant.py"), suite)
    out = subprocess.run([sys.executable, "-m", "pytest", str(suite), "-q", "-p", "no:cacheprovider",
                          "--rootdir", str(root)],
                         env=env, cwd=str(root), capture_output=True, text=True, timeout=1800)
    tail = "\n".join(out.stdout.splitlines()[-15:])
    print(tail)
    assert out.returncode == 0, tail + out.stderr[-2000:]
    assert " passed" in tail and "failed" not in tail
