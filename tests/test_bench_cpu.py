"""bench.py and the package's Python modules on the CPU: no name is used
that nothing defines, and the reference arm (the reference's CPU solver on
the host cores) prints its JSON line."""
import ast
import builtins
import glob
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SOURCES = ["bench.py", "__graft_entry__.py"] + sorted(glob.glob(os.path.join(ROOT, "lattice_microbes_b200", "*.py")))


def _bound_names(tree):
    names = set(dir(builtins)) | {"__file__", "__name__", "__doc__"}
    for node in ast.walk(tree):
        if isinstance(node, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
            names.add(node.name)
        elif isinstance(node, ast.arg):
            names.add(node.arg)
        elif isinstance(node, ast.Name) and isinstance(node.ctx, (ast.Store, ast.Del)):
            names.add(node.id)
        elif isinstance(node, (ast.Import, ast.ImportFrom)):
            for a in node.names:
                names.add((a.asname or a.name).split(".")[0])
        elif isinstance(node, ast.ExceptHandler) and node.name:
            names.add(node.name)
        elif isinstance(node, (ast.Global, ast.Nonlocal)):
            names.update(node.names)
        elif isinstance(node, ast.MatchAs) and node.name:
            names.add(node.name)
    return names


@pytest.mark.parametrize("path", SOURCES, ids=os.path.basename)
def test_no_undefined_names(path):
    path = os.path.join(ROOT, path)
    tree = ast.parse(open(path).read(), path)
    bound = _bound_names(tree)
    missing = sorted({(n.id, n.lineno) for n in ast.walk(tree)
                      if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load) and n.id not in bound})
    assert not missing, "names used but never defined: %s" % missing


def test_reference_arm_prints_its_line():
    sys.path.insert(0, ROOT)
    from tests import ref_cpu_lib
    if not ref_cpu_lib.available():
        pytest.skip("reference CPU solvers not built")
    env = dict(os.environ, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--cpu-sample-time", "1e-4"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "site-steps/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0
