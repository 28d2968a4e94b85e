"""The shipped package never reaches the oracle: no module of public_b200 imports it, and importing
every module (the C-ABI binding, the closure, slabs, autograd, the study scripts) leaves it unloaded."""
import ast
import glob
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_no_package_module_imports_the_oracle():
    bad = []
    for path in glob.glob(os.path.join(ROOT, "public_b200", "*.py")):
        for node in ast.walk(ast.parse(open(path).read())):
            names = []
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom) and node.module:
                names = [node.module]
            bad += [(os.path.basename(path), n) for n in names if n.split(".")[0] == "oracle"]
    assert not bad, bad


def test_importing_the_package_leaves_the_oracle_unloaded():
    mods = sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(ROOT, "public_b200", "*.py"))
                  if not p.endswith("__main__.py"))
    code = ("import importlib, sys\n"
            f"for m in {mods!r}:\n"
            "    importlib.import_module('public_b200.' + m if m != '__init__' else 'public_b200')\n"
            "print(sorted(k for k in sys.modules if k == 'oracle' or k.startswith('oracle.')))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "[]", r.stdout
