"""Install lightsmith (the reference) into ``baseline/_ref`` for the reference arm of ``bench.py`` and for the
tests that run lightsmith's own code (its plugin registry, its drivers and run loop, its CPU engine).

The offline install the benchmark contract names,

    python -m pip install --no-index --no-build-isolation --find-links /opt/wheelhouse --target baseline/_ref <lightsmith>

fails here: lightsmith builds with hatchling (its pyproject.toml, ``[build-system]``), which the offline
wheelhouse does not hold. lightsmith is pure Python and its wheel is its ``src/lightsmith`` package as it is
(``[tool.hatch.build.targets.wheel] packages = ["src/lightsmith"]``), so this recipe lays the wheel's content
out by hand: ``baseline/_ref/lightsmith`` is an unmodified copy of the package. lightsmith imports
``array_api_compat``, which is not installed either; the small stand-in under ``tests/golden/shim`` goes beside
it. ``baseline/_ref`` is ignored by git and travels with the working tree to the GPU host.

    python baseline/install_ref.py [--src <lightsmith checkout>]
"""

from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
TARGET = os.path.join(HERE, "_ref")
SHIM = os.path.join(REPO, "tests", "golden", "shim", "array_api_compat")


def _tree_digest(root: str) -> str:
    h = hashlib.sha256()
    for d, dirs, files in sorted(os.walk(root)):
        dirs[:] = sorted(x for x in dirs if x != "__pycache__")
        for f in sorted(files):
            if f.endswith(".pyc"):
                continue
            p = os.path.join(d, f)
            h.update(os.path.relpath(p, root).encode())
            with open(p, "rb") as fh:
                h.update(fh.read())
    return h.hexdigest()[:16]


def pip_install(src: str) -> tuple[bool, str]:
    """The contract's offline pip install (from a copy: the build may write into the source tree)."""
    tmp = "/tmp/lightsmith-src-copy"
    shutil.rmtree(tmp, ignore_errors=True)
    shutil.copytree(src, tmp, ignore=shutil.ignore_patterns(".git", "__pycache__"))
    cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation", "--find-links",
           "/opt/wheelhouse", "--target", TARGET, "--no-deps", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    shutil.rmtree(tmp, ignore_errors=True)
    tail = (r.stdout + r.stderr).strip().splitlines()
    return r.returncode == 0, tail[-1] if tail else ""


def install(src: str) -> str:
    pkg = os.path.join(src, "src", "lightsmith")
    if not os.path.isdir(pkg):
        raise SystemExit(f"no lightsmith package under {src}/src")
    ok, why = pip_install(src)
    how = "pip install --no-index (offline wheelhouse)"
    if not ok or not os.path.isdir(os.path.join(TARGET, "lightsmith")):
        how = f"wheel layout by hand (pip install failed: {why})"
        dst = os.path.join(TARGET, "lightsmith")
        shutil.rmtree(dst, ignore_errors=True)
        os.makedirs(TARGET, exist_ok=True)
        shutil.copytree(pkg, dst, ignore=shutil.ignore_patterns("__pycache__", "*.pyc"))
    shim_dst = os.path.join(TARGET, "array_api_compat")
    shutil.rmtree(shim_dst, ignore_errors=True)
    shutil.copytree(SHIM, shim_dst, ignore=shutil.ignore_patterns("__pycache__", "*.pyc"))
    version = "unknown"
    for line in open(os.path.join(src, "pyproject.toml")):
        if line.startswith("version"):
            version = line.split("=", 1)[1].strip().strip('"')
            break
    digest = _tree_digest(os.path.join(TARGET, "lightsmith"))
    note = f"lightsmith {version}\nhow: {how}\npackage sha256[:16]: {digest}\n"
    with open(os.path.join(TARGET, "INSTALLED.txt"), "w") as f:
        f.write(note)
    return note


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=os.environ.get("LIGHTSMITH_CHECKOUT", "/root/reference"))
    print(install(ap.parse_args().src), end="")


if __name__ == "__main__":
    main()
