import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def golden_cases(prefix="engine_"):
    return sorted(f[len(prefix):-4] for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


@pytest.fixture(scope="session")
def golden():
    from lightsmith_b200 import plan as P

    cache = {}

    def load(name):
        if name not in cache:
            cache[name] = P.load(os.path.join(GOLDEN, name + ".npz"))
        return cache[name]
    return load


@pytest.fixture(scope="module")
def plugin(tmp_path_factory):
    """lightsmith (the reference install) with this package installed as a plugin: a distribution declaring the
    entry point (as pyproject.toml does) on sys.path, and lightsmith's registry reloaded from the entry points;
    yields the plugin module (``lightsmith_b200.backend``)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sys.path.insert(0, GOLDEN)
    from refsrc import add_to_path

    if not add_to_path():
        pytest.skip("lightsmith (the reference install, baseline/_ref) not available")
    from lightsmith.backends import base as ls_base

    d = tmp_path_factory.mktemp("site")
    info = d / "lightsmith_b200-0.1.0.dist-info"
    info.mkdir()
    (info / "METADATA").write_text("Metadata-Version: 2.1\nName: lightsmith-b200\nVersion: 0.1.0\n")
    (info / "entry_points.txt").write_text(
        "[lightsmith.backends]\nlightsmith-fdtd-b200 = lightsmith_b200.backend:B200FDTD\n")
    with pytest.MonkeyPatch.context() as mp:
        mp.syspath_prepend(str(d))
        mp.setattr(ls_base, "_REGISTRY", dict(ls_base._REGISTRY))
        mp.setattr(ls_base, "_PLUGINS_LOADED", False)
        from lightsmith_b200 import backend as B

        assert ls_base.get_backend("fdtd", kind="scattering") is B.B200FDTD
        yield B
