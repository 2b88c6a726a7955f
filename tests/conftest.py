import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "langevinmedium.jl_b200"
PKG_NAME = "langevinmedium_b200"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def load_pkg():
    """Import the package directory langevinmedium.jl_b200 (its name is not an identifier)."""
    if PKG_NAME in sys.modules:
        return sys.modules[PKG_NAME]
    spec = importlib.util.spec_from_file_location(PKG_NAME, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[PKG_NAME] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); the driver runs these with -m gpu")


@pytest.fixture(scope="session")
def lmb():
    pkg = load_pkg()
    if not pkg.capi.LIB_PATH.exists():          # a fresh checkout: build the in-tree library first
        spec = importlib.util.spec_from_file_location("_lim_build", PKG_DIR / "build.py")
        b = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(b)
        b.build()
    return pkg


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle
