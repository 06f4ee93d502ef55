import importlib.util
import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "oceanwave3d-fortran90_b200"
# the tests call the probes of include/ow3d_test.h: load the testing build of
# the library (the same objects as libow3d.so, with the probes exported)
os.environ.setdefault("OW3D_TEST_BUILD", "1")


def load_package():
    """Import the package directory (its name is not a Python identifier)."""
    if "ow3d_b200" in sys.modules:
        return sys.modules["ow3d_b200"]
    spec = importlib.util.spec_from_file_location("ow3d_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ow3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def reference_decks():
    """Folder of the reference's example input decks, from the
    OW3D_REFERENCE_DECKS environment variable (None when unset: the tests
    that read those decks are then skipped)."""
    import os
    d = os.environ.get("OW3D_REFERENCE_DECKS")
    return pathlib.Path(d) if d else None


def load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    sys.path.insert(0, str(ROOT / "tests"))


@pytest.fixture(scope="session")
def ow3d():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()
