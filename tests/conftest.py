"""Shared test setup: loads the package (directory suli-openmp_b200) as `suli_b200`, puts
oracle/ on the path, and registers the `gpu` marker.  GPU tests call the CUDA library
through its C-ABI and check it against the CPU oracle (oracle/, test infrastructure)."""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "suli-openmp_b200"


def load_pkg():
    if "suli_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("suli_b200", PKG_DIR / "__init__.py",
                                                      submodule_search_locations=[str(PKG_DIR)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["suli_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["suli_b200"]


load_pkg()
if str(ROOT / "oracle") not in sys.path:
    sys.path.insert(0, str(ROOT / "oracle"))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls libsuli_gpu.so")


# Run order: the C++ driver's GPU test first (it starts its own processes on the GPU, so it
# runs before this process holds a CUDA context, whatever the GPU's compute mode), then the
# per-step hot path, then the reference's optional features (bottom obstacles, wave inflow,
# restart and field files), and the no-allocation entry point last, so that a run stopping at
# its first failure (-x) has covered everything before the failing part.
OPTIONAL_FEATURE_FILES = ("test_obstacle.py", "test_waves.py", "test_fileio.py")


def pytest_collection_modifyitems(session, config, items):
    def rank(item):
        name = pathlib.Path(str(item.fspath)).name
        if name == "test_driver_gpu.py":
            return -1
        if name == "test_zz_no_alloc.py":
            return 2
        return 1 if name in OPTIONAL_FEATURE_FILES else 0
    items.sort(key=rank)   # stable: file and test order kept within each group


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle
