"""pytest configuration: the `gpu` marker, and loaders for the package (which
lives in the `tesserae.jl_b200/` folder) and the CPU oracle."""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def load_package():
    if "tesserae_b200" in sys.modules:
        return sys.modules["tesserae_b200"]
    pkg = ROOT / "tesserae.jl_b200"
    spec = importlib.util.spec_from_file_location("tesserae_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tesserae_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle_module():
    if str(ROOT / "oracle") not in sys.path:
        sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def tb():
    return load_package()


@pytest.fixture(scope="session")
def oracle(tb):
    return load_oracle_module().Oracle(tb._abi)


@pytest.fixture(scope="session")
def ctx(tb):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tesserae_b200 import runtime
    c = runtime.Context(0)
    yield c
    c.close()
