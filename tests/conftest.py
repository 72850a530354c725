"""Shared test set-up: registers the `gpu` marker and loads the product
package (directory p3-miden_b200/) under the import name p3_miden_b200."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(Path(__file__).resolve().parent))


def load_product():
    if "p3_miden_b200" in sys.modules:
        return sys.modules["p3_miden_b200"]
    pkg = ROOT / "p3-miden_b200"
    spec = importlib.util.spec_from_file_location("p3_miden_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["p3_miden_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def product():
    return load_product()


@pytest.fixture(scope="session")
def gpu_ctx(product):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = product.Context(0)
    yield ctx
    ctx.close()
