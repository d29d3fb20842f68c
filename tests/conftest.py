"""Shared test setup: loads the package (its directory name has a hyphen, so it is
loaded by path), registers the `gpu` marker, and makes sure the oracle is built."""
from __future__ import annotations

import importlib.util
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    if "drone_race_b200" in sys.modules:
        return sys.modules["drone_race_b200"]
    pkg_dir = ROOT / "drone-race_b200"
    spec = importlib.util.spec_from_file_location("drone_race_b200", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["drone_race_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


drb = load_package()

from oracle import oracle as O  # noqa: E402

O.set_abi(drb.abi)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on the B200 box)")


def _ensure_oracle():
    if not O.PORT_LIB.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "port"], check=True)
    ref_src = O.reference_dir()
    if ref_src.exists() and not all(O.ref_available(v) for v in ("nth2_spline", "nth2_dense", "nth8_spline")):
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "-j4", "ref"], check=True)
    if ref_src.exists() and not (O.REF_DIR / "libengine_dropin.so").exists() and drb.abi.LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "engine"], check=True)
    if ref_src.exists() and not (O.REF_DIR / "libadapter_gate.so").exists() and drb.abi.LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "adapter_gate"], check=True)


_ensure_oracle()


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("a CUDA GPU is required for -m gpu tests")
    return True
