import os
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "tests"))
sys.path.insert(0, str(REPO / "gpu-ibs_b200" / "python"))
sys.path.insert(0, str(REPO / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu() -> bool:
    try:
        import ibs_b200
        return ibs_b200.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def case_root(tmp_path_factory):
    return tmp_path_factory.mktemp("cases")


@pytest.fixture(scope="session")
def build_case(case_root):
    import corpus
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = corpus.build_case(name, case_root)
        return cache[name]
    return get


@pytest.fixture(scope="session")
def native_shim():
    """tests/native/fold_shim.so: the window-statistics fold of
    gpu-ibs_b200/csrc/ibs_core.cuh, the minimizer key map of mz_core.cuh and
    the wide-code reader of wide_core.cuh compiled for the host."""
    src = REPO / "tests" / "native" / "fold_shim.cpp"
    out = REPO / "tests" / "native" / "fold_shim.so"
    deps = [src, REPO / "gpu-ibs_b200/csrc/ibs_core.cuh", REPO / "gpu-ibs_b200/csrc/mz_core.cuh",
            REPO / "gpu-ibs_b200/csrc/wide_core.cuh"]
    if not out.exists() or out.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        cuda_inc = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out), str(src),
                        f"-I{REPO / 'gpu-ibs_b200' / 'csrc'}", f"-I{cuda_inc}"], check=True)
    import ctypes
    return ctypes.CDLL(str(out))
