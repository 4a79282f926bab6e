"""The C ABI libraries load and export every symbol their headers declare
(no compute calls, so this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(ipg_[a-z0-9_]+)\s*\(", text))


def test_runtime_exports_header():
    import ipregel_b200 as ip
    if not os.path.exists(ip.RUNTIME_PATH):
        pytest.skip("runtime not built")
    lib = ctypes.CDLL(ip.RUNTIME_PATH)
    declared = _declared("ipregel_b200.h")
    assert declared, "no declarations found"
    assert set(ip.RUNTIME_SYMBOLS) == declared
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_app_libraries_export_reference_interface():
    import ipregel_b200 as ip
    libs = sorted(glob.glob(os.path.join(ip.LIB_DIR, "app*.so")))
    if not libs:
        pytest.skip("application libraries not built")
    host_abi = _declared(os.path.join("ipregel_b200", "host.cuh"))
    host_abi = {s for s in host_abi if s.startswith("ipg_app_")}
    assert host_abi <= set(ip.APP_SYMBOLS)
    for path in libs:
        lib = ctypes.CDLL(path)
        missing = [s for s in ip.APP_SYMBOLS if not hasattr(lib, s)]
        assert not missing, (path, missing)


def test_every_version_is_built():
    import ipregel_b200 as ip
    if not os.path.exists(ip.RUNTIME_PATH):
        pytest.skip("runtime not built")
    for app in ("cc", "sssp"):
        for v in ip.VERSIONS:
            assert os.path.exists(ip.app_library(app, v)), (app, v)
    for v in ("combiner", "single_broadcast"):
        assert os.path.exists(ip.app_library("pagerank", v))


def test_product_does_not_import_oracle():
    """The product package has no path into the oracle (no CPU fallback)."""
    for path in glob.glob(os.path.join(ROOT, "ipregel_b200", "**", "*.py"), recursive=True):
        src = open(path).read()
        assert "oracle" not in re.sub(r"#.*", "", src).replace('"""', ""), path


def test_probe_library_is_apart_from_the_runtime():
    """The benchmark's measurement probe lives in its own library: the runtime
    exports none of it, and the probe library exports what its header says."""
    import ipregel_b200 as ip
    if not os.path.exists(ip.PROBE_PATH):
        pytest.skip("probe library not built")
    declared = _declared("ipregel_b200_probe.h")
    assert declared == set(ip.PROBE_SYMBOLS)
    probe = ctypes.CDLL(ip.PROBE_PATH)
    assert all(hasattr(probe, s) for s in declared)
    runtime = ctypes.CDLL(ip.RUNTIME_PATH)
    assert not any(hasattr(runtime, s) for s in declared)
