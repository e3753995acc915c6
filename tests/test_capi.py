"""CPU checks of the C ABI boundary: the library builds, loads and exports
exactly the entry points include/strata_b200.h declares (no compute calls)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "strata_b200.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(strata_[a-z0-9_]+)\s*\(", text))


@pytest.fixture(scope="module")
def lib_path():
    import importlib.util
    spec = importlib.util.spec_from_file_location("sk_build", ROOT / "strata-k_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("strata_transitive_closure_bool", "strata_shortest_paths_trop", "strata_count_triangles",
              "strata_count_4cliques", "strata_intern_terms", "strata_mssp_trop", "strata_op_sort"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_and_binding_matches_header(lib_path):
    from strata_b200 import _lib as L
    lib = L.load(lib_path)
    assert set(L.SIGNATURES) == declared_symbols()
    assert lib.strata_version().decode().startswith("strata-b200")


def test_library_built_for_sm100a_only():
    """Every object and the link step get exactly one -gencode: sm_100a."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("sk_build_flags", ROOT / "strata-k_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert mod.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    gencodes = [mod.NVFLAGS[i + 1] for i, f in enumerate(mod.NVFLAGS) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"]
    assert not any(f.startswith(("-arch", "--gpu-architecture")) for f in mod.NVFLAGS)


def test_context_without_device_reports_not_built(lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    from strata_b200 import _lib as L
    lib = L.load(lib_path)
    ctx = L.ctxp()
    assert lib.strata_ctx_create(0, 0, C.byref(ctx)) == L.E_NOT_BUILT
    assert lib.strata_last_error(None).decode() == "no context"


def test_engine_raises_not_built_without_device(lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    import strata_b200 as S
    with pytest.raises(S.NotBuilt):
        S.Engine(0)
