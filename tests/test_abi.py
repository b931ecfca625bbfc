"""The C-ABI library loads and exports every entry point the header declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "shinobi_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(shn_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("shn_ctx_create", "shn_scene_create", "shn_grid_build", "shn_trace_closest",
                 "shn_trace_any", "shn_trace_primary", "shn_trace_ao", "shn_pt_render",
                 "shn_exclusive_scan_u32", "shn_compact_u32", "shn_sort_keys_u64"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from shinobi_b200 import _abi
    lib = _abi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.shn_abi_version() == 1
    assert lib.shn_status_string(4) == b"bounded device wait gave up"


def test_python_signatures_cover_header():
    from shinobi_b200 import _abi
    assert set(declared_functions()) == set(_abi.SIGNATURES)


def test_grid_params_defaults_follow_reference():
    import shinobi_b200 as shn
    p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL)
    assert (p.lambda_, p.top_divisor, p.min_res, p.leaf_threshold) == (5.0, 6, 2, 16)
    assert abs(p.lambda_leaf - 1.2) < 1e-7
    q = shn.grid_params(shn.SHN_GRID_UNIFORM)
    assert (q.lambda_, q.top_divisor, q.min_res) == (5.0, 1, 1)


def test_ctx_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        return
    from shinobi_b200 import _abi
    lib = _abi.load()
    h = ctypes.c_void_p()
    st = lib.shn_ctx_create(0, 0, ctypes.byref(h))
    assert st != 0 and not h.value
