"""The C-ABI library loads without a GPU and exports every symbol include/*.h declares."""
import ctypes
import os
import re

from wadjet_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^WG_API\s+[\w\s\*]+?\b(wg_\w+)\s*\(", text, flags=re.M))
    return names


def test_header_declares_the_operator_contract():
    names = declared_symbols()
    for must in ("wg_filter_execute", "wg_join_build_append", "wg_join_probe", "wg_agg_consume", "wg_agg_merge",
                 "wg_agg_finalize", "wg_agg_emit", "wg_pipeline_run", "wg_ledger_stats"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    assert declared_symbols() == set(_abi.SIGNATURES)


def test_version_and_errors_without_gpu():
    import wadjet_b200 as wg
    assert b"sm_100a" in wg.lib.wg_version()
    # a NULL context is rejected on the host before any device work
    assert wg.lib.wg_ctx_synchronize(None) == _abi.WG_E_INVALID
    assert b"NULL" in wg.lib.wg_last_error()
