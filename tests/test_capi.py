"""The C ABI library loads and exports every symbol include/mt_masstree.h
declares (no device calls: this runs without a GPU)."""
import ctypes
import os
import re

from indexingpu_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdrs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    names = set()
    for h in hdrs:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(mt_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["mt_create", "mt_destroy", "mt_find", "mt_insert", "mt_update", "mt_erase", "mt_scan",
              "mt_mixed_batch", "mt_sync", "mt_stats"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_status_strings():
    lib = _lib.load()
    assert lib.mt_status_string(0) == b"ok"
    assert b"exhausted" in lib.mt_status_string(1)


def test_flag_values_match_header():
    """The Python mirror passes the same flag bits that mt_masstree.h defines."""
    from indexingpu_b200 import masstree

    src = open(os.path.join(ROOT, "include", "mt_masstree.h")).read()
    defined = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define MT_(FLAG_\w+)\s+(\d+)u", src)}
    assert "FLAG_REMOVE_EMPTY_LAYERS" in defined and "FLAG_MERGE" in defined
    for name, value in defined.items():
        assert getattr(masstree, name) == value, name
    assert len(set(defined.values())) == len(defined)
