"""The C ABI: libhpic.so loads on a machine without a GPU and exports every
function include/hpic.h declares (no compute is called here)."""
import ctypes
import os
import re

import hpic

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "hpic.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)  # drop comments
    text = re.sub(r"//[^\n]*", " ", text)
    names = set()
    # a declaration: return type, name hp_*, '(' ... ');'
    for m in re.finditer(r"(?:^|[;}\n])\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(hp_\w+)\s*\(([^;{]*?)\)\s*;", text):
        names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_operators():
    names = declared_functions()
    for op in ("hp_Field", "hp_Move", "hp_SortBoundary", "hp_MCC", "hp_Deposit", "hp_step", "hp_case_create",
               "hp_batch_create", "hp_server_create", "hp_Deposit_noalloc", "hp_step_kernels"):
        assert op in names, op
    assert len(names) > 40


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(hpic.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared in include/hpic.h but not exported: {missing}"
