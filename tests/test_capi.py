"""The C-ABI libraries load without a GPU and export every symbol that
include/ipcb.h and include/ipcb_direct.h declare (no compute calls here)."""
import ctypes
import os
import re

from ipc_warp_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols(header="ipcb.h"):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ipcb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(_native.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_table_covers_header():
    assert sorted(_native.SIGNATURES) == header_symbols()


def test_sizes_and_args_without_gpu():
    L = _native.lib()
    assert L.ipcb_version() == 1
    assert L.ipcb_lbvh_bytes(1000) > 1000 * 64
    assert L.ipcb_sort_workspace_u32(10) > 0
    assert L.ipcb_bsr_workspace(100, 10, 10) > 100 * 8
    # argument validation happens before any launch
    assert L.ipcb_sort_pairs_u32(None, None, -1, 8, None, 0, None) == 1
    assert L.ipcb_contact_hessian(5, None, None, 0, 0, 1.0, None, None, None, None, None, None) == 1
    assert L.ipcb_contact_hessian_after(1, None, None, -1, 0, None, 1.0, None, None, None, None, None, None) == 1
    # line-search accumulator fold and body-block inverses: refused before any launch
    assert L.ipcb_acc_fold(None, None, 1, None) == 1
    assert L.ipcb_acc_fold(ctypes.c_void_p(16), None, 2, None) == 1
    assert L.ipcb_acc_fold(ctypes.c_void_p(16), ctypes.c_void_p(16), -1, None) == 1
    assert L.ipcb_group_jacobi(-1, 1, None, None, None, 0, None, None, None) == 1
    assert L.ipcb_group_jacobi(4, 2, None, None, None, 0, None, None, None) == 1
    assert L.ipcb_group_jacobi(4, 0, None, None, None, 0, None, None, None) == 0  # nothing to do
    # contact BSR: negative counts mean "read on the device" and need the lists' count words
    assert L.ipcb_contact_bsr_workspace(10, 5) > L.ipcb_contact_bsr_workspace(1, 5)
    ee = _native.Contacts(None, None, None, None, None, None, 4)  # capacity 4, no count word
    pt = _native.Contacts(None, None, None, None, None, None, 4)
    nnz, st = ctypes.c_int(), ctypes.c_int()
    assert L.ipcb_contact_bsr(ctypes.byref(ee), -1, ctypes.byref(pt), -1, 8, None, None, 0, ctypes.byref(nnz),
                              None, None, ctypes.byref(nnz), ctypes.byref(st), None, 0, None) == 1
    assert L.ipcb_contact_bsr(ctypes.byref(ee), 5, ctypes.byref(pt), 0, 8, None, None, 0, ctypes.byref(nnz),
                              None, None, ctypes.byref(nnz), ctypes.byref(st), None, 0, None) == 1  # 5 > capacity


def test_direct_library_exports_header_symbols():
    from ipc_warp_b200 import direct

    lib = direct.lib()
    syms = header_symbols("ipcb_direct.h")
    assert len(syms) == 7
    assert not [s for s in syms if not hasattr(lib, s)]
    assert sorted(direct.SIGNATURES) == syms
    # argument validation before any device work
    assert lib.ipcb_direct_analyze(None, 0, 0, None, None, 0, 0, None) == 1
    assert lib.ipcb_direct_factor(None, None, None) == 1


def _header_arity(header="ipcb.h"):
    """{name: number of parameters} from the C declarations."""
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(ipcb_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_argument_counts_match_header():
    arity = _header_arity()
    wrong = {name: (len(args), arity[name]) for name, (_, args) in _native.SIGNATURES.items()
             if name in arity and len(args) != arity[name]}
    assert not wrong, wrong
