"""The C ABI library loads and exports every function include/n2w.h declares."""
import ctypes as C
import re

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include" / "n2w.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(n2w_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_core_entry_points():
    names = declared_functions()
    for required in ["n2w_bvh_create", "n2w_bvh_query_device", "n2w_bvh_query_device_masked",
                     "n2w_wos_estimate", "n2w_wos_pure_samples", "n2w_wos_prefix_samples", "n2w_wos_combine",
                     "n2w_reduce_samples", "n2w_mesh_bumpy_sphere_ref", "n2w_last_error"]:
        assert required in names


def test_library_exports_every_declared_symbol(n2w):
    lib = C.CDLL(str(n2w.LIB_PATH))
    missing = [name for name in declared_functions() if not hasattr(lib, name)]
    assert not missing, f"libn2w.so lacks {missing}"


def test_python_binding_covers_header(n2w):
    bound = set(n2w.EXPORTED)
    missing = [name for name in declared_functions() if name not in bound]
    assert not missing, f"ctypes binding lacks {missing}"


def test_error_path_sets_message(n2w):
    from n2w._lib import lib

    st = lib.n2w_mesh_bumpy_sphere_ref(2, 8, C.c_float(0.1), C.byref(C.c_void_p()))
    assert st == 1
    assert b"stacks >= 4" in lib.n2w_last_error()


def test_abi_version(n2w):
    from n2w._lib import lib

    assert lib.n2w_abi_version() == 1
