"""The C-ABI library loads without a GPU and exports every function include/photon_cuda.h declares."""
import re

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include" / "photon_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(pe_[a-z_0-9]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for required in ("pe_device_create", "pe_device_set_scene", "pe_device_render", "pe_device_destroy",
                     "pe_last_error", "pe_scene_build"):
        assert required in names


def test_library_exports_every_declared_symbol(pe):
    lib = pe._capi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol(pe):
    assert set(declared_functions()) <= set(pe._capi.SIGNATURES), set(declared_functions()) - set(pe._capi.SIGNATURES)


def test_abi_version(pe):
    header = (ROOT / "include" / "photon_cuda.h").read_text()
    want = int(re.search(r"#define PE_ABI_VERSION (\d+)", header).group(1))
    assert pe._capi.load().pe_abi_version() == want


def test_device_create_reports_error_without_crashing(pe):
    errs = []
    dev = pe.create_device("cuda:99", errs)
    assert dev is None and errs
    assert pe.create_device("vulkan:0", errs) is None
