"""The drop-in RenderDevice adapter builds against the reference's headers and links: the library
that carries it (with the reference engine and its RenderSession driver) loads and resolves
libphoton_cuda.so from the package folder.  No GPU call is made here."""
import ctypes
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402


@pytest.mark.skipif(not oracle.adapter_available(), reason="oracle/_ref/libpe_adapter.so not built")
def test_adapter_library_loads_and_exports_the_session_driver():
    lib = ctypes.CDLL(str(oracle.ADAPTER_LIB))
    for name in ("ref_session_cuda", "ref_session_cuda_update", "ref_scene_create", "ref_render"):
        assert hasattr(lib, name), name
    maps = pathlib.Path("/proc/self/maps").read_text()
    assert "photon-engine_b200/libphoton_cuda.so" in maps
