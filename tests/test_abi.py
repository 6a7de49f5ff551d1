"""CPU checks of the boundary: libgvdb2.so loads and exports every symbol
include/gvdb2.h declares; the oracle library loads.  No compute calls."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def built_lib():
    import build as gbuild
    return gbuild.build()


def test_header_declares_entry_points():
    from gvdb2 import declared_symbols
    names = declared_symbols()
    for must in ("gvdb2_rebuild_topology", "gvdb2_update_atlas", "gvdb2_insert_points_subcell", "gvdb2_scatter_density",
                 "gvdb2_gather_density", "gvdb2_update_apron", "gvdb2_update_apron_faces", "gvdb2_scatter_kernel",
                 "gvdb2_gather_kernel", "gvdb2_scatter_kernel_backward", "gvdb2_gather_kernel_backward"):
        assert must in names
    assert len(names) >= 38


def test_library_exports_every_declared_symbol(built_lib):
    from gvdb2 import declared_symbols
    lib = ctypes.CDLL(built_lib)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_library_is_sm100a_only(built_lib):
    # the kernels are built for sm_100a alone: no compatibility PTX, no other SASS
    import build as gbuild
    assert gbuild.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_wrapper_binds_every_symbol(built_lib):
    from gvdb2 import _lib, declared_symbols
    L = _lib.lib()
    for n in declared_symbols():
        assert getattr(L, n) is not None


def test_create_without_device_reports_not_available(built_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from gvdb2 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.gvdb2_create(ctypes.byref(h), 0) == 8  # GVDB2_ERR_NOT_AVAILABLE
    assert not h.value


def test_null_handle_is_an_argument_error(built_lib):
    from gvdb2 import _lib
    L = _lib.lib()
    assert L.gvdb2_update_atlas(None) == 1
    assert L.gvdb2_destroy(None) == 0


def test_oracle_loads(oracle_mod):
    o = oracle_mod.Oracle()
    o.configure(3, 3, 3, 3, 3)
    o.add_channel(0, 1)
    assert o.tile_res() == 10


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "gvdb-voxels_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in txt and "liboracle" not in txt and "gvdb_oracle" not in txt, f


def test_cpp_facade_compiles_and_links(built_lib, tmp_path):
    """The C++ drop-in facade compiles against the header and links to the library."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    src = tmp_path / "use.cpp"
    src.write_text(
        '#include "gvdb2_volume.hpp"\n'
        "int main(int argc, char**) {\n"
        "  if (argc > 5) { gvdb2::VolumeGVDB v(0); v.Configure(3,3,3,3,3); v.AddChannel(0, GVDB2_T_FLOAT, 1);\n"
        "    v.RebuildTopology(0, 2.0f); v.UpdateAtlas(); v.UpdateApron(); }\n"
        "  return 0; }\n")
    out = tmp_path / "use"
    libdir = os.path.dirname(built_lib)
    r = subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(out),
                        "-L", libdir, "-lgvdb2", f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_wrapper_argument_counts_match_header():
    """Every ctypes binding passes as many arguments as the header declares:
    a binding slip would otherwise show only on a GPU."""
    import re
    from gvdb2 import _lib
    txt = re.sub(r"/\*.*?\*/", "", open(_lib.HEADER).read(), flags=re.S)
    decls = dict(re.findall(r"GVDB2_API\s+[\w\s\*]*?\b(gvdb2_\w+)\s*\(([^)]*)\)\s*;", txt))
    assert decls, "no declarations parsed"
    for name, params in decls.items():
        p = params.strip()
        n = 0 if p in ("", "void") else p.count(",") + 1
        if name in _lib._SIGS:
            assert len(_lib._SIGS[name]) == n, f"{name}: header takes {n} arguments, binding {len(_lib._SIGS[name])}"
