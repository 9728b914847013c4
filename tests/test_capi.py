"""The C-ABI library loads and exports every symbol declared in include/*.h (no compute calls)."""
import ctypes
import re
from pathlib import Path

import pytest

from conftest import ROOT, gpu_available

INCLUDE = ROOT / "include"


def declared_functions():
    names = []
    for h in sorted(INCLUDE.glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cfsa_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "cfsa_ns_create" in names and "cfsa_ns_piso_step" in names
    assert "cfsa_mesh_cylinder" in names
    assert len(names) > 40


def test_library_exports_every_declared_symbol(cf):
    lib = ctypes.CDLL(str(cf.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol(cf):
    import inspect

    src = inspect.getsource(cf)
    missing = [n for n in declared_functions() if f'"{n}"' not in src]
    assert not missing, missing


def test_headers_compile_as_c(tmp_path):
    import subprocess

    src = tmp_path / "t.c"
    src.write_text('#include "cfsa_ns.h"\n#include "cfsa_mesh.h"\nint main(void){return 0;}\n')
    gcc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", f"-I{INCLUDE}", "-c", str(src), "-o",
                    str(tmp_path / "t.o")], check=True)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_create_without_device_fails_cleanly(cf):
    m = cf.Mesh.cylinder(4.0, 1.0, 1, 2)
    m.setupBoundaryConditions()
    s = cf.NavierStokesSolver()
    with pytest.raises(cf.CfsaError) as e:
        s.initialize(m, cf.Fluid(1060.0, 0.004))
    assert e.value.code == cf.CUDA_ERROR
