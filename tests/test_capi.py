"""The C ABI without a GPU: libnsph.so loads, exports every entry point that
include/nsph.h declares, and the ctypes mirrors of its structs have the C
layout (checked by compiling the header with gcc)."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "nsph.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return re.findall(r"^NSPH_API\s+[\w\s\*]+?\b(nsph_\w+)\s*\(", text, flags=re.M)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "nsph_sph_step" in names and "nsph_grid_build" in names and "nsph_integrate_particles" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    from newton_sph_dev_b200 import _build, _lib

    _build.build()
    lib = ctypes.CDLL(str(_lib.lib_path()))
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in nsph.h but not exported"
    # every binding in _lib has a declaration
    assert {n for n, _, _ in _lib.SIGNATURES} == set(declared_functions())
    # host-only entry points work without a GPU
    lib.nsph_version.restype = ctypes.c_int
    assert lib.nsph_version() >= 1
    lib.nsph_status_string.restype = ctypes.c_char_p
    assert lib.nsph_status_string(2) == b"capacity exceeded"


def test_library_exports_nothing_else():
    from newton_sph_dev_b200 import _build, _lib

    _build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.lib_path())], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("nm unavailable")
    exported = {ln.split()[-1] for ln in out.stdout.splitlines() if " T " in ln}
    ours = {s for s in exported if s.startswith("nsph_")}
    assert ours == set(declared_functions())


def _c_layout(struct: str, fields: list[str]) -> list[int]:
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"nsph.h\"\nint main(void){\n"
    src += f'printf("%zu\\n", sizeof({struct}));\n'
    for f in fields:
        src += f'printf("%zu\\n", offsetof({struct}, {f}));\n'
    src += "return 0;}\n"
    tmp = Path("/tmp/nsph_layout_check.c")
    tmp.write_text(src)
    exe = Path("/tmp/nsph_layout_check")
    subprocess.run(["gcc", f"-I{REPO / 'include'}", str(tmp), "-o", str(exe)], check=True)
    return [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]


@pytest.mark.parametrize("pyname,cname", [("NsphSphParams", "nsph_sph_params"), ("NsphGridView", "nsph_grid_view"),
                                          ("NsphContactParams", "nsph_contact_params"),
                                          ("NsphRaycastCamera", "nsph_raycast_camera"),
                                          ("NsphShape", "nsph_shape"), ("NsphSoftContacts", "nsph_soft_contacts"),
                                          ("NsphSoftContactParams", "nsph_soft_contact_params")])
def test_struct_layouts_match_header(pyname, cname):
    from newton_sph_dev_b200 import _lib

    cls = getattr(_lib, pyname)
    fields = [f for f, _ in cls._fields_]
    c = _c_layout(cname, fields)
    assert c[0] == ctypes.sizeof(cls)
    assert c[1:] == [getattr(cls, f).offset for f in fields]


def test_oracle_camera_layout_matches_header():
    from oracle.oracle import RaycastCamera

    fields = [f for f, _ in RaycastCamera._fields_]
    c = _c_layout("nsph_raycast_camera", fields)
    assert c[0] == ctypes.sizeof(RaycastCamera)
    assert c[1:] == [getattr(RaycastCamera, f).offset for f in fields]


def test_oracle_params_layout_matches_header():
    from oracle.oracle import SphParams32

    fields = [f for f, _ in SphParams32._fields_]
    c = _c_layout("nsph_sph_params", fields)
    assert c[0] == ctypes.sizeof(SphParams32)
    assert c[1:] == [getattr(SphParams32, f).offset for f in fields]


def test_solver_refuses_cpu_models():
    from conftest import lattice_scene

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg = lattice_scene((4, 4, 4), device="cpu")
    with pytest.raises(RuntimeError, match="CUDA"):
        SolverSPH(model, cfg)
