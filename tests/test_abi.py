"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute call: runs without a GPU)."""
import ctypes
import pathlib
import re
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def header_symbols():
    syms = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        syms += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(tb_\w+)\s*\(", text, flags=re.M)
    return sorted(set(syms))


def ensure_built(tb):
    lib = tb._abi.LIB_PATH
    if not lib.exists():
        subprocess.run(["make", "-C", str(lib.parent)], check=True, stdout=subprocess.DEVNULL)
    return lib


def test_header_matches_bindings(tb):
    assert header_symbols() == sorted(tb._abi.declared_symbols())


def test_library_exports_every_declared_symbol(tb):
    lib = ctypes.CDLL(str(ensure_built(tb)))
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_loader(tb):
    ensure_built(tb)
    lib = tb._abi.load_library()
    assert lib.tb_last_error(None) == b"null context"
    assert lib.tb_launch_count(None) == 0


def test_struct_sizes_match_header(tb):
    # Compile a tiny C probe of the POD layouts and compare with ctypes.
    src = ROOT / "include" / "tesserae_b200.h"
    probe = (
        f'#include "{src}"\n#include <stdio.h>\n#include <stddef.h>\n'
        "int main(){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(tb_mesh), sizeof(tb_particles),"
        " sizeof(tb_grid), sizeof(tb_partition), sizeof(tb_weights), sizeof(tb_step_params));}\n")
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = pathlib.Path(d) / "p.c"
        c.write_text(probe)
        exe = pathlib.Path(d) / "p"
        subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
        sizes = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    a = tb._abi
    assert sizes == [ctypes.sizeof(s) for s in (a.tb_mesh, a.tb_particles, a.tb_grid, a.tb_partition,
                                                a.tb_weights, a.tb_step_params)]


def test_tape_bytes_arithmetic():
    """tb_tape_bytes (no device call): the whole tape is nsteps slots; a
    checkpointed tape is its checkpoints plus one segment of slots."""
    import numpy as np
    import tesserae_b200 as tb
    from tesserae_b200 import runtime
    mesh = tb.CartesianMesh(1 / 16, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    n = 1000
    slot = runtime.tape_slot_bytes(mesh, n, np.float32)
    assert slot > n * (13 * 4 + 9 * 8)
    assert runtime.tape_bytes(mesh, n, np.float32, 50, 1) == 50 * slot
    ck = runtime.tape_bytes(mesh, n, np.float32, 50, 10)
    assert slot * 10 < ck < 50 * slot
    assert runtime.tape_bytes(mesh, n, np.float64, 50, 1) > 50 * slot
    assert runtime.tape_bytes(mesh, n, np.float32, 50, 1, apic=True) > 50 * slot
    with pytest.raises(ValueError):
        runtime.tape_bytes(mesh, n, np.float32, 50, 0)
