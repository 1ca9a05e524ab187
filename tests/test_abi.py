"""The C-ABI library loads on a CPU-only host and exports every function
declared in include/*.h (no compute calls)."""
import ctypes
import re
from pathlib import Path

import graphene_b200._lib as L

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(gr_[a-z0-9_]+)\s*\(",
                             text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_functions():
    names = declared_functions()
    assert "gr_spmv" in names and "gr_solve" in names and "gr_solver_create" in names
    assert len(names) >= 30


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(str(L.LIB_PATH))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_header():
    assert declared_functions() <= set(L.SIGNATURES), set(declared_functions()) - set(L.SIGNATURES)


def test_error_reporting_without_gpu():
    lib = L.lib()
    rc = lib.gr_host_matrix_poisson(0, 1, 1, 1, 0, 0, ctypes.byref(ctypes.c_void_p()))
    assert rc == L.GR_EINVAL
    assert b"positive" in lib.gr_last_error()
    assert lib.gr_version() >= 1


def test_c_client_of_host_entry_points(tmp_path):
    """tests/abi_host_example.c, compiled with gcc against the header and
    linked with the library, runs the host-side entry points from plain C."""
    import subprocess
    exe = tmp_path / "abi_host_example"
    lib_dir = Path(L.LIB_PATH).parent
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "abi_host_example.c"), "-L", str(lib_dir),
                    "-lgraphene_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"
