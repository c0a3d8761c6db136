"""The C ABI (CPU only, no GPU calls): the headers in include/ compile as C, every function
they declare is exported by the matching library, the libraries load without a GPU, and no
library links or names the oracle (the checker must never be on the product path)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, pgb

INC = os.path.join(ROOT, "include")
HEADERS = {
    "pgb_g5.h": ["libpg5.so", "libpg5sym.so", "libpg5_newton.so"],
    "pgb_g5table.h": ["libpg5table.so"],
    "pgb_g6.h": ["libpg6.so", "libpg6_newton.so"],
    "pgb_bhtree.h": ["libpgbtree.so"],
}


def declared_functions(header, symmetric=False):
    src = open(os.path.join(INC, header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    # keep the branch of #ifdef PGB_SYMMETRIC that applies
    out, keep = [], [True]
    for line in src.splitlines():
        s = line.strip()
        if s.startswith("#ifdef PGB_SYMMETRIC"):
            keep.append(symmetric)
            continue
        if s.startswith("#else") and len(keep) > 1:
            keep[-1] = not keep[-1]
            continue
        if s.startswith("#endif") and len(keep) > 1:
            keep.pop()
            continue
        if all(keep):
            out.append(line)
    text = "\n".join(out)
    names = re.findall(r"^\s*(?:extern\s+)?(?:void|int|long long|double|float|pgbt_tree)\s+\**\s*(\w+)\s*\(", text, re.M)
    return sorted(set(names))


@pytest.mark.parametrize("header", sorted(HEADERS))
def test_header_compiles_as_c(header, tmp_path):
    src = tmp_path / "t.c"
    src.write_text(f'#include "{header}"\nint main(void) {{ return 0; }}\n')
    for sym in (False, True):
        cmd = ["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", INC, str(src)]
        if sym:
            cmd.insert(1, "-DPGB_SYMMETRIC")
        subprocess.run(cmd, check=True)


@pytest.mark.parametrize("header,lib", [(h, l) for h, ls in sorted(HEADERS.items()) for l in ls])
def test_every_declared_function_is_exported(header, lib):
    path = pgb.ffi.lib_path(lib)
    L = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    names = declared_functions(header, symmetric=(lib == "libpg5sym.so"))
    assert len(names) > 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    if header == "pgb_g5table.h":
        C.c_float.in_dll(L, "Force_table")   # the exported table data symbol


def test_reference_symbol_sets_are_covered():
    """Every function the reference libraries export is exported by the drop-in too."""
    from oracle import oracle as O
    pairs = [("libpg5_ref.so", "libpg5.so"), ("libpg5table_ref.so", "libpg5table.so"),
             ("libquad_ref.so", "libpg5.so"), ("libpg6_ref.so", "libpg6.so"),
             ("libpg5sym_ref.so", "libpg5sym.so")]
    internal = {"GravityKernel", "GravityKernel0", "c_GravityKernel", "c_GravityKernel0", "gravity_kernel",
                "gravity_kernel_future", "gravity_kernel2", "gravity_kernels", "gravity_kerneln",
                "gravity_kernel2n", "rsqrt", "drsqrt", "rsqrt_bias", "get_dtime"}
    checked = 0
    for ref, ours in pairs:
        if not O.ref_available(ref):
            continue
        out = subprocess.run(["nm", "-D", "--defined-only", O.ref_path(ref)], capture_output=True, text=True).stdout
        names = {l.split()[-1] for l in out.splitlines() if " T " in l}
        names = {n for n in names if n not in internal and not n.startswith("avx_")}
        L = C.CDLL(pgb.ffi.lib_path(ours), mode=os.RTLD_LOCAL | os.RTLD_NOW)
        missing = sorted(n for n in names if not hasattr(L, n))
        assert not missing, (ours, missing)
        checked += 1
    if checked == 0:
        pytest.skip("reference not built")


@pytest.mark.parametrize("lib", ["libpg5.so", "libpg5sym.so", "libpg5table.so", "libpg6.so", "libpgbtree.so"])
def test_product_does_not_use_the_oracle(lib):
    out = subprocess.run(["nm", "-D", pgb.ffi.lib_path(lib)], capture_output=True, text=True).stdout
    assert "orc_" not in out
    ldd = subprocess.run(["ldd", pgb.ffi.lib_path(lib)], capture_output=True, text=True).stdout
    assert "oracle" not in ldd and "_ref" not in ldd


def test_sources_do_not_reference_the_oracle():
    csrc = os.path.join(ROOT, "phantom-grape_b200", "csrc")
    for name in os.listdir(csrc):
        txt = open(os.path.join(csrc, name)).read()
        assert "pg_oracle" not in txt and "liboracle" not in txt, name
