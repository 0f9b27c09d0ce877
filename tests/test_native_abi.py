"""The C-ABI library: it loads, exports every function the header declares, and the ctypes
mirrors of the header's structs have the C compiler's layout (no GPU needed)."""

from __future__ import annotations

import ctypes
import re
import shutil
import subprocess

import pytest

from conftest import REPO
from grg_spmv_b200.backends.b200 import _native as nat

HEADER = REPO / "include" / "grg_b200.h"


def _declared_functions() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"^(?:int|size_t)\s+(grg_b200_\w+)\s*\(", text, flags=re.M))


def test_library_exports_every_declared_function():
    lib = nat.load_library()
    declared = _declared_functions()
    assert declared == set(nat.EXPORTED_SYMBOLS)
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.grg_b200_abi_version() == nat.ABI_VERSION


def test_header_constants_match_binding():
    text = HEADER.read_text()

    def define(name):
        return int(re.search(rf"#define {name} (0x[0-9A-Fa-f]+|\d+)u?", text).group(1), 0)

    assert define("GRG_B200_ABI_VERSION") == nat.ABI_VERSION
    assert define("GRG_B200_SEG_START") == nat.SEG_START
    assert define("GRG_B200_SRC_SHIFT") == nat.SRC_SHIFT
    assert define("GRG_B200_ID_MASK") == nat.ID_MASK
    assert define("GRG_B200_NARROW_VARIANTS") == nat.NARROW_VARIANTS
    assert define("GRG_B200_MAX_SLOT_BUCKETS") == nat.MAX_SLOT_BUCKETS
    assert define("GRG_B200_LAUNCH_PDL") == nat.LAUNCH_PDL
    assert define("GRG_B200_DEVICE_WAIT_TIMEOUT") == nat.DEVICE_WAIT_TIMEOUT


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
@pytest.mark.parametrize("struct,cname", [(nat.Level, "grg_b200_level"), (nat.TraverseArgs, "grg_b200_traverse_args")])
def test_struct_layout_matches_c(tmp_path, struct, cname):
    fields = [f[0] for f in struct._fields_]
    src = tmp_path / "layout.c"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "grg_b200.h"', "int main(void) {",
             f'  printf("size %zu\\n", sizeof({cname}));']
    lines += [f'  printf("{f} %zu\\n", offsetof({cname}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{HEADER.parent}", str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    assert int(out["size"]) == ctypes.sizeof(struct)
    for f in fields:
        assert int(out[f]) == getattr(struct, f).offset, f


def test_invalid_arguments_fail_before_any_launch():
    lib = nat.load_library()
    args = nat.TraverseArgs()
    args.k = 0
    status = lib.grg_b200_traverse(ctypes.byref(args), None)
    assert status == nat.ERR_INVALID
    assert "k must be >= 1" in nat.last_error(lib)
    args.k = 4
    args.ld_state = 4
    args.state = 16
    args.narrow_variant = 17
    assert lib.grg_b200_traverse(ctypes.byref(args), None) == nat.ERR_INVALID
    assert "narrow_variant" in nat.last_error(lib)


def test_ring_create_rejects_bad_sizes():
    lib = nat.load_library()
    ring = ctypes.c_void_p()
    assert lib.grg_b200_ring_create(0, 0, ctypes.byref(ring)) == nat.ERR_INVALID


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_mixed_storage_sizes_match_c(tmp_path):
    """The Python sizes of mixed buffers equal GRG_B200_MIX_BYTES (the runtime allocates with them)."""
    cases = [(1, 4), (3, 4), (5, 8), (1000, 12), (999_983, 36)]
    src = tmp_path / "mix.c"
    lines = ["#include <stdio.h>", '#include "grg_b200.h"', "int main(void) {",
             '  printf("%d\\n", (int)GRG_B200_MIXED);']
    lines += [f'  printf("%lld\\n", (long long)GRG_B200_MIX_BYTES({r}, {ld}));' for r, ld in cases]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "mix"
    subprocess.run(["gcc", f"-I{HEADER.parent}", str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert out[0] == nat.MIXED
    assert out[1:] == [nat.mix_bytes(r, ld) for r, ld in cases]
    assert [nat.mix_ld(k) for k in (1, 3, 4, 5, 32, 33)] == [4, 4, 4, 8, 32, 36]
