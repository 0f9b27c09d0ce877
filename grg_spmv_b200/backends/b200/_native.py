"""ctypes binding of ``libgrg_b200.so`` (declared in ``include/grg_b200.h``) and its build.

The library is built in-tree (``grg_spmv_b200/libgrg_b200.so``) by ``build_library()``; the
B200 runtime refuses to start without it — there is no CPU or PyTorch fallback.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path
import subprocess
import threading

PACKAGE_DIR = Path(__file__).resolve().parents[2]
REPO_DIR = PACKAGE_DIR.parent
LIB_PATH = PACKAGE_DIR / "libgrg_b200.so"
SOURCES = (PACKAGE_DIR / "csrc" / "grg_b200.cu",)
HEADER_DIR = REPO_DIR / "include"
ABI_VERSION = 14

NVCC_FLAGS = (
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
)

# Status codes, enums and entry coding (grg_b200.h).
OK, ERR_INVALID, ERR_CUDA, ERR_UNSUPPORTED = 0, 1, 2, 3
F64, F32, MIXED = 0, 1, 2
MAX_SLOT_BUCKETS = 8
LAUNCH_PDL = 1
SCHEDULE_LEVELS, SCHEDULE_DATAFLOW = 0, 1
DEVICE_WAIT_TIMEOUT = 6
UP, DOWN = 0, 1
INIT_NONE, INIT_VECTOR, INIT_XTX, INIT_MATRIX = 0, 1, 2, 3
BIAS_NONE, BIAS_VECTOR, BIAS_XTX = 0, 1, 2
SEG_START = 0x80000000


def mix_plane(nbytes: int) -> int:
    """GRG_B200_MIX_PLANE: a plane's bytes rounded up to 16."""
    return (int(nbytes) + 15) // 16 * 16


def mix_bytes(rows: int, ld: int) -> int:
    """GRG_B200_MIX_BYTES: one mixed buffer (float hi plane, then int16 lo plane)."""
    return mix_plane(int(rows) * int(ld) * 4) + mix_plane(int(rows) * int(ld) * 2)


def mix_ld(k: int) -> int:
    """Leading dimension of mixed storage for k columns (a multiple of 4)."""
    return (int(k) + 3) // 4 * 4


SRC_SHIFT = 29
SRC_STATE, SRC_INPUT, SRC_MISS, SRC_NULL = 0, 1, 2, 3
ID_MASK = 0x1FFFFFFF
MAX_ID = 0x1FFFFFFF
NARROW_VARIANTS = 17


class Level(ctypes.Structure):
    _fields_ = [
        ("row_begin", ctypes.c_int64),
        ("num_rows", ctypes.c_int64),
        ("num_entries", ctypes.c_int64),
        ("num_heavy", ctypes.c_int64),
        ("heavy_threshold", ctypes.c_int32),
        ("ring_slot", ctypes.c_int32),
        ("blob", ctypes.c_void_p),
        ("blob_bytes", ctypes.c_int64),
        ("off_row_ptr", ctypes.c_int64),
        ("off_heavy", ctypes.c_int64),
        ("off_row_ids", ctypes.c_int64),
        ("off_entries", ctypes.c_int64),
        ("list_align", ctypes.c_int32),
        ("num_slot_buckets", ctypes.c_int32),
        ("slot_pos", ctypes.c_int64 * 8),
        ("slot_entry", ctypes.c_int64 * 8),
        ("slot_width", ctypes.c_int32 * 8),
        ("short_rows", ctypes.c_int64),
    ]


class TraverseArgs(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int32),
        ("direction", ctypes.c_int32),
        ("init_mode", ctypes.c_int32),
        ("bias_mode", ctypes.c_int32),
        ("emit_all_nodes", ctypes.c_int32),
        ("by_individual", ctypes.c_int32),
        ("use_miss", ctypes.c_int32),
        ("exact_order", ctypes.c_int32),
        ("k", ctypes.c_int64),
        ("num_nodes", ctypes.c_int64),
        ("num_samples", ctypes.c_int64),
        ("num_mutations", ctypes.c_int64),
        ("num_individuals", ctypes.c_int64),
        ("state", ctypes.c_void_p),
        ("ld_state", ctypes.c_int64),
        ("input", ctypes.c_void_p),
        ("ld_input", ctypes.c_int64),
        ("output", ctypes.c_void_p),
        ("ld_output", ctypes.c_int64),
        ("miss", ctypes.c_void_p),
        ("ld_miss", ctypes.c_int64),
        ("init_vector", ctypes.c_void_p),
        ("init_matrix", ctypes.c_void_p),
        ("ld_init", ctypes.c_int64),
        ("node_perm", ctypes.c_void_p),
        ("inv_node_perm", ctypes.c_void_p),
        ("xtx_node", ctypes.c_void_p),
        ("endpoint_bias", ctypes.c_void_p),
        ("sample_to_individual", ctypes.c_void_p),
        ("ind_ptr", ctypes.c_void_p),
        ("ind_samples", ctypes.c_void_p),
        ("sel_mut_ptr", ctypes.c_void_p),
        ("sel_mut_idx", ctypes.c_void_p),
        ("sel_miss_ptr", ctypes.c_void_p),
        ("sel_miss_idx", ctypes.c_void_p),
        ("level0_rows", ctypes.c_int64),
        ("num_levels", ctypes.c_int32),
        ("levels", ctypes.POINTER(Level)),
        ("ring", ctypes.c_void_p),
        ("slot_buffers", ctypes.POINTER(ctypes.c_void_p)),
        ("slot_bytes", ctypes.POINTER(ctypes.c_int64)),
        ("num_slots", ctypes.c_int32),
        ("error_word", ctypes.c_void_p),
        ("narrow_variant", ctypes.c_int32),
        ("heavy_variant", ctypes.c_int32),
        ("mix_scratch", ctypes.c_void_p),
        ("mix_scratch_bytes", ctypes.c_int64),
        ("narrow_split", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("dataflow_sync", ctypes.c_void_p),
        ("launch_flags", ctypes.c_int32),
        ("persist_ctas", ctypes.c_int32),
        ("fuse_entries", ctypes.c_int64),
    ]


class RowopArgs(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_int64),
        ("k", ctypes.c_int64),
        ("ld", ctypes.c_int64),
        ("src", ctypes.c_void_p),
        ("dst", ctypes.c_void_p),
        ("miss_in", ctypes.c_void_p),
        ("miss_scale", ctypes.c_void_p),
        ("pre_scale", ctypes.c_void_p),
        ("col_sub", ctypes.c_void_p),
        ("sub_scale", ctypes.c_void_p),
        ("post_scale", ctypes.c_void_p),
        ("miss_out", ctypes.c_void_p),
        ("miss_out_scale", ctypes.c_void_p),
        ("col_sums", ctypes.c_int32),
        ("sum_weight", ctypes.c_void_p),
        ("partials", ctypes.c_void_p),
        ("sums", ctypes.c_void_p),
    ]


ROWOP_MAX_BLOCKS = 1184


def rowop_blocks(rows: int) -> int:
    """GRG_B200_ROWOP_BLOCKS: row blocks (and rows of partial sums) of a rowop call."""
    return min((int(rows) + 255) // 256, ROWOP_MAX_BLOCKS)


EXPORTED_SYMBOLS = (
    "grg_b200_abi_version",
    "grg_b200_last_error",
    "grg_b200_ring_create",
    "grg_b200_ring_destroy",
    "grg_b200_seed_up",
    "grg_b200_run_level",
    "grg_b200_output_up",
    "grg_b200_output_down",
    "grg_b200_emit_all",
    "grg_b200_traverse",
    "grg_b200_traverse_static",
    "grg_b200_rowop",
)

_lock = threading.Lock()
_lib = None


def build_library(*, force: bool = False, verbose: bool = False) -> Path:
    """Compile ``libgrg_b200.so`` for sm_100a with nvcc (cross-compiles without a GPU)."""
    newest = max(p.stat().st_mtime for p in (*SOURCES, HEADER_DIR / "grg_b200.h"))
    if not force and LIB_PATH.exists() and LIB_PATH.stat().st_mtime >= newest:
        return LIB_PATH
    nvcc = os.environ.get("NVCC", "nvcc")
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *NVCC_FLAGS, f"-I{HEADER_DIR}", "-o", str(tmp), *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    tmp.replace(LIB_PATH)
    return LIB_PATH


def load_library():
    """Load the library once; raises if it is missing or was built for another ABI."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with grg_spmv_b200.backends.b200.build_library() "
                "(the B200 backend has no CPU fallback)"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name in EXPORTED_SYMBOLS:
            getattr(lib, name)
        lib.grg_b200_abi_version.restype = ctypes.c_int
        lib.grg_b200_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        lib.grg_b200_last_error.restype = ctypes.c_size_t
        lib.grg_b200_ring_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        lib.grg_b200_ring_destroy.argtypes = [ctypes.c_void_p]
        for name in ("grg_b200_seed_up", "grg_b200_output_up", "grg_b200_output_down", "grg_b200_emit_all", "grg_b200_traverse",
                     "grg_b200_traverse_static"):
            getattr(lib, name).argtypes = [ctypes.POINTER(TraverseArgs), ctypes.c_void_p]
            getattr(lib, name).restype = ctypes.c_int
        lib.grg_b200_rowop.argtypes = [ctypes.POINTER(RowopArgs), ctypes.c_void_p]
        lib.grg_b200_rowop.restype = ctypes.c_int
        lib.grg_b200_run_level.argtypes = [ctypes.POINTER(TraverseArgs), ctypes.POINTER(Level), ctypes.c_void_p]
        lib.grg_b200_run_level.restype = ctypes.c_int
        version = int(lib.grg_b200_abi_version())
        if version != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {version}, expected {ABI_VERSION}; rebuild it")
        _lib = lib
        return lib


def last_error(lib) -> str:
    buf = ctypes.create_string_buffer(1024)
    lib.grg_b200_last_error(buf, len(buf))
    return buf.value.decode("utf-8", errors="replace")


def check(lib, status: int, what: str) -> None:
    if int(status) != OK:
        raise RuntimeError(f"{what} failed with status {int(status)}: {last_error(lib)}")


__all__ = [
    "EXPORTED_SYMBOLS",
    "LIB_PATH",
    "Level",
    "RowopArgs",
    "TraverseArgs",
    "build_library",
    "check",
    "last_error",
    "load_library",
]
