"""Static checks of ``bench.py`` that need no GPU.

Its GPU paths only run on a B200, so a name error there would first show at measurement time.
These checks parse the file and flag, in every top-level function, names that are read but
never bound (locally, as a module global or builtin), and locals that shadow a module-level
function (which turns every earlier use of that function into an UnboundLocalError).  The
CPU-only helpers are also called directly.
"""

from __future__ import annotations

import ast
import builtins
from pathlib import Path
import sys

import pytest

BENCH = Path(__file__).resolve().parents[1] / "bench.py"


def _module_names(tree: ast.Module) -> set[str]:
    names = set()
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)):
            names.add(node.name)
        elif isinstance(node, (ast.Import, ast.ImportFrom)):
            names.update((a.asname or a.name).split(".")[0] for a in node.names)
        elif isinstance(node, ast.Assign):
            names.update(t.id for t in node.targets if isinstance(t, ast.Name))
    return names


def _functions(tree: ast.Module):
    return [node for node in tree.body if isinstance(node, ast.FunctionDef)]


def _bound_in(func: ast.FunctionDef) -> set[str]:
    bound = {a.arg for a in func.args.args + func.args.kwonlyargs}
    for node in ast.walk(func):
        if isinstance(node, (ast.Import, ast.ImportFrom)):
            bound.update((a.asname or a.name).split(".")[0] for a in node.names)
        elif isinstance(node, ast.Name) and isinstance(node.ctx, ast.Store):
            bound.add(node.id)
        elif isinstance(node, (ast.FunctionDef, ast.Lambda)):
            if isinstance(node, ast.FunctionDef):
                bound.add(node.name)
            bound.update(a.arg for a in node.args.args + node.args.kwonlyargs)
        elif isinstance(node, ast.ExceptHandler) and node.name:
            bound.add(node.name)
    return bound


def test_bench_functions_bind_every_name_they_read():
    tree = ast.parse(BENCH.read_text())
    module = _module_names(tree) | set(dir(builtins))
    for func in _functions(tree):
        used = {n.id for n in ast.walk(func) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load)}
        assert not used - _bound_in(func) - module, f"{func.name} reads unbound names {sorted(used - _bound_in(func) - module)}"


def test_bench_locals_do_not_shadow_module_functions():
    tree = ast.parse(BENCH.read_text())
    functions = {f.name for f in _functions(tree)}
    for func in _functions(tree):
        stored = {n.id for n in ast.walk(func) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Store)}
        assert not stored & functions, f"{func.name} assigns {sorted(stored & functions)}, which are module functions"


def test_bench_cpu_helpers(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    sys.path.insert(0, str(BENCH.parent))
    import bench

    args = bench.parse_args()
    assert args.k == 8 and args.e2e_inflight == 8 and args.pdl == "auto" and args.slots == "none"
    spec = bench.large_spec(0.1)
    assert (spec.num_samples, spec.num_nodes, spec.num_mutations, spec.num_levels) == (100_000, 6_000_000, 2_000_000, 60)

    class Level:
        def __init__(self, rows, entries, heavy=0, ring_slot=-1):
            self.num_rows, self.num_entries, self.num_heavy, self.ring_slot = rows, entries, heavy, ring_slot

    levels = [Level(10, 100), Level(10, 100), Level(0, 0), Level(10, 100), Level(10, 10_000, heavy=2), Level(10, 100)]
    assert bench.traversal_level_launches(levels, True, 0) == 5
    assert bench.traversal_level_launches(levels, False, 0) == 6  # heavy rows apart: a second launch
    assert bench.traversal_level_launches(levels, True, 1000) == 3  # one run of three, the big level, a single
    with pytest.raises(SystemExit):
        monkeypatch.setattr(sys, "argv", ["bench.py", "--slots", "sideways"])
        bench.parse_args()
