"""Every name bench.py reads is defined somewhere in it (an assignment, an
argument, an import, a function or class, a builtin): a cheap check over the
source's syntax tree that catches a name left behind by an edit in one of the
benchmark's workloads, which only a GPU run would otherwise reach."""
from __future__ import annotations

import ast
import builtins
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def undefined_names(path: Path) -> set[str]:
    tree = ast.parse(path.read_text())
    defined = set(dir(builtins)) | {"__file__", "__name__"}
    for node in ast.walk(tree):
        if isinstance(node, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
            defined.add(node.name)
        elif isinstance(node, ast.Import):
            defined.update((a.asname or a.name).split(".")[0] for a in node.names)
        elif isinstance(node, ast.ImportFrom):
            defined.update(a.asname or a.name for a in node.names)
        elif isinstance(node, ast.Name) and isinstance(node.ctx, (ast.Store, ast.Del)):
            defined.add(node.id)
        elif isinstance(node, ast.arg):
            defined.add(node.arg)
        elif isinstance(node, ast.ExceptHandler) and node.name:
            defined.add(node.name)
    used = {n.id for n in ast.walk(tree) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load)}
    return used - defined


def test_bench_reads_no_undefined_name():
    assert undefined_names(ROOT / "bench.py") == set()


def test_the_check_finds_a_planted_undefined_name(tmp_path):
    p = tmp_path / "planted.py"
    p.write_text("def f(a):\n    return a + lanes\n")
    assert undefined_names(p) == {"lanes"}
