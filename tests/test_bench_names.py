"""Static check of bench.py and kernel_bench.py: every name a function reads is bound.

The workload paths of bench.py (cross, batched, learned) run only on a GPU, so a
name left over from another workload's code would first fail there, after the
solve.  This walks each top-level function's syntax tree and reports loads of
names that are neither bound in the function (arguments, assignments, imports,
loop and comprehension targets, nested definitions) nor at module level nor
builtins.
"""
import ast
import builtins
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bound_in(node):
    names = set()
    for n in ast.walk(node):
        if isinstance(n, ast.Name) and isinstance(n.ctx, (ast.Store, ast.Del)):
            names.add(n.id)
        elif isinstance(n, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
            names.add(n.name)
        elif isinstance(n, ast.arg):
            names.add(n.arg)
        elif isinstance(n, (ast.Import, ast.ImportFrom)):
            for a in n.names:
                names.add((a.asname or a.name).split(".")[0])
        elif isinstance(n, ast.ExceptHandler) and n.name:
            names.add(n.name)
        elif isinstance(n, (ast.Global, ast.Nonlocal)):
            names.update(n.names)
    return names


@pytest.mark.parametrize("path", ["bench.py", os.path.join("slepc_b200", "kernel_bench.py")])
def test_bench_functions_read_only_bound_names(path):
    with open(os.path.join(ROOT, path)) as f:
        tree = ast.parse(f.read())
    module = set(dir(builtins))
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
            module.add(node.name)
        else:
            module |= _bound_in(node)
    missing = []
    for fn in tree.body:
        if not isinstance(fn, (ast.FunctionDef, ast.AsyncFunctionDef)):
            continue
        local = _bound_in(fn)
        for n in ast.walk(fn):
            if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load) and n.id not in local and n.id not in module:
                missing.append(f"{fn.name}:{n.lineno}: {n.id}")
    assert not missing, missing
