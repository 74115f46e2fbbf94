"""Scripts that GPU tests run in a child process (``python -c SCRIPT``) are
strings, so neither the import of the test module nor a linter sees an
undefined name in them; the child would only fail on the GPU.  This CPU test
compiles every such script and checks that each global name it reads is
imported, assigned or a builtin."""
import ast
import builtins
import symtable
from pathlib import Path

import pytest

TESTS = Path(__file__).resolve().parent


def _child_scripts():
    """Module-level string constants whose name starts with CHILD in tests/*.py."""
    found = []
    for path in sorted(TESTS.glob("test_*.py")):
        tree = ast.parse(path.read_text(), filename=str(path))
        for node in tree.body:
            if not isinstance(node, ast.Assign) or not isinstance(node.value, ast.Constant):
                continue
            if not isinstance(node.value.value, str):
                continue
            for target in node.targets:
                if isinstance(target, ast.Name) and target.id.startswith("CHILD"):
                    found.append((f"{path.name}:{target.id}", node.value.value))
    return found


def _undefined_globals(source, name):
    table = symtable.symtable(source, name, "exec")
    defined = {s.get_name() for s in table.get_symbols() if s.is_assigned() or s.is_imported()}
    missing = set()

    def walk(t):
        for s in t.get_symbols():
            if (s.is_global() or t.get_type() == "module") and s.is_referenced():
                n = s.get_name()
                if n not in defined and not hasattr(builtins, n):
                    missing.add(n)
        for child in t.get_children():
            walk(child)

    walk(table)
    return missing


SCRIPTS = _child_scripts()


def test_child_scripts_are_found():
    assert any(name.startswith("test_checked_build_gpu.py") for name, _ in SCRIPTS)


@pytest.mark.parametrize("name,source", SCRIPTS, ids=[n for n, _ in SCRIPTS])
def test_child_script_compiles_and_defines_every_name(name, source):
    compile(source, name, "exec")
    assert _undefined_globals(source, name) == set()


def test_the_check_catches_a_missing_import():
    assert _undefined_globals("import json\nx = np.zeros(3)\n", "t") == {"np"}
