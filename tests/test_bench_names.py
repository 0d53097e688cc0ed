"""bench.py's legs run only on a GPU box, and some (the multi-scene
workload, the multi-GPU path) only when asked for; much of the package's
Python runs only with a device too. A name that a function uses but nothing
defines would surface there as a NameError at run time. This resolves every
such name statically, on the CPU: each name a function reads that is not
local, not a parameter and not bound in an enclosing function must be bound
at module level or be a builtin."""
from __future__ import annotations

import builtins
import glob
import os
import symtable

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def unresolved(path: str) -> list[str]:
    src = open(path).read()
    top = symtable.symtable(src, path, "exec")
    module_names = {s.get_name() for s in top.get_symbols()
                    if s.is_assigned() or s.is_imported() or s.is_namespace()}
    known = module_names | set(dir(builtins)) | {"__file__", "__name__", "__spec__"}
    missing = []

    def walk(table):
        for child in table.get_children():
            if child.get_type() == "function":
                for sym in child.get_symbols():
                    if sym.is_referenced() and sym.is_global() and sym.get_name() not in known:
                        missing.append(f"{child.get_name()}: {sym.get_name()}")
            walk(child)

    walk(top)
    return missing


def python_sources():
    files = ["bench.py", "__graft_entry__.py"]
    for pattern in ("parallax_b200/*.py", "oracle/*.py", "tests/*.py"):
        files += sorted(os.path.relpath(f, ROOT) for f in glob.glob(os.path.join(ROOT, pattern)))
    return files


def test_every_name_the_python_sources_use_is_defined():
    missing = {f: m for f in python_sources() if (m := unresolved(os.path.join(ROOT, f)))}
    assert missing == {}


def test_the_check_finds_an_undefined_name(tmp_path):
    bad = tmp_path / "bad.py"
    bad.write_text("def outer():\n    def inner():\n        return frames[0]\n    return inner\n")
    assert unresolved(str(bad)) == ["inner: frames"]
