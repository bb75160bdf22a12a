"""Record the reference's public Python API as a fixture.

Parses (never imports) the reference package's sources -- src/python/spyker/
__init__.py, module.py, sparse.py and utils.py -- and writes
tests/golden/api_surface.json: the names the package exports and, for every
public function, class constructor and public method defined in those
modules, its parameter names in order with the source text of each default.
tests/test_api_surface.py checks spyker_b200 against it, so a user of the
reference finds the same names, argument order and defaults.

Usage: python tests/golden/make_api_surface.py [reference checkout]
(default: $SPYKER_REFERENCE, else ../reference next to the repository).  The
fixture is committed; nothing else reads the reference tree.
"""

from __future__ import annotations

import ast
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _params(fn: ast.FunctionDef, drop_self: bool) -> list:
    a = fn.args
    pos = a.posonlyargs + a.args
    defaults = [None] * (len(pos) - len(a.defaults)) + [ast.unparse(d) for d in a.defaults]
    out = [[p.arg, d] for p, d in zip(pos, defaults)]
    if a.vararg:
        out.append(["*" + a.vararg.arg, None])
    for p, d in zip(a.kwonlyargs, a.kw_defaults):
        out.append([p.arg, None if d is None else ast.unparse(d)])
    if drop_self and out and out[0][0] in ("self", "cls"):
        out = out[1:]
    return out


def _module_api(path: str) -> dict:
    tree = ast.parse(open(path).read())
    api = {}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and not node.name.startswith("_"):
            api[node.name] = {"kind": "function", "params": _params(node, False)}
        elif isinstance(node, ast.ClassDef) and not node.name.startswith("_"):
            methods = {}
            for m in node.body:
                if isinstance(m, ast.FunctionDef) and (not m.name.startswith("_") or m.name in ("__init__", "__call__")):
                    if any(isinstance(d, ast.Name) and d.id == "property" for d in m.decorator_list):
                        methods[m.name] = {"kind": "property"}
                        continue
                    if any(isinstance(d, ast.Attribute) and d.attr == "setter" for d in m.decorator_list):
                        continue
                    methods[m.name] = {"kind": "method", "params": _params(m, True)}
            api[node.name] = {"kind": "class", "methods": methods}
    return api


def _exports(path: str) -> list:
    names = []
    for node in ast.parse(open(path).read()).body:
        if isinstance(node, ast.ImportFrom):
            names += [a.asname or a.name for a in node.names]
        elif isinstance(node, ast.Import):
            names += [(a.asname or a.name).split(".")[-1] for a in node.names]
    return sorted(n for n in set(names) if not n.startswith("_"))


def main(ref: str) -> None:
    pkg = os.path.join(ref, "src", "python", "spyker")
    out = {
        "source": "src/python/spyker/{__init__,module,sparse,utils}.py of ShahriarRezghi/Spyker",
        "exports": _exports(os.path.join(pkg, "__init__.py")),
        "module": _module_api(os.path.join(pkg, "module.py")),
        "sparse": _module_api(os.path.join(pkg, "sparse.py")),
        "utils": _module_api(os.path.join(pkg, "utils.py")),
    }
    with open(os.path.join(HERE, "api_surface.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    default = os.environ.get("SPYKER_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
    main(sys.argv[1] if len(sys.argv) > 1 else default)
