"""spyker_b200 against the reference's public Python API (the committed
fixture tests/golden/api_surface.json, made by make_api_surface.py from the
reference sources): every exported name exists, and every public function,
constructor and method takes the reference's parameters in the reference's
order with the reference's defaults (extra trailing parameters of our own, and
defaults for parameters the reference requires, are allowed), so code written
against ``import spyker`` runs unchanged."""

import ast
import inspect
import json
import os

import pytest

import spyker_b200 as spyker
from spyker_b200 import sparse, utils

HERE = os.path.dirname(os.path.abspath(__file__))
SURFACE = json.load(open(os.path.join(HERE, "golden", "api_surface.json")))

# Reference utilities for formats this build leaves out (image files need
# stb, absent from the reference tree as well).
NOT_BUILT = {("utils", "read_image"), ("utils", "write_image")}


def _value(text):
    try:
        return ast.literal_eval(text)
    except ValueError:
        return text


def _check(ours, want, where, method=False):
    got = list(inspect.signature(ours).parameters.values())
    if method and got and got[0].name in ("self", "cls"):
        got = got[1:]
    names = []
    for p in got:
        if p.kind == p.VAR_POSITIONAL:
            names.append("*" + p.name)
        elif p.kind != p.VAR_KEYWORD:
            names.append(p.name)
    ref_names = [n for n, _ in want]
    assert names[: len(ref_names)] == ref_names, f"{where}: parameters {names} != reference {ref_names}"
    for (name, default), p in zip(want, got):
        if default is None or name.startswith("*"):
            continue  # required there; a default here keeps every reference call valid
        assert p.default is not inspect.Parameter.empty, f"{where}: {name} needs the default {default}"
        assert p.default == _value(default), f"{where}: {name}={p.default!r}, reference {default}"
    for p in got[len(ref_names):]:
        assert p.kind == p.VAR_KEYWORD or p.default is not inspect.Parameter.empty, \
            f"{where}: extra parameter {p.name} must have a default"


def test_exports():
    missing = [n for n in SURFACE["exports"] if not hasattr(spyker, n)]
    assert missing == []


def _cases():
    mods = {"module": spyker, "sparse": sparse, "utils": utils}
    for mod, api in (("module", SURFACE["module"]), ("sparse", SURFACE["sparse"]), ("utils", SURFACE["utils"])):
        for name, entry in sorted(api.items()):
            if (mod, name) in NOT_BUILT:
                continue
            if entry["kind"] == "function":
                yield pytest.param(mods[mod], name, None, entry["params"], id=f"{mod}.{name}")
            else:
                for meth, m in sorted(entry["methods"].items()):
                    yield pytest.param(mods[mod], name, meth, m, id=f"{mod}.{name}.{meth}")


@pytest.mark.parametrize("where,name,method,want", list(_cases()))
def test_signature(where, name, method, want):
    assert hasattr(where, name), f"{name} missing"
    obj = getattr(where, name)
    if method is None:
        _check(obj, want, name)
        return
    if want["kind"] == "property":
        assert isinstance(inspect.getattr_static(obj, method), property), f"{name}.{method} is not a property"
        return
    assert hasattr(obj, method), f"{name}.{method} missing"
    _check(getattr(obj, method), want["params"], f"{name}.{method}", method=True)
