"""Write tests/golden/closures_table.json from the reference's Python surface.

    python tests/golden/make_closures_table.py [path/to/python/rdb/closures.py]

Reads python/rdb/closures.py of the reference as text and parses it with
`ast` (nothing of it is imported or executed).  For every class it records
the keyword defaults of __init__ and every `config.<group>.<knob> = ...`
assignment of its apply()/_apply(): the knob, and whether the value is a
keyword of the constructor (`{"kw": name}`), a constant (`{"const": v}`) or
another expression (`{"expr": source}`).  tests/test_closures_mirror.py checks
the mirror in roundabout_b200/config.py against this table.
"""
from __future__ import annotations

import ast
import json
import sys
from pathlib import Path

DEFAULT_SRC = Path("/root/reference/python/rdb/closures.py")
OUT = Path(__file__).resolve().parent / "closures_table.json"


def _self_attr(node):
    """`self.x`, possibly wrapped in float()/int()/bool(): 'x', else None."""
    if isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in ("float", "int", "bool") \
            and len(node.args) == 1:
        node = node.args[0]
    if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id == "self":
        return node.attr
    return None


def _config_target(node):
    """`config.<group>.<knob>`: 'group.knob', else None."""
    if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Attribute) and \
            isinstance(node.value.value, ast.Name) and node.value.value.id == "config":
        return f"{node.value.attr}.{node.attr}"
    return None


def table(src: Path) -> dict:
    tree = ast.parse(src.read_text())
    out = {}
    for cls in tree.body:
        if not isinstance(cls, ast.ClassDef):
            continue
        entry = {"defaults": {}, "assigns": []}
        # self.<attr> = <kw> in __init__ (attribute names can differ from keywords)
        attr_of_kw = {}
        for fn in cls.body:
            if not isinstance(fn, ast.FunctionDef):
                continue
            if fn.name == "__init__":
                args = fn.args.args[1:]
                defs = fn.args.defaults
                for a, d in zip(args[len(args) - len(defs):], defs):
                    entry["defaults"][a.arg] = ast.literal_eval(d)
                for st in ast.walk(fn):
                    if isinstance(st, ast.Assign):
                        targets = st.targets[0].elts if isinstance(st.targets[0], ast.Tuple) else st.targets
                        values = st.value.elts if isinstance(st.value, ast.Tuple) else [st.value]
                        for t, v in zip(targets, values):
                            if isinstance(t, ast.Attribute) and isinstance(v, ast.Name):
                                attr_of_kw[t.attr] = v.id
                            elif isinstance(t, ast.Attribute) and isinstance(v, ast.Call) and v.args and \
                                    isinstance(v.args[0], ast.Name):
                                attr_of_kw[t.attr] = v.args[0].id
            if fn.name in ("apply", "_apply"):
                for st in ast.walk(fn):
                    if isinstance(st, ast.Assign) and len(st.targets) == 1:
                        knob = _config_target(st.targets[0])
                        if knob is None:
                            continue
                        attr = _self_attr(st.value)
                        if attr is not None:
                            entry["assigns"].append([knob, {"kw": attr_of_kw.get(attr, attr)}])
                        else:
                            try:
                                entry["assigns"].append([knob, {"const": ast.literal_eval(st.value)}])
                            except ValueError:
                                entry["assigns"].append([knob, {"expr": ast.unparse(st.value)}])
        out[cls.name] = entry
    return out


if __name__ == "__main__":
    src = Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_SRC
    OUT.write_text(json.dumps(table(src), indent=1, sort_keys=True) + "\n")
    print(f"wrote {OUT}")
