"""Regenerate ``tests/golden/golden.json`` from the reference's own files.

Give it the reference's checkout (read only), as an argument or in the
environment variable CELLWEAVE_REFERENCE:

    python tests/golden/make_golden.py PATH_TO_CELLWEAVE_CHECKOUT

It reads, and records with their source locations:
  * the network files under examples/networks/ (parsed with tomllib, with
    ``extends`` chains merged as NetworkSpec::merge_onto does,
    crates/core/src/network.rs:269-283);
  * the RAS/ERK golden table of crates/engine/src/network.rs:869-879;
  * the Hill-free term-slope cases of network.rs:1071-1155 are restated in the
    tests themselves, since they are formulas, not captured numbers.
The JSON is committed so the tests never read the reference at run time.
"""
import json
import os
import re
import sys
import tomllib

REF = None  # the reference checkout, set by main()
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def load_chain(path, seen=()):
    here = os.path.realpath(path)
    if here in seen:
        raise ValueError(f"a network extends itself round a loop: {path}")
    with open(path, "rb") as fh:
        spec = tomllib.load(fh)
    parent = spec.get("extends")
    if parent is None:
        spec.pop("extends", None)
        return spec
    base = load_chain(os.path.join(os.path.dirname(path), parent), seen + (here,))
    nodes = list(base.get("nodes", []))
    for node in spec.get("nodes", []):
        for k, existing in enumerate(nodes):
            if existing["name"] == node["name"]:
                nodes[k] = node
                break
        else:
            nodes.append(node)
    return {"nodes": nodes, "roles": spec.get("roles") or base.get("roles"),
            "mechanics": spec.get("mechanics") or base.get("mechanics")}


def rk4_table():
    src = open(os.path.join(REF, "crates/engine/src/network.rs")).read().splitlines()
    rows = []
    for lineno in range(869, 880):  # network.rs:869-879, 1-based
        line = src[lineno - 1]
        m = re.match(r"\s*\((\d+),\s*([\d.]+),\s*([\d.]+),\s*\[([^\]]*)\]\),", line)
        if m:
            vals = [float(v) for v in m.group(4).split(",")]
            rows.append({"steps": int(m.group(1)), "o2": float(m.group(2)), "egf": float(m.group(3)),
                         "expected": vals, "source": f"crates/engine/src/network.rs:{lineno}"})
    assert len(rows) == 9, rows
    return rows


def main(argv=None):
    global REF
    argv = sys.argv[1:] if argv is None else argv
    REF = argv[0] if argv else os.environ.get("CELLWEAVE_REFERENCE")
    if not REF or not os.path.isdir(os.path.join(REF, "crates", "engine")):
        sys.exit("usage: make_golden.py PATH_TO_CELLWEAVE_CHECKOUT (or set CELLWEAVE_REFERENCE)")
    nets = {}
    ndir = os.path.join(REF, "examples/networks")
    for name in sorted(os.listdir(ndir)):
        if name.endswith(".toml"):
            nets[name[:-5]] = load_chain(os.path.join(ndir, name))
    golden = {
        "networks": nets,
        "networks_source": "examples/networks/*.toml",
        "ras_erk_rk4": rk4_table(),
        "ras_erk_reference_volume": 200,
        "mechanics": {"free_target_after_40": 299, "capped_target_after_40": 240, "cap": 1.2, "lambda": 50.0,
                      "source": "crates/engine/src/network.rs:893-902, 951-965"},
        "reach": {"volume_order3": [26, 9.0], "volume_order2": [18, 5.0], "plane_order2": [8, 3.0],
                  "plane_order3": [12, 5.0], "source": "crates/engine/src/cpm.rs:1868-1883"},
    }
    with open(OUT, "w") as fh:
        json.dump(golden, fh, indent=1, sort_keys=True)
    print(OUT)


if __name__ == "__main__":
    main()
