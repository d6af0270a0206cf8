"""Configuration files of the reference examples' shapes, for timing the
configuration runner (``python -m cellweave_b200 DIR/NAME.toml``).

Writes into DIR the RAS/ERK network of golden.json as ``ras-erk.toml`` and
three scenarios with the sizes and rates of the reference's spheroid, cord
and spheroid-3d examples (examples/spheroid.toml, cord.toml,
spheroid-3d.toml; the 3D one with the RAS/ERK network in place of its soft
variant, which golden.json does not hold):

    python tests/golden/make_scenarios.py DIR
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def network_toml(spec):
    lines = []
    for node in spec["nodes"]:
        lines += ["[[nodes]]", f'name = "{node["name"]}"', f'initial = {node["initial"]}', "terms = ["]
        for t in node["terms"]:
            kv = ", ".join(f'{k} = "{v}"' if isinstance(v, str) else f"{k} = {v}" for k, v in t.items())
            lines.append(f"  {{ {kv} }},")
        lines.append("]")
    lines.append("[roles]")
    lines += [f'{k} = "{v}"' for k, v in spec["roles"].items()]
    lines.append("[mechanics]")
    lines += [f"{k} = {v}" for k, v in spec["mechanics"].items()]
    return "\n".join(lines) + "\n"


SCENARIOS = {
    "spheroid": ("width = 800\nheight = 800\nmcs = 626\ntemperature = 10.0\nsnapshot_interval = 25\n"
                 'output_dir = "out-spheroid"\noxygen_uptake = 0.00002\nnetwork = "ras-erk.toml"\n'
                 '[oxygen_source]\nkind = "bath"\n'),
    "cord": ("width = 300\nheight = 300\nmcs = 3000\ntemperature = 10.0\nsnapshot_interval = 50\n"
             'output_dir = "out-cord"\noxygen_uptake = 0.00002\nnetwork = "ras-erk.toml"\n'
             '[oxygen_source]\nkind = "vessel"\nradius = 6\n'),
    "spheroid3d": ("width = 320\nheight = 320\ndepth = 320\nmax_cells = 200000\nmcs = 1500\ntemperature = 10.0\n"
                   'snapshot_interval = 20\noutput_dir = "out-spheroid3d"\noxygen_uptake = 0.0001024\n'
                   'debris_loss = 0.024\nsweeps_per_step = 4\ncontact_order = 3\nnetwork = "ras-erk.toml"\n'
                   "[cycle]\nmedian = 20.0\nspread = 0.3\n[still_medium]\ndiffusion = 0.606\n"),
}


def main(out):
    os.makedirs(out, exist_ok=True)
    spec = json.load(open(os.path.join(HERE, "golden.json")))["networks"]["ras-erk"]
    with open(os.path.join(out, "ras-erk.toml"), "w") as fh:
        fh.write(network_toml(spec))
    for name, text in SCENARIOS.items():
        with open(os.path.join(out, f"{name}.toml"), "w") as fh:
            fh.write(text)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else ".")
