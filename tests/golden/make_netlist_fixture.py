"""Collect the reference's netlist input files (testbin/mainTests/**/
netlist_surfaces.dat and .xml) into one fixture, so the netlist readers and
the circuits they describe can be tested without a reference checkout.  Run
once where a checkout exists:

    python tests/golden/make_netlist_fixture.py /path/to/reference/checkout

Writes netlist_inputs.json: {path relative to testbin/mainTests: file text},
one entry per distinct file text.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    base = os.path.join(ref, "testbin", "mainTests")
    seen, out = set(), {}
    for root, _, files in sorted(os.walk(base)):
        for name in sorted(files):
            if name not in ("netlist_surfaces.dat", "netlist_surfaces.xml"):
                continue
            path = os.path.join(root, name)
            with open(path) as f:
                text = f.read()
            if text in seen:
                continue
            seen.add(text)
            out[os.path.relpath(path, base)] = text
    with open(os.path.join(HERE, "netlist_inputs.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(len(out), "files")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
