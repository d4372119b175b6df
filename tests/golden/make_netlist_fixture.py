"""Collect the reference's netlist input files (testbin/mainTests/**/
netlist_surfaces.dat and .xml) into one fixture, so the netlist readers and
the circuits they describe can be tested without a reference checkout.  Run
once where a checkout exists:

    python tests/golden/make_netlist_fixture.py /path/to/reference/checkout

Writes netlist_inputs.json: {path relative to testbin/mainTests: file text},
one entry per distinct file text; netlist_periodic_tables.json: the
(time, value) tables ("<source>.dat" beside the input) that the inputs'
prescribedPeriodicFlow / prescribedPeriodicPressure controls name; and
netlist_closed_loops.json: per case directory with a
netlist_closed_loop_downstream.xml, that file's text, the netlist_surfaces
file beside it, its solver.inp and that file's "List of Netlist LPN
Surfaces".
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    base = os.path.join(ref, "testbin", "mainTests")
    seen, out, tables = set(), {}, {}
    for root, _, files in sorted(os.walk(base)):
        for name in sorted(files):
            if name not in ("netlist_surfaces.dat", "netlist_surfaces.xml"):
                continue
            path = os.path.join(root, name)
            with open(path) as f:
                text = f.read()
            for src in re.findall(r"prescribedPeriodic(?:Flow|Pressure)\s*(?:</type>\s*<source>)?\s*(\w+)", text):
                tpath = os.path.join(root, src + ".dat")
                if os.path.exists(tpath):
                    with open(tpath) as f:
                        tables[os.path.relpath(tpath, base)] = f.read()
            if text in seen:
                continue
            seen.add(text)
            out[os.path.relpath(path, base)] = text
    loops = {}
    for root, _, files in sorted(os.walk(base)):
        if "netlist_closed_loop_downstream.xml" not in files or "solver.inp" not in files:
            continue
        surf = [n for n in ("netlist_surfaces.xml", "netlist_surfaces.dat") if n in files]
        with open(os.path.join(root, "solver.inp")) as f:
            lists = [ln.split(":", 1)[1].split("#")[0].split() for ln in f
                     if ln.split(":", 1)[0].strip().lower() == "list of netlist lpn surfaces"]
        if not surf:
            continue
        with open(os.path.join(root, surf[0])) as f:
            surfaces = f.read()
        with open(os.path.join(root, "netlist_closed_loop_downstream.xml")) as f:
            downstream = f.read()
        with open(os.path.join(root, "solver.inp")) as f:
            loops[os.path.relpath(root, base)] = {
                "downstream": downstream, "surfaces_file": surf[0], "surfaces": surfaces,
                "srfids": [int(t) for t in lists[0]] if lists else [], "solver_inp": f.read()}
    with open(os.path.join(HERE, "netlist_closed_loops.json"), "w") as f:
        json.dump(loops, f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "netlist_inputs.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "netlist_periodic_tables.json"), "w") as f:
        json.dump(tables, f, indent=1, sort_keys=True)
    print(len(out), "files,", len(tables), "periodic tables,", len(loops), "closed-loop cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
