"""Extracts the reference's known-answer values into known_answers.json.

The reference (asmelko/paraPhysiCell) cannot be built here: its paraBioFVM,
pugixml and googletest submodules are absent. Its unit tests
(test/test.cpp) still carry known answers as text. This script reads them
from the reference source tree and writes the committed fixture, so the
numbers in the fixture have a scripted provenance:

- host_velocity_solver.simple (test/test.cpp:141-191): the x/y/z velocity
  of cell 1 after one force pass, per dimensionality;
- host_velocity_solver.complex (test/test.cpp:265-320): expected neighbour
  counts;
- host_neighbors_solver.grid (test/test.cpp:333-400): parameter grid;
- cell_container.add_and_remove (test/test.cpp:52-115): volumes and
  velocities after each removal;
- host_interactions_solver.{attack,dead_phagocytosis,phagocytosis,fusion}
  (test/test.cpp:402-560): each case's cells (definition, position, rates,
  dead flag), the number of interaction calls and the asserted flags and
  damage.

Usage: python tests/golden/make_golden.py path/to/reference
(or with the path in the environment variable PPC_REFERENCE_ROOT)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    src = open(os.path.join(ref, "test", "test.cpp")).read()

    # velocities: "if (dims == 3) expected = X; else if (dims == 2) expected = Y; else expected = Z;"
    m = re.search(r"if \(dims == 3\)\s*expected = ([0-9.eE+-]+);\s*else if \(dims == 2\)\s*expected = ([0-9.eE+-]+);"
                  r"\s*else\s*expected = ([0-9.eE+-]+);", src)
    assert m, "known-answer block not found"
    simple = {"3": m.group(1), "2": m.group(2), "1": m.group(3)}

    counts = [int(x) for x in re.findall(r"states\.neighbors\[(?:\d)\]\.size\(\), (\d+)\)", src)]
    assert len(counts) == 3, counts

    m = re.search(r"INSTANTIATE_TEST_SUITE_P\(neis, host_neighbors_solver,\s*testing::Combine\(testing::Values\(([^)]*)\),"
                  r" testing::Values\(([^)]*)\), testing::Values\(([^)]*)\)\)\)", src)
    assert m, "grid parameters not found"
    grid = {
        "dims": [int(x) for x in m.group(1).split(",")],
        "cells_in_one_voxel": [int(x) for x in m.group(2).split(",")],
        "adhesion": [int(x) for x in m.group(3).split(",")],
    }
    m = re.search(r"TEST_P\(host_neighbors_solver, grid\).*?cartesian_mesh mesh\(dims, \{ 0, 0, 0 \}, \{ (\d+), (\d+), (\d+) \},"
                  r" \{ (\d+), (\d+), (\d+) \}\);.*?radius\(\) = (\d+);", src, re.S)
    assert m, "grid mesh not found"
    grid["mesh_max"] = [int(m.group(i)) for i in (1, 2, 3)]
    grid["diffusion_voxel"] = [int(m.group(i)) for i in (4, 5, 6)]
    grid["radius"] = float(m.group(7))

    block = src[src.index("TEST(cell_container, add_and_remove)"): src.index("void update_cell_for_velocity")]
    removes = []
    for part in block.split("cont.remove_agent(")[1:]:
        seg = part.split("}")[0]
        vols = [float(x) for x in re.findall(r"volumes\[\d\], (\d+)\)", seg)]
        vels = [float(x) for x in re.findall(r"velocities\[\d\], (\d+)\)", seg)]
        removes.append({"removed": part.split(")")[0], "volumes": vols, "velocities": vels})

    interactions = {}
    for name in ("attack", "dead_phagocytosis", "phagocytosis", "fusion"):
        start = src.index(f"TEST(host_interactions_solver, {name})")
        nxt = src.find("TEST(", start + 5)
        body = src[start: nxt if nxt > 0 else len(src)]
        m = re.search(r"cartesian_mesh mesh\((\d), \{ ([^}]*) \}, \{ ([^}]*) \}, \{ ([^}]*) \}\);", body)
        case = {"dims": int(m.group(1)), "mesh_min": [int(x) for x in m.group(2).split(",")],
                "mesh_max": [int(x) for x in m.group(3).split(",")], "cells": [], "asserts": []}
        names = []
        for cm in re.finditer(r"auto (c\d) = cont\.create_cell\((?:\*e->cell_definitions\[(\d)\]|e->cell_defaults\(\))\);",
                              body):
            names.append(cm.group(1))
            case["cells"].append({"definition": int(cm.group(2) or 0), "rates": {}, "rate_rows": {}})
        for pm in re.finditer(r"(c\d)->assign_position\(\{ ([^}]*) \}\);", body):
            case["cells"][names.index(pm.group(1))]["position"] = [float(x) for x in pm.group(2).split(",")]
        for rm in re.finditer(r"(c\d)->phenotype\.cell_interactions\.(\w+)\(\)\[(\d)\] = (\d+);", body):
            rows = case["cells"][names.index(rm.group(1))]["rate_rows"]
            rows.setdefault(rm.group(2), {})[rm.group(3)] = float(rm.group(4))
        for rm in re.finditer(r"(c\d)->phenotype\.cell_interactions\.(\w+)\(\) = (\d+);", body):
            case["cells"][names.index(rm.group(1))]["rates"][rm.group(2)] = float(rm.group(3))
        for dm in re.finditer(r"(c\d)->phenotype\.death\.dead\(\) = (\d);", body):
            case["cells"][names.index(dm.group(1))]["dead"] = int(dm.group(2))
        case["calls"] = len(re.findall(r"is\.update_cell_cell_interactions\(\*e\);", body))
        for am in re.finditer(r"ASSERT_(EQ|NE)\((c\d)->flag\(\), cell_state_flag::(\w+)\);", body):
            case["asserts"].append({"cell": names.index(am.group(2)), "field": "flag", "op": am.group(1),
                                    "value": am.group(3)})
        for am in re.finditer(r"ASSERT_(EQ|NE)\((c\d)->state\.damage\(\), (\d+)\);", body):
            case["asserts"].append({"cell": names.index(am.group(2)), "field": "damage", "op": am.group(1),
                                    "value": float(am.group(3))})
        assert case["cells"] and case["asserts"] and case["calls"] >= 1, name
        interactions[name] = case
    m = re.search(r"default_env\(microenvironment& m, index_t cell_defs_count = (\d+)\)", src)
    defs_count = int(m.group(1))

    out = {
        "source": "reference test/test.cpp (asmelko/paraPhysiCell), read as text",
        "host_velocity_solver_simple": {"expected_velocity_cell1": simple,
                                        "lines": "test/test.cpp:141-191"},
        "host_velocity_solver_complex": {"neighbor_counts": counts, "lines": "test/test.cpp:265-320"},
        "host_neighbors_solver_grid": dict(grid, lines="test/test.cpp:333-400"),
        "cell_container_add_and_remove": {"after_removals": removes, "lines": "test/test.cpp:52-115"},
        "host_interactions_solver": {"cases": interactions, "cell_definitions": defs_count,
                                     "lines": "test/test.cpp:36-50,402-560"},
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PPC_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py path/to/reference (or set PPC_REFERENCE_ROOT)")
    main(root)
