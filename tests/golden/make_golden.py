"""Generates the golden fixtures under tests/golden/ from the reference tree.

Run where a reference checkout exists, with REFERENCE_ROOT set to its root
(required; the script exits otherwise); the GPU box never runs this script.

Outputs:
  square8k_mesh.npz          positions (float32, V x 3) and 0-based faces (int32, F x 3)
                             of resources/models/square8K.obj, degenerate faces dropped
                             as src/Utils/mesh_reader.cpp:170-177 does.
  example2_energy_frame30.json  the frame-30 VBD energy logs pasted in
                             documents/example2_async_convergence.py:78-84
                             (sync: 101 values, async: 102 values).
  heft2002.json              the 10-task / 3-processor DAG and computation matrix of
                             examples/example1_heft2002.cpp:43-72 with the makespan and
                             speedups quoted in README.md:25-31.
  square40k_faces.json       SHA-256 of the 0-based int32 face array of
                             resources/models/square40K.obj plus its vertex bounds.
"""
import ast
import hashlib
import json
import os
import re
import sys

import numpy as np

REF = os.environ.get("REFERENCE_ROOT")
HERE = os.path.dirname(os.path.abspath(__file__))


def read_obj(path):
    pos, faces = [], []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                pos.append([float(t[1]), float(t[2]), float(t[3])])
            elif t[0] == "f":
                ids = [int(tok.split("/")[0]) - 1 for tok in t[1:4]]
                if len(set(ids)) == 3:
                    faces.append(ids)
    return np.asarray(pos, dtype=np.float32), np.asarray(faces, dtype=np.int32)


def energy_lists():
    src = open(os.path.join(REF, "documents/example2_async_convergence.py")).read()
    out = {}
    for name in ("list_sync", "list_async"):
        m = re.search(name + r"\s*=\s*(\[.*?\])", src, re.S)
        out[name] = [float(v) for v in ast.literal_eval(m.group(1))]
    return out


def heft_case():
    src = open(os.path.join(REF, "examples/example1_heft2002.cpp")).read()
    edges = [[int(a), int(b), float(w)] for a, b, w in
             re.findall(r"set_connect\(tid_(\d+),\s*tid_(\d+),\s*([\d.]+)f\)", src)]
    comp = {}
    for t, row in re.findall(r"computation_matrix\[tid_(\d+)\]\s*=\s*\{([^}]*)\}", src):
        comp[int(t)] = [float(v) for v in row.split(",")]
    readme = open(os.path.join(REF, "README.md")).read()
    m = re.search(r"should be (\d+)", readme)
    makespan = float(m.group(1)) if m else None
    speedups = [float(v) for v in re.findall(r"([0-9]+\.[0-9]+)%", readme)[:3]]
    return {"tasks": sorted(comp), "edges": edges,
            "computation": [comp[t] for t in sorted(comp)],
            "communication_speed": [[0, 1, 1], [1, 0, 1], [1, 1, 0]],
            "makespan": makespan, "speedups_percent": speedups}


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("set REFERENCE_ROOT to the root of a libAtsSim checkout")
    pos, faces = read_obj(os.path.join(REF, "resources/models/square8K.obj"))
    np.savez_compressed(os.path.join(HERE, "square8k_mesh.npz"), positions=pos, faces=faces)
    json.dump(energy_lists(), open(os.path.join(HERE, "example2_energy_frame30.json"), "w"), indent=1)
    json.dump(heft_case(), open(os.path.join(HERE, "heft2002.json"), "w"), indent=1)
    p40, f40 = read_obj(os.path.join(REF, "resources/models/square40K.obj"))
    json.dump({"num_verts": int(p40.shape[0]), "num_faces": int(f40.shape[0]),
               "faces_sha256": hashlib.sha256(np.ascontiguousarray(f40).tobytes()).hexdigest(),
               "bounds_min": p40.min(0).tolist(), "bounds_max": p40.max(0).tolist()},
              open(os.path.join(HERE, "square40k_faces.json"), "w"), indent=1)
    print("fixtures written to", HERE, file=sys.stderr)


if __name__ == "__main__":
    main()
