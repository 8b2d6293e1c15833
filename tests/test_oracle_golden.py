"""Pins the CPU oracle to libAtsSim's own published output.

documents/example2_async_convergence.py:78-80 lists the energy of frame 30 of the
synchronous VBD run of examples/example2_async_iter.cpp (square8K.obj, 100
iterations, k = 1e4, k_b = 5e-3 x 0.5, 0.01 kg per vertex, h = 1/60) before the
first iteration and after each of the 100. The log keeps inertia + stretch only
(the bending term is computed and discarded, example2_async_iter.cpp:832-846).
The values are printed with 6 significant digits.
"""
import json
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_frame30_energy_trajectory(oracle):
    m = np.load(os.path.join(GOLD, "square8k_mesh.npz"))
    pos, faces = m["positions"], m["faces"]
    mass = np.full(len(pos), 0.01, np.float32)
    s = oracle.Scene(pos, faces, mass, oracle.reference_pins(pos), k_stretch=1e4, k_bend=2.5e-3,
                     iterations=100, threads=1)
    s.run(30)
    e, _ = s.frame(log_energy=True, with_bending=False)
    gold = np.array(json.load(open(os.path.join(GOLD, "example2_energy_frame30.json")))["list_sync"])
    assert e.shape == gold.shape == (101,)
    # 6 significant digits printed: half an ulp of the print is 5e-4 at 4xx.x
    assert np.max(np.abs(e - gold)) < 1e-3
    assert np.max(np.abs(e - gold) / gold) < 3e-6
    # monotone descent, like the published curve
    assert (np.diff(e) < 0).all()


def test_heft_fixture_values():
    d = json.load(open(os.path.join(GOLD, "heft2002.json")))
    assert d["makespan"] == 91.0
    assert d["speedups_percent"] == [39.56, 42.86, 57.14]
    assert len(d["edges"]) == 15 and len(d["computation"]) == 10
