"""The Launcher API (include/ats_launcher.hpp) through C++ driver programs.

HEFT known answer of examples/example1_heft2002.cpp / README.md:25-31 (makespan 91,
speedups 39.56 / 42.86 / 57.14 %), and the VBD task graph of
examples/example2_async_iter.cpp:1305-1384 launched through the scheduler with a CUDA
implementation, which must give exactly the positions of ats_frame.
"""
import json
import os
import subprocess

import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def programs(ats):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "cpp"))
    from build_programs import build_programs
    return build_programs()


def heft_input(d):
    lines = [f"3 {len(d['computation'])} {len(d['edges'])}"]
    lines += [" ".join(str(c) for c in row) for row in d["computation"]]
    lines += [f"{a} {b} {w}" for a, b, w in d["edges"]]
    return "\n".join(lines) + "\n"


def test_heft_2002_known_answer(programs):
    d = json.load(open(os.path.join(GOLD, "heft2002.json")))
    r = subprocess.run([programs["heft_case"]], input=heft_input(d), capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    assert out["makespan"] == d["makespan"] == 91.0
    assert out["speedups_percent"] == d["speedups_percent"]
    # 10 tasks + added root and terminal, all launched in schedule order
    assert out["launched"] == 12
    # every task starts after its predecessors finish
    sched = {t: (p, s, e) for t, p, s, e in out["schedule"]}
    for a, b, _ in d["edges"]:
        assert sched[b][1] >= sched[a][2] - 1e-6


def test_heft_rejects_cycles(programs):
    d = json.load(open(os.path.join(GOLD, "heft2002.json")))
    d = dict(d, edges=d["edges"] + [[10, 1, 1.0]])
    r = subprocess.run([programs["heft_case"]], input=heft_input(d), capture_output=True, text=True, timeout=60)
    assert r.returncode == 3
    assert "cycle" in r.stderr


def _vbd_dag(programs, mode, n=24, iters=6, frames=3):
    r = subprocess.run([programs["vbd_dag"], str(n), str(iters), str(frames), mode], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    return json.loads(lines[-1]), lines


@pytest.mark.gpu
def test_vbd_task_graph_single_device_modes(programs):
    """Every task on the B200 (the CUDA solver through the C ABI) gives exactly the
    frames of ats_frame; every task on the host (the oracle's per-step entry points)
    gives exactly the oracle's frames."""
    gpu, _ = _vbd_dag(programs, "gpu")
    assert gpu["status"] == 0 and gpu["rel_l2_vs_gpu_alone"] == 0.0
    assert gpu["max_displacement"] > 1e-3
    cpu, _ = _vbd_dag(programs, "cpu")
    assert cpu["status"] == 0 and cpu["rel_l2_vs_oracle_alone"] == 0.0
    # 2 cloths x (predict + 6 x 4 colours + last node + update) + root + terminal
    assert gpu["tasks"] == 2 * (1 + 6 * 4 + 2) + 2


@pytest.mark.gpu
def test_vbd_task_graph_split_between_cpu_and_b200(programs):
    """The HEFT schedule puts colour sweeps on both the host (oracle) and the B200
    (CUDA). Hetero runs both devices at once, ordered by CUDA events and host
    counters; FakeHetero runs the same schedule one task at a time. Their positions
    are bit-identical, and close to either device alone."""
    fake, _ = _vbd_dag(programs, "fake")
    het, _ = _vbd_dag(programs, "hetero")
    for out in (fake, het):
        assert out["status"] == 0
        assert out["sweeps_on_cpu"] > 0 and out["sweeps_on_gpu"] > 0
        assert out["cross_device_waits"] > 0
        assert out["rel_l2_vs_gpu_alone"] < 1e-4 and out["rel_l2_vs_oracle_alone"] < 1e-4
    assert het["digest"] == fake["digest"]
    # the Hetero launch measured every launch event (GPU by CUDA events) for the refit
    assert het["measured_events"] == het["launch_events"]


@pytest.mark.gpu
def test_vbd_task_graph_profiled_costs(programs):
    out, lines = _vbd_dag(programs, "profiled")
    prof = json.loads(lines[0])["profiled"]
    # one measured row per distinct (function id, colour) on both devices
    assert len(prof) == 3 + 4 and all(c >= 0 for row in prof for c in row[2:])
    sweeps = [row for row in prof if row[0] == "id_vbd_all_in_one"]
    assert all(row[2] > 0 and row[3] > 0 for row in sweeps)
    assert out["status"] == 0 and out["rel_l2_vs_gpu_alone"] < 1e-4


@pytest.mark.gpu
def test_async_two_copy_iteration_through_scheduler(programs):
    """example2's asynchronous iteration driven by the scheduler: fork
    (id_xpbd_copy_to_cpu_gpu), K iterations on each device's own copy, merge
    (id_xpbd_read_and_solve_conflict, ats_async_merge), R rounds per frame. The chains
    of a round run concurrently in Hetero and one at a time in FakeHetero, with
    bit-identical results; the merged trajectory stays close to plain VBD with the
    same total iterations."""
    rounds, k, frames = 3, 4, 3
    outs = {}
    for mode in ("fake", "hetero"):
        r = subprocess.run([programs["async_dag"], "24", str(rounds), str(k), str(frames), mode], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs[mode] = json.loads(r.stdout.strip().splitlines()[-1])
    for out in outs.values():
        assert out["status"] == 0
        assert out["merges"] == rounds * frames
        assert out["sweeps_on_cpu"] > 0 and out["sweeps_on_gpu"] > 0 and out["cross_device_waits"] > 0
        assert out["max_displacement"] > 1e-3
        assert out["rel_l2_vs_plain"] < 5e-2
    assert outs["hetero"]["digest"] == outs["fake"]["digest"]


def test_launch_modes_on_host_devices(programs):
    # the HEFT 2002 DAG on two host-only "devices" (the first two cost columns); every
    # mode runs each task it owns once, after its predecessors, on the mode's device
    d = json.load(open(os.path.join(GOLD, "heft2002.json")))
    text = "\n".join([f"2 {len(d['computation'])} {len(d['edges'])}"] +
                     [" ".join(str(c) for c in row[:2]) for row in d["computation"]] +
                     [f"{a} {b} {w}" for a, b, w in d["edges"]]) + "\n"
    r = subprocess.run([programs["launch_modes"]], input=text, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    proc = {t + 1: p for t, p in enumerate(out["proc"])}
    assert set(proc.values()) == {0, 1}  # the schedule uses both devices
    n = len(d["computation"])
    for mode, m in out["modes"].items():
        assert m["status"] == 0, mode
        runs = [(t, dev) for t, dev in m["log"] if dev != 2]
        tasks = [t for t, _ in runs]
        assert len(tasks) == len(set(tasks)), mode
        own = {"partial_cpu": {t for t in proc if proc[t] == 0}, "partial_gpu": {t for t in proc if proc[t] == 1}}
        assert set(tasks) == own.get(mode, set(range(1, n + 1))), mode
        where = dict(runs)
        expect_dev = {"cpu": lambda t: 0, "sequence_hetero": lambda t: 0, "gpu": lambda t: 1,
                      "partial_cpu": lambda t: 0, "partial_gpu": lambda t: 1}.get(mode, lambda t: proc[t])
        assert all(dev == expect_dev(t) for t, dev in runs), mode
        pos = {t: i for i, (t, _) in enumerate(m["log"]) if t}
        for a, b, _ in d["edges"]:
            if a in pos and b in pos:
                assert pos[a] < pos[b], (mode, a, b)
                # a host task waits for a device predecessor: a drain lies between them
                if mode in ("hetero", "fake_hetero") and where[a] == 1 and where[b] == 0:
                    assert any(t == 0 and dev == 2 for t, dev in m["log"][pos[a] + 1:pos[b]]), (mode, a, b)
    # work left on device 1 is drained once at the end of a launch
    assert out["modes"]["gpu"]["drains"] == 1 and out["modes"]["cpu"]["drains"] == 0


@pytest.mark.parametrize("mode", ["sequence", "fake", "hetero"])
def test_example2_scheduler_sequence(programs, mode):
    """examples/example2_async_iter.cpp:1305-1460 written against ats_launcher.hpp: the
    reference's ids (id_additional_root = 0, predict 62, vbd_all_in_one 54, last node
    45, update 66 in launcher.h:14-221), every task run once, each cluster's iterations
    in order, predict first and the velocity update last."""
    iters, clusters = 3, 4
    r = subprocess.run([programs["example2_sequence"], str(iters), str(clusters), mode], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert "Task of each processor" in r.stdout  # print_schedule_to_graph_xpbd
    out = json.loads(lines[-1])
    assert out["status"] == 0
    assert out["ids"] == {"predict": 62, "vbd": 54, "last": 45, "update": 66, "root": 0}
    runs = out["runs"]
    assert len(runs) == 1 + iters * clusters + 2
    assert runs[0][0] == 62 and runs[-1][0] == 66 and runs[-2][0] == 45
    seen = {}
    for i, (f, it, c, dev) in enumerate(runs):
        if f == 54:
            seen[(it, c)] = i
            if it > 0:
                assert seen[(it - 1, c)] < i
    assert len(seen) == iters * clusters
    devices = {dev for f, it, c, dev in runs}
    assert devices == ({0} if mode == "sequence" else {0, 1})


def test_hetero_launch_wait_is_bounded(programs):
    """A device task that takes longer than the launch's wait limit ends the Hetero
    launch with LaunchWaitTimeout (status 1) and a message, instead of blocking: the
    failure is made on the host (a slow implementation), not on a GPU."""
    r = subprocess.run([programs["example2_sequence"], "3", "4", "timeout"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["status"] == 1
    assert "in time" in r.stderr or "too long" in r.stderr
