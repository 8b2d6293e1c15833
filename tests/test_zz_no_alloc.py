"""ats_energy_noalloc: the energy entry point for callers that cannot allocate.

Programs whose device memory comes from their own allocator, or whose frame loop
cannot pay for cudaMalloc, hand in their own device arrays; the call keeps its
partial sums in the library's static device scratch. Its result must equal the
handle-based ats_energy on the same state, on consecutive calls (the scratch keeps
the previous call's contents), and oversize inputs are refused before any launch.
This file is collected last so that a stop-at-first-failure run has already run
every other test.
"""
import numpy as np
import pytest

from libatssim_b200 import configs

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_noalloc_energy_matches_handle_energy_twice(ats):
    import torch

    insts, prm = configs.c0()
    inst = insts[0]
    rng = np.random.RandomState(11)
    x0 = (inst.positions + 1e-3 * rng.standard_normal(inst.positions.shape)).astype(np.float32)
    v0 = (0.2 * rng.standard_normal(inst.positions.shape)).astype(np.float32)
    cloth = ats.Cloth(insts, **prm)
    cloth.set_state(x0, v0)
    cloth.predict()
    cloth.vbd_iterations(2)
    xm = cloth.positions()
    ref = cloth.energy()

    topo = ats.Topology(inst)
    edges, bending = topo.edges()
    rest, q = topo.rest()
    t = {k: _dev(torch, a) for k, a in dict(x=xm, xs=x0, v=v0, m=inst.mass, f=inst.fixed, e=edges, L=rest,
                                            b=bending, q=q).items()}
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    for call in range(2):
        out.fill_(float("nan"))
        ats.energy_noalloc(t["x"].data_ptr(), t["xs"].data_ptr(), t["v"].data_ptr(), t["m"].data_ptr(),
                           t["f"].data_ptr(), inst.num_verts, t["e"].data_ptr(), t["L"].data_ptr(), len(edges),
                           t["b"].data_ptr(), t["q"].data_ptr(), len(bending), inst.k_stretch, inst.k_bend,
                           (0.0, -9.8, 0.0), prm["implicit_dt"], out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-12 * np.abs(ref).sum()), (call, got, ref)


def test_noalloc_energy_rejects_oversize_inputs(ats):
    too_many = 8388608 + 1
    dummy = 1  # never dereferenced: the size check comes before any launch
    with pytest.raises(ats.AtsError) as e:
        ats.energy_noalloc(dummy, dummy, dummy, dummy, dummy, too_many, dummy, dummy, 0, dummy, dummy, 0,
                           1.0, 1.0, (0.0, 0.0, 0.0), 0.01, dummy)
    assert e.value.status == ats.ATS_ERR_INVALID
    assert b"8388608" in ats.lib().ats_last_error()
