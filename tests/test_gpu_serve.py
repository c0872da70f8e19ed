"""Continuous-batching server: results alone and in the mix agree.

Each job's energy when it runs alone (one job on the GPU at a time) and when
it shares the GPU with the rest of a stream must agree to 1e-9 Eh (same SCF
protocol and precision form on both sides; only the order of the FP64 atomic
sums differs).  Admission never exceeds the slot count."""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [False, True])
def test_served_results_match_alone(graphs):
    from hfcode_b200 import serve
    jobs_mix = serve.make_stream(10, rate=0.0, seed=4242, max_alkane=5, max_water=4)
    srv = serve.Server(hbm_budget=32 << 30, max_slots=4, fp32_cutoff=1e-7, graphs=graphs)
    out = srv.serve(jobs_mix, realtime=False)
    assert out["failed"] == 0 and out["not_converged"] == 0, out["errors"]
    assert 1 <= srv.peak_active <= 4
    jobs_alone = serve.make_stream(10, rate=0.0, seed=4242, max_alkane=5, max_water=4)
    solo = serve.Server(hbm_budget=32 << 30, max_slots=1, fp32_cutoff=1e-7)
    serve.serve_sequential(jobs_alone, solo)
    for a, b in zip(sorted(jobs_mix, key=lambda j: j.jid), sorted(jobs_alone, key=lambda j: j.jid)):
        assert a.name == b.name
        assert abs(a.energy - b.energy) < 1e-9, (a.name, a.energy, b.energy)


@pytest.mark.gpu
def test_admission_waits_for_memory():
    from hfcode_b200 import serve
    jobs = serve.make_stream(6, rate=0.0, seed=7, max_alkane=4, max_water=3)
    srv = serve.Server(hbm_budget=1, max_slots=8)  # budget below any footprint -> one job at a time?
    for j in jobs:
        srv.prepare(j)
    # a budget that fits exactly the two largest footprints admits at most two jobs at once
    fps = sorted(j.footprint for j in jobs)
    srv = serve.Server(hbm_budget=fps[-1] + fps[-2], max_slots=8)
    out = srv.serve(jobs, realtime=False)
    assert out["failed"] == 0, out["errors"]
    assert srv.peak_in_use <= fps[-1] + fps[-2]
    assert srv.peak_active <= 6
