"""Continuous-batching server: results alone and in the mix agree, and
admission by device-memory footprint holds jobs back.

Each job's energy when it runs alone (one job on the GPU at a time) and when
it shares the GPU with the rest of a stream must agree to 1e-9 Eh (same SCF
protocol and precision form on both sides; only the order of the FP64 atomic
sums differs).  With the device step every job's state (density, Fock,
DIIS history, screening tables) stays on the GPU."""
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("step,graphs", [("device", False), ("host", False), ("host", True)])
def test_served_results_match_alone(step, graphs):
    from hfcode_b200 import serve
    jobs_mix = serve.make_stream(10, rate=0.0, seed=4242, max_alkane=5, max_water=4)
    srv = serve.Server(hbm_budget=32 << 30, max_slots=4, fp32_cutoff=1e-7, graphs=graphs, step=step)
    out = srv.serve(jobs_mix, realtime=False)
    assert out["failed"] == 0 and out["not_converged"] == 0, out["errors"]
    assert srv.peak_active >= 2   # the jobs did share the GPU
    assert srv.peak_active <= 4   # never more than the slots
    jobs_alone = serve.make_stream(10, rate=0.0, seed=4242, max_alkane=5, max_water=4)
    solo = serve.Server(hbm_budget=32 << 30, max_slots=1, fp32_cutoff=1e-7, step=step)
    serve.serve_sequential(jobs_alone, solo)
    for a, b in zip(sorted(jobs_mix, key=lambda j: j.jid), sorted(jobs_alone, key=lambda j: j.jid)):
        assert a.name == b.name
        assert abs(a.energy - b.energy) < 1e-9, (a.name, a.energy, b.energy)


@pytest.mark.gpu
def test_admission_waits_for_memory():
    """Three copies of one job against a budget of one job's estimated
    footprint: the second is admitted only after the first has released its
    memory, and so on (FIFO); against three footprints they overlap."""
    from hfcode_b200 import serve
    base = serve.make_stream(1, rate=0.0, seed=7, max_alkane=4, max_water=3)[0]
    probe = serve.Server(hbm_budget=1 << 40, max_slots=8)
    probe.prepare(base)
    fp = base.footprint

    def jobs():
        return [serve.Job(i, base.name, base.mol, 0.0) for i in range(3)]

    tight = serve.Server(hbm_budget=fp, max_slots=8)
    js = jobs()
    out = tight.serve(js, realtime=False)
    assert out["failed"] == 0, out["errors"]
    assert tight.peak_active == 1
    order = sorted(js, key=lambda j: j.admitted)
    for prev, nxt in zip(order, order[1:]):
        assert nxt.admitted >= prev.finished - 1e-6, (prev.finished, nxt.admitted)
    assert tight.peak_in_use <= fp
    roomy = serve.Server(hbm_budget=3 * fp, max_slots=8)
    out = roomy.serve(jobs(), realtime=False)
    assert out["failed"] == 0, out["errors"]
    assert roomy.peak_active >= 2


@pytest.mark.gpu
def test_job_larger_than_budget_is_refused():
    from hfcode_b200 import serve
    js = serve.make_stream(2, rate=0.0, seed=11, max_alkane=3, max_water=2)
    srv = serve.Server(hbm_budget=1 << 20, max_slots=2)  # 1 MiB: below any job
    out = srv.serve(js, realtime=False)
    assert out["failed"] == 2
    assert all("exceeds" in j.error for j in js)
