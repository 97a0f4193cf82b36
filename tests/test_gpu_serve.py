"""Serving (hf_server_*): continuous batching. Each scenario's result must be
bit-identical alone and in the mix, whatever was admitted alongside it and
whenever; admission respects the HBM budget."""
import numpy as np
import pytest

from tests.gpu_util import exact_fraction

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import serve, workloads
    return serve, workloads


def scn(workloads, n, seed, t_end, peak=60.0):
    s = workloads.valley(n=n, dx=5.0, seed=seed, peak=peak, t_end=t_end)
    s.max_dt = 5.0
    return s


def alone(workloads, s):
    with workloads.simulation_for(s) as sim:
        sim.run_until(s.t_end)
        return sim.states(), sim.steps()


def test_results_same_alone_and_in_the_mix(gpu):
    serve, workloads = gpu
    a, b, c, d = (scn(workloads, 40, 1, 50.0), scn(workloads, 70, 2, 30.0),
                  scn(workloads, 17, 3, 40.0), scn(workloads, 96, 4, 25.0))
    results = {}
    with serve.Server(hbm_budget_bytes=1 << 30, max_slots=8) as srv:
        ids = {srv.try_admit(a): "a", srv.try_admit(b): "b"}
        srv.advance(5)                      # a and b run alone for a while
        ids[srv.try_admit(c)] = "c"         # c joins mid-flight
        while len(results) < 4:
            srv.advance(3)
            for slot in srv.finished():
                results[ids[slot]] = srv.collect(slot)
                if "d" not in ids.values():  # d takes a freed slot
                    ids[srv.try_admit(d)] = "d"
    for name, s in zip("abcd", (a, b, c, d)):
        r = results[name]
        ref, steps = alone(workloads, s)
        assert r["status"] == 0 and r["t"] == s.t_end and r["steps"] == steps
        assert exact_fraction(r["state"], ref) == 1.0, name


def test_admission_respects_budget(gpu):
    serve, workloads = gpu
    s1, s2, s3 = scn(workloads, 64, 5, 10.0), scn(workloads, 64, 6, 10.0), scn(workloads, 64, 7, 10.0)
    per = 8 * 64 * 64 * 8
    with serve.Server(hbm_budget_bytes=2 * per + 100, max_slots=8) as srv:
        assert srv.try_admit(s1) is not None and srv.try_admit(s2) is not None
        assert srv.try_admit(s3) is None            # over budget
        used, occ = srv.usage()
        assert used == 2 * per and occ == 2
        while not srv.finished():
            srv.advance(8)
        srv.collect(srv.finished()[0])
        assert srv.try_admit(s3) is not None        # fits once memory is freed


def test_arrival_stream(gpu):
    serve, workloads = gpu
    reqs = serve.request_stream(12, rate=200.0, seed=3, sides=(16, 32, 48), horizon_min=5.0,
                                horizon_max=20.0, max_dt=2.0)
    out = serve.serve_stream(reqs, hbm_budget_bytes=1 << 28, chunk=4, keep_state=True)
    assert out["n"] == 12 and out["failed"] == 0
    assert 0 < out["latency_p50"] <= out["latency_p99"]
    for r in reqs[:3]:
        s = r.make()
        ref, steps = alone(workloads, s)
        assert r.result["steps"] == steps
        assert exact_fraction(r.result["state"], ref) == 1.0


def test_solo_scenarios_same_alone_and_in_the_mix(gpu):
    """Scenarios of at least 512 tiles of 32 x 32 (736 x 736 and up) run their
    stages as their own launches beside the batched ones; the graphs are
    captured again whenever such a scenario is admitted or collected. Large
    and small scenarios joining and leaving mid-flight: every result equals
    its lone solve bit for bit."""
    serve, workloads = gpu
    big1, big2 = scn(workloads, 736, 11, 30.0, peak=200.0), scn(workloads, 768, 12, 20.0, peak=200.0)
    small1, small2 = scn(workloads, 40, 13, 50.0), scn(workloads, 90, 14, 25.0)
    results = {}
    with serve.Server(hbm_budget_bytes=1 << 32, max_slots=8) as srv:
        ids = {srv.try_admit(big1): "big1", srv.try_admit(small1): "small1"}
        srv.advance(4)
        ids[srv.try_admit(big2)] = "big2"     # a second large scenario joins mid-flight
        while len(results) < 4:
            srv.advance(3)
            for slot in srv.finished():
                results[ids[slot]] = srv.collect(slot)
                if "small2" not in ids.values():
                    ids[srv.try_admit(small2)] = "small2"
    for name, s in (("big1", big1), ("big2", big2), ("small1", small1), ("small2", small2)):
        r = results[name]
        ref, steps = alone(workloads, s)
        assert r["status"] == 0 and r["t"] == s.t_end and r["steps"] == steps, name
        assert exact_fraction(r["state"], ref) == 1.0, name
