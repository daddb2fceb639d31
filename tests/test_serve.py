"""Serving-loop scheduling (admission under an HBM budget, slots, retirement, latency) on the host,
with the device solve replaced by a stand-in that converges after a set number of outer iterations."""
import numpy as np

from babelsim_b200 import serve


class FakeMesh:
    def __init__(self, n_cells, n_faces):
        self.n_cells = n_cells
        self.owner = np.zeros(n_faces, dtype=np.int32)

    def close(self):
        pass


class FakeReport:
    def __init__(self, it, done):
        self.iterations = it
        self.converged = done
        self.status = 0 if done else 1


class FakeSim:
    def __init__(self, needed, trace, rid):
        self.needed, self.it, self.trace, self.rid = needed, 0, trace, rid

    def iterate(self, k):
        self.it += k
        self.trace.append(self.rid)
        return FakeReport(self.it, self.it >= self.needed)

    def fields(self):
        return None, None, None

    def close(self):
        pass


class Clock:
    """A clock that advances one unit per reading, so arrivals are reached deterministically."""
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1.0
        return self.t


def _server(budget, slots, needed, trace):
    srv = serve.Server(ctx=None, hbm_budget=budget, slots=slots, batched=False)
    srv._start = lambda req: (FakeMesh(req.mesh.n_cells, 1), FakeSim(needed[req.id], trace, req.id))
    return srv


def test_admission_respects_slots_budget_and_order():
    reqs = [serve.Request(i, arrival=0.0, mesh=FakeMesh(1000 * (i + 1), 3000 * (i + 1))) for i in range(5)]
    need = {r.id: 3 for r in reqs}
    one = serve.device_bytes(1000, 3000)
    budget = serve.device_bytes(1000, 3000) + serve.device_bytes(2000, 6000)  # the first two fit together
    trace = []
    srv = _server(budget, slots=4, needed=need, trace=trace)
    res = srv.run(reqs, clock=Clock())
    assert [r.id for r in res] == list(range(5))
    assert all(r.converged and r.iterations == 3 for r in res[:2])
    admitted = [e[1] for e in srv.log if e[0] == "admitted"]
    assert admitted[:2] == [0, 1]
    # request 4 needs more than the whole budget: rejected, never admitted
    assert ("rejected", 4, serve.device_bytes(5000, 15000)) in srv.log and 4 not in admitted
    # at no time is more admitted than the budget
    live, peak = 0, 0
    for kind, rid, val in srv.log:
        if kind == "admitted":
            live += val
        elif kind == "retired":
            live -= serve.device_bytes(1000 * (rid + 1), 3000 * (rid + 1))
        peak = max(peak, live)
    assert peak <= budget and one > 0


def test_round_robin_and_refill():
    reqs = [serve.Request(i, arrival=0.0, mesh=FakeMesh(100, 300)) for i in range(3)]
    trace = []
    srv = _server(10**12, slots=2, needed={0: 2, 1: 4, 2: 1}, trace=trace)
    res = srv.run(reqs, clock=Clock())
    # 0 and 1 alternate; 2 takes 0's slot when 0 retires
    assert trace[:4] == [0, 1, 0, 1]
    assert trace[4] == 1 and 2 in trace[4:6]
    assert [r.iterations for r in res] == [2, 4, 1]
    assert all(r.latency > 0 for r in res)
    s = serve.summary(res, wall=10.0)
    assert s["solves"] == 3 and s["converged"] == 3 and s["p99_latency_s"] >= s["p50_latency_s"]


def test_device_bytes_grows_with_size():
    assert serve.device_bytes(10**6, 7 * 10**6) > 10 * serve.device_bytes(10**5, 7 * 10**5) * 0.99


class _SizedMesh:
    def __init__(self, n):
        self.n_cells = n


def _stream(n=40, seed=3):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(0.1, n))
    return [serve.Request(i, float(t[i]), _SizedMesh(int(rng.integers(4000, 100000))), max_iterations=100)
            for i in range(n)]


def test_shards_partition_the_stream_and_balance_work():
    reqs = _stream()
    for world in (1, 2, 3, 4):
        shards = [serve.shard(reqs, world, r) for r in range(world)]
        ids = sorted(q.id for s in shards for q in s)
        assert ids == list(range(len(reqs)))
        loads = [sum(q.mesh.n_cells * q.max_iterations for q in s) for s in shards]
        biggest = max(q.mesh.n_cells * q.max_iterations for q in reqs)
        assert max(loads) - min(loads) <= biggest
        for s in shards:
            assert [q.arrival for q in s] == sorted(q.arrival for q in s)


def _shard_worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    mine = [q.id for q in serve.shard(_stream(), world, rank)]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out.put(gathered)
    dist.destroy_process_group()


def test_two_ranks_agree_on_the_partition_over_gloo():
    """Two processes (gloo, the multi-GPU launch shape without GPUs) each compute their shard of the
    same seeded stream; the gathered shards are disjoint and cover it."""
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(gathered[0] + gathered[1]) == list(range(40)) and not set(gathered[0]) & set(gathered[1])


class FakeBatch:
    """A cohort's segmented solve: member k converges after needed[k] outer iterations and then
    keeps its report (a converged segment is frozen)."""
    def __init__(self, needed, trace, ids):
        self.needed, self.it, self.trace, self.ids = needed, 0, trace, ids

    def iterate(self, k):
        self.it += k
        self.trace.append(tuple(self.ids))
        return FakeReport(self.it, self.it >= max(self.needed))

    def segment_report(self, k):
        it = min(self.it, self.needed[k])
        return FakeReport(it, it >= self.needed[k])

    def fields(self):
        return None, None, None

    def close(self):
        pass


def test_batched_cohorts_admit_as_slots_free_and_retire_members_individually():
    reqs = [serve.Request(i, arrival=0.0 if i < 3 else 6.0, mesh=FakeMesh(1000, 3000)) for i in range(5)]
    need = {0: 2, 1: 5, 2: 3, 3: 2, 4: 2}
    trace = []
    srv = serve.Server(ctx=None, hbm_budget=10 * serve.device_bytes(1000, 3000), slots=3, batched=True)

    def start(members):
        ids = [r.id for r, _, _ in members]
        return serve._Cohort(list(members), FakeMesh(1000 * len(ids), 1), FakeBatch([need[i] for i in ids], trace, ids),
                             np.arange(len(ids) + 1) * 1000, [False] * len(ids))
    srv._start_cohort = start
    res = srv.run(reqs, clock=Clock())
    assert [r.id for r in res] == list(range(5))
    assert all(r.converged for r in res)
    assert [r.iterations for r in res] == [2, 5, 3, 2, 2]
    # the first three arrive together and form one cohort; the later two join as slots free up
    assert trace[0] == (0, 1, 2)
    cohorts = {t for t in trace}
    assert (0, 1, 2) in cohorts and any(3 in t for t in cohorts) and any(4 in t for t in cohorts)
    # never more than three requests admitted and unretired at once
    live = peak = 0
    for kind, rid, _ in srv.log:
        live += 1 if kind == "admitted" else (-1 if kind == "retired" else 0)
        peak = max(peak, live)
    assert peak <= 3
