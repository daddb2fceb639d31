"""Serving loop on the GPU: each request's result is the same alone and in the mix, and the
loop retires every request.

In the mix, requests admitted together run as one block-diagonal cohort whose pressure
systems share one persistent launch; each member's CTA share depends only on its own size
(while the cohort fits the grid), so its arithmetic, and therefore its result, is bit for bit
the one it has alone.  Against the unbatched path (its own launches on the whole grid, so a
different dot-product order in the pressure solves) results agree to 1e-7 relative L2."""
import numpy as np
import pytest

from babelsim_b200 import meshgen, serve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def _requests():
    meshes = [meshgen.cavity_2d(8), meshgen.cavity_2d(10), meshgen.warped_box(4), meshgen.voronoi_cube(5, 0.3, 7)]
    return [serve.Request(i, arrival=0.0, mesh=m, speed=0.5 + 0.5 * i, nu=10 ** (-2 - 0.3 * i), max_iterations=25,
                          tolerance=1e-4) for i, m in enumerate(meshes)]


def test_results_alone_and_in_the_mix_agree(ctx):
    reqs = _requests()
    alone = [serve.Server(ctx, slots=1, keep_fields=True).run([r])[0] for r in reqs]
    srv = serve.Server(ctx, slots=3, keep_fields=True)
    mix = srv.run(reqs)
    assert [r.id for r in mix] == [0, 1, 2, 3]
    for a, b in zip(alone, mix):
        assert a.iterations == b.iterations and a.converged == b.converged
        assert np.array_equal(a.U, b.U) and np.array_equal(a.p, b.p)
    # the first three ran as one cohort: their outer iterations were shared launches
    assert srv.batched
    # three slots: the fourth request waited for a retirement
    admitted = [e[1] for e in srv.log if e[0] == "admitted"]
    assert admitted == [0, 1, 2, 3]
    first_retired = next(i for i, e in enumerate(srv.log) if e[0] == "retired")
    assert srv.log.index(("admitted", 3, serve.device_bytes(reqs[3].mesh.n_cells, len(reqs[3].mesh.owner)))) > first_retired


def test_budget_queues_and_rejects(ctx):
    reqs = _requests()
    sizes = [serve.device_bytes(r.mesh.n_cells, len(r.mesh.owner)) for r in reqs]
    budget = max(sizes[:3])  # one at a time for the first three; the Voronoi cube may not fit at all
    srv = serve.Server(ctx, hbm_budget=budget, slots=4)
    res = srv.run(reqs)
    assert len(res) == 4
    for kind, rid, val in srv.log:
        if kind == "admitted":
            assert val <= budget
    rejected = {e[1] for e in srv.log if e[0] == "rejected"}
    assert rejected == {i for i, s in enumerate(sizes) if s > budget}


def test_batched_and_unbatched_serving_agree(ctx):
    reqs = _requests()
    batched = serve.Server(ctx, slots=4, keep_fields=True).run(reqs)
    each = serve.Server(ctx, slots=4, keep_fields=True, batched=False).run(reqs)
    for a, b in zip(batched, each):
        assert a.converged == b.converged
        assert abs(a.iterations - b.iterations) <= 1
        assert np.linalg.norm(a.U - b.U) <= 1e-7 * np.linalg.norm(b.U)
        assert np.linalg.norm(a.p - b.p) <= 1e-7 * np.linalg.norm(b.p)
