"""Serving loop for steady SIMPLE requests (continuous batching at outer-iteration granularity).

Each request carries a case description: a polyhedral mesh, the lid (or inlet) speed
and the viscosity.  The server admits arrived requests in arrival order while the
device-memory estimate of everything admitted stays within the HBM budget and a
slot is free, keeps every admitted solve's fields, matrices and AMG hierarchy
resident on the device, and retires a solve when it converges (or reaches its
iteration cap), freeing its slot and memory for the next admission.

Batched (the default): the requests admitted together form a cohort, one
block-diagonal batch (meshgen.concatenate + bsg_simple_set_segments) whose outer
iteration is one set of kernel launches for all its members, with every member's
pressure systems solved side by side in one persistent launch.  Requests that
arrive while cohorts run are admitted into a new cohort as slots and memory free
up; the cohorts advance one outer iteration each in turn.  A member's arithmetic
is the same as alone except for the order of its pressure-solve dot products (its
CTA share of the launch), so its result equals its solo result within rounding
as long as both take the same number of outer iterations.  Unbatched: every
request is its own solve, advanced one outer iteration each in turn.

The reference serves no requests: its unit of work is one `babelsim-solve` run per
case (src/runtime/application.cpp:238-272), which is the per-request semantics here.
"""
from __future__ import annotations

import heapq
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    id: int
    arrival: float              # seconds after the stream starts
    mesh: object                # meshgen.PolyMesh (six patches; lid on patch 3)
    speed: float = 1.0          # lid speed
    nu: float = 1e-2            # kinematic = dynamic viscosity (density 1)
    max_iterations: int = 200
    tolerance: float = 1e-5     # momentum / velocity / pressure-change tolerance of the outer loop


@dataclass
class Result:
    id: int
    cells: int
    arrival: float
    admitted: float
    finished: float
    iterations: int
    converged: bool
    U: np.ndarray | None = None
    p: np.ndarray | None = None

    @property
    def latency(self):
        return self.finished - self.arrival


def device_bytes(n_cells: int, n_faces: int) -> int:
    """Device-memory estimate of one resident SIMPLE solve: geometry (152 B per face,
    40 B per cell), fields and workspaces (~60 doubles per cell), two LDU systems on
    the cell-to-face pattern, the AMG hierarchy with its SELL copies (~1.6x the
    level-0 matrix), the SELL copy of the momentum matrix (~1.3x its off-diagonal
    entries, 12 B each), the per-slot records of the diffusion face pass (64 B per
    face) and Krylov workspaces."""
    matrix = 8 * n_cells + 12 * 2 * n_faces
    return int(152 * n_faces + 40 * n_cells + 480 * n_cells + 2 * matrix + 1.6 * (matrix + 8 * 2 * n_faces) +
               1.3 * 12 * 2 * n_faces + 64 * n_faces + 16 * 8 * n_cells)


def shard(requests: list[Request], world: int, rank: int) -> list[Request]:
    """This rank's requests when a stream is served by `world` GPUs, each with its own admission
    loop and no data exchanged between them: in arrival order, every request goes to the rank with
    the least predicted work so far (cells x iteration cap; ties to the lower rank).  Every rank
    computes the same assignment from the same stream, so the shards partition it."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    load = [0.0] * world
    mine = []
    for r in sorted(requests, key=lambda q: (q.arrival, q.id)):
        k = min(range(world), key=lambda i: (load[i], i))
        load[k] += float(r.mesh.n_cells) * r.max_iterations
        if k == rank:
            mine.append(r)
    return mine


@dataclass
class _Active:
    req: Request
    mesh: object
    sim: object
    admitted: float
    bytes: int
    iterations: int = 0


@dataclass
class _Cohort:
    members: list               # [(Request, admitted, bytes)]
    mesh: object
    sim: object
    cells: np.ndarray           # cell offsets of the members in the concatenated mesh
    done: list                  # per member: retired


@dataclass
class Server:
    ctx: object
    hbm_budget: int = 150 * 2**30
    slots: int = 8
    keep_fields: bool = False
    solver_precision: int = 0
    batched: bool = True
    log: list = field(default_factory=list)
    trace: bool = False         # also print every log entry to stderr as it happens

    def _note(self, entry):
        self.log.append(entry)
        if self.trace:
            import sys
            print("serve:", *entry, file=sys.stderr, flush=True)

    def _simple(self, mesh, nu, tolerance):
        import babelsim_b200 as bsg
        opts = bsg.options("linear", "greenGauss", "upwind", "orthogonal")
        return bsg.Simple(mesh, 1.0, nu, 0.7, 0.3, 1, 1e-6, tolerance, tolerance, tolerance, opts, opts,
                          bsg.solver_config("bcgs", "bjacobi", 1e-14, 1e-8, 1000),
                          bsg.solver_config("cg", "hypre", 1e-14, 1e-8, 1000, precision=self.solver_precision))

    @staticmethod
    def _lid(sim, patch0, speed):
        for patch in range(6):
            sim.set_boundary("U", patch0 + patch, "fixedValue", (speed, 0.0, 0.0) if patch == 3 else (0.0, 0.0, 0.0))
            sim.set_boundary("p", patch0 + patch, "zeroGradient")

    def _start(self, req: Request):
        import babelsim_b200 as bsg
        m = bsg.Mesh.from_polyhedral(self.ctx, req.mesh)
        sim = self._simple(m, req.nu, req.tolerance)
        self._lid(sim, 0, req.speed)
        sim.set_fields(np.zeros((m.n_cells, 3)), np.zeros(m.n_cells))
        return m, sim

    def _start_cohort(self, members) -> _Cohort:
        import babelsim_b200 as bsg
        from . import meshgen
        reqs = [r for r, _, _ in members]
        poly, cells, patches = meshgen.concatenate([r.mesh for r in reqs])
        m = bsg.Mesh.from_polyhedral(self.ctx, poly)
        sim = self._simple(m, reqs[0].nu, reqs[0].tolerance)
        sim.set_segments(cells, [r.nu for r in reqs])
        for k, r in enumerate(reqs):
            self._lid(sim, int(patches[k]), r.speed)
        sim.set_fields(np.zeros((m.n_cells, 3)), np.zeros(m.n_cells))
        return _Cohort(list(members), m, sim, cells, [False] * len(reqs))

    def run(self, requests: list[Request], clock=time.perf_counter) -> list[Result]:
        """Serve `requests` (arrival times relative to the call) and return one Result each."""
        if self.batched:
            return self._run_batched(requests, clock)
        return self._run_each(requests, clock)

    def _run_batched(self, requests: list[Request], clock) -> list[Result]:
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        queue: list[tuple[float, int, Request]] = []
        cohorts: list[_Cohort] = []
        results: list[Result] = []
        used = 0
        busy = 0   # admitted requests not yet retired
        t0 = clock()
        i = 0
        while i < len(pending) or queue or cohorts:
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                heapq.heappush(queue, (pending[i].arrival, pending[i].id, pending[i]))
                i += 1
            # admission in arrival order under the slot count and the memory budget; the requests
            # admitted now form one cohort (requests of one cohort share the outer tolerance)
            members = []
            while queue and busy + len(members) < self.slots:
                req = queue[0][2]
                need = device_bytes(req.mesh.n_cells, len(req.mesh.owner))
                if need > self.hbm_budget:
                    heapq.heappop(queue)
                    results.append(Result(req.id, req.mesh.n_cells, req.arrival, now, now, 0, False))
                    self._note(("rejected", req.id, need))
                    continue
                if used + need > self.hbm_budget or (members and req.tolerance != members[0][0].tolerance):
                    break
                heapq.heappop(queue)
                used += need
                members.append((req, clock() - t0, need))
                self._note(("admitted", req.id, need))
            if members:
                cohorts.append(self._start_cohort(members))
                busy += len(members)
            if not cohorts:
                if i < len(pending):  # idle until the next arrival
                    wait = pending[i].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            # one outer iteration of every cohort, in admission order
            for c in list(cohorts):
                c.sim.iterate(1)
                fields = None
                for k, (req, admitted, need) in enumerate(c.members):
                    if c.done[k]:
                        continue
                    rep = c.sim.segment_report(k)
                    if rep.converged or rep.status == 2 or rep.iterations >= req.max_iterations:
                        c.done[k] = True
                        U = p = None
                        if self.keep_fields:
                            if fields is None:
                                fields = c.sim.fields()
                            a, b = int(c.cells[k]), int(c.cells[k + 1])
                            U, p = fields[0][a:b].copy(), fields[1][a:b].copy()
                        used -= need
                        busy -= 1
                        results.append(Result(req.id, req.mesh.n_cells, req.arrival, admitted, clock() - t0,
                                              rep.iterations, bool(rep.converged), U, p))
                        self._note(("retired", req.id, rep.iterations))
                if all(c.done):
                    c.sim.close()
                    c.mesh.close()
                    cohorts.remove(c)
        return sorted(results, key=lambda r: r.id)

    def _run_each(self, requests: list[Request], clock) -> list[Result]:
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        queue: list[tuple[float, int, Request]] = []
        active: list[_Active] = []
        results: list[Result] = []
        used = 0
        t0 = clock()
        i = 0
        turn = 0
        while i < len(pending) or queue or active:
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                heapq.heappush(queue, (pending[i].arrival, pending[i].id, pending[i]))
                i += 1
            # admission in arrival order under the slot count and the memory budget
            while queue and len(active) < self.slots:
                req = queue[0][2]
                need = device_bytes(req.mesh.n_cells, len(req.mesh.owner))
                if need > self.hbm_budget:
                    heapq.heappop(queue)
                    results.append(Result(req.id, req.mesh.n_cells, req.arrival, now, now, 0, False))
                    self._note(("rejected", req.id, need))
                    continue
                if used + need > self.hbm_budget:
                    break
                heapq.heappop(queue)
                m, sim = self._start(req)
                used += need
                active.append(_Active(req, m, sim, clock() - t0, need))
                self._note(("admitted", req.id, need))
            if not active:
                if i < len(pending):  # idle until the next arrival
                    wait = pending[i].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            # one outer iteration of every active solve, in admission order
            done = []
            for a in active:
                rep = a.sim.iterate(1)
                a.iterations = rep.iterations
                if rep.converged or rep.status == 2 or a.iterations >= a.req.max_iterations:
                    done.append((a, rep))
            for a, rep in done:
                U = p = None
                if self.keep_fields:
                    U, p, _ = a.sim.fields()
                a.sim.close()
                a.mesh.close()
                used -= a.bytes
                active.remove(a)
                results.append(Result(a.req.id, a.req.mesh.n_cells, a.req.arrival, a.admitted, clock() - t0,
                                      a.iterations, bool(rep.converged), U, p))
                self._note(("retired", a.req.id, a.iterations))
            turn += 1
        return sorted(results, key=lambda r: r.id)


def summary(results: list[Result], wall: float) -> dict:
    lat = np.array([r.latency for r in results if r.finished > r.admitted or r.iterations > 0])
    cells = sum(r.cells * r.iterations for r in results)
    return {"solves": len(results), "solves_per_s": len(results) / wall,
            "p50_latency_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if lat.size else None,
            "converged": int(sum(r.converged for r in results)), "cell_iters_per_s": cells / wall}
