#!/usr/bin/env python3
"""Benchmark of the MLS-MPM soil step on B200: particle-steps/s.

Workload (default): the plain large rigid-wheel rut, 2,000,000 particles on a
128^3 grid (dx = 1/128) with the M1 PIC-rigid cylinder (R = 0.1 m, width
0.08 m, 5 kg, 2 rad/s, 0.1 m/s), dt = 5e-5 s; one step = P2G, grid update,
M1 coupler, G2P. Synthetic seeded inputs (no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--forms plain,batched,served,adjoint]

Beside the headline plain step the line carries the two other forms of the
metric (one GPU only): "batched" (256 uneven box-drop scenes stepped
together) and "served" (Poisson request streams into the continuous-batching
server, with p50/p99 latency), each with the plain per-scene loop on the same
scenes and the ratio to it.

N > 1 runs N independent replicas (one per GPU, launched by torchrun); the
path has no inter-GPU exchange, so there is no collective on the data path.
Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MPM particle-steps/s on 1 B200, batched+served vs plain; p50/p99 solve latency"
UNIT = "particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=int, default=2_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--math", choices=["fast", "ieee"], default=None,
                    help="SVD arithmetic of the fused step (default: the library default)")
    ap.add_argument("--sort-interval", type=int, default=None)
    ap.add_argument("--variant", type=int, default=None, help="launch shape of the fused kernel")
    ap.add_argument("--forms", default="plain,batched,served,adjoint",
                    help="comma list: plain (the headline wheel rut), batched (256 uneven scenes), "
                         "served (Poisson request stream), adjoint (differentiable tine pass)")
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--serve-rates", default="200,10", help="arrival rates (req/s) of the served runs")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# rank / process-group plumbing (replicas only: barrier + max over ranks)

class Ranks:
    def __init__(self, n_gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.pg is None and self.world > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------

def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# The sources that build and launch the plain solver's fused kernel: its
# translation unit and the headers it includes, and the World and solver code
# that choose its launch (variant, CTA order). The batched, served, coupler
# and adjoint sources do not change that kernel or its traffic.
FUSED_SOURCES = ("basements_b200/csrc/bm_kernels.cu", "basements_b200/csrc/bm_internal.h",
                 "basements_b200/csrc/bm_math.cuh", "basements_b200/csrc/bm_world.cu",
                 "basements_b200/csrc/bm_world.h", "basements_b200/csrc/bm_solver.cu",
                 "basements_b200/csrc/bm_solver_impl.h", "include/bm_mpm.h")


def kernel_sources_hash() -> str:
    """sha256 of the sources of the plain solver's fused kernel
    (FUSED_SOURCES), the key under which its ncu traffic figure is recorded."""
    import hashlib
    h = hashlib.sha256()
    files = sorted(os.path.join(ROOT, f) for f in FUSED_SOURCES)
    for f in files:
        h.update(os.path.basename(f).encode())
        h.update(open(f, "rb").read())
    return h.hexdigest()


def kernel_traffic(kernel: str):
    """DRAM bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)
    of `kernel` at this workload, from profiles/traffic.json, only when that
    capture was made from the same library sources; otherwise None."""
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(tp):
        return None
    rec = json.load(open(tp))
    if rec.get("sources_sha256") != kernel_sources_hash():
        return None
    return rec.get(kernel)


def bytes_per_unit(n_particles: int, touched_nodes: int):
    """Algorithmic bytes of one step (FP32 SoA): per particle 248 B (P2G reads
    x,v,C,F,m,V0 = 26 floats; G2P reads x,F = 12 and writes x,v,C,F = 24) and
    per touched node 80 B (P2G flush 7 floats, update reads 7 / writes 3, G2P
    reads 3). Per kernel: P2G 104 B/particle + 28 B/node, grid update 40 B/node,
    G2P 144 B/particle + 12 B/node; the fused G2P(n) + P2G(n+1) kernel does
    the work of both: 248 B/particle + 40 B/node."""
    return {
        "step": 248 * n_particles + 80 * touched_nodes,
        "p2g": 104 * n_particles + 28 * touched_nodes,
        "grid_update": 40 * touched_nodes,
        "g2p": 144 * n_particles + 12 * touched_nodes,
        "g2p2g": 248 * n_particles + 40 * touched_nodes,
    }


def run_ours(args, ranks: Ranks):
    import basements_b200 as bm
    from basements_b200 import scenes

    if ranks.world > 1:
        bm.set_device(ranks.local)
    sc = scenes.wheel_rut(n_keep=args.particles)
    body = sc.bodies[0]
    s = bm.MPMSolver(sc.dx, domain=sc.domain)
    s.set_material(sc.E, sc.nu, sc.rho)
    s.set_plastic_alpha(sc.alpha)
    s.add_particles(sc.position, None, sc.mass)
    if args.math:
        s.set_math_mode(args.math == "fast")
    if args.sort_interval is not None:
        s.set_sort_interval(args.sort_interval)
    if args.variant is not None:
        s.set_launch_variant(args.variant)

    def collider(step):
        return bm.make_collider(**body.at_time(step * sc.dt).as_tuple())

    # warm-up (untimed)
    for i in range(args.warmup):
        s.step_coupled(sc.dt, [collider(i)], read_reactions=False)
    st, _ = s.sync()
    if st != 0:
        raise RuntimeError(f"warm-up reported status {st}")
    # touched nodes (for the algorithmic byte count)
    s.p2g(sc.dt)
    touched = int((s.get_grid()["mass"] > 0).sum())
    s.grid_update(sc.dt)
    s.g2p(sc.dt)
    step0 = args.warmup + 1

    # timed region: K coupled steps, inputs resident in HBM (208 MB of particle
    # state, larger than the 126 MB L2), CUDA events on the solver's stream
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    idx = ranks.local if ranks.world > 1 else 0
    sampler = ClockSampler(vis[idx] if idx < len(vis) and vis[idx] else str(idx))
    s.sync()
    suspects0 = s.light_node_suspects()
    ranks.barrier()
    sampler.start()
    s.timer_start()
    for i in range(args.steps):
        s.step_coupled(sc.dt, [collider(step0 + i)], read_reactions=False)
    ms = s.timer_stop()
    clocks = sampler.stop()
    ranks.barrier()
    st, esc = s.sync()
    if st != 0:
        raise RuntimeError(f"timed steps reported status {st} ({esc} escaped writes)")
    suspects = s.light_node_suspects() - suspects0
    ms_max = ranks.max(ms)
    per_step_ms = ms_max / args.steps
    value = sc.n * args.steps * ranks.world / (ms_max / 1e3)
    # per-kernel times: the same number of steps again, each phase between two
    # CUDA events on the solver stream (the events add gaps of their own, so
    # this pass is not the timed one)
    s.profile(True)
    s.profile_reset()
    step1 = step0 + args.steps
    s.timer_start()
    for i in range(args.steps):
        s.step_coupled(sc.dt, [collider(step1 + i)], read_reactions=False)
    ms_profiled = s.timer_stop()
    prof = s.profile_read()
    s.profile(False)
    st, esc = s.sync()
    if st != 0:
        raise RuntimeError(f"profiled steps reported status {st} ({esc} escaped writes)")
    suspects = s.light_node_suspects() - suspects0  # over both passes

    # roofline of the dominant kernel
    bpu = bytes_per_unit(sc.n, touched)
    kernels = {k: v for k, v in prof.items() if v[1] > 0}
    dom = max(kernels, key=lambda k: kernels[k][0])
    dom_ms = kernels[dom][0] / kernels[dom][1]
    peak, peak_kind = measured_peak_hbm()
    alg = bpu.get(dom)
    achieved = (alg / (dom_ms / 1e3)) / 1e9 if alg else None
    traffic = kernel_traffic(dom)
    kernel_ms_per_step = sum(v[0] for v in kernels.values()) / args.steps
    launches = sum(v[1] for k, v in kernels.items() if k != "grid_clear")
    launches += 2 * kernels.get("bin_sort", (0, 0))[1]  # key + scan + permute per sort
    # a folded grid update is the update plus the three light-node repair
    # kernels (which return at once unless a suspect was found)
    launches += 3 * kernels.get("grid_update", (0, 0))[1]
    step_roof_gbs = bpu["step"] / (per_step_ms / 1e3) / 1e9

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded wheel-rut sand bed)",
        "config": {"workload": "wheel_rut plain large rigid-wheel rut: 2M particles, 128^3 grid dx=1/128, "
                               "M1 cylinder R=0.1 w=0.08 5kg, dt=5e-5",
                   "particles": sc.n, "grid": sc.grid, "touched_nodes": touched,
                   "parallelism": f"replicas{ranks.world}", "l2": "inputs larger than L2 (208 MB particle state)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "kernel_ms": dom_ms,
                     "step_achieved_gbs": step_roof_gbs, "step_frac": step_roof_gbs / peak,
                     "bytes_per_particle_step": bpu["step"] / sc.n},
        "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in kernels.items()},
        # where a step's time goes: the sum of the phases' event-timed
        # durations per step against the step, the rest being the gaps
        # between launches and small copies
        # (both from the profiled pass), and the unprofiled step beside them:
        # the events themselves add to the profiled step
        "step_breakdown_ms": {"step": per_step_ms, "step_profiled": ms_profiled / args.steps,
                              "phases_sum": kernel_ms_per_step,
                              "gaps": ms_profiled / args.steps - kernel_ms_per_step},
        "clocks": clocks,
        "gpu_launches": int(launches),
        # nodes of the timed and profiled steps where the fused kernel's
        # light-node rule could have missed a force record; each such step's
        # grid was redone unfolded on the device (exact)
        "light_node_suspects": int(suspects),
    }
    s.close()
    if not args.no_e2e:
        out["e2e"] = run_e2e(args, sc, ranks)
    return out


def run_e2e(args, sc, ranks: Ranks):
    """The same job through the public C ABI from host arrays: upload of the
    particles, K coupled steps each taking the collider from the host and
    returning the reaction to the host (synchronous), download of the final
    positions and velocities."""
    import basements_b200 as bm

    body = sc.bodies[0]
    colliders = [bm.make_collider(**body.at_time(i * sc.dt).as_tuple()) for i in range(args.steps)]
    pos = np.ascontiguousarray(sc.position)
    mass = np.ascontiguousarray(sc.mass)
    # warm the library / context once outside the timed region (a read
    # included: the process keeps the pinned read-back chunks)
    w = bm.MPMSolver(sc.dx, domain=sc.domain)
    w.add_particles(pos[:1024], None, mass[:1024])
    w.step_coupled(sc.dt, [colliders[0]])
    w.get_particles(("position",))
    w.close()
    ranks.barrier()
    t0 = time.perf_counter()
    s = bm.MPMSolver(sc.dx, domain=sc.domain)
    s.set_material(sc.E, sc.nu, sc.rho)
    s.set_plastic_alpha(sc.alpha)
    t1 = time.perf_counter()
    s.add_particles(pos, None, mass)
    t2 = time.perf_counter()
    s.step_coupled(sc.dt, [colliders[0]])
    t3 = time.perf_counter()
    for i in range(1, args.steps):
        s.step_coupled(sc.dt, [colliders[i]])
    t4 = time.perf_counter()
    out = s.get_particles(("position", "velocity"))
    el = time.perf_counter() - t0
    phases = {"create_ms": (t1 - t0) * 1e3, "upload_ms": (t2 - t1) * 1e3, "first_step_ms": (t3 - t2) * 1e3,
              "steps_ms": (t4 - t3) * 1e3, "download_ms": (t0 + el - t4) * 1e3}
    s.close()
    el = ranks.max(el)
    n = sc.n
    h2d = n * 16 + args.steps * 76
    d2h = n * 24 + args.steps * 28
    assert np.isfinite(out["position"]).all()
    return {"value": n * args.steps * ranks.world / el, "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "what": "upload + K synchronous coupled steps (host collider in, host reaction out) + download",
            "host_phases": phases}


def _host_body_step(body: dict, force, torque, gravity, dt):
    """The reference TimeIntegrator step (integrator.h:19-57) on a host body,
    with the identity body-space inverse inertia the reference scenarios leave
    in place: v += (m g + F)/m dt, w += tau dt, x += v dt, q += dt/2 (0,w) q."""
    m = body["mass"]
    v = [body["linear_velocity"][i] + (gravity[i] * m + float(force[i])) / m * dt for i in range(3)]
    w = [body["angular_velocity"][i] + float(torque[i]) * dt for i in range(3)]
    body["linear_velocity"], body["angular_velocity"] = tuple(v), tuple(w)
    body["center"] = tuple(body["center"][i] + v[i] * dt for i in range(3))
    qw, qx, qy, qz = body["orientation"]
    wx, wy, wz = w
    dq = (-wx * qx - wy * qy - wz * qz, wx * qw + wy * qz - wz * qy, -wx * qz + wy * qw + wz * qx,
          wx * qy - wy * qx + wz * qw)
    q = [body["orientation"][k] + 0.5 * dt * dq[k] for k in range(4)]
    n = sum(c * c for c in q) ** 0.5
    body["orientation"] = tuple(c / n for c in q) if n >= 1e-6 else (1.0, 0.0, 0.0, 0.0)


def plain_scene_loop(scs, steps, warmup: int = 3):
    """The plain per-scene loop: the scenes one after another through the
    drop-in solver API, each stepped `steps` times after `warmup` untimed
    steps. A dynamic body takes the reaction back to the host every step and
    is integrated there, as the reference's coupling harness does
    (bench_compare_all.cpp:104-116). Host-clock time, synchronised at both
    ends of each scene's timed steps (the loop's host round trips are part of
    what it costs). Returns (particle-steps/s, particle-steps, seconds)."""
    import basements_b200 as bm

    work, secs = 0, 0.0
    for sc in scs:
        s = bm.MPMSolver(sc.dx, domain=sc.domain)
        s.set_material(sc.E, sc.nu, sc.rho)
        s.set_plastic_alpha(sc.alpha)
        s.set_floor_friction(sc.floor_friction)
        s.set_gravity(sc.gravity)
        s.add_particles(sc.position, None, sc.mass)
        body = dict(sc.bodies[0].as_tuple()) if sc.bodies else None

        def one():
            if body is None:
                s.step(sc.dt)
            else:
                f, t, _ = s.step_coupled(sc.dt, [bm.make_collider(**body)])[0]
                _host_body_step(body, f, t, sc.gravity, sc.dt)

        for _ in range(warmup):
            one()
        s.sync()
        t0 = time.perf_counter()
        for _ in range(sc.steps if steps is None else steps):
            one()
        st, _ = s.sync()
        secs += time.perf_counter() - t0
        if st != 0:
            raise RuntimeError(f"plain loop: scene {sc.name} reported status {st}")
        work += sc.n * (sc.steps if steps is None else steps)
        s.close()
    return work / secs, work, secs


def run_batched(args):
    """Batched form: 256 box-drop scenes of uneven size (grid side in
    {32,48,64,96}, 8k-400k particles, dynamic boxes) in one batch: one
    persistent launch per phase over the scene table, CUDA-graph chunks,
    launch shape and sort interval chosen by the autotuner. K steps timed with
    CUDA events on the batch stream, inputs resident (GBs, beyond L2)."""
    import basements_b200 as bm
    from basements_b200 import scenes

    scs = [scenes.box_drop_scene(i) for i in range(args.batch_scenes)]
    n_tot = sum(sc.n for sc in scs)
    b = bm.Batch(scs)
    b.step(1)
    # each candidate timed over at least 64 steps (shorter trials let noise of
    # a percent or two pick the sort interval)
    tune = b.autotune(trial_steps=64)
    for _ in range(args.warmup):
        b.step(1)
    b.sync()
    # a whole number of sort intervals, so that the regrouping is counted at
    # the rate it runs (a window shorter than the interval may hold none)
    K = max(1, int(tune.get("sort_interval") or 1))
    steps = K * ((args.steps + K - 1) // K)
    b.timer_start()
    b.step(steps)
    ms = b.timer_stop()
    st, bad, esc = b.sync()
    if st != 0:
        raise RuntimeError(f"batched: scene {bad} reported status {st}")
    # per-phase breakdown from a few eager steps after the timed region
    b.profile(True)
    b.profile_reset()
    prof_steps = 4
    b.step(prof_steps)
    phases = {k: round(v[0] / prof_steps, 4) for k, v in b.profile_read().items() if v[1] > 0}
    b.profile(False)
    b.close()
    value = n_tot * steps / (ms / 1e3)
    loop_steps = min(args.steps, 50)
    loop_rate, loop_work, loop_secs = plain_scene_loop(scs, loop_steps)
    return {"workload": f"{len(scs)} box-drop scenes, grid side in {{32,48,64,96}}, 8k-400k particles "
                        "(log-uniform, 8 ppc), friction angle 25-40 deg, E 1e5-1e6 Pa, dynamic M1 box",
            "scenes": len(scs), "particles": n_tot, "value": value, "unit": UNIT, "steps": steps,
            "ms_per_step": ms / steps,
            "timing": "CUDA events on the batch stream, over a whole number of sort intervals",
            "phases_ms_per_step_eager": phases,
            "autotune": tune,
            "plain_loop": {"value": loop_rate, "unit": UNIT, "steps_per_scene": loop_steps,
                           "seconds": loop_secs,
                           "what": "same scenes one after another through bm_solver_step_coupled, reaction "
                                   "read back and the body integrated on the host every step (host clock)"},
            "speedup_vs_plain_loop": value / loop_rate,
            "cpu_baseline": _aggregate_or_none(args, "box_drop", list(range(len(scs))))}


def _aggregate_or_none(args, gen, seeds):
    if args.no_cpu_baseline:
        return None
    from oracle import oracle as O
    kind = O.reference_or_port()
    if not O.available(kind):
        return None
    # one scene per core, at most 64 processes (a few hundred MB each)
    cores = min(os.cpu_count() or 1, 64)
    return cpu_aggregate(gen, seeds[:cores], kind)


def run_served(args):
    """Served form: Poisson request streams into the continuous-batching
    server (bm_server_*), one per arrival rate; each request is a seeded
    scene of 10k-1M particles on a 32-128 grid for 100-2000 steps, half with a
    dynamic box or cylinder. Reported per rate: throughput = particle-steps of
    all requests / (last completion - first arrival), host clock, and the
    server's p50/p99 submit-to-result latency of the timed requests (the server's
    own percentiles also count the untimed warm-up requests). The plain
    per-request loop runs the same requests one after another through the
    drop-in solver API."""
    import basements_b200 as bm
    from basements_b200 import scenes

    rates = [float(r) for r in args.serve_rates.split(",") if r]
    runs = []
    base_seed = 0
    all_reqs = []
    for ri, rate in enumerate(rates):
        reqs = [scenes.serve_request_scene(base_seed + i) for i in range(args.serve_requests)]
        base_seed += args.serve_requests
        all_reqs += reqs
        rng = np.random.default_rng(77 + ri)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        arrivals -= arrivals[0]
        srv = bm.Server()
        # untimed warm-up: the same requests for 2 steps each, so that the
        # server's device memory pool and pinned read-back blocks have grown
        # to this stream's sizes (a long-running server keeps and reuses them)
        warm = [srv.submit(sc, 2) for sc in reqs]
        for r in warm:
            if srv.wait(r, timeout_ms=600_000) != 0:
                raise RuntimeError("served: warm-up request failed")
            srv.release(r)
        st0 = srv.stats()
        work = sum(sc.n * sc.steps for sc in reqs)
        ids = []
        t0 = time.perf_counter()
        for sc, at in zip(reqs, arrivals):
            d = t0 + at - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(sc, sc.steps))
        for r in ids:
            if srv.wait(r, timeout_ms=600_000) != 0:
                raise RuntimeError(f"served: request {r} did not complete")
        el = time.perf_counter() - t0
        lat = [srv.result(r)["latency_ms"] for r in ids]
        st = srv.stats()
        srv.close()
        busy = st["busy_seconds"] - st0["busy_seconds"]
        runs.append({"rate_req_s": rate, "requests": len(reqs), "particle_steps": work,
                     "value": work / el, "unit": UNIT, "seconds": el,
                     "p50_latency_ms": float(np.percentile(lat, 50)), "p99_latency_ms": float(np.percentile(lat, 99)),
                     "server_p50_ms": st["p50_latency_ms"], "server_p99_ms": st["p99_latency_ms"],
                     "worker_busy_rate": (st["particle_steps"] - st0["particle_steps"]) / max(busy, 1e-9),
                     "iterations": st["iterations"] - st0["iterations"], "peak_bytes": st["peak_bytes"],
                     "host_seconds": {k: st[k] - st0[k] for k in ("admit_seconds", "step_seconds", "retire_seconds")}})
    # the first rate's requests, each for all of its steps, one after another
    loop_rate, _, loop_secs = plain_scene_loop(all_reqs[:args.serve_requests], None)
    best = max(r["value"] for r in runs)
    return {"workload": "Poisson request stream: grid 32-128, 10k-1M particles (log-uniform, capped to fit "
                        "the grid), 100-2000 steps, friction angle 25-40 deg, half with a dynamic box or "
                        "cylinder; admission by a 150 GB HBM budget",
            "runs": runs, "value": best, "unit": UNIT,
            "plain_loop": {"value": loop_rate, "unit": UNIT, "steps_per_request": "all (100-2000)",
                           "seconds": loop_secs,
                           "what": "the first rate's requests one after another through the drop-in solver "
                                   "(host clock, body integrated on the host every step)"},
            "speedup_vs_plain_loop": best / loop_rate,
            "cpu_baseline": _aggregate_or_none(args, "serve", list(range(args.serve_requests)))}


def run_adjoint(args):
    """Differentiable form: the tine pass (262,144 particles on the 64^3 grid,
    200 steps at dt = 1e-4, 16 waypoints, checkpoints every 20 steps). The
    forward records the run, the backward returns dL/d waypoint for the soft
    heightfield loss. CUDA events on the solver stream around each pass (the
    backward includes the upload of dL/dx and the download of the result)."""
    import basements_b200 as bm
    from basements_b200 import scenes

    sc, body, wp, target = scenes.tine_pass()
    s = bm.MPMSolver(sc.dx, domain=sc.domain)
    s.set_material(sc.E, sc.nu, sc.rho)
    s.set_plastic_alpha(sc.alpha)
    s.add_particles(sc.position, None, sc.mass)
    tape = bm.Tape(s, 20)
    col = bm.make_collider(**body.as_tuple())
    x0 = s.get_particles(("position", "velocity", "F", "C"))
    fwd, bwd = [], []
    for it in range(args.warmup + 3):
        s.set_particles(0, position=x0["position"], velocity=x0["velocity"], F=x0["F"], C_=x0["C"])
        s.sync()
        s.timer_start()
        tape.forward(sc.dt, sc.steps, col, wp)
        f_ms = s.timer_stop()
        L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
        s.timer_start()
        gw = tape.backward(g)["dL_dwaypoints"]
        b_ms = s.timer_stop()
        if it >= args.warmup:
            fwd.append(f_ms)
            bwd.append(b_ms)
    assert np.isfinite(gw).all()
    f_ms, b_ms = float(np.median(fwd)), float(np.median(bwd))
    work = sc.n * sc.steps
    tape.close()
    s.close()
    return {"workload": "tine pass: 262,144 particles, 64^3 grid, 200 steps at dt=1e-4, 16 waypoints, "
                        "soft-heightfield L2 loss, checkpoints every 20 steps",
            "forward_ms": f_ms, "backward_ms": b_ms, "loss": L,
            "value": work / ((f_ms + b_ms) / 1e3), "unit": UNIT + " (forward + backward)",
            "backward_over_forward": b_ms / f_ms, "timing": "CUDA events on the solver stream, median of 3",
            "gradient_check": "tests/test_gpu_adjoint.py (FP64 central differences)"}


def host_cpu():
    """The host's logical core count and CPU model (from /proc/cpuinfo)."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "model": model}


def _cpu_scene_worker(job):
    """One process of the aggregate CPU baseline: the reference's own solver
    (coupler and integrator included) on one scene for `steps` steps, as the
    reference's harness runs a scene (bench_compare_all.cpp:104-116)."""
    kind, gen, seed, steps = job
    from basements_b200 import scenes
    from oracle import oracle as O

    sc = scenes.box_drop_scene(seed) if gen == "box_drop" else scenes.serve_request_scene(seed)
    c = O.CpuSolver(kind, sc.dx)
    c.set_material(sc.E, sc.nu, sc.rho)
    c.set_plastic_alpha(sc.alpha)
    c.set_gravity(sc.gravity)
    c.set_floor_friction(sc.floor_friction)
    c.add_particles(sc.position, None, sc.mass)
    t0 = time.perf_counter()
    if sc.bodies:
        c.run_dynamic_body(O.collider(**sc.bodies[0].as_tuple()), sc.gravity, sc.dt, steps)
    else:
        c.step(sc.dt, steps)
    el = time.perf_counter() - t0
    c.close()
    return sc.n * steps, el, sc.n


def cpu_aggregate(gen: str, seeds, kind: str, work_per_scene: float = 8e6):
    """Aggregate CPU baseline of a many-scene workload: the reference's solver
    in one process per host core (spawned, so that no process inherits a CUDA
    context), each on one scene of the sample for about work_per_scene
    particle-steps. Returns particle-steps of all processes / wall time of the
    whole pool."""
    import concurrent.futures as cf
    import multiprocessing as mp

    from basements_b200 import scenes

    make = scenes.box_drop_scene if gen == "box_drop" else scenes.serve_request_scene
    jobs = []
    for seed in seeds:
        n = make(seed).n
        jobs.append((kind, gen, seed, max(1, int(round(work_per_scene / max(n, 1))))))
    procs = min(os.cpu_count() or 1, len(jobs))
    t0 = time.perf_counter()
    with cf.ProcessPoolExecutor(max_workers=procs, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_cpu_scene_worker, jobs))
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    return {"value": work / wall, "unit": UNIT, "cores": procs,
            "kind": "reference" if kind == "ref" else "port",
            "sample": f"{len(jobs)} scenes of the workload ({gen} seeds {seeds[0]}..{seeds[-1]}), one process "
                      f"per core, ~{work_per_scene:.0e} particle-steps each ({wall:.1f} s wall)",
            "host": host_cpu()}


def cpu_reference_rate(sc, n_steps: int, kind: str):
    """Times the reference's own CPU MPMSolver (oracle/_ref, else the pinned
    float restatement) on the wheel-rut scene: P2G, update_grid, M1 apply,
    G2P per step, single thread (the reference has no threading)."""
    from oracle import oracle as O

    body = sc.bodies[0]
    c = O.CpuSolver(kind, sc.dx)
    c.set_material(sc.E, sc.nu, sc.rho)
    c.set_plastic_alpha(sc.alpha)
    c.add_particles(sc.position, None, sc.mass)
    t0 = time.perf_counter()
    for i in range(n_steps):
        c.p2g(sc.dt)
        c.grid_update(sc.dt)
        c.m1_apply(O.collider(**body.at_time(i * sc.dt).as_tuple()), sc.dt)
        c.g2p(sc.dt)
    el = time.perf_counter() - t0
    c.close()
    return sc.n * n_steps / el, el


def run_reference(args, ranks: Ranks):
    from basements_b200 import scenes
    from oracle import oracle as O

    kind = O.reference_or_port()
    sc = scenes.wheel_rut(n_keep=args.particles)
    # each step is a bounded sample: the full 2M-particle coupled step (~3 s
    # on one core); warm-up steps are not timed
    n_timed = max(1, min(args.steps, 3))
    n_warm = min(args.warmup, 1)
    if n_warm:
        cpu_reference_rate(sc, n_warm, kind)
    rate, el = cpu_reference_rate(sc, n_timed, kind)
    sample = f"{n_timed} coupled steps of the {sc.n}-particle wheel-rut scene"
    cb = {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference" if kind == "ref" else "port",
          "sample": sample, "host": host_cpu()}
    return {"metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": ranks.world,
            "steps": n_timed, "warmup": n_warm, "ms_per_step": el * 1e3 / n_timed, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded wheel-rut sand bed)",
            "config": {"workload": "wheel_rut plain large rigid-wheel rut: 2M particles, 128^3 grid dx=1/128, "
                                   "M1 cylinder R=0.1 w=0.08 5kg, dt=5e-5", "particles": sc.n,
                       "parallelism": "1 host thread (the reference is single-threaded)"},
            "cpu_baseline": cb,
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    ranks = Ranks(args.gpus)
    try:
        if args.impl == "reference":
            if ranks.rank == 0:
                print(json.dumps(run_reference(args, ranks)), flush=True)
            return
        forms = set(f for f in args.forms.split(",") if f)
        out = run_ours(args, ranks)
        if ranks.world == 1 and "batched" in forms:
            out["batched"] = run_batched(args)
        if ranks.world == 1 and "served" in forms:
            out["served"] = run_served(args)
            sv = out["served"]
            # what bounds the served-over-loop ratio: the plain loop already
            # runs the large requests near the kernel's rate, so even a server
            # at the batched kernel's rate would be this many times the loop
            if "batched" in out:
                sv["fraction_of_batched_rate"] = sv["value"] / out["batched"]["value"]
                sv["ratio_ceiling_at_batched_rate"] = out["batched"]["value"] / sv["plain_loop"]["value"]
        if ranks.world == 1 and "adjoint" in forms:
            out["adjoint"] = run_adjoint(args)
        if ranks.rank == 0 and not args.no_cpu_baseline:
            from basements_b200 import scenes
            from oracle import oracle as O
            kind = O.reference_or_port()
            if O.available(kind):
                sc = scenes.wheel_rut(n_keep=args.particles)
                rate, el = cpu_reference_rate(sc, 3, kind)
                out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": 1,
                                       "kind": "reference" if kind == "ref" else "port",
                                       "sample": f"3 coupled steps of the {sc.n}-particle wheel-rut scene "
                                                 f"({el:.1f} s, 1 thread: the reference is single-threaded)",
                                       "host": host_cpu()}
        if ranks.rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
