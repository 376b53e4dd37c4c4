#!/usr/bin/env python
"""bench.py -- density + force particle-updates/s on one or more B200s.

Workload (the lattice-100 density + force configuration): the close-packed unit-box
lattice with npartx = 100 (1,403,000 particles), 1% of particles (seeded uniform pick)
with h scaled by U[0.65, 1.35], velocities N(0, 0.1^2) per component, u = 1,
gamma = 5/3, alpha_AV = 1, beta = 2, alphau = 0, cubic kernel, hfact 1.2, tolh 1e-4,
open boundaries (the reference driver's boundary choice).  Synthetic, seeded.

A step is one density solve (tree + Newton-Raphson + gradient sweep) followed by one
force pass, both through the library's C-ABI.  Particle-updates per step = the sum over
Newton iterations of the particles updated + the live particles of the force pass.

  value   device-timed, inputs resident in HBM (no host transfers in the timed region)
  e2e     the same step through the C-ABI from pinned host buffers, with every step's
          uploads (POS, HSML, VEL, ACCEL, THERMO) and downloads (HSML, DENS_OUT,
          GRAD_OUT, FORCE_OUT) inside the timed region
Multi-GPU: one process per GPU (torchrun), each an independent replica of the workload
(the path has no exchange step); value = all ranks' updates / the slowest rank's time.

--impl reference times the CPU oracle (the reference cannot be built here: its
Cornerstone dependency is absent) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "density+force particle-updates/s (lattice 100 + jiggle)"
UNIT = "particle-updates/s"
FLOP_PER_DENSITY_PAIR = 30.0
FLOP_PER_NR_UPDATE = 30.0
BYTES_PER_DENSITY_UPDATE = 56.0


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                              device_id=torch.device("cuda", local))
        dist = td
    return rank, world, local, dist


def barrier(dist, local):
    if dist is not None:
        import torch
        t = torch.zeros(1, device=f"cuda:{local}")
        dist.all_reduce(t)
        torch.cuda.synchronize(local)


def max_over_ranks(dist, local, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, local, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t)
    return float(t.item())


class ClockSampler:
    """nvidia-smi sampled every 100 ms during the timed region."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(gpu), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.count(",") >= 9]
        os.unlink(self.f.name)
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].strip() == "Active"})
        busy = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)]
        return {"sm_mhz": statistics.median(busy or sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def workload(npartx):
    from cosmosphere_b200 import inputs
    return inputs.lattice100_workload(npartx)


def cpu_oracle_step(p, threads=0):
    """One density (+gradients) + force step of the CPU oracle; returns (updates, seconds)."""
    from oracle import oracle as O
    o = O.Oracle(threads=threads)
    n = p.n
    vel = np.stack([p["vx"], p["vy"], p["vz"]])
    t0 = time.perf_counter()
    st = o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], vel=vel, acc=np.zeros((3, n)), max_iter=100)
    assert st == 0, st
    o.force(np.stack([p["pro2"], p["cs"], p["alpha"], p["u"]]), beta=2.0, alphau=0.0)
    dt = time.perf_counter() - t0
    upd = float(o.array("activePerIter").sum() + o.scalar("nAlive"))
    return upd, dt, O.max_threads()


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary, if any."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get(kernel)
    return None


A_FLOOR = 0.1   # per-particle relative |a| errors are taken where |a| >= A_FLOOR x rms |a|


def mixed_accuracy(c, p, n, pos, hsml, vel, acc, thermo, outs, hfact=1.2):
    """Max / rms errors of the mixed form against the FP64 form, same inputs, same GPU."""
    from cosmosphere_b200 import capi
    res = {}
    for mode in (0, 1):
        c.set_precision(bool(mode))
        c.upload(capi.POS, pos, n); c.upload(capi.HSML, hsml, n)
        c.upload(capi.VEL, vel, n); c.upload(capi.ACCEL, acc, n)
        c.density(n, p["pmass"], tolh=1e-4, hfact=hfact, periodic_box=p.get("box"))
        c.upload(capi.THERMO, thermo, n, sorted_=True)
        c.force(n, p["pmass"], beta=2.0, alphau=0.0)
        res[mode] = {k: c.download(k, n).copy() for k in outs}
    c.set_precision(False)
    r0, r1 = res[0], res[1]
    rel = lambda a, b: np.abs(a - b) / np.abs(b)
    f0, f1 = r0[capi.FORCE_OUT][:3], r1[capi.FORCE_OUT][:3]
    amag = np.sqrt((f0 ** 2).sum(0))
    da = np.sqrt(((f1 - f0) ** 2).sum(0))
    rms_a = float(np.sqrt((amag ** 2).mean()))
    eh, er = rel(r1[capi.HSML][0], r0[capi.HSML][0]), rel(r1[capi.DENS_OUT][0], r0[capi.DENS_OUT][0])
    # per-particle relative |a| error where |a| is not near zero: |a| at least A_FLOOR x rms |a|
    big = amag >= A_FLOOR * rms_a
    ea = da[big] / amag[big]
    return {"vs": "plain FP64 form (bit-exact with the FP64 oracle)",
            "h_max_rel": float(eh.max()), "h_rms_rel": float(np.sqrt((eh ** 2).mean())),
            "rho_max_rel": float(er.max()), "rho_rms_rel": float(np.sqrt((er ** 2).mean())),
            "a_max_rel_to_rms_a": float(da.max() / rms_a), "a_rms_rel_to_rms_a": float(np.sqrt((da ** 2).mean()) / rms_a),
            "a_max_rel": float(ea.max()) if ea.size else None,
            "a_rms_rel": float(np.sqrt((ea ** 2).mean())) if ea.size else None,
            "a_rel_floor": f"particles with |a| >= {A_FLOOR} x rms |a| ({int(big.sum())} of {n})"}


def run_ensemble(args, rank, world, local, dist):
    """The batched-ensemble workload: 256 sets (log-uniform 1e4..5e5 particles, periodic
    uniform boxes and Plummer spheres), density / Newton-Raphson only.  Batched solves
    (plain and mixed) against 256 sequential plain FP64 single-set solves on the same GPU.
    On N GPUs the sets are packed onto the ranks by particle count (no exchange step);
    each rank times its own share and the job's time is the slowest rank's."""
    from cosmosphere_b200 import autotune, capi, inputs, shard
    sizes = inputs.ensemble_sizes(args.nsets)
    shares = shard.pack_sets(sizes, world)
    mine = shares[rank]
    sets = inputs.ensemble_sets(args.nsets, only=mine)
    n_all = int(sizes.sum())
    c = capi.Cosmo()
    c.set_device(local)
    res = {}
    outs = {}
    tuned = {}
    for mode in ("fp64", "mixed"):
        c.set_precision(mode == "mixed")
        untuned_ms = None
        if args.autotune == "on":
            # per size class, on this rank's sets, before anything is timed
            w0 = time.perf_counter()
            table = autotune.tune(sets, max_particles=args.tune_particles)
            table, t_tab, t_def = autotune.confirm(sets, table)
            tuned[mode] = {"seconds": time.perf_counter() - w0, "confirm_s": {"tuned": t_tab, "default": t_def},
                           "kept": "tuned" if table.entries else "default", **table.to_json()}
            b = capi.Batch(sets)
            b.set_staging(False)          # the untuned form: the library's default feed
            b.upload()
            for _ in range(args.warmup):
                assert b.density(final_rho=True) == 0
            tu = 0.0
            for _ in range(args.steps):
                assert b.density(final_rho=True) == 0
                tu += b.scalar("t_total")
            untuned_ms = 1e3 * shard.reduce_scalar(dist, tu, "max", device=f"cuda:{local}" if dist else None) / args.steps
        b = capi.Batch(sets)
        if args.autotune == "on":
            table.apply(b)
        b.upload()
        for _ in range(args.warmup):
            assert b.density(final_rho=True) == 0
        t = 0.0
        upd = 0.0
        tnr = 0.0
        barrier(dist, local)
        for _ in range(args.steps):
            assert b.density(final_rho=True) == 0
            t += b.scalar("t_total")
            tnr += b.scalar("t_nr")
            upd += b.scalar("updates")
        t_max = shard.reduce_scalar(dist, t, "max", device=f"cuda:{local}" if dist else None)
        upd_all = shard.reduce_scalar(dist, upd, "sum", device=f"cuda:{local}" if dist else None)
        # end to end: upload + solve + download through the batch C-ABI
        barrier(dist, local)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            b.upload()
            assert b.density(final_rho=True) == 0
            out = b.download()
        we = shard.reduce_scalar(dist, (time.perf_counter() - w0) / args.steps, "max",
                                 device=f"cuda:{local}" if dist else None)
        outs[mode] = out
        res[mode] = {"value": upd_all / t_max, "ms_per_solve": 1e3 * t_max / args.steps, "e2e_ms_per_solve": 1e3 * we,
                     "e2e_value": upd_all / args.steps / we,
                     "ms_newton_loop_graph": 1e3 * tnr / args.steps, "graph": b.scalar("graph") == 1.0,
                     "updates_per_solve": upd_all / args.steps, "iters": b.scalar("itersRun"),
                     "leaves_rank0": b.scalar("nLeaves"), "ms_per_solve_untuned": untuned_ms}
    c.set_precision(False)
    # sequential plain FP64 single-set solves
    tseq = 0.0
    useq = 0.0
    barrier(dist, local)
    for p in sets:
        c.arrays_init(p.n)
        c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
        c.upload(capi.HSML, p["h"])
        c.mark(5)
        assert c.density_status(p.n, p["pmass"], periodic_box=p.get("box"), with_gradients=False) == 0
        c.mark(6)
        tseq += c.elapsed(5, 6)
        useq += float(c.array("activePerIter").sum())
    tseq = shard.reduce_scalar(dist, tseq, "max", device=f"cuda:{local}" if dist else None)
    useq = shard.reduce_scalar(dist, useq, "sum", device=f"cuda:{local}" if dist else None)
    h0, r0 = np.concatenate(outs["fp64"][0]), np.concatenate(outs["fp64"][1])
    h1, r1 = np.concatenate(outs["mixed"][0]), np.concatenate(outs["mixed"][1])
    live = h0 > 0
    eh = shard.reduce_scalar(dist, float(np.max(np.abs(h1[live] / h0[live] - 1))), "max",
                             device=f"cuda:{local}" if dist else None)
    er = shard.reduce_scalar(dist, float(np.max(np.abs(r1[live] / r0[live] - 1))), "max",
                             device=f"cuda:{local}" if dist else None)
    if rank == 0:
        line = {"metric": f"batched density particle-updates/s ({args.nsets}-set ensemble)",
                "value": res["mixed"]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": res["mixed"]["ms_per_solve"], "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                "config": {"workload": f"{args.nsets} sets, log-uniform 1e4..5e5 particles, even: periodic uniform "
                                       "box, odd: Plummer r<20; h = 1.2 x spacing x U[0.8,1.2]; cubic; density/NR "
                                       "loop as one CUDA graph + rho at the converged h; launch parameters "
                                       + ("autotuned per size class" if args.autotune == "on" else "default"),
                           "particles": n_all,
                           "parallelism": f"sets packed on {world} GPU(s), largest first onto the least-loaded "
                                          f"(imbalance {shard.imbalance(sizes, shares):.3f})"},
                "e2e": {"value": res["mixed"]["e2e_value"], "unit": UNIT, "h2d_bytes_per_step": 8 * 4 * n_all,
                        "d2h_bytes_per_step": 8 * 3 * n_all},
                "batched_mixed": res["mixed"], "batched_fp64": res["fp64"],
                "sequential_fp64": {"value": useq / tseq, "ms_total": 1e3 * tseq, "updates": useq,
                                    "how": "one single-set plain FP64 solve per set through the C-ABI, device-timed"},
                "speedup_mixed_batched_vs_sequential_fp64": (res["mixed"]["value"]) / (useq / tseq),
                "speedup_mixed_vs_fp64_batched": res["mixed"]["value"] / res["fp64"]["value"],
                "accuracy_mixed_vs_fp64": {"h_max_rel": eh, "rho_max_rel": er},
                "autotune_rank0": tuned or None,
                "roofline": None, "cpu_baseline": None, "gpu_launches": None}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def profile_ensemble(args, local):
    """For ncu: the ensemble's sets solved as one batch, --warmup + --steps times, with the
    Newton loop driven from the host (each iteration's launches visible to the profiler),
    in the precision --precision names (fp64 or mixed), with the default launch parameters
    or (--autotune on) tuned ones; prints the last solve's counters."""
    from cosmosphere_b200 import autotune, capi, inputs
    sets = inputs.ensemble_sets(args.nsets)
    c = capi.Cosmo()
    c.set_device(local)
    c.set_precision(args.precision == "mixed")
    table = autotune.tune(sets, max_particles=args.tune_particles) if args.autotune == "on" else None
    b = capi.Batch(sets)
    if table is not None:
        table.apply(b)
    b.upload()
    for _ in range(args.warmup + args.steps):
        assert b.density(final_rho=True, graph=False) == 0
    print(json.dumps({"profile_solves": args.warmup + args.steps,
                      **{k: b.scalar(k) for k in ["t_total", "t_nr", "t_build", "itersRun", "nLeaves", "updates"]}}),
          flush=True)


def _served_fp64_loop(reqs):
    """The plain FP64 one-request-at-a-time loop through the C-ABI: per request upload,
    density, thermo, force and download of every output; a continuation drifts its set's
    positions on the host by v dt (wrapped in a periodic box) and restarts Newton from the
    set's last h.  Returns per-request service seconds, updates and (h, rho)."""
    from cosmosphere_b200 import capi
    c = capi.Cosmo()
    c.set_precision(False)
    last = {}
    serv, upd, res = [], [], []
    for k, e in enumerate(reqs):
        j = k if e["kind"] == "new" else e["of"]
        f = reqs[j]
        p, n = f["p"], f["n"]
        if e["kind"] == "new":
            pos, h = f["pos3"], np.ascontiguousarray(p["h"])
        else:
            pos, h = last[j]
            pos = pos + f["vel3"] * e["dt"]
            if p.get("box") is not None:
                pos = np.where(pos >= 1.0, pos - 1.0, np.where(pos < 0.0, pos + 1.0, pos))
        box = p.get("box")
        outs = {capi.HSML: np.empty((1, n)), capi.DENS_OUT: np.empty((2, n)), capi.GRAD_OUT: np.empty((3, n)),
                capi.FORCE_OUT: np.empty((6, n))}
        t0 = time.perf_counter()
        c.arrays_init(n)
        c.upload(capi.POS, pos, n)
        c.upload(capi.HSML, h, n)
        c.upload(capi.VEL, f["vel3"], n)
        c.upload(capi.ACCEL, np.zeros((3, n)), n)
        c.density(n, p["pmass"], tolh=1e-4, hfact=1.2, periodic_box=box)
        c.upload(capi.THERMO, f["thermo4"], n, sorted_=True)
        c.force(n, p["pmass"], beta=2.0, alphau=0.0, disc=0, pdv=1, shock=1)
        for slot, buf in outs.items():
            c.download(slot, n, buf)
        serv.append(time.perf_counter() - t0)
        upd.append(float(c.array("activePerIter").sum() + c.scalar("nAlive")))
        last[j] = (pos, outs[capi.HSML][0].copy())
        res.append((outs[capi.HSML][0], outs[capi.DENS_OUT][0]))
    return serv, upd, res


def _served_run(reqs, arrivals, slots, budget_gb):
    """Submit the requests to the served form at their arrival times (seconds after the
    start); returns per-request latency, updates, (h, rho) and the makespan."""
    from cosmosphere_b200 import capi
    srv = capi.Server(slots=slots, budget_gb=budget_gb)
    rid = []
    try:
        t0 = time.perf_counter()
        for k, e in enumerate(reqs):
            dly = t0 + arrivals[k] - time.perf_counter()
            if dly > 0:
                time.sleep(dly)
            if e["kind"] == "new":
                p = e["p"]
                rid.append(srv.submit({"x": p["x"], "y": p["y"], "z": p["z"], "h": p["h"], "pmass": p["pmass"],
                                       "vx": p["vx"], "vy": p["vy"], "vz": p["vz"]}, e["thermo4"],
                                      box=p.get("box"), hfact=1.2, keep=True))
            else:
                rid.append(srv.cont(rid[e["of"]], e["dt"]))
        res, lat, upd, subm, done = [], [], [], [], []
        for r in rid:
            st, o = srv.wait(r)
            if st != 1:
                raise RuntimeError(f"served request {r} ended with status {st}")
            res.append((o["h"], o["dens"][0]))
            lat.append(srv.stat(r, "latency"))
            upd.append(srv.stat(r, "updates"))
            subm.append(srv.stat(r, "submit"))
            done.append(srv.stat(r, "done"))
        info = {"max_inflight": srv.server_stat("max_inflight"), "evicted": srv.server_stat("evicted"),
                "rejected": srv.server_stat("rejected"), "resident_sets_at_end": srv.server_stat("resident_sets"),
                "device_bytes_at_end": srv.server_stat("device_bytes")}
        makespan = max(done) - min(subm)
    finally:
        srv.stop()
    return lat, upd, res, makespan, info


def run_served(args, rank, world, local, dist):
    """The served stream: requests with particle counts log-uniform in [5e3, 2e6] from the
    lattice / periodic-uniform / Plummer generators, 30% continuing a device-resident set
    (drift by v dt, dt = 0.1 min(h/c_s), Newton warm-started from the last h), admitted
    against an HBM budget, mixed precision; against the plain FP64 one-request-at-a-time
    loop through the C-ABI."""
    from cosmosphere_b200 import capi, inputs, shard
    # on N GPUs each rank serves its share of the stream (new sets packed by particle
    # count, continuations with their set); latencies are gathered, the job's makespan is
    # the slowest rank's
    skeleton = inputs.served_requests(args.nreq, seed=42, only=[])
    owner = shard.pack_requests(skeleton, world)
    mine = [k for k in range(len(skeleton)) if owner[k] == rank]
    tg = time.perf_counter()
    full = inputs.served_requests(args.nreq, seed=42, only=mine)
    tg = time.perf_counter() - tg
    local_of = {k: i for i, k in enumerate(mine)}
    reqs = []
    for k in mine:
        e = dict(full[k])
        if e["kind"] == "cont":
            e["of"] = local_of[e["of"]]
        reqs.append(e)
    dev = f"cuda:{local}" if dist else None
    c = capi.Cosmo()
    c.set_device(local)
    # warm-up: the CUDA context and the FP64 loop's buffers at the largest size
    big = max((e for e in reqs if e["kind"] == "new"), key=lambda e: e["n"])
    _served_fp64_loop([big])
    serv, upd64, res64 = _served_fp64_loop(reqs)
    total_upd = float(np.sum(upd64))
    sum_local_serv = float(np.sum(serv))
    cap64 = total_upd / sum_local_serv
    # Poisson arrivals at `load` x the FP64 loop's request rate
    rate = args.serve_load * len(reqs) / float(np.sum(serv))
    rng = np.random.default_rng(7)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    arrivals -= arrivals[0]
    # the FP64 loop's latencies under the same arrivals (one request at a time, FIFO)
    lat64, free = [], 0.0
    for a, s_ in zip(arrivals, serv):
        start = max(a, free)
        free = start + s_
        lat64.append(free - a)
    make64 = free - arrivals[0]
    c.set_precision(True)
    # warm-up: one saturated pass of the whole stream, so the device memory pool and the
    # pinned scalar blocks hold what the stream needs (a long-running server's state)
    _served_run(reqs, np.zeros(len(reqs)), args.slots, args.budget_gb)
    lat, upd, res, makespan, info = _served_run(reqs, arrivals, args.slots, args.budget_gb)
    # saturated: every request at t = 0
    lat_b, upd_b, _, make_b, info_b = _served_run(reqs, np.zeros(len(reqs)), args.slots, args.budget_gb)
    c.set_precision(False)
    red = lambda v, op: shard.reduce_scalar(dist, v, op, device=dev)
    eh = red(max(float(np.max(np.abs(a[0] / b[0] - 1.0))) for a, b in zip(res, res64)), "max")
    er = red(max(float(np.max(np.abs(a[1] / b[1] - 1.0))) for a, b in zip(res, res64)), "max")
    nnew = int(red(sum(1 for e in reqs if e["kind"] == "new"), "sum"))
    nall = int(red(len(reqs), "sum"))
    bytes_in = red(sum(8 * e["n"] * 11 for e in reqs if e["kind"] == "new"), "sum")
    bytes_out = red(sum(8 * 12 * reqs[k if e["kind"] == "new" else e["of"]]["n"] for k, e in enumerate(reqs)), "sum")
    pnew = int(red(sum(e["n"] for e in reqs if e["kind"] == "new"), "sum"))
    lat, lat_b, lat64 = (shard.gather_floats(dist, v, world) for v in (lat, lat_b, lat64))
    serv = shard.gather_floats(dist, serv, world)
    pct = lambda a, q: float(np.percentile(np.asarray(a) * 1e3, q))
    thr_stream = red(float(np.sum(upd)), "sum") / red(makespan, "max")
    thr_sat = red(float(np.sum(upd_b)), "sum") / red(make_b, "max")
    makespan, make_b, make64 = red(makespan, "max"), red(make_b, "max"), red(make64, "max")
    total_upd = red(total_upd, "sum")
    cap64 = total_upd / red(sum_local_serv, "max")
    rate = red(rate, "sum")
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {"metric": "served density+force particle-updates/s (Poisson stream, 5e3..2e6 particles)",
            "value": thr_sat, "unit": UNIT, "n_gpus": world, "steps": nall, "warmup": 1,
            "ms_per_step": 1e3 * make_b / nall, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"{nall} requests ({nnew} new sets, {nall - nnew} continuations), "
                                   "counts log-uniform 5e3..2e6 from lattice+jiggle / periodic uniform box / "
                                   "Plummer (cubic), density(NR+gradients)+force, dt = 0.1 min(h/c_s)",
                       "particles_new": pnew,
                       "slots": args.slots, "hbm_budget_gb": args.budget_gb,
                       "offered_load": f"Poisson at {args.serve_load} x the FP64 loop's request rate "
                                       f"({rate:.1f} req/s over all GPUs)",
                       "parallelism": f"requests packed on {world} GPU(s) by particle count, continuations "
                                      "with their set",
                       "input_generation_s": tg},
            "e2e": {"value": thr_sat, "unit": UNIT, "h2d_bytes_per_step": bytes_in / nall,
                    "d2h_bytes_per_step": bytes_out / nall,
                    "how": "every request through the served C-ABI from host buffers: copy at submission, "
                           "H2D, solve, D2H of all outputs"},
            "served_mixed": {"stream": {"p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "max_ms": pct(lat, 100),
                                        "throughput": thr_stream, "makespan_s": makespan, **info},
                             "saturated": {"throughput": thr_sat, "makespan_s": make_b, "p50_ms": pct(lat_b, 50),
                                           "p99_ms": pct(lat_b, 99), **info_b}},
            "fp64_loop": {"stream": {"p50_ms": pct(lat64, 50), "p99_ms": pct(lat64, 99), "max_ms": pct(lat64, 100),
                                     "throughput": total_upd / make64, "makespan_s": make64},
                          "capacity": cap64, "service_p50_ms": pct(serv, 50), "service_p99_ms": pct(serv, 99),
                          "how": "plain FP64, one request at a time through the C-ABI, wall-timed per request; "
                                 "stream latencies from the same arrivals, FIFO"},
            "speedup_saturated_vs_fp64_loop": thr_sat / cap64,
            "accuracy_mixed_vs_fp64": {"h_max_rel": eh, "rho_max_rel": er},
            "roofline": None, "cpu_baseline": None, "gpu_launches": None}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_reference(args, rank, world, local, dist):
    """The CPU arm: the oracle port of the path, all host threads, a bounded sample."""
    if rank != 0:
        return
    sample_npx = args.ref_npartx
    p = workload(sample_npx)
    for _ in range(args.warmup):
        cpu_oracle_step(p)
    upd = 0.0
    t = 0.0
    cores = 0
    for _ in range(args.steps):
        u, dt, cores = cpu_oracle_step(p)
        upd += u
        t += dt
    v = upd / t
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": lattice_label(sample_npx), "particles": p.n, "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "same_config": sample_npx == args.npartx,
                             "sample": (f"the workload itself ({p.n} particles), one density+force step of the "
                                        "CPU oracle (FP64, OpenMP, all host threads) per step")
                                       if sample_npx == args.npartx else
                                       f"lattice-{sample_npx} instance of the lattice-100 generator ({p.n} "
                                       "particles), one density+force step per step"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--npartx", type=int, default=100)
    ap.add_argument("--periodic", action="store_true",
                    help="lattice workloads: solve in the unit periodic box [0,1)^3 instead of open boundaries")
    ap.add_argument("--ref-npartx", type=int, default=100,
                    help="lattice size of the CPU arm's workload (default: the timed workload itself)")
    ap.add_argument("--no-forms", action="store_true",
                    help="lattice100: leave out the batched-ensemble and served-stream legs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                    help="both: plain FP64 (the headline value) and mixed in one run")
    ap.add_argument("--workload", default="lattice100", choices=["lattice100", "plummer", "ensemble", "served", "file"])
    ap.add_argument("--input-file", default=None, help="file: a particle file in the reference's Fortran layout")
    ap.add_argument("--jiggle", action="store_true", help="file: perturb h of ~1%% of the particles first")
    ap.add_argument("--plummer-n", type=int, default=2000000)
    ap.add_argument("--nreq", type=int, default=64, help="served: requests in the stream")
    ap.add_argument("--slots", type=int, default=4, help="served: worker slots")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: HBM budget")
    ap.add_argument("--serve-load", type=float, default=0.9,
                    help="served: Poisson rate as a multiple of the FP64 loop's request rate")
    ap.add_argument("--nsets", type=int, default=256)
    ap.add_argument("--autotune", default="on", choices=["on", "off"],
                    help="ensemble: tune the batched form per size class before timing")
    ap.add_argument("--tune-particles", type=float, default=2.0e6,
                    help="ensemble: particles in the sample of each size class the tuner times")
    ap.add_argument("--profile", action="store_true",
                    help="for ncu: set up, run --warmup and --steps device-resident steps, print nothing else")
    args = ap.parse_args()
    if not args.profile:
        args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        # host cores only: rank 0 times the CPU arm, the other ranks exit at once; no
        # process group is needed for that
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0, None)
        return
    rank, world, local, dist = dist_setup(args)
    if args.workload == "ensemble":
        if args.profile:
            profile_ensemble(args, local)
        else:
            run_ensemble(args, rank, world, local, dist)
        return
    if args.workload == "served":
        run_served(args, rank, world, local, dist)
        return

    if args.workload == "file":
        run_file(args, rank, world, local, dist)
        return
    if args.workload == "plummer":
        run_particles(args, rank, world, local, dist, plummer_workload(args.plummer_n), quintic=True,
                      metric="density+force particle-updates/s (Plummer 2M, quintic)",
                      label=f"Plummer a=1 r<20, {args.plummer_n} particles, h = (m/rho)^(1/3) x lognormal(0.3), "
                            "|v| = 0.5 v_circ, u = 0.05, quintic, hfact 1.0, density(NR+gradients)+force, open")
        return
    p = workload(args.npartx)
    if args.periodic:
        p["box"] = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
    run_particles(args, rank, world, local, dist, p, quintic=False, metric=METRIC,
                  label=lattice_label(args.npartx, args.periodic))


def lattice_label(npx, periodic=False):
    return (f"lattice {npx} + 1% h-jiggle U[0.65,1.35], density(NR+gradients)+force, cubic, "
            + ("unit periodic box" if periodic else "open boundaries"))


def run_file(args, rank, world, local, dist):
    """A particle file in the reference's Fortran record layout (a dump with x, y, z, h
    and pmass): density / Newton-Raphson solves through the C-ABI, plain FP64 and mixed,
    in particle-updates/s (Newton updates), as the reference's standalone driver times it.
    With --jiggle, h of ~1% of the particles is perturbed first as that driver does."""
    from cosmosphere_b200 import capi, dumpio, inputs
    if not args.input_file:
        raise SystemExit("--workload file needs --input-file PATH")
    p = dumpio.read_particles(args.input_file)
    if args.jiggle:
        inputs.jiggle_ref(p["h"], 42)
    n = p.n
    c = capi.Cosmo()
    c.set_device(local)
    pos = np.ascontiguousarray(np.stack([p["x"], p["y"], p["z"]]))
    h0 = np.ascontiguousarray(p["h"])
    hout = np.empty(n)
    res = {}
    for mode in ("fp64", "mixed"):
        c.set_precision(mode == "mixed")
        c.arrays_init(n)
        for _ in range(args.warmup):
            c.upload(capi.POS, pos, n); c.upload(capi.HSML, h0, n)
            c.density(n, p["pmass"])
        t = upd = 0.0
        barrier(dist, local)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            c.upload(capi.POS, pos, n); c.upload(capi.HSML, h0, n)
            c.mark(0)
            c.density(n, p["pmass"])
            c.mark(1)
            c.download(capi.HSML, n, hout)
            t += c.elapsed(0, 1)
            upd += float(c.array("activePerIter").sum())
        we = time.perf_counter() - w0
        res[mode] = {"value": sum_over_ranks(dist, local, upd) / max_over_ranks(dist, local, t),
                     "e2e_value": sum_over_ranks(dist, local, upd) / max_over_ranks(dist, local, we),
                     "ms_per_solve": 1e3 * t / args.steps, "iters": len(c.array("activePerIter"))}
    c.set_precision(False)
    if rank == 0:
        print(json.dumps({
            "metric": "density particle-updates/s (particle file)", "value": res["fp64"]["value"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["fp64"]["ms_per_solve"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": os.path.basename(args.input_file),
            "config": {"workload": f"{args.input_file}: {n} particles, pmass {p['pmass']:.6e}"
                                   + (", jiggled" if args.jiggle else "") + "; density/NR only",
                       "particles": n, "parallelism": f"replicas x{world}"},
            "e2e": {"value": res["fp64"]["e2e_value"], "unit": UNIT, "h2d_bytes_per_step": 32 * n,
                    "d2h_bytes_per_step": 8 * n},
            "plain_fp64": res["fp64"], "mixed": res["mixed"],
            "roofline": None, "cpu_baseline": None, "gpu_launches": None}), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def plummer_workload(n, seed=42):
    """The clustered deep-tree workload: a Plummer sphere (a = 1, r < 20) of n particles,
    h = hfact (m / rho_Plummer)^(1/3) x lognormal(0.3) with hfact 1.0, velocities isotropic
    at 0.5 x the circular speed, u = 0.05, gamma = 5/3, alpha_AV = 1 (quintic kernel)."""
    from cosmosphere_b200 import inputs
    p = inputs.plummer(n, rmax=20.0, hfact=1.0, lnsigma=0.3, vfrac=0.5, seed=seed)
    th = inputs._thermo(p, 0.05, hfact=1.0)
    p["pro2"], p["cs"], p["alpha"], p["u"] = th[0], th[1], th[2], th[3]
    p["hfact"] = 1.0
    return p


def measure(args, c, p, mixed, hfact, dist, local, profile=False):
    """Device-resident and end-to-end timing of density + force steps of one precision."""
    from cosmosphere_b200 import capi
    n = p.n
    pm = p["pmass"]
    box = p.get("box")
    pos = np.ascontiguousarray(np.stack([p["x"], p["y"], p["z"]]))
    hsml = np.ascontiguousarray(p["h"])
    vel = np.ascontiguousarray(np.stack([p["vx"], p["vy"], p["vz"]]))
    acc = np.zeros((3, n))
    thermo = np.ascontiguousarray(np.stack([p["pro2"], p["cs"], p["alpha"], p["u"]]))
    outs = {capi.HSML: np.empty((1, n)), capi.DENS_OUT: np.empty((2, n)), capi.GRAD_OUT: np.empty((3, n)),
            capi.FORCE_OUT: np.empty((6, n))}
    for a in [pos, hsml, vel, acc, thermo] + list(outs.values()):
        c.pin(a)
    c.arrays_init(n)
    c.set_precision(mixed)

    def upload_inputs():
        c.upload(capi.POS, pos, n)
        c.upload(capi.HSML, hsml, n)
        c.upload(capi.VEL, vel, n)
        c.upload(capi.ACCEL, acc, n)

    def step_resident():
        c.density(n, pm, tolh=1e-4, hfact=hfact, periodic_box=box)
        c.force(n, pm, beta=2.0, alphau=0.0, disc=0, pdv=1, shock=1)

    def step_e2e():
        upload_inputs()
        c.density(n, pm, tolh=1e-4, hfact=hfact, periodic_box=box)
        c.upload(capi.THERMO, thermo, n, sorted_=True)
        c.force(n, pm, beta=2.0, alphau=0.0, disc=0, pdv=1, shock=1)
        for slot, buf in outs.items():
            c.download(slot, n, buf)

    # inputs resident; THERMO gathered into Hilbert order once (every step sorts the same input)
    upload_inputs()
    c.density(n, pm, tolh=1e-4, hfact=hfact, periodic_box=box)
    c.upload(capi.THERMO, thermo, n, sorted_=True)
    for _ in range(args.warmup):
        step_resident()
    if profile:
        for _ in range(args.steps):
            step_resident()
        c.sync()
        return {"nr_iterations": len(c.array("activePerIter"))}
    barrier(dist, local)
    c.sync()
    launches0 = c.launches()
    upd_step = 0.0
    t_nr = t_fk = t_gk = 0.0
    pairs = nr_upd = 0.0
    nr_launches = 0
    c.mark(0)
    for _ in range(args.steps):
        step_resident()
        act = c.array("activePerIter")
        upd_step = float(act.sum() + c.scalar("nAlive"))
        nr_upd += float(act.sum())
        nr_launches += len(act)
        t_nr += c.scalar("t_nrkern")
        t_gk += c.scalar("t_gradkern")
        t_fk += c.scalar("t_fkern")
        pairs += c.scalar("pairsDensity")
    c.mark(1)
    t_dev = c.elapsed(0, 1)
    c.sync()
    barrier(dist, local)
    launches = c.launches() - launches0
    t_max = max_over_ranks(dist, local, t_dev)
    upd_total = sum_over_ranks(dist, local, upd_step * args.steps)
    # end to end through the C-ABI
    for _ in range(args.warmup):
        step_e2e()
    barrier(dist, local)
    c.sync()
    c.mark(2)
    w0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    c.mark(3)
    t_e2e_dev = c.elapsed(2, 3)
    t_e2e_wall = time.perf_counter() - w0
    barrier(dist, local)
    t_e2e = max_over_ranks(dist, local, max(t_e2e_dev, t_e2e_wall))
    res = {"value": upd_total / t_max, "ms_per_step": 1e3 * t_max / args.steps,
           "e2e_value": upd_total / t_e2e, "e2e_ms_per_step": 1e3 * t_e2e / args.steps,
           "updates_per_step": upd_step, "nr_iterations": len(act), "launches": launches,
           "kernel_ms_per_step": {"density_nr": 1e3 * t_nr / args.steps, "gradient": 1e3 * t_gk / args.steps,
                                  "force": 1e3 * t_fk / args.steps},
           "t_nr": t_nr, "nr_upd": nr_upd, "pairs": pairs, "nr_launches": nr_launches,
           "h2d": 8 * n * (3 + 1 + 3 + 3 + 4), "d2h": 8 * n * (1 + 2 + 3 + 6)}
    c.set_precision(False)
    for a in [pos, hsml, vel, acc, thermo] + list(outs.values()):
        c.unpin(a)
    return res


def newton_cap_report(c, p, hfact):
    """The same density solve with the Newton cap at 10 iterations (the iteration cap the
    specification names; the library's default is the reference's built 100): whether it
    converges within 10, and how many particles are left unconverged if not."""
    from cosmosphere_b200 import capi
    n = p.n
    c.set_precision(False)
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    st10 = c.density_status(n, p["pmass"], tolh=1e-4, hfact=hfact, max_iter=10, with_gradients=False)
    unconv10 = int(c.scalar("unconverged")) if st10 == 1 else 0
    act10 = [int(a) for a in c.array("activePerIter")]
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    st100 = c.density_status(n, p["pmass"], tolh=1e-4, hfact=hfact, max_iter=100, with_gradients=False)
    return {"cap": 10, "status": "converged" if st10 == 0 else ("unconverged" if st10 == 1 else f"status {st10}"),
            "unconverged_particles": unconv10, "active_per_iteration": act10,
            "iterations_to_converge_with_cap_100": int(c.scalar("itersRun")) if st100 == 0 else None}


def run_form_legs(args):
    """The batched-ensemble and served-stream forms, each run as its own bench.py process
    on this GPU after the lattice-100 timing; their headline figures are carried on this
    line (their full lines come from --workload ensemble / served)."""
    out = {}
    legs = {"batched_ensemble": ["--workload", "ensemble", "--steps", "3", "--warmup", "1"],
            "served_stream": ["--workload", "served"]}
    for name, extra in legs.items():
        t0 = time.perf_counter()
        r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "1", *extra],
                           capture_output=True, text=True, timeout=900)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not lines:
            out[name] = {"error": (r.stderr or r.stdout).strip().splitlines()[-1:] or ["no output"]}
            continue
        d = json.loads(lines[-1])
        d["wall_s"] = time.perf_counter() - t0
        if name == "batched_ensemble":
            out[name] = {"metric": d["metric"], "value": d["value"], "unit": d["unit"], "config": d["config"],
                         "speedup_mixed_batched_vs_sequential_fp64": d["speedup_mixed_batched_vs_sequential_fp64"],
                         "speedup_mixed_vs_fp64_batched": d["speedup_mixed_vs_fp64_batched"],
                         "batched_mixed_ms_per_solve": d["batched_mixed"]["ms_per_solve"],
                         "batched_fp64_ms_per_solve": d["batched_fp64"]["ms_per_solve"],
                         "sequential_fp64_ms_total": d["sequential_fp64"]["ms_total"],
                         "accuracy_mixed_vs_fp64": d["accuracy_mixed_vs_fp64"], "steps": d["steps"],
                         "wall_s": d["wall_s"]}
        else:
            sm, fl = d["served_mixed"], d["fp64_loop"]
            out[name] = {"metric": d["metric"], "value": d["value"], "unit": d["unit"], "config": d["config"],
                         "p50_ms": sm["stream"]["p50_ms"], "p99_ms": sm["stream"]["p99_ms"],
                         "fp64_loop_p50_ms": fl["stream"]["p50_ms"], "fp64_loop_p99_ms": fl["stream"]["p99_ms"],
                         "speedup_saturated_vs_fp64_loop": d["speedup_saturated_vs_fp64_loop"],
                         "accuracy_mixed_vs_fp64": d["accuracy_mixed_vs_fp64"], "requests": d["steps"],
                         "wall_s": d["wall_s"]}
    return out


def run_particles(args, rank, world, local, dist, p, quintic, metric, label):
    """One set of particles: the plain FP64 form (the headline value) and the mixed form,
    with the mixed form's error against FP64 on the same inputs."""
    from cosmosphere_b200 import capi
    c = capi.Cosmo(quintic=quintic)
    c.set_device(local)
    n = p.n
    hfact = p.get("hfact", 1.2)
    if args.profile:
        r = measure(args, c, p, args.precision == "mixed", hfact, dist, local, profile=True)
        print(json.dumps({"profile_steps": args.steps, "particles": n, **r}), flush=True)
        return
    accuracy = None
    if args.precision in ("mixed", "both"):
        pos = np.ascontiguousarray(np.stack([p["x"], p["y"], p["z"]]))
        hsml = np.ascontiguousarray(p["h"])
        vel = np.ascontiguousarray(np.stack([p["vx"], p["vy"], p["vz"]]))
        acc = np.zeros((3, n))
        thermo = np.ascontiguousarray(np.stack([p["pro2"], p["cs"], p["alpha"], p["u"]]))
        outs = {capi.HSML: np.empty((1, n)), capi.DENS_OUT: np.empty((2, n)), capi.GRAD_OUT: np.empty((3, n)),
                capi.FORCE_OUT: np.empty((6, n))}
        c.arrays_init(n)
        accuracy = mixed_accuracy(c, p, n, pos, hsml, vel, acc, thermo, outs, hfact)
    clocks = ClockSampler(local)
    time.sleep(0.3)
    plain = measure(args, c, p, False, hfact, dist, local) if args.precision in ("fp64", "both") else None
    mixed = measure(args, c, p, True, hfact, dist, local) if args.precision in ("mixed", "both") else None
    clk = clocks.stop()
    head = plain if plain is not None else mixed
    # roofline of the Newton density kernel (the largest single kernel of the step)
    fp64_peak = c.fp64_peak_tflops()
    flops = FLOP_PER_DENSITY_PAIR * head["pairs"] + FLOP_PER_NR_UPDATE * head["nr_upd"]
    achieved = flops / head["t_nr"] / 1e12
    peaks, src = measured_peaks()
    hbm_achieved = BYTES_PER_DENSITY_UPDATE * head["nr_upd"] / head["t_nr"] / 1e9
    kname = ("Newton stage, per iteration: density_nr_kernel + newton_rows_kernel + density_row_kernel "
             "+ plan_items_kernel, timed together by CUDA events")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not quintic:
        same = args.ref_npartx == args.npartx and args.workload == "lattice100"
        cp = p if same else workload(args.ref_npartx)
        u, dt, cores = cpu_oracle_step(cp)
        cpu = {"value": u / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "same_config": same,
               "sample": (f"the timed workload itself ({cp.n} particles), one density+force step of the CPU "
                          "oracle (FP64, OpenMP, all host threads)") if same else
                         (f"lattice-{args.ref_npartx} instance of the same generator ({cp.n} particles), "
                          "one density+force step of the CPU oracle (FP64, OpenMP)")}
    forms = None
    if rank == 0 and world == 1 and args.workload == "lattice100" and not args.no_forms and not quintic:
        forms = run_form_legs(args)
    cap10 = None
    if args.workload == "plummer":
        cap10 = newton_cap_report(c, p, hfact)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    strip = lambda r: None if r is None else {k: v for k, v in r.items()
                                              if k not in ("t_nr", "nr_upd", "pairs", "nr_launches", "h2d", "d2h")}
    line = {
        "metric": metric, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if plain is not None else "f32+f64", "data": "synthetic",
        "precision": "fp64" if plain is not None else "mixed",
        "config": {"workload": label, "particles": n, "particles_per_gpu": n,
                   "nr_iterations": head["nr_iterations"], "updates_per_step": head["updates_per_step"],
                   "parallelism": f"replicas x{world}", "l2": "working set above the 126 MB L2 (no flush needed)"},
        "e2e": {"value": head["e2e_value"], "unit": UNIT, "h2d_bytes_per_step": head["h2d"],
                "d2h_bytes_per_step": head["d2h"], "ms_per_step": head["e2e_ms_per_step"]},
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": hbm_achieved, "peak": peaks.get("hbm_gbs"),
                     "unit": "GB/s", "frac": hbm_achieved / peaks.get("hbm_gbs"), "peak_source": src,
                     "byte_convention": "56 B per particle-update (read x, y, z, h; write h, rho, dh, flag)",
                     "algorithmic_bytes_per_iteration": BYTES_PER_DENSITY_UPDATE * head["nr_upd"]
                                                        / max(1, head["nr_launches"]),
                     "traffic": (ncu_traffic("newton_stage_per_iteration")
                                 if args.workload == "lattice100" and args.npartx == 100 and not quintic
                                 and not args.periodic else None),
                     "traffic_note": "DRAM bytes per Newton iteration assembled from one-kernel ncu captures "
                                     "(profiles/traffic.json, method in its note); above the algorithmic bytes "
                                     "because the Newton rows (r^2 per pair) are written once and streamed by the "
                                     "later iterations",
                     "fp64": {"achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                              "flop_convention": "30 FLOP per accepted pair + 30 per Newton update",
                              "peak_source": "FP64 FMA microkernel run in this bench "
                                             "(MEASURED_PEAKS.json has no FP64 figure)"},
                     "launch_ms": 1e3 * head["t_nr"] / max(1, head["nr_launches"])},
        "kernel_ms_per_step": head["kernel_ms_per_step"],
        "plain_fp64": strip(plain),
        "mixed": None if mixed is None else {**strip(mixed),
                                             "speedup_vs_plain": (mixed["value"] / plain["value"]) if plain else None,
                                             "accuracy_vs_fp64": accuracy},
        "cpu_baseline": cpu,
        "forms": forms,
        "newton_cap_10": cap10,
        "clocks": clk,
        "gpu_launches": head["launches"],
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
