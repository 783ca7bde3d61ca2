"""Benchmark: impurity solves/s of the large single-solve workload on B200.

Workload (aim_n12): single-orbital Anderson impurity with 11 bath sites
(nsite 12), U = 3, half filling, bath eps ~ U(-2,2), V ~ U(0.1,1) from seed
12; ground state over the 9 sectors n_up, n_dn in {5,6,7} (largest dimension
C(12,6)^2 = 853,776) with 300 Lanczos steps, then the Green's function: c
and c^+ Lanczos runs of 300 steps on the impurity orbital and the continued
fraction on 2048 Matsubara points (beta = 100).  A step is one full solve
(ground_state + cluster_green_ftn of the reference).  Inputs are synthetic
and seeded: the reference quotes no data set.

  value      solves/s, device time (CUDA events on the solver's stream) of
             each solve, L2 flushed (a 256 MiB write) between timed solves
  e2e        the same through the C ABI with host buffers: the model and the
             frequency grid copied in, the ground-state vector (gs%vec),
             G_cl and the Lanczos coefficients copied out, every step
  roofline   the persistent Lanczos kernel: algorithmic bytes / its measured
             device time against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (restatement of the reference's algorithm) on
             this host's cores, on a bounded sample of the workload
  plain_gpu  the reference's Lanczos structure run kernel by kernel on the
             same GPU (the one-solve-at-a-time drop-in comparator)
  hv         standalone H.v (edzt_hx) at nsite 12/14/16: GB/s at 16 B per
             state against the measured HBM peak
  batched    the batched form: the first --batched instances of the seeded
             256-instance draw (nsite ~ U{8..14}) in one edzt_solve_batch call
             per GPU (on N GPUs each rank solves its cost-balanced share),
             solves/s, with the plain engine's solves/s on the same instances
             (one per nsite timed, weighted by counts)
  served     the served form (one GPU): --served requests of the workload's
             nsite 8..16 distribution, Poisson arrivals at 200/s (saturation),
             through edzt_server's request loop: solves/s and p50/p99 latency
             from arrival to result; a second run below saturation (half the
             measured throughput) with the small requests' p50 against their
             solve-alone time; the plain engine's solves/s on the same requests

--impl reference times the CPU oracle on all host threads (the reference
itself is Fortran + MPI + MKL and cannot be built here).
"""

from __future__ import annotations

import argparse
import importlib
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "dmft-ed-zt_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "impurity solves/s (nsite 12, 9 sectors, 300 Lanczos steps, G on 2048 Matsubara points)"
UNIT = "solves/s"
FALLBACK_HBM_GBS = 6650.0


def load_pkg():
    name = "dmft_ed_zt_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload():
    load_pkg()
    cfgs = importlib.import_module("dmft_ed_zt_b200.configs")
    return cfgs.aim_n12()


def config_dict(cfg, n_gpus):
    return {"workload": "aim_n12 single impurity solve", "nsite": 12, "norb": 1, "nbath": 11,
            "sectors": "n_up,n_dn in {5,6,7}", "max_dim": 853776, "lanczos_steps": cfg["maxnstep"],
            "nw": cfg["nw"], "beta": cfg["beta"], "parallelism": f"replicas x{n_gpus}",
            "l2": "flushed between timed solves (256 MiB write)"}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"edzt_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs (the oracle: test infrastructure, used here only as the baseline)
# ---------------------------------------------------------------------------
def plain_estimate(pkg, s, items, omega, maxnstep):
    """Plain one-solve-at-a-time GPU engine time per solve, measured on one
    item per nsite and weighted by the items' nsite counts."""
    import numpy as np
    import torch
    by_ns = {}
    for it in items:
        by_ns.setdefault(it["model"].nsite, []).append(it)
    s.set_engine(pkg.ENGINE_PLAIN)
    total = 0.0
    per_ns = {}
    try:
        for ns, group in sorted(by_ns.items()):
            it = group[0]
            s.set_model(it["model"])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.solve(it["sectors"], maxnstep, omega, nspin=it.get("nspin", 1), seed=it.get("seed", 0))
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            per_ns[int(ns)] = round(1000 * dt, 2)
            total += dt * len(group)
    finally:
        s.set_engine(pkg.ENGINE_FUSED)
    return len(items) / total, per_ns


def batched_leg(pkg, s, cfgs, n, dist=None, rank=0, world=1):
    """The batched form: the first n instances of the seeded 256-instance draw
    (nsite ~ U{8..14}, 9 or 4 sectors within one electron of half filling,
    nspin 2: 4 c/c^+ runs each).  On one GPU one edzt_solve_batch call; on N
    GPUs every rank solves its cost-balanced share (replicas.sharded_batch)
    and the results are gathered, with the time taken as the max over
    ranks."""
    import numpy as np
    import torch
    replicas = importlib.import_module("dmft_ed_zt_b200.replicas")
    insts = cfgs.batch(256)[:n]
    omega = pkg.matsubara(2048, 100.0)
    costs = [replicas.instance_cost(i, 300) for i in insts]
    mine = replicas.my_units(costs, rank, world)
    s.solve_batch([insts[i] for i in mine[:2]] or insts[:2], 300, omega)   # warm-up (tables, pool)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    res, mine = replicas.sharded_batch(lambda lst: s.solve_batch(lst, 300, omega), insts, 300, rank, world, dist)
    torch.cuda.synchronize()
    dt = replicas.max_over_ranks(time.perf_counter() - t0, dist, device="cuda")
    out = {"value": n / dt, "unit": "solves/s", "instances": n, "seconds": dt, "n_gpus": world,
           "nsite_counts_8_to_14": np.bincount([i["model"].nsite for i in insts], minlength=15)[8:15].tolist(),
           "sample": (f"all 256 seeded instances (seed 4)" if n >= 256 else
                      f"first {n} of the 256 seeded instances (seed 4)") +
                     (", wall clock of one call, synchronised" if world == 1 else
                      f", split over {world} GPUs by cost (LPT), max over ranks of each rank's synchronised "
                      "wall clock, results gathered")}
    if rank == 0:
        plain, per_ns = plain_estimate(pkg, s, insts, omega, 300)
        out["plain_gpu"] = {"value": plain, "unit": "solves/s", "ms_per_solve_by_nsite": per_ns,
                            "how": "one instance per nsite timed on one GPU, weighted by counts"}
    return out


def _served_requests(pkg, cfgs, n, seed, nsite_max):
    import numpy as np
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        ns = int(rng.integers(8, nsite_max + 1))
        nb = ns - 1
        U = float(rng.uniform(1.0, 4.0))
        ek = rng.uniform(-2.0, 2.0, nb)
        V = rng.uniform(0.1, 1.0, nb)
        m = pkg.Model(1, nb, np.zeros((1, 2)), np.stack([ek, ek], 1), np.stack([V, V], 1).reshape(1, nb, 2),
                      U=U, mu=U / 2)
        reqs.append(dict(model=m, sectors=cfgs.near_half_sectors(ns), nspin=2, seed=int(rng.integers(1 << 40))))
    return reqs, rng


def _serve_run(pkg, s, reqs, arrivals, omega):
    sv = pkg.Server(s, 300, omega)
    try:
        _, lat, total = pkg.serve(sv, reqs, arrivals)
    finally:
        sv.close()
    return lat, total


def served_leg(pkg, s, cfgs, n, seed=5, nsite_max=16, sub=12):
    """The served form, requests of the workload's distribution: nsite ~
    U{8..nsite_max}, random U, J = 0, bath as the batched form, nspin 2,
    through edzt_server's request loop (pkg.serve), latency from arrival to
    result.
      saturation    n requests, Poisson arrivals at 200/s (seed 5): solves/s,
                    p50/p99 overall and by nsite
      sub-saturation  `sub` requests of a second draw (seed 6), Poisson at
                    half the measured saturation throughput: p50/p99, and the
                    p50 of the small requests (nsite <= 11) against their
                    solve-alone time (edzt_solve on the same request)
    with the plain engine's solves/s on the saturation requests (one request
    per nsite timed, weighted by counts)."""
    import numpy as np
    import torch
    omega = pkg.matsubara(2048, 100.0)
    reqs, rng = _served_requests(pkg, cfgs, n, seed, nsite_max)
    arrivals = np.cumsum(rng.exponential(1.0 / 200.0, n))
    arrivals -= arrivals[0]
    warm = _served_requests(pkg, cfgs, 2, 99, 10)[0]                 # warm-up: tables, pool, kernels
    _serve_run(pkg, s, warm, [0.0, 0.0], omega)
    lat, total = _serve_run(pkg, s, reqs, arrivals, omega)
    ns = np.array([r["model"].nsite for r in reqs])
    by_ns = {int(k): round(float(np.percentile(lat[ns == k], 50)) * 1000, 1) for k in sorted(set(ns.tolist()))}
    rate_sat = n / total
    # below saturation
    sreqs, srng = _served_requests(pkg, cfgs, sub, seed + 1, nsite_max)
    offered = 0.5 * rate_sat
    sarr = np.cumsum(srng.exponential(1.0 / offered, sub))
    sarr -= sarr[0]
    slat, stotal = _serve_run(pkg, s, sreqs, sarr, omega)
    sns = np.array([r["model"].nsite for r in sreqs])
    small = np.nonzero(sns <= 11)[0]
    alone = []
    for i in small:
        r = sreqs[i]
        s.set_model(r["model"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.solve(r["sectors"], 300, omega, nspin=2, seed=r["seed"])
        torch.cuda.synchronize()
        alone.append(time.perf_counter() - t0)
    sub_out = {"requests": sub, "offered_rate_per_s": offered, "seconds": stotal,
               "latency_ms": {"p50": float(np.percentile(slat, 50) * 1000), "p99": float(np.percentile(slat, 99) * 1000)}}
    if small.size:
        sub_out["small_requests"] = {
            "count": int(small.size), "p50_ms": float(np.percentile(slat[small], 50) * 1000),
            "alone_p50_ms": float(np.percentile(alone, 50) * 1000),
            "ratio": float(np.percentile(slat[small], 50) / np.percentile(alone, 50)),
            "how": "nsite <= 11; alone = edzt_solve of the same request on the idle GPU, host wall clock"}
    plain, per_ns = plain_estimate(pkg, s, reqs, omega, 300)
    return {"value": rate_sat, "unit": "solves/s", "requests": n, "seconds": total,
            "latency_ms": {"p50": float(np.percentile(lat, 50) * 1000), "p99": float(np.percentile(lat, 99) * 1000)},
            "p50_ms_by_nsite": by_ns, "offered_rate_per_s": 200.0, "sub_saturation": sub_out,
            "plain_gpu": {"value": plain, "unit": "solves/s", "ms_per_solve_by_nsite": per_ns,
                          "how": "one request per nsite timed, weighted by counts"},
            "sample": f"{n} requests, nsite ~ U{{8..{nsite_max}}}, Poisson 200/s (seed 5); the sub-saturation "
                      f"run: {sub} requests (seed 6) at half the measured throughput"}


def hv_leg(pkg, s, peak):
    """Standalone H.v (edzt_hx, y = H x) on the half-filled sector of a
    single-orbital impurity at nsite 12, 14, 16: device time per H.v (CUDA
    events on the library's stream, median of 5 after 2 warm-up), achieved
    GB/s at 16 B per state (x read, y written) against the measured peak."""
    import numpy as np
    import torch
    stream = torch.cuda.ExternalStream(s.stream_ptr(), device=torch.device("cuda", torch.cuda.current_device()))
    out = {}
    for ns in (12, 14, 16):
        nb = ns - 1
        rng = np.random.default_rng(ns)
        m = pkg.Model(1, nb, np.zeros((1, 2)), np.stack([rng.uniform(-2, 2, nb)] * 2, 1),
                      np.stack([rng.uniform(0.1, 1, nb)] * 2, 1).reshape(1, nb, 2), U=3.0, mu=1.5)
        s.set_model(m)
        n = s.dim(ns // 2, ns // 2)
        x = torch.rand(n, dtype=torch.float64, device="cuda")
        y = torch.empty_like(x)
        ts = []
        for it in range(7):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.hx(ns // 2, ns // 2, x, y)
            e1.record(stream)
            e1.synchronize()
            if it >= 2:
                ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        gbs = 16.0 * n / (ms / 1000.0) / 1e9
        out[f"nsite{ns}"] = {"dim": int(n), "ms": ms, "achieved_GBs": gbs, "frac": gbs / peak if peak else None}
        del x, y
    return out


def read_traffic(path):
    """DRAM bytes per k_lanczos launch (dram__bytes_read.sum + dram__bytes_write.sum
    from one ncu capture of this workload), from the `bytes_per_launch:` line of
    the committed profile summary; None when there is none."""
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def cpu_solve_sample(cfg, threads=None, steps=None):
    """Times the oracle on a bounded sample and extrapolates to one full solve.

    Sample: the reference's diag_lanczos (coefficient pass, eigenvector pass
    and residual) on the largest sector (6,6) plus the c and c^+
    Green's-function runs.  A full solve runs diag_lanczos on all 9 sectors,
    so the sector time is scaled by sum(dim)/dim(6,6).  steps (< the
    workload's 300) times runs of steps/2 and steps Lanczos steps instead and
    extrapolates each part linearly to 300 (every step costs one H.v and the
    same vector updates; the rest of a run is a fixed cost)."""
    from oracle import oracle as O
    O.build()
    if threads:
        O.set_num_threads(threads)
    m = cfg["model"]
    o = O.Oracle(m.norb, m.nbath, m.em, m.ek, m.vmk, m.U, m.Up, m.Jex, m.Jp, m.mu)
    dims = [o.dim(u, d) for u, d in cfg["sectors"]]
    big = (6, 6)
    omega = O.matsubara(cfg["nw"], cfg["beta"])
    N = cfg["maxnstep"]
    t_start = time.perf_counter()

    def timed(n):
        t0 = time.perf_counter()
        r = o.diag_lanczos(*big, n, seed=0, stream=4)
        t1 = time.perf_counter()
        o.green_diag(*big, r["vec"], r["e0"], 1, 1, n, omega)
        t2 = time.perf_counter()
        return t1 - t0, t2 - t1

    if steps and steps < N:
        n1, n2 = steps // 2, steps
        (d1, g1), (d2, g2) = timed(n1), timed(n2)
        t_diag = d2 + (d2 - d1) * (N - n2) / (n2 - n1)
        t_green = g2 + (g2 - g1) * (N - n2) / (n2 - n1)
        how = f"[{n1} and {n2} steps, extrapolated linearly to {N}]"
    else:
        t_diag, t_green = timed(N)
        how = f"[{N} steps + eigenvector pass]"
    t_solve = t_diag * sum(dims) / o.dim(*big) + t_green
    sample = (f"diag_lanczos of sector (6,6) {how} + c/c^+ Green's runs, "
              f"scaled by sum(dim)/dim(6,6) = {sum(dims) / o.dim(*big):.3f} to one 9-sector solve")
    return 1.0 / t_solve, O.num_threads(), sample, time.perf_counter() - t_start


class OracleSolve:
    """One impurity solve of the workload on the CPU oracle, cut into the
    pieces the reference runs one after another: diag_lanczos of each sector
    (coefficient pass, eigenvector pass and residual; src/ground_state.f90:
    30-73 with src/lanczos_solver.f90:20-90), keeping the lowest as
    ground_state does, then the Green's-function runs of cluster_green_ftn
    (c^+ and c Lanczos runs and the continued fraction on the Matsubara grid;
    src/dmft_green.f90:47-260).  run_piece() runs the next piece; a solve is
    len(sectors) + 1 pieces."""

    def __init__(self, cfg):
        from oracle import oracle as O
        O.build()
        self.O = O
        m = cfg["model"]
        self.o = O.Oracle(m.norb, m.nbath, m.em, m.ek, m.vmk, m.U, m.Up, m.Jex, m.Jp, m.mu)
        self.sectors = list(cfg["sectors"])
        self.maxnstep = cfg["maxnstep"]
        self.omega = O.matsubara(cfg["nw"], cfg["beta"])
        self.pieces = len(self.sectors) + 1
        self.next = 0
        self.solves = 0
        self._reset()

    def _reset(self):
        self.best, self.best_e, self.best_vec = -1, float("inf"), None

    def run_piece(self):
        i = self.next
        if i < len(self.sectors):
            nu, nd = self.sectors[i]
            r = self.o.diag_lanczos(nu, nd, self.maxnstep, seed=0, stream=i)
            tie = 1.0e-10 * max(1.0, abs(self.best_e))
            if self.best < 0 or r["e0"] < self.best_e - tie:
                self.best, self.best_e, self.best_vec = i, r["e0"], r["vec"]
        else:
            nu, nd = self.sectors[self.best]
            self.o.cluster_green_ftn(1, nu, nd, self.best_vec, self.best_e, self.maxnstep, self.omega)
            self.solves += 1
            self._reset()
        self.next = (i + 1) % self.pieces

    def warm(self):
        """A short untimed run: 20 Lanczos steps of the smallest sector."""
        nu, nd = min(self.sectors, key=lambda s: self.o.dim(*s))
        self.o.lanczos_iteration(nu, nd, self.O.start_vector(0, 99, self.o.dim(nu, nd)), 20)


def run_reference(args):
    """The reference's algorithm on this host's CPU cores: the oracle (a CPU
    restatement of the reference's Fortran, which cannot be built here) on
    all host threads.  Each step is one piece of a whole solve in the
    reference's order (a sector's diag_lanczos, or the Green's-function runs
    that end a solve); every timed piece is run in full, with no
    extrapolation.  value = whole solves completed in the timed region / the
    time of the pieces they consist of (with --steps a multiple of the
    pieces per solve, that is every timed step).  Warm-up steps are a short
    20-step Lanczos run each, not pieces of a solve."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = workload()
    ref = OracleSolve(cfg)
    for _ in range(args.warmup):
        ref.warm()
    piece_s = []
    solve_s = []
    acc = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        last = ref.next == ref.pieces - 1
        ref.run_piece()
        dt = time.perf_counter() - t0
        piece_s.append(dt)
        acc += dt
        if last:
            solve_s.append(acc)
            acc = 0.0
    if solve_s:
        value = len(solve_s) / sum(solve_s)
    else:                                # fewer steps than one solve: pieces done / pieces per solve
        value = (len(piece_s) / ref.pieces) / sum(piece_s)
    cores = ref.O.num_threads()
    sample = (f"{len(piece_s)} pieces of whole solves (each a sector's 300-step diag_lanczos with its "
              f"eigenvector pass, or the c/c^+ Green's runs; {ref.pieces} pieces per solve): "
              f"{len(solve_s)} whole solves timed in full, no extrapolation")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(piece_s) / len(piece_s),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config_dict(cfg, 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "solve_seconds": solve_s,
            "note": "CPU restatement of the reference's Fortran algorithm (the reference needs a Fortran "
                    "compiler, MPI, MKL and ARPACK, none of which exist on this image); a step is one piece "
                    "of a solve, warm-up steps are 20-step Lanczos runs"}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    pkg = load_pkg()
    if local == 0:                       # one make per node; the other ranks wait for it
        pkg.build()
    if dist is not None:
        dist.barrier()
    cfg = workload()
    m = cfg["model"]
    sectors = cfg["sectors"]
    K, W = args.steps, args.warmup
    nw, maxn = cfg["nw"], cfg["maxnstep"]
    omega_h = pkg.matsubara(nw, cfg["beta"])

    s = pkg.Solver(local)
    stream = torch.cuda.ExternalStream(s.stream_ptr(), device=torch.device("cuda", local))
    omega_d = torch.tensor(omega_h, device="cuda")
    G_d = torch.zeros(2 * nw * m.norb, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    import ctypes as C
    L = pkg.load_library()
    sec = np.ascontiguousarray(np.asarray(sectors, dtype=np.int32).reshape(-1, 2))
    em, ek, vmk = m.fortran_arrays()
    isec, e0 = C.c_int(), C.c_double()

    def solve_device():
        s.set_model(m)
        s._check(L.edzt_solve(s._h, len(sec), sec.ctypes.data, maxn, C.c_uint64(0), 1, nw,
                              omega_d.data_ptr(), C.byref(isec), C.byref(e0), G_d.data_ptr(), None))

    # ---- device-timed solves -------------------------------------------------
    for _ in range(W):
        solve_device()
    torch.cuda.synchronize()
    s.reset_stats()
    launches0 = s.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    lat = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    for _ in range(K):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        solve_device()
        ev1.record(stream)
        ev1.synchronize()
        lat.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = s.launch_count() - launches0
    ks = s.kernel_stats()
    # whether the solves ran an eigenvector pass (a launch over the winning
    # sector alone) or took the eigenvector from the scan's kept pairs
    eig_pass = any(e["states"] in [float(s.dim(u, d)) for u, d in sectors] for e in s.launch_log())
    total_ms = sum(lat)
    replicas = importlib.import_module("dmft_ed_zt_b200.replicas")
    total_ms = replicas.max_over_ranks(total_ms, dist, device="cuda")
    value = world * K / (total_ms / 1000.0)

    # ---- end to end through the C ABI with host buffers ---------------------
    gsvec_h = np.zeros(max(s.dim(u, d) for u, d in sectors))
    G_h = np.zeros(2 * nw * m.norb)
    coeffs_h = np.zeros(m.norb * 2 * 4 * maxn)
    es_h = np.zeros(len(sec))

    def solve_host():
        s._check(L.edzt_set_model(s._h, m.norb, m.nbath, em.ctypes.data, ek.ctypes.data, vmk.ctypes.data,
                                  m.U, m.Up, m.Jex, m.Jp, m.mu))
        s._check(L.edzt_ground_state(s._h, len(sec), sec.ctypes.data, maxn, C.c_uint64(0), C.byref(isec),
                                     C.byref(e0), gsvec_h.ctypes.data, es_h.ctypes.data))
        s._check(L.edzt_cluster_green_ftn(s._h, 1, maxn, nw, omega_h.ctypes.data, G_h.ctypes.data,
                                          coeffs_h.ctypes.data))

    for _ in range(min(W, 3)):
        solve_host()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e2e_ms = 0.0
    for _ in range(K):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solve_host()
        torch.cuda.synchronize()
        e2e_ms += 1000.0 * (time.perf_counter() - t0)
    e2e_ms = replicas.max_over_ranks(e2e_ms, dist, device="cuda")
    gs_dim = int(L.edzt_gs_dim(s._h))
    h2d = (em.nbytes + ek.nbytes + vmk.nbytes + sec.nbytes + omega_h.nbytes)
    d2h = 8 * gs_dim + G_h.nbytes + coeffs_h.nbytes + es_h.nbytes + 8
    e2e = {"value": world * K / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "timing": "host wall clock around each C-ABI solve, synchronised"}

    # ---- plain one-kernel-per-step GPU Lanczos (the comparator) -------------
    plain = None
    if not args.skip_plain and rank == 0:
        s.set_engine(pkg.ENGINE_PLAIN)
        solve_device()
        torch.cuda.synchronize()
        pl = []
        for _ in range(max(1, min(K, 2))):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            solve_device()
            ev1.record(stream)
            ev1.synchronize()
            pl.append(ev0.elapsed_time(ev1))
        s.set_engine(pkg.ENGINE_FUSED)
        # Lanczos state-steps of a solve in each engine: the plain engine runs
        # the eigenvector pass of every sector as the reference does, the
        # fused engine only the winner's (or none: the eigenvector from the
        # scan's kept pairs), so part of the ratio is skipped work
        dims = [s.dim(u, d) for u, d in sectors]
        gdim = sum(s.dim(u + du, d + dd) for (u, d) in [max(sectors, key=lambda q: s.dim(*q))]
                   for du, dd in ((1, 0), (-1, 0)))
        plain_steps = sum(2 * maxn * x for x in dims) + maxn * gdim
        fused_steps = sum(maxn * x for x in dims) + (maxn * max(dims) if eig_pass else 0) + maxn * gdim
        ratio = (1000.0 * len(pl) / sum(pl))
        plain = {"value": ratio, "unit": UNIT, "ms_per_solve": sum(pl) / len(pl),
                 "engine": "one kernel per BLAS-1 step + H.v kernels, host reads of every reduction, "
                           "eigenvector pass for every sector (the reference's structure)",
                 "state_steps_per_solve": plain_steps, "fused_state_steps_per_solve": fused_steps,
                 "skipped_work_factor": plain_steps / fused_steps}

    # ---- roofline of the persistent Lanczos kernel ---------------------------
    peak, peak_src = measured_peak()
    achieved = ks["bytes"] / (ks["ms"] / 1000.0) / 1e9 if ks["ms"] > 0 else 0.0
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if peak else None, "traffic": None,
                "kernel": "k_lanczos (persistent fused Lanczos)", "peak_source": peak_src,
                "launches": ks["launches"], "avg_launch_ms": ks["ms"] / max(ks["launches"], 1),
                "algorithmic_bytes_per_launch": ks["bytes"] / max(ks["launches"], 1),
                "eigenvector": "eigenvector pass" if eig_pass else "from the scan's kept Lanczos pairs",
                "note": "24 B/state per coefficient step, 40 B/state per eigenvector step; the "
                        "ground-state scan (9 sectors, 252 MB of pair buffers and D) exceeds L2, the "
                        "eigenvector and Green's-function launches are L2-resident"}
    roofline["traffic"] = read_traffic(args.traffic_file)
    # the launches of one solve separately, told apart by the states they
    # carry: the ground-state scan (every sector), the eigenvector pass of the
    # winner (absent when the scan kept its Lanczos pairs), the c/c^+ runs
    log = s.launch_log()
    scan_states = float(sum(s.dim(u, d) for u, d in sectors))
    kinds = {}
    for e in log:
        kinds.setdefault(e["states"], []).append(e)
    per = []
    for st_, ent in kinds.items():
        if st_ == scan_states:
            name = f"ground-state scan ({len(sectors)} sectors, {maxn} steps)"
        elif st_ in [float(s.dim(u, d)) for u, d in sectors]:
            name = "eigenvector pass (winning sector)"
        else:
            name = f"c / c^+ runs (excitation sectors, {maxn} steps)"
        ms = sum(e["ms"] for e in ent) / len(ent)
        by = sum(e["bytes"] for e in ent) / len(ent)
        gbs = by / (ms / 1000.0) / 1e9 if ms > 0 else 0.0
        per.append({"launch": name, "launches": len(ent), "avg_ms": ms, "algorithmic_bytes": by,
                    "achieved_GBs": gbs, "frac": gbs / peak if peak else None, "states": st_,
                    "pair_and_D_bytes": 40.0 * st_})
    if per:
        roofline["per_launch"] = per

    hv = hv_leg(pkg, s, peak) if (world == 1 and not args.skip_hv) else None
    batched = served = None
    if args.batched > 0:
        cfgs = importlib.import_module("dmft_ed_zt_b200.configs")
        batched = batched_leg(pkg, s, cfgs, args.batched, dist, rank, world)
    if world == 1 and args.served > 0:
        cfgs = importlib.import_module("dmft_ed_zt_b200.configs")
        served = served_leg(pkg, s, cfgs, args.served, nsite_max=args.served_nsite_max, sub=args.served_sub)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        v, cores, sample, _ = cpu_solve_sample(cfg)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        lat_sorted = sorted(lat)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": config_dict(cfg, world),
                "latency_ms": {"p50": float(np.percentile(lat_sorted, 50)),
                               "p99": float(np.percentile(lat_sorted, 99)),
                               "each": [round(float(x), 3) for x in lat]},
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu,
                "plain_gpu": plain, "hv": hv, "batched": batched, "served": served, "clocks": clk, "e0": e0.value}
        print(json.dumps(line))
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_case(spec, steps):
    """Small single-kernel workloads for ncu captures and kernel A/B timing,
    on the half-filled sector of the hv leg's single-orbital model at nsite NS:
      hx:NS   four y = H x calls (k_hx); the last one is timed
      lz:NS   lanczos_iteration of 5, then of `steps` steps (k_lanczos); the
              second launch is timed
      solve   one impurity solve of the bench workload (nsite 12, 9 sectors)
    Prints one JSON line with the device time (CUDA events) of the timed part."""
    import numpy as np
    import torch

    pkg = load_pkg()
    s = pkg.Solver(0)
    kind, _, arg = spec.partition(":")
    out = {"case": spec}
    if kind == "solve":
        cfg = workload()
        s.set_model(cfg["model"])
        omega = pkg.matsubara(cfg["nw"], cfg["beta"])
        s.solve(cfg["sectors"], cfg["maxnstep"], omega, nspin=1, seed=0)
        s.reset_stats()
        s.solve(cfg["sectors"], cfg["maxnstep"], omega, nspin=1, seed=0)
        st = s.kernel_stats()
        out.update(k_lanczos_ms=st["ms"], launches=st["launches"])
    else:
        ns = int(arg)
        nb = ns - 1
        rng = np.random.default_rng(ns)
        m = pkg.Model(1, nb, np.zeros((1, 2)), np.stack([rng.uniform(-2, 2, nb)] * 2, 1),
                      np.stack([rng.uniform(0.1, 1, nb)] * 2, 1).reshape(1, nb, 2), U=3.0, mu=1.5)
        s.set_model(m)
        n = s.dim(ns // 2, ns // 2)
        out["dim"] = int(n)
        if kind == "hx":
            stream = torch.cuda.ExternalStream(s.stream_ptr())
            x = torch.rand(n, dtype=torch.float64, device="cuda")
            y = torch.empty_like(x)
            for _ in range(3):
                s.hx(ns // 2, ns // 2, x, y)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.hx(ns // 2, ns // 2, x, y)
            e1.record(stream)
            e1.synchronize()
            out["k_hx_ms"] = e0.elapsed_time(e1)
        elif kind == "lz":
            v0 = np.random.default_rng(0).random(n)
            s.lanczos_iteration(ns // 2, ns // 2, v0, 5)
            s.reset_stats()
            s.lanczos_iteration(ns // 2, ns // 2, v0, steps)
            st = s.kernel_stats()
            out.update(steps=steps, k_lanczos_ms=st["ms"], ns_per_state_step=st["ms"] * 1e6 / (n * (steps + 1)))
        else:
            raise SystemExit(f"unknown case {spec}")
    s.close()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-hv", action="store_true")
    ap.add_argument("--batched", type=int, default=256, help="instances of the batched leg (0: skip)")
    ap.add_argument("--served", type=int, default=32, help="requests of the served leg (0: skip)")
    ap.add_argument("--served-nsite-max", type=int, default=16, choices=range(8, 17),
                    help="largest nsite of the served leg's requests (the workload's 16 by default)")
    ap.add_argument("--served-sub", type=int, default=12, help="requests of the served leg's sub-saturation run")
    ap.add_argument("--traffic-file", default=os.path.join(ROOT, "profiles", "k_lanczos_aim_n12_dram.txt"))
    ap.add_argument("--case", default=None, help="run one small profiling case (hx:NS, lz:NS, solve) and exit")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case, args.steps)
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
