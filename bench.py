"""Benchmark of the granular hot path: particle-steps/s on the 1M-sphere
Hertz/history + rolling-friction hopper with a triangulated mesh wall.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload hopper|pour] [--n N] [--settle S]

Own arm: the workload is generated (seeded), uploaded, set up and settled for
S steps, then W warm-up steps run untimed and K steps are timed with CUDA
events on the engine's stream, bracketed by a barrier and device syncs.
``value`` = particles x K / device time (whole job, summed over ranks).
Multi-GPU: every rank runs an independent replica (different seed) -- the
domain-decomposed multi-GPU path is not built, see DESIGN.md.

Reference arm (--impl reference): the CPU oracle (a restatement of the
reference's own CPU algorithm) on rank 0, on the host cores, timed on a
bounded number of steps of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "liggghts-public_b200", "python"))

METRIC = "particle-steps/s @1M spheres Hertz/history+mesh, 1 B200 vs plain FP64 GPU & host-CPU ref"
UNIT = "particle-steps/s"


def parse():
    return parse_list(None)


def parse_list(argv):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--workload", default="hopper", choices=["hopper", "pour", "drum", "sq"])
    ap.add_argument("--n", type=int, default=0, help="particle count (default: 1M hopper, 20k pour)")
    ap.add_argument("--settle", type=int, default=200, help="untimed settling steps before warm-up")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--precision", default="split", choices=["split", "fp64"],
                    help="precision of the headline arm (split: FP32 contact math on FP64 state)")
    ap.add_argument("--fp64-steps", type=int, default=-1,
                    help="timed steps of the plain FP64 form on the same state (-1: as many as --steps, 0: skip)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args(argv)


def make_workload(args, seed_offset=0):
    import gb2_scenarios as S
    if args.workload == "drum":
        n = args.n or 1_000_000
        length = 0.85 * (n / 8_000_000)
        sc = S.drum(n=n, seed=7 + seed_offset, length=max(length, 0.05), n_ax=max(8, int(121 * length / 0.85)))
        ntri = len(sc["fixes"][1]["nodes"])
        desc = ("drum-%d: spheres r U(0.8, 1.2) mm, Hertz/history, 0.5 m drum (length scaled to the particle "
                "count for a 35%% fill of the 8M/0.85 m configuration), %d triangles, fix move/mesh rotate 2 rad/s, "
                "dt 5e-6" % (n, ntri))
        return sc, desc, {"n_particles": n, "triangles": ntri}
    if args.workload == "hopper":
        n = args.n or 1_000_000
        sc = S.hopper(n=n, seed=2024 + seed_offset, gap=0.01, vmax=0.05)
        ntri = len(sc["fixes"][1]["nodes"])
        desc = ("hopper-%d: %d polydisperse spheres (lognormal r, median 1 mm, sigma 0.25, clip 0.5-2 mm), "
                "Hertz/history + rolling cdt, conical mesh hopper %d triangles (60 deg, 30 mm outlet), "
                "plane catch floor, dt 5e-6" % (n, n, ntri))
        return sc, desc, {"n_particles": n, "triangles": ntri}
    n = args.n or 20000
    sc = S.sphere_pour(n=n, seed=12345 + seed_offset)
    desc = "sphere-pour-%d: monodisperse r=1 mm, Hertz/history, periodic x/y, plane floor, dt 1e-5" % n
    return sc, desc, {"n_particles": n, "triangles": 0}


# --------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.p = None
        self.out = None
        try:
            self.out = open(os.devnull if False else "/tmp/gb2_clocks_%d.csv" % os.getpid(), "w")
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                       "-i", str(device), "-lms", "250"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.out.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.out.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.out.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- roofline

def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(kernel, n, cen, nfix_plane, nfix_mesh, split=False):
    """Algorithmic HBM bytes per launch (model in DESIGN.md): owned-atom
    records, list indices and shear history that must cross HBM once;
    neighbour-state gathers are served from L2 and not counted."""
    avg = lambda k: 0.5 * (cen[0][k] + cen[1][k])
    if kernel == "k_pair_step":
        # own x,v,w,r,m,type 92 + list counts 8 + touch mask 16 + xhold 24 + x,v,w out 72
        # (+ the 32-byte FP32 kinematics record written in split precision)
        per_atom = 92 + 8 + 16 + 24 + 72 + (32 if split else 0) + nfix_plane * 1 + nfix_mesh * 4
        b = n * per_atom + avg("nlist") * 4 + avg("nrev") * 4 + avg("ntouch") * (52 + 25)
        b += avg("nwall_touch") * 48 + avg("nmesh_cand") * 4 + avg("nmesh_touch") * 52
        return b
    if kernel == "k_pair_main":
        per_atom = 92 + 48 + 4 + 48 + 48 + nfix_plane * 1 + nfix_mesh * 4
        b = n * per_atom + avg("nlist") * 4 + avg("ntouch") * 52
        b += avg("nwall_touch") * 48 + avg("nmesh_cand") * 4 + avg("nmesh_touch") * 52
        return b
    if kernel == "k_pair_reverse":
        return n * (92 + 4 + 48) + avg("nrev") * 4 + avg("ntouch") * 24
    raise ValueError(kernel)


def load_traffic(kernel, workload):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            d = json.load(fh)
        e = d.get(workload, {}).get(kernel)
        return e
    except Exception:
        return None


# --------------------------------------------------------------- CPU oracle

def run_oracle_sample(sc, target_s, max_steps):
    """Time the oracle (single thread) on sc: setup + 2 warm-up steps untimed,
    then steps until ~target_s of CPU time (at most max_steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.Oracle(sc)
    o.setup()
    o.run(2)
    t0 = time.perf_counter()
    o.run(1)
    one = time.perf_counter() - t0
    k = int(max(1, min(max_steps, target_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    o.run(k)
    dt = time.perf_counter() - t0 + one
    n = len(sc["atoms"]["tag"])
    return n * (k + 1) / dt, k + 1


# --------------------------------------------------------------- arms

def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        else:   # host-only runs (tests of the multi-rank plumbing)
            dist.init_process_group("gloo", timeout=timedelta(seconds=60))
        return ws, rank, local, dist
    return 1, 0, 0, None


def barrier(dist):
    if dist is not None:
        dist.barrier()


def allmax(dist, x):
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _ref_worker(argv, seconds, barrier, out):
    """One replica of the reference arm: the oracle port (the reference's
    algorithm, single-threaded) on the workload, timed for ~`seconds`."""
    args = parse_list(argv)
    sc, desc, extra = make_workload(args)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.Oracle(sc)
    o.setup()
    o.run(min(args.settle, 200))
    o.run(min(args.warmup, 3))
    n = len(sc["atoms"]["tag"])
    barrier.wait()
    k, t0 = 0, time.perf_counter()
    while k < max(args.steps, 1):
        o.run(1)
        k += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    out.put((n * k / dt, k, dt))


def reference_arm(args):
    """The reference's CPU path (the oracle port: its algorithm, restated in
    C, single-threaded like the reference without MPI) on all host cores the
    process may use: one replica per core on the same workload, timed
    together; value = the replicas' summed particle-steps/s."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    n_est = args.n or (20_000 if args.workload == "pour" else 1_000_000)
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 8 << 30
    per = 400 + 900 * n_est          # bytes per replica (measured ~0.84 GB at 1M atoms)
    nproc = max(1, min(cores, int(0.6 * avail // per)))
    ctx = mp.get_context("spawn")
    barrier, out = ctx.Barrier(nproc), ctx.Queue()
    seconds = 20.0
    procs = [ctx.Process(target=_ref_worker, args=(sys.argv[1:], seconds, barrier, out)) for _ in range(nproc)]
    for p in procs:
        p.start()
    res = [out.get() for _ in range(nproc)]
    for p in procs:
        p.join()
    val = sum(r[0] for r in res)
    k = min(r[1] for r in res)
    dt = max(r[2] for r in res)
    sc, desc, extra = make_workload(args)
    settle, w = min(args.settle, 200), min(args.warmup, 3)
    sample = ("%s; oracle port, %d single-threaded replicas on %d host cores, each after %d settle + %d warm-up "
              "steps, ~%.0f s timed together (>= %d steps each)" % (desc, nproc, cores, settle, w, seconds, k))
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": ws, "steps": k, "warmup": w,
        "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": dict({"workload": desc, "settle_steps": settle}, **extra),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": nproc, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def state_scenario(sc, a):
    """Scenario whose x, v, omega are a downloaded engine state (by tag)."""
    out = dict(sc)
    order = np.argsort(a["tag"])
    idx = a["tag"][order] - 1
    out["atoms"] = dict(sc["atoms"])
    for k in ("x", "v", "omega"):
        arr = np.zeros_like(sc["atoms"][k])
        arr[idx] = a[k][order]
        out["atoms"][k] = arr
    return out


PROFILE_EVERY = 16   # per-kernel CUDA events on every 16th step of the timed window


def timed_window(eng, steps, dist, device, clocks=True):
    """Device-timed window of `steps` steps: CUDA events at its ends give the
    window time; per-kernel CUDA events on every PROFILE_EVERY-th step give
    each kernel's average launch time (the events serialise the pair step
    and its dependent tail kernel on those steps only)."""
    eng.sync()
    cen0 = eng.census()
    st0 = eng.stats()
    sampler = ClockSampler(device) if clocks else None
    barrier(dist)
    eng.sync()
    eng.set_profiling(True, every=PROFILE_EVERY)
    eng.timer_start()
    eng.run(steps)
    ms = eng.timer_stop()
    eng.sync()
    barrier(dist)
    clk = sampler.stop() if sampler else None
    st1 = eng.stats()
    eng.set_profiling(False)
    cen1 = eng.census()
    kt = {k: st1[k] - st0[k] for k in ("t_integrate", "t_pair_main", "t_pair_tail", "t_forward", "t_rebuild")}
    npm = st1["n_pair_main"] - st0["n_pair_main"]
    return {"ms": allmax(dist, ms), "clocks": clk, "cen": (cen0, cen1), "kt": kt, "npm": npm,
            "kernel_ms_per_step": dict({k: v / max(npm, 1) for k, v in kt.items()},
                                       note="CUDA events on every %dth step of the timed window (%d steps timed)"
                                            % (PROFILE_EVERY, npm)),
            "launches": st1["kernel_launches"] - st0["kernel_launches"],
            "rebuilds": st1["nsteps_rebuild"] - st0["nsteps_rebuild"],
            "growth": st1["ngrow"] - st0["ngrow"],
            "capacities": {k: st1[k] for k in ("maxneigh", "maxpartner", "maxrev", "maxmesh")}}


def own_arm(args):
    ws, rank, local, dist = dist_init()
    import granb200
    split = args.precision == "split"
    prec = granb200.PREC_SPLIT if split else granb200.PREC_FP64
    sc, desc, extra = make_workload(args, seed_offset=rank)
    n = len(sc["atoms"]["tag"])
    eng = granb200.Engine(sc, precision=prec, device=local)
    eng.setup()
    eng.run(args.settle)
    if args.fp64_steps < 0:
        args.fp64_steps = args.steps
    # the settled state the timed window starts from (warm-up aside): the FP64
    # arm and the end-to-end run start from it too
    start_state = state_scenario(sc, eng.atoms()) if (args.fp64_steps > 0 and split) or not args.no_e2e else None
    eng.run(max(args.warmup, 3))
    W = timed_window(eng, args.steps, dist, local)
    ms_max = W["ms"]
    value = n * args.steps * ws / (ms_max * 1e-3)

    # roofline of the dominant kernel
    nfix_plane = sum(1 for f in sc["fixes"] if f["kind"] == "wall_plane")
    nfix_mesh = sum(1 for f in sc["fixes"] if f["kind"] == "wall_mesh")
    dom = "k_pair_step"
    dom_ms = W["kt"]["t_pair_main"] / max(W["npm"], 1)
    ab = algorithmic_bytes(dom, n, W["cen"], nfix_plane, nfix_mesh, split)
    peak, peak_kind = peaks()
    achieved = ab / (dom_ms * 1e-3) / 1e9
    traffic = load_traffic(dom + ("_split" if split else ""), args.workload)
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": traffic["bytes_per_launch"] if traffic else None,
            "algorithmic_bytes_per_launch": ab, "avg_launch_ms": dom_ms,
            "timing": "pair-step launches timed with CUDA events on every %dth step of the timed window"
                      % PROFILE_EVERY}

    pdesc = ("split (FP32 contact math on FP64-differenced positions and FP64 overlap, Kahan FP32 pair sums; "
             "FP64 walls, gravity, integration)" if split else "fp64 (bit-exact to the oracle)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 contact / f64 state" if split else "f64", "data": "synthetic",
        "config": dict({"workload": desc, "settle_steps": args.settle, "precision": pdesc,
                        "l2": "inputs larger than L2 (per-step working set > 126 MB at 1M particles)",
                        "parallelism": "replicas x%d" % ws if ws > 1 else "single GPU"}, **extra),
        "roofline": roof,
        "gpu_launches": W["launches"],
        "clocks": W["clocks"],
        "kernel_ms_per_step": W["kernel_ms_per_step"],
        "census": {k: 0.5 * (W["cen"][0][k] + W["cen"][1][k]) for k in W["cen"][0]},
        "rebuilds": W["rebuilds"],
        "capacity_growth_in_window": W["growth"],
        "capacities": W["capacities"],
    }

    # the plain FP64 form on the same starting state (same settle, warm-up)
    if start_state is not None and args.fp64_steps > 0 and split:
        e64 = granb200.Engine(start_state, precision=granb200.PREC_FP64, device=local)
        e64.setup()
        e64.run(max(args.warmup, 3))
        W64 = timed_window(e64, args.fp64_steps, dist, local, clocks=False)
        v64 = n * args.fp64_steps * ws / (W64["ms"] * 1e-3)
        line["fp64_gpu"] = {"value": v64, "unit": UNIT, "steps": args.fp64_steps,
                            "ms_per_step": W64["ms"] / args.fp64_steps,
                            "kernel_ms_per_step": W64["kernel_ms_per_step"],
                            "note": "bit-exact FP64 path from the same settled state (same settle and warm-up "
                                    "steps, %d timed steps; split window %d)" % (args.fp64_steps, args.steps)}
        line["split_over_fp64"] = value / v64
        e64.close()
        del e64

    # end to end through the C ABI: host arrays in, setup, run, host arrays out
    if not args.no_e2e:
        sc2 = start_state
        barrier(dist)
        t0 = time.perf_counter()
        e2 = granb200.Engine(sc2, precision=prec, device=local)
        t1 = time.perf_counter()
        e2.setup()
        t2 = time.perf_counter()
        e2.run(args.steps)
        e2.sync()
        t3 = time.perf_counter()
        out = e2.atoms()
        e2.sync()
        t4 = time.perf_counter()
        dt = t4 - t0
        dt = allmax(dist, dt)
        h2d = n * (3 * 3 * 8 + 2 * 8 + 2 * 4) + sum(f["nodes"].size * 8 for f in sc["fixes"] if f["kind"] == "wall_mesh")
        d2h = n * (5 * 3 * 8 + 4)
        line["e2e"] = {"value": n * args.steps * ws / dt, "unit": UNIT,
                       "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                       "includes": "context create, materials, atom + mesh upload, Verlet setup, %d steps from the "
                                   "settled state the timed window starts from, download of x/v/omega/f/torque"
                                   % args.steps,
                       "seconds": {"create_upload": t1 - t0, "setup": t2 - t1, "run": t3 - t2, "download": t4 - t3}}
        del e2, out

    # CPU baseline: the oracle on this rank's state at the start of the window
    if rank == 0 and ws == 1 and not args.no_cpu:
        sc3 = state_scenario(sc, eng.atoms())
        cval, ck = run_oracle_sample(sc3, args.cpu_seconds, 200)
        line["cpu_baseline"] = {"value": cval, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": "oracle port, 1 thread, same %d-particle state as the GPU window end, "
                                          "setup + 2 untimed steps, %d timed steps" % (n, ck)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def sq_arm(args):
    """Superquadric packing: plain first-contact solve against the learned
    initial guess, same particles, same steps, device-timed."""
    import granb200
    import gb2_scenarios as S
    n = args.n or 200_000
    t0 = time.perf_counter()
    tr = granb200.MlpTrainer()
    info = tr.make_data(1_000_000, seed=1)
    tr.init(seed=2)
    l0, l1 = tr.train(epochs=4, batch=4096, lr=2e-3)
    ev = tr.evaluate(100_000, seed=99)
    train_s = time.perf_counter() - t0
    solve = tr.time_solves(400_000, seed=123)   # first-contact solves alone, same pairs both ways
    params = tr.params()
    sc = S.sq_packing(n=n, seed=11)
    res = {}
    for name, learned in (("plain", None), ("learned", params)):
        e = granb200.SqEngine(sc, learned=learned)
        e.setup()
        e.run(args.settle)
        e.run(max(args.warmup, 3))
        c0 = e.counters()
        ms = e.run_timed(args.steps)
        c1 = e.counters()
        res[name] = {"ms_per_step": ms / args.steps, "value": n * args.steps / (ms * 1e-3),
                     "newton_iters": c1["iters"] - c0["iters"], "newton_solves": c1["solves"] - c0["solves"],
                     "pairs_solved": c1["pairs_solved"] - c0["pairs_solved"],
                     "learned_accepted": c1["learned_used"] - c0["learned_used"],
                     "learned_rejected": c1["learned_rejected"] - c0["learned_rejected"]}
        e.close()
    line = {
        "metric": "particle-steps/s @200k superquadrics, learned vs plain initial guess", "unit": UNIT,
        "value": res["learned"]["value"], "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["learned"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 contact solve, bf16 MLP", "data": "synthetic",
        "config": {"workload": "sq-packing-%d: half-axes U(1,2) mm, blockiness U(2,8), random orientations, "
                               "Hertz/history, dt 1e-5, random velocities +-1 m/s" % n,
                   "settle_steps": args.settle},
        "plain": res["plain"], "learned": res["learned"],
        "learned_over_plain": res["learned"]["value"] / res["plain"]["value"],
        "first_contact_solve": dict(solve, note="contact-point solve of fresh pairs near contact (a new "
                                                "contact's first solve), plain homotopy vs learned guess with "
                                                "homotopy fallback, each launch timed alone; a launch lasts as "
                                                "long as its slowest pairs (those both methods fail on after "
                                                "the iteration cap)"),
        "training": {"samples": info["valid"], "plain_iters_per_sample": info["plain_iters"],
                     "plain_solves_per_sample": info["plain_solves"], "loss_first": l0, "loss_last": l1,
                     "seconds": train_s, "held_out": ev},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "sq":
        sq_arm(args)
    else:
        own_arm(args)


if __name__ == "__main__":
    main()
