"""Benchmark of the granular hot path: particle-steps/s on the 1M-sphere
Hertz/history + rolling-friction hopper with a triangulated mesh wall.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload hopper|pour|drum|bed|sq] [--particles N]

Own arm: the workload is generated (seeded; the default is the packed
conical hopper at the start of its discharge), uploaded and set up; W
warm-up steps run untimed and K steps are timed with CUDA events on the
engine's stream, bracketed by a barrier and device syncs.  ``value`` =
particles x K / device time (whole job, summed over ranks).  The headline
arm computes in FP64 and is bit-exact with the reference; beside it the
line reports, from the same generated state: the split-precision form
(FP32 contact math), a longer window in which neighbour rebuilds happen
(rebuild cost per step, and the kernel timings the roofline uses), the
end-to-end time through the C ABI with host buffers, and the reference's
CPU time on one core.  Multi-GPU: every rank runs an independent replica
(different seed); the spatially decomposed multi-GPU path is not built.

Reference arm (--impl reference): the reference itself (LIGGGHTS built
from its own sources as oracle/_ref/lmp_ref) on the same generated state,
written as a read_data file with its STL mesh and input script; W warm-up
steps, then K steps timed by the reference's own "Loop time"; one
single-threaded replica per host core the memory allows (no MPI on the
box), value = the replicas' summed particle-steps/s.  Rank 0 alone runs it.
"""
import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "liggghts-public_b200", "python"))

METRIC = "particle-steps/s @1M spheres Hertz/history+mesh, 1 B200 vs plain FP64 GPU & host-CPU ref"
UNIT = "particle-steps/s"
# the default workload's state must hold config 2's work when the window starts
FLOOR_TOUCH_PER_ATOM = 2.0
FLOOR_MESH_CONTACTS = 10_000


def parse():
    return parse_list(None)


def parse_list(argv):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--workload", default="hopper", choices=["hopper", "pour", "drum", "bed", "sq"])
    ap.add_argument("--particles", type=int, default=0, help="particle count (default: the configuration's)")
    ap.add_argument("--settle", type=int, default=0, help="sq arm: untimed settling steps before warm-up")
    ap.add_argument("--long-steps", type=int, default=2000,
                    help="steps of the longer window with neighbour rebuilds (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU time of the baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=60.0, help="reference arm: target timed seconds")
    ap.add_argument("--roofline-steps", type=int, default=32,
                    help="steps right after the headline window with every pair-step launch timed (roofline)")
    ap.add_argument("--force-frames", type=int, default=0,
                    help="FP64 vs split force error on this many frames of the FP64 run (restarts of its state)")
    ap.add_argument("--frame-every", type=int, default=10, help="steps between force-error frames")
    ap.add_argument("--sq-reps", type=int, default=3, help="sq arm: timed windows per arm (median reported)")
    ap.add_argument("--no-split", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args(argv)


def make_workload(args, seed_offset=0):
    """(scenario, description, config extras) of the selected workload."""
    import gb2_scenarios as S
    if args.workload == "drum":
        n = args.particles or 8_000_000
        sc = S.drum_config3(n=n, seed=7 + seed_offset)
        ntri = len(sc["fixes"][1]["nodes"])
        desc = ("drum-%d: %d spheres r U(0.8, 1.2) mm, density 2700, E 1e7, nu 0.45, e 0.5, mu 0.4, Hertz/history, "
                "0.5 m drum (length for a 35%% fill), %d triangles, fix move/mesh rotate 2 rad/s, dt 5e-6"
                % (n, n, ntri))
        return sc, desc, {"n_particles": n, "triangles": ntri}
    if args.workload == "bed":
        n = args.particles or 20_000_000
        sc = S.bed_config5(n=n, seed=5 + seed_offset)
        ntri = len(sc["fixes"][1]["nodes"])
        desc = ("bed-%d: %d spheres r 0.5 mm in a 0.2 x 0.2 x 0.5 m box, flat floor plus a %d-triangle bumpy plate, "
                "Hertz/history, dt 2e-6" % (n, n, ntri))
        return sc, desc, {"n_particles": n, "triangles": ntri}
    if args.workload == "hopper":
        n = args.particles or 1_000_000
        sc = S.hopper_packed(n=n, seed=2024 + seed_offset)
        ntri = len(sc["fixes"][1]["nodes"])
        desc = ("hopper-%d: %d polydisperse spheres (lognormal r, median 1 mm, sigma 0.25, clip 0.5-2 mm), "
                "Hertz/history + rolling cdt, conical mesh hopper %d triangles (60 deg, 30 mm outlet), plane catch "
                "floor, dt 5e-6; packed at the start of its discharge" % (n, n, ntri))
        return sc, desc, {"n_particles": n, "triangles": ntri}
    n = args.particles or 20000
    sc = S.sphere_pour(n=n, seed=12345 + seed_offset)
    desc = "sphere-pour-%d: monodisperse r=1 mm, Hertz/history, periodic x/y, plane floor, dt 1e-5" % n
    return sc, desc, {"n_particles": n, "triangles": 0}


def shared_config(args, desc, extra):
    """The config both arms print (identical keys and values)."""
    return dict({"workload": desc, "state": "generated state, %d warm-up steps, then the timed steps" % args.warmup,
                 "l2": "inputs larger than L2 (per-step working set > 126 MB)"}, **extra)


# --------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.p = None
        self.out = None
        try:
            self.out = open("/tmp/gb2_clocks_%d.csv" % os.getpid(), "w")
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                       "-i", str(device), "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
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


def algorithmic_bytes(n, cen, nfix_plane, nfix_mesh, split=False):
    """Algorithmic HBM bytes per launch of k_pair_step: the owned atoms' own
    records, list indices and shear history that must cross HBM once;
    neighbour-state gathers are served from L2 and not counted."""
    avg = lambda k: 0.5 * (cen[0][k] + cen[1][k])
    # own x,v,w,r,m,type 92 + list counts 8 + touch mask 16 + xhold 24 + x,v,w out 72
    # (+ the 32-byte FP32 kinematics record written in split precision)
    per_atom = 92 + 8 + 16 + 24 + 72 + (32 if split else 0) + nfix_plane * 1 + nfix_mesh * 4
    b = n * per_atom + avg("nlist") * 4 + avg("nrev") * 4 + avg("ntouch") * (52 + 25)
    b += avg("nwall_touch") * 48 + avg("nmesh_cand") * 4 + avg("nmesh_touch") * 52
    return b


def load_traffic(kernel, workload):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            d = json.load(fh)
        return d.get(workload, {}).get(kernel)
    except Exception:
        return None


# --------------------------------------------------------------- the reference binary

def ref_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    return ref


LOOP_RE = re.compile(r"Loop time of ([0-9.eE+-]+) on \d+ procs for (\d+) steps with (\d+) atoms")


def write_reference_input(sc, warmup, steps, wd):
    """read_data file, STL meshes and input script of the scenario in the
    reference's grammar: `run warmup` (setup included) then `run steps`."""
    ref = ref_module()
    ref.write_data(os.path.join(wd, "data.txt"), sc)
    lines = ref.script(sc, wd, [max(warmup, 0), steps], None, thermo=0)
    path = os.path.join(wd, "in.bench")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path


def run_reference_replicas(script, wd, nproc):
    """nproc copies of lmp_ref on the script at once; per replica (atoms,
    steps, loop seconds) of its last run."""
    ref = ref_module()
    procs = []
    for r in range(nproc):
        scr = os.path.join(wd, "screen%d.txt" % r)
        procs.append((subprocess.Popen([ref.LMP, "-in", script, "-log", "none", "-screen", scr],
                                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, cwd=wd), scr))
    out = []
    for p, scr in procs:
        _, err = p.communicate()
        txt = open(scr).read() if os.path.exists(scr) else ""
        loops = LOOP_RE.findall(txt)
        if p.returncode != 0 or len(loops) < 2:
            raise RuntimeError("lmp_ref failed (rc %d): %s %s" % (p.returncode, err.decode()[-500:], txt[-1500:]))
        t, k, n = loops[-1]
        out.append((int(n), int(k), float(t)))
    return out


def reference_steps_cap(n, steps, seconds):
    """Timed steps of a reference replica: K, capped so a replica's window
    stays near `seconds` at ~3e6 particle-steps/s per core (the reference's
    measured rate on the packed 1M hopper, one core)."""
    est = n / 3.0e6
    return max(1, min(steps, int(seconds / max(est, 1e-9))))


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def avail_bytes():
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 8 << 30


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


def reference_arm(args):
    """The reference (lmp_ref) on all host cores the memory allows: one
    single-threaded replica per core, all on the same generated state, W
    warm-up steps then the timed steps; value = summed particle-steps/s from
    each replica's own "Loop time"."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc, desc, extra = make_workload(args)
    n = len(sc["atoms"]["tag"])
    ref = ref_module()
    cores = host_cores()
    k = reference_steps_cap(n, args.steps, args.ref_seconds)
    W0 = max(args.warmup, 3)
    line = {"metric": METRIC, "unit": UNIT, "n_gpus": ws, "steps": k, "warmup": W0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": shared_config(argparse.Namespace(warmup=W0), desc, extra)}
    if not ref.available():
        line.update({"value": None, "unavailable": "reference binary oracle/_ref/lmp_ref not built"})
        print(json.dumps(line), flush=True)
        return
    per = 250e6 + 900.0 * n          # resident bytes per replica (511 MB measured at 1M atoms)
    nproc = max(1, min(cores, int(0.7 * avail_bytes() // per)))
    wd = tempfile.mkdtemp(prefix="gb2bench_ref_")
    try:
        script = write_reference_input(sc, W0, k, wd)
        res = run_reference_replicas(script, wd, nproc)
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    val = sum(na * ka / ta for na, ka, ta in res)
    tmax = max(t for _, _, t in res)
    sample = ("%s; LIGGGHTS-PUBLIC 3.8.0 built from its sources (oracle/_ref/lmp_ref, g++ -O2, serial with MPI "
              "stubs), %d single-threaded replicas on %d host cores at once, each %d warm-up + %d timed steps "
              "(\"Loop time\")" % (desc, nproc, cores, W0, k))
    line.update({"value": val, "ms_per_step": 1e3 * tmax / k,
                 "cpu_baseline": {"value": val, "unit": UNIT, "cores": nproc, "kind": "reference", "sample": sample},
                 "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


PROFILE_EVERY = 16   # per-kernel CUDA events on every 16th step of a window


def force_frames(sc, eng, nframes, every, device, g=9.81):
    """Force error of the split-precision path on frames of an FP64 run.
    Every `every` steps the FP64 run's state is downloaded (atoms, pair,
    wall and mesh contact histories, mesh nodes) and restarted into a fresh
    FP64 and a fresh split context; each computes the forces at that state
    (setup, shear history not advanced) and they are compared atom by atom.
    Per frame: max |df| / max |f|, the RMS ratio, and the 99.9th percentile
    and maximum of the per-atom error |df_i| / (|f_i| + m_i g) (torques:
    |dt_i| / (|t_i| + r_i m_i g)), all with max-norm over components."""
    import granb200
    frames = []
    for fr in range(nframes):
        eng.run(every)
        snap = eng.snapshot(sc)
        sc2 = granb200.restart_scenario(sc, snap["atoms"], {i: m["nodes"] for i, m in snap["meshes"].items()})
        res = {}
        for prec in (granb200.PREC_FP64, granb200.PREC_SPLIT):
            e = granb200.Engine(sc2, precision=prec, device=device)
            e.restore(snap)
            e.setup()
            a = e.atoms()
            order = np.argsort(a["tag"])
            res[prec] = {k: a[k][order] for k in ("f", "torque", "tag")}
            e.close()
            del e
        f64, f32 = res[granb200.PREC_FP64]["f"], res[granb200.PREC_SPLIT]["f"]
        t64, t32 = res[granb200.PREC_FP64]["torque"], res[granb200.PREC_SPLIT]["torque"]
        at = sc2["atoms"]
        o = np.argsort(at["tag"])
        mg = np.asarray(at["rmass"])[o] * g
        rad = np.asarray(at["radius"])[o]
        df = np.abs(f32 - f64).max(axis=1)
        dt = np.abs(t32 - t64).max(axis=1)
        ef = df / (np.abs(f64).max(axis=1) + mg)
        et = dt / (np.abs(t64).max(axis=1) + rad * mg)
        frames.append({"frame": fr, "rel_max_force": float(df.max() / max(np.abs(f64).max(), 1e-300)),
                       "rel_rms_force": float(np.sqrt((df ** 2).mean() / max((np.abs(f64).max(axis=1) ** 2).mean(),
                                                                             1e-300))),
                       "atom_p999_force": float(np.percentile(ef, 99.9)), "atom_max_force": float(ef.max()),
                       "atom_p999_torque": float(np.percentile(et, 99.9)), "atom_max_torque": float(et.max())})
        print("frame %d: %s" % (fr, frames[-1]), file=sys.stderr, flush=True)
    keys = [k for k in frames[0] if k != "frame"]
    return {"frames": len(frames), "steps_between": every,
            "max_over_frames": {k: max(f[k] for f in frames) for k in keys},
            "median_over_frames": {k: float(np.median([f[k] for f in frames])) for k in keys},
            "method": force_frames.__doc__.split("\n\n")[0].replace("\n", " ").strip(),
            "per_frame": frames}


def timed_window(eng, steps, dist, device, clocks=True, profile=True, every=PROFILE_EVERY):
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
    if profile:
        eng.set_profiling(True, every=every)
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
                                       note="CUDA events on every %dth step of the window (%d steps sampled)"
                                            % (every, npm)),
            "launches": st1["kernel_launches"] - st0["kernel_launches"],
            "rebuilds": st1["nsteps_rebuild"] - st0["nsteps_rebuild"],
            "growth": st1["ngrow"] - st0["ngrow"],
            "capacities": {k: st1[k] for k in ("maxneigh", "maxpartner", "maxrev", "maxmesh")}}


def long_window(eng, steps, dist, device):
    """A longer window continuing the run: neighbour rebuilds happen here.
    Rebuild cost per step = the device time of the sampled rebuild steps'
    rebuild kernels, scaled to all rebuilds, over the window's steps."""
    W = timed_window(eng, steps, dist, device, clocks=False)
    nreb = max(W["rebuilds"], 0)
    out = {"steps": steps, "ms_per_step": W["ms"] / steps, "rebuilds": nreb,
           "kernel_ms_per_step": W["kernel_ms_per_step"], "census_start": W["cen"][0], "census_end": W["cen"][1],
           "launches": W["launches"], "capacity_growth": W["growth"],
           "rebuild_ms_each": W["kt"]["t_rebuild"] / nreb if nreb else None,
           "rebuild_ms_per_step": W["kt"]["t_rebuild"] / steps,
           "note": "every rebuild timed with CUDA events (rebuild kernels, device time); the other kernels on "
                   "every %dth step" % PROFILE_EVERY}
    return out, W


def check_floors(args, n, cen):
    """The default workload must hold config 2's work at the window start."""
    if args.workload != "hopper" or n < 1_000_000:
        return None
    ok = cen["ntouch"] >= FLOOR_TOUCH_PER_ATOM * n and cen["nmesh_touch"] >= FLOOR_MESH_CONTACTS
    if not ok:
        raise SystemExit("bench: the timed state lacks config 2's work: %d touching pairs (need %d), %d mesh "
                         "contacts (need %d)" % (cen["ntouch"], FLOOR_TOUCH_PER_ATOM * n, cen["nmesh_touch"],
                                                 FLOOR_MESH_CONTACTS))
    return {"touching_pairs_per_atom_min": FLOOR_TOUCH_PER_ATOM, "mesh_contacts_min": FLOOR_MESH_CONTACTS,
            "met": True}


def own_arm(args):
    ws, rank, local, dist = dist_init()
    import granb200
    sc, desc, extra = make_workload(args, seed_offset=rank)
    n = len(sc["atoms"]["tag"])
    nfix_plane = sum(1 for f in sc["fixes"] if f["kind"] in ("wall_plane", "wall_cylinder"))
    nfix_mesh = sum(1 for f in sc["fixes"] if f["kind"] == "wall_mesh")
    W0 = max(args.warmup, 3)

    # headline: FP64, bit-exact with the reference
    eng = granb200.Engine(sc, precision=granb200.PREC_FP64, device=local)
    eng.setup()
    eng.run(W0)
    cen_start = eng.census()
    floors = check_floors(args, n, cen_start)
    W = timed_window(eng, args.steps, dist, local)
    value = n * args.steps * ws / (W["ms"] * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": W0,
        "ms_per_step": W["ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": shared_config(argparse.Namespace(warmup=W0), desc, extra),
        "precision": "fp64: IEEE FP64 throughout, FMA contraction off, bit-exact with the reference",
        "parallelism": "replicas x%d (no data-path collective)" % ws if ws > 1 else "single GPU",
        "gpu_launches": W["launches"],
        "clocks": W["clocks"],
        "kernel_ms_per_step": W["kernel_ms_per_step"],
        "census_window_start": cen_start,
        "census_floors": floors,
        "rebuilds": W["rebuilds"],
        "capacity_growth_in_window": W["growth"],
        "capacities": W["capacities"],
    }

    # roofline: right after the headline window (the same state), every
    # pair-step launch of a short window timed with CUDA events
    dom = "k_pair_step"
    peak, peak_kind = peaks()
    if args.roofline_steps > 0:
        WR = timed_window(eng, args.roofline_steps, dist, local, clocks=False, every=1)
        kt_src, npm, cen_src, src = WR["kt"], WR["npm"], WR["cen"], "%d steps right after the headline window" % (
            args.roofline_steps)
    else:
        kt_src, npm, cen_src, src = W["kt"], W["npm"], W["cen"], "headline window (every %dth step)" % PROFILE_EVERY
    dom_ms = kt_src["t_pair_main"] / max(npm, 1)
    ab = algorithmic_bytes(n, cen_src, nfix_plane, nfix_mesh, False)
    achieved = ab / (dom_ms * 1e-3) / 1e9 if npm > 0 and dom_ms > 0 else None
    traffic = load_traffic(dom, args.workload)
    # the capture's DRAM bytes belong to its own state (census at capture):
    # the ratio to the algorithmic bytes is taken there, and the per-launch
    # traffic of this window is that ratio times this window's algorithmic bytes
    t_ratio = None
    if traffic and traffic.get("algorithmic_bytes_at_capture"):
        t_ratio = traffic["bytes_per_launch"] / traffic["algorithmic_bytes_at_capture"]
    line["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak if achieved else None, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                        "traffic": t_ratio * ab if t_ratio and ab else None,
                        "traffic_over_algorithmic": t_ratio,
                        "algorithmic_bytes_per_launch": ab, "avg_launch_ms": dom_ms, "sampled_launches": npm,
                        "timing": "every pair-step launch timed with CUDA events over the %s" % src}
    if traffic:
        line["roofline"]["traffic_source"] = (traffic.get("capture", "") + "; measured %d bytes at a state of %d "
                                              "algorithmic bytes, scaled to this window by its algorithmic bytes"
                                              % (traffic["bytes_per_launch"],
                                                 traffic.get("algorithmic_bytes_at_capture", 0)))

    # longer FP64 window with rebuilds
    if args.long_steps > 0:
        lw, WL = long_window(eng, args.long_steps, dist, local)
        line["long_window"] = lw
        dl = WL["kt"]["t_pair_main"] / max(WL["npm"], 1)
        abl = algorithmic_bytes(n, WL["cen"], nfix_plane, nfix_mesh, False)
        lw["pair_step_roofline"] = {"avg_launch_ms": dl, "algorithmic_bytes_per_launch": abl,
                                    "achieved_gbs": abl / (dl * 1e-3) / 1e9 if WL["npm"] and dl > 0 else None,
                                    "frac": abl / (dl * 1e-3) / 1e9 / peak if WL["npm"] and dl > 0 else None}

    # FP64 vs split force error on frames of the FP64 run
    if args.force_frames > 0:
        line["force_error_frames"] = force_frames(sc, eng, args.force_frames, args.frame_every, local)
    eng.close()
    del eng

    # split precision from the same generated state (same warm-up)
    if not args.no_split:
        e32 = granb200.Engine(sc, precision=granb200.PREC_SPLIT, device=local)
        e32.setup()
        e32.run(W0)
        W32 = timed_window(e32, args.steps, dist, local, clocks=False)
        v32 = n * args.steps * ws / (W32["ms"] * 1e-3)
        line["split_gpu"] = {"value": v32, "unit": UNIT, "steps": args.steps, "ms_per_step": W32["ms"] / args.steps,
                             "kernel_ms_per_step": W32["kernel_ms_per_step"],
                             "precision": "FP32 contact math on FP64-differenced positions and FP64 overlap, Kahan "
                                          "FP32 pair sums; FP64 walls, gravity, integration"}
        line["split_over_fp64"] = v32 / value
        if args.long_steps > 0:
            lw32, _ = long_window(e32, args.long_steps, dist, local)
            line["split_gpu"]["long_window"] = lw32
            if "long_window" in line:
                line["split_over_fp64_long"] = line["long_window"]["ms_per_step"] / lw32["ms_per_step"]
        e32.close()
        del e32

    # end to end through the C ABI: pinned host arrays in, setup, K steps, host arrays out
    if not args.no_e2e:
        a = sc["atoms"]
        host = {}
        for k in ("x", "v", "omega"):
            host[k] = granb200.pinned_empty((n, 3))
            host[k][:] = a[k]
        for k in ("radius", "rmass"):
            host[k] = granb200.pinned_empty((n,))
            host[k][:] = a[k]
        for k in ("type", "tag"):
            host[k] = granb200.pinned_empty((n,), np.int32)
            host[k][:] = a[k]
        out = {k: granb200.pinned_empty((n, 3)) for k in ("x", "v", "omega", "f", "torque")}
        out["tag"] = granb200.pinned_empty((n,), np.int32)
        sc2 = dict(sc)
        sc2["atoms"] = dict(a, **host)
        barrier(dist)
        t0 = time.perf_counter()
        e2 = granb200.Engine(sc2, precision=granb200.PREC_FP64, device=local)
        t1 = time.perf_counter()
        e2.setup()
        e2.sync()
        t2 = time.perf_counter()
        e2.run(args.steps)
        e2.sync()
        t3 = time.perf_counter()
        e2.atoms(out)
        t4 = time.perf_counter()
        dt = allmax(dist, t4 - t0)
        h2d = n * (3 * 3 * 8 + 2 * 8 + 2 * 4) + sum(f["nodes"].size * 8 for f in sc["fixes"] if f["kind"] == "wall_mesh")
        d2h = n * (5 * 3 * 8 + 4)
        line["e2e"] = {"value": n * args.steps * ws / dt, "unit": UNIT,
                       "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                       "includes": "context create, materials, atom + mesh upload from pinned host memory, Verlet "
                                   "setup, %d FP64 steps from the generated state, download of x/v/omega/f/torque/tag "
                                   "into pinned host memory" % args.steps,
                       "seconds": {"create_upload": t1 - t0, "setup": t2 - t1, "run": t3 - t2, "download": t4 - t3}}
        e2.close()
        del e2

    # CPU baseline: the reference itself on one core, same generated state
    if rank == 0 and ws == 1 and not args.no_cpu:
        ref = ref_module()
        if ref.available():
            k = reference_steps_cap(n, args.steps, args.cpu_seconds)
            wd = tempfile.mkdtemp(prefix="gb2bench_cpu_")
            try:
                script = write_reference_input(sc, W0, k, wd)
                (na, ka, ta), = run_reference_replicas(script, wd, 1)
            finally:
                shutil.rmtree(wd, ignore_errors=True)
            line["cpu_baseline"] = {"value": na * ka / ta, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": "lmp_ref (the reference built from its sources), 1 process, same "
                                              "generated %d-particle state, %d warm-up + %d timed steps (\"Loop "
                                              "time\")" % (n, W0, ka)}
        else:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": "reference binary not built"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def sq_arm(args):
    """Superquadric packing: plain first-contact solve against the learned
    initial guess, same particles, same steps, device-timed."""
    import granb200
    import gb2_scenarios as S
    n = args.particles or 200_000
    settle = args.settle or 100
    t0 = time.perf_counter()
    tr = granb200.MlpTrainer()
    # ~5M labelled pairs: the oriented boxes of about 65% of the candidate
    # pairs intersect, and only those are kept
    info = tr.make_data(7_800_000, seed=1)
    tr.init(seed=2)
    l0, l1 = tr.train(epochs=4, batch=4096, lr=2e-3)
    ev = tr.evaluate(100_000, seed=99)
    train_s = time.perf_counter() - t0
    solve = tr.time_solves(400_000, seed=123)   # first-contact solves alone, same pairs both ways
    params = tr.params()
    sc = S.sq_packing(n=n, seed=11)
    res = {}
    # each arm is timed args.sq_reps times, alternating, every time from a
    # fresh engine on the same particles (the work is identical run to run:
    # same iteration and solve counts); the median window is reported
    runs = {"plain": [], "learned": []}
    for rep in range(max(1, args.sq_reps)):
        for name, learned in (("plain", None), ("learned", params)):
            e = granb200.SqEngine(sc, learned=learned)
            e.setup()
            e.run(settle)
            e.run(max(args.warmup, 3))
            c0 = e.counters()
            sampler = ClockSampler(0)
            time.sleep(0.3)   # the sampler's first reading lands inside the window
            ms = e.run_timed(args.steps)
            clk = sampler.stop()
            c1 = e.counters()
            runs[name].append((ms, clk, {
                "newton_iters": c1["iters"] - c0["iters"], "newton_solves": c1["solves"] - c0["solves"],
                "pairs_solved": c1["pairs_solved"] - c0["pairs_solved"],
                "learned_accepted": c1["learned_used"] - c0["learned_used"],
                "learned_rejected": c1["learned_rejected"] - c0["learned_rejected"]}))
            e.close()
    for name, rr in runs.items():
        order = sorted(range(len(rr)), key=lambda q: rr[q][0])
        ms, clk, cnt = rr[order[len(rr) // 2]]
        res[name] = dict({"ms_per_step": ms / args.steps, "value": n * args.steps / (ms * 1e-3),
                          "ms_per_step_runs": [r[0] / args.steps for r in rr], "clocks": clk}, **cnt)
    line = {
        "metric": "particle-steps/s @200k superquadrics, learned vs plain initial guess", "unit": UNIT,
        "value": res["learned"]["value"], "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["learned"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 contact solve, bf16 MLP", "data": "synthetic",
        "config": {"workload": "sq-packing-%d: half-axes U(1,2) mm, blockiness U(2,8), random orientations, "
                               "Hertz/history, dt 1e-5, random velocities +-1 m/s" % n,
                   "settle_steps": settle},
        "plain": res["plain"], "learned": res["learned"],
        "learned_over_plain": res["learned"]["value"] / res["plain"]["value"],
        "first_contact_solve": dict(solve, note="contact-point solve of fresh pairs near contact (a new "
                                                "contact's first solve), plain homotopy vs learned guess with "
                                                "homotopy fallback, each launch timed alone"),
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
