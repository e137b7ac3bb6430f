"""Benchmark of the per-turn weak-weak tracking loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload uniform|single|uneven|beam_ion|beam_ion_mlp|slice_fbii]

Default workload (the uniform multi-bunch configuration): all 416 buckets
filled at 0.5 nC, 2e4 macroparticles per bunch (8.32e6, 400 MB of FP64
coordinates, larger than the 126 MB L2 so no flush is needed), long-range
resistive wall over a 50-turn history plus a longitudinal HOM, quantum
excitation on.  One step is one turn of the whole ring.

b200 arm: `value` is device-timed (CUDA events on the context's stream)
throughput with the beam resident in HBM; `e2e` goes through mbt_track, the
host-buffer C-ABI call, with the beam uploaded from pinned host memory and
statistics and beam downloaded inside the timed region; `roofline` times the
particle-pass kernel alone with CUDA events between the kernels of a turn.
With N GPUs every rank tracks its own independent ring (replicas, weak
scaling); the time is the max over ranks.

reference arm: the reference's own CPU code (oracle/_ref, the reference's
sources compiled unmodified; the C restatement in oracle/ when that library
is absent) on the host cores, bunches split across one process per core.

slice_fbii: the reference's slice model (BunchModel = STRONG) with fast
beam-ion interaction (include/mbt_ws.h) on the 200-bunch train, 47 slices per
bunch; metric turns/s of the whole ring, the reference arm its own
functions on one core (its ion train passes bunch to bunch in sequence).
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import re
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFS = os.path.join(ROOT, "tests", "confs")
WORKLOADS = {
    "uniform": ("uniform_fill.conf", {}, "uniform fill: 416 bunches x 2e4 macroparticles, long-range RW "
                                         "(50-turn history) + HOM, quantum excitation on"),
    "single": ("single_bunch.conf", {"EnableQuantum": 1}, "single bunch: 1e5 macroparticles, broadband "
                                                          "resonator in 3 planes, quantum excitation on"),
    "uneven": ("uneven_fill.conf", {}, "uneven fill: 321 bunches incl. 5 nC camshaft, RW + HOM + RF "
                                       "feedback, quantum excitation on"),
    "beam_ion": ("beam_ion.conf", {}, "beam-ion weak-strong: 200-bunch train x 5e4 macroparticles, CO at "
                                      "1 nTorr, 20 interaction points, 1000 macro-ions per passage per point, "
                                      "Faddeeva-based Bassetti-Erskine fields"),
    "beam_ion_mlp": ("beam_ion.conf", {}, "beam-ion weak-strong: 200-bunch train x 5e4 macroparticles, CO at "
                                          "1 nTorr, 20 interaction points, 1000 macro-ions per passage per "
                                          "point, learned field (tensor-core MLP, 1% audit)"),
    "combined": ("combined.conf", {}, "combined: uneven fill (321 bunches incl. 5 nC camshaft, macroparticles "
                                      "proportional to charge, 2e3..1e5, 8e6 in all), RW + HOM + RF feedback with a "
                                      "generator loop (gain 10, one-turn delay), beam-ion (CO 1 nTorr, 20 points, 1000 "
                                      "macro-ions per passage per point) with the learned field and a 1% audit, "
                                      "quantum excitation on"),
    "slice_fbii": ("slice_fbii.conf", {"Nslc": 23, "Np": 5000, "Iring": 84.6, "NrevTot": 1000, "NrevMon": 100},
                   "slice model (BunchModel = STRONG) with fast beam-ion interaction: 200-bunch train, 47 "
                   "slices x 25 grid points per bunch (1175 macro-ions), long-range RW over 10 turns"),
}
SLICE_FLOP_PER_PULL = 40   # FP64 operations of one ion-slice pull in the reference's expressions
BEAM_ION_CPU_SCALE = 100   # the CPU sample keeps 1/100 of the electrons and of the ions
BYTES_PER_MP_TURN = 96   # 6 FP64 coordinates read and written per macroparticle per turn
METRIC = "macroparticle-turns/s"


def conf_path(workload, tmpdir):
    from oracle.binding import conf_with
    name, over, _ = WORKLOADS[workload]
    src = os.path.join(CONFS, name)
    over = dict(over)
    if "uneven" in name or workload == "combined":
        over["filling"] = os.path.join(CONFS, "uneven_fill.txt")
    if "beam_ion" in name or workload == "slice_fbii":
        over["filling"] = os.path.join(CONFS, "beam_ion_fill.txt")
    if not over:
        return src
    return conf_with(src, os.path.join(tmpdir, name), **over)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(workload):
    """DRAM bytes per particle-pass launch from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "turn_map_%s_fill.md" % workload)
    if not os.path.exists(p):
        p = os.path.join(ROOT, "profiles", "turn_map_%s.md" % workload)
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.out = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ CPU side

def _cpu_worker(args):
    """One host process: bunches [lo, hi) of the ring for `turns` turns;
    returns the wall time of each turn.  Loads the reference's library
    (oracle/_ref) or the C restatement (oracle/), never libmbt."""
    kind, conf, lo, hi, turns = args
    sys.path.insert(0, ROOT)
    import numpy as np
    from oracle.binding import Oracle, Reference, beam_ion_section
    if kind == "beam_ion":
        # no reference code exists for this stage: the C restatement, its
        # ring and bunches as the reference's own parser reads the file
        p, bucket, npb, ib, Gl, Gv, Gh = Reference(conf, private=False).oracle_inputs()
        bi = beam_ion_section(conf)
        bi.ions_per_passage = max(1, bi.ions_per_passage // BEAM_ION_CPU_SCALE)
        O = Oracle(p, bucket, np.maximum(2, npb // BEAM_ION_CPU_SCALE), ib, Gl, Gv, Gh)
        O.generate_beam()
        O.prepare()
        O.enable_beam_ion(bi)
        step = lambda: O.lib.orc_run(O.h, 1, None, None, None, 0)   # noqa: E731
    elif kind == "reference":
        R = Reference(conf, bunch_range=(lo, hi), private=False)
        R.prepare()
        step = lambda: R.lib.refh_run(1, None, None, 0)   # noqa: E731
    else:
        p, bucket, npb, ib, Gl, Gv, Gh = Reference(conf, private=False).oracle_inputs()
        O = Oracle(p, bucket, npb, ib, Gl, Gv, Gh)
        O.set_range(lo, hi)
        O.generate_beam()
        O.prepare()
        step = lambda: O.lib.orc_run(O.h, 1, None, None, None, 0)   # noqa: E731
    times = []
    for _ in range(turns):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    return times


def _ring_probe(conf):
    """(bunches, macroparticles per bunch) as the reference's own parser
    reads the file (a spawned process; libmbt is not loaded)."""
    sys.path.insert(0, ROOT)
    from oracle.binding import Reference
    R = Reference(conf, private=False)
    return int(R.nb), [int(x) for x in R.np]


def cpu_kind():
    from oracle import binding
    if binding.build_reference() is not None:
        return "reference"
    binding.build_oracle()
    return "port"


def cpu_run(workload, turns, tmpdir, cores=None):
    """Time `turns` turns of the whole ring on the host cores (bunches split
    over one process per core).  Returns (per-turn seconds list, info).
    Every process is spawned and loads only the reference's library or the
    C restatement."""
    conf = conf_path(workload, tmpdir)
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        nb, npb = pool.apply(_ring_probe, (conf,))
    particles = int(sum(npb))
    if workload.startswith("beam_ion"):
        # no reference code for this stage: the C restatement (oracle) on one
        # core, 1/BEAM_ION_CPU_SCALE of the electrons and ions, the time per
        # turn scaled back up (the work is linear in both counts)
        with ctx.Pool(1) as pool:
            res = pool.map(_cpu_worker, [("beam_ion", conf, 0, nb, turns)])
        per_turn = [x * BEAM_ION_CPU_SCALE for x in res[0]]
        return per_turn, {"kind": "port", "cores": 1, "bunches": nb, "particles": particles,
                          "np_per_bunch": npb[0], "scaled": BEAM_ION_CPU_SCALE}
    if cores is None:
        cores = len(os.sched_getaffinity(0))
    procs = max(1, min(cores, nb))
    edges = [round(i * nb / procs) for i in range(procs + 1)]
    kind = cpu_kind()
    jobs = [(kind, conf, edges[i], edges[i + 1], turns) for i in range(procs)]
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, jobs)
    per_turn = [max(r[t] for r in res) for t in range(turns)]
    info = {"kind": kind, "cores": procs, "bunches": nb, "particles": particles, "np_per_bunch": npb[0]}
    return per_turn, info


# ------------------------------------------------------------ GPU side

def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def run_b200(args):
    import numpy as np
    import torch
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from mbtrack_b200 import api
    import tempfile
    tmp = tempfile.mkdtemp()
    conf = conf_path(args.workload, tmp)
    cfg = api.Config(conf)
    np_model = args.np_per_bunch or cfg.params.np_model
    npart = int(cfg.nbunch * np_model)

    # CPU baseline first (spawned processes; rank 0 at N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        per_turn, info = cpu_run(args.workload, args.cpu_turns, tmp)
        t = float(np.mean(per_turn[1:])) if len(per_turn) > 1 else per_turn[0]
        cpu = {"value": npart / t, "unit": METRIC, "cores": info["cores"], "kind": info["kind"],
               "sample": "%d turns of the whole ring (%d bunches x %d macroparticles) split over %d "
                         "processes, one per core; first turn dropped; time = slowest process"
                         % (args.cpu_turns, info["bunches"], info["np_per_bunch"], info["cores"])}
        if info.get("scaled"):
            cpu["sample"] = ("%d turns of the C restatement (no reference code exists for this stage) on one "
                             "core with 1/%d of the electrons and of the macro-ions, time scaled by %d; first "
                             "turn dropped" % (args.cpu_turns, info["scaled"], info["scaled"]))

    tiles = None
    if args.workload in ("uneven", "combined"):
        # macroparticles proportional to the bunch charge, clamped to
        # 2e3 .. 1e5, about 8e6 in total
        frac = np.asarray(cfg.ib_frac, dtype=np.float64)
        lo, hi = 1.0, 1e7
        for _ in range(100):
            k = math.sqrt(lo * hi)
            tot = np.clip(np.rint(k * frac), 2000, 100000).sum()
            lo, hi = (k, hi) if tot < 8e6 else (lo, k)
        npb = np.clip(np.rint(k * frac), 2000, 100000).astype(np.int32)
        trk = api.Tracker(cfg.params, cfg.bucket, npb, cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh,
                          seed=1000 + rank)
        npart = int(npb.sum())
    else:
        trk = api.Tracker.from_config(cfg, np_per_bunch=np_model, seed=1000 + rank)
    trk.generate_beam(77 + rank)
    bi_info = None
    if args.workload.startswith("beam_ion") or args.workload == "combined":
        bi = cfg.beam_ion()
        bi.surrogate = 1 if args.workload in ("beam_ion_mlp", "combined") else 0
        if args.n_ip:
            bi.n_ip = args.n_ip
        if args.ions_per_passage:
            bi.ions_per_passage = args.ions_per_passage
        trk.enable_beam_ion(bi)
        bi_info = {"n_ip": bi.n_ip, "ions_per_passage": bi.ions_per_passage,
                   "field_evaluations_per_turn": bi.n_ip * (bi.ions_per_passage * cfg.nbunch * (cfg.nbunch - 1) // 2
                                                            + (npart - int(trk.np[0])))}
        if bi.surrogate:
            mlp = api.Mlp(seed=31 + rank)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tr = dict(api.MLP_TRAIN, steps=args.mlp_steps or api.MLP_TRAIN["steps"])
            hist = mlp.train(seed=32 + rank, **tr)
            torch.cuda.synchronize()
            bi_info["training"] = dict(tr, seconds=time.perf_counter() - t0, final_loss=float(hist[-1]))
            trk.use_mlp(mlp)
    init_stats = trk.prepare()
    if args.workload in ("uneven", "combined"):
        tiles = [int(x) for x in trk.autotune(trial_turns=10 if args.workload == "uneven" else 2)]
    trk.run(args.warmup, stats=False)
    if bi_info is not None and bi_info.get("training"):
        trk.beam_ion_audit()   # reset the audit counters before the timed region

    # timed region: device time of K turns (CUDA events inside mbt_run_turns)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        stats = trk.run(args.steps, stats=True)
    torch.cuda.synchronize()
    dev_ms = float(trk.timing()[0][3])
    t_local = dev_ms / 1e3
    if dist:
        tt = torch.tensor([t_local], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
        dist.barrier()
    else:
        t_max = t_local
    value = world * npart * args.steps / t_max

    audit = trk.beam_ion_audit() if (bi_info is not None and bi_info.get("training")) else None
    # per-kernel device times (events between the four kernels of a turn)
    prof = trk.profile(args.profile_turns)
    k1_ms = float(prof[0])
    if bi_info is not None:
        bi_ms = trk.beam_ion_timing()
        bi_info["stage_ms_per_turn"] = bi_ms
        bi_info["kernels_ms_per_turn"] = dict(zip(("frames", "ions", "clouds", "kick"),
                                                  [float(v) for v in trk.beam_ion_kernel_times()]))
        bi_info["field_evaluations_per_s"] = bi_info["field_evaluations_per_turn"] / (bi_ms * 1e-3)
        if audit is not None:
            bi_info["audit"] = {"audited": int(audit[0]), "max_rel_error": float(audit[1]),
                                "rms_rel_error": float(audit[2]), "faddeeva_fallbacks": int(audit[3]),
                                "tensor_failures": int(audit[4]),
                                "fallback_fraction": int(audit[3]) / float(bi_info["field_evaluations_per_turn"]
                                                                           * args.steps)}
            # network FLOPs: 2 x (3x128 + 2x128x128 + 128x2) per evaluation
            tfl = 66816.0 * bi_info["field_evaluations_per_turn"] / (bi_ms * 1e-3) / 1e12
            bi_info["network_tflops"] = tfl
        if args.workload == "combined":
            bi_info.update(combined_extras(args, cfg, trk, mlp, init_stats, tiles, tmp))
        elif args.growth_turns > 0 and bi.surrogate:
            bi_info["growth_check"] = growth_check(cfg, mlp, args.growth_turns)
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_MP_TURN * npart / (k1_ms * 1e-3) / 1e9
    traffic = profile_traffic(args.workload)

    # end to end through mbt_track with pinned host buffers
    e2e_turns = args.e2e_turns if bi_info is None else min(args.e2e_turns, 5)
    pinned = torch.empty(6 * npart, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    host[:] = trk.get_all()
    st_pinned = torch.empty(e2e_turns * cfg.nbunch * 12, dtype=torch.float64, pin_memory=True)
    st_host = st_pinned.numpy()
    e2e_t = []
    for _ in range(args.e2e_steps + 1):
        t0 = time.perf_counter()
        trk.track(host, e2e_turns, st_host)
        e2e_t.append(time.perf_counter() - t0)
    e2e_sec = float(np.mean(e2e_t[1:]))
    if dist:
        tt = torch.tensor([e2e_sec], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_sec = float(tt.item())
    e2e_value = world * npart * e2e_turns / e2e_sec
    ok = bool(np.all(np.isfinite(stats)))
    trk.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    _, name_over, desc = WORKLOADS[args.workload]
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "bunches": int(cfg.nbunch), "np_per_bunch": int(np_model),
                   "macroparticles": npart, "turns_per_step": 1, "noise": "Philox4x32-10 counter RNG",
                   "l2": "beam of %.0f MB > 126 MB L2, no flush" % (npart * 48 / 1e6),
                   "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": (None if traffic is None else
                                        "dram__bytes_read.sum + dram__bytes_write.sum of one launch from the "
                                        "committed ncu summary in profiles/ (not measured by this run)"),
                     "kernel": "turn_map (particle pass)", "peak_source": peak_kind,
                     "bytes_per_launch": BYTES_PER_MP_TURN * npart, "launch_ms": k1_ms},
        "kernels_ms_per_turn": {"turn_map": k1_ms, "bunch_reduce": float(prof[1]),
                                "ring_scan": float(prof[2]), "bunch_wakes": float(prof[3])},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 6 * 8 * npart,
                "d2h_bytes_per_step": 6 * 8 * npart + e2e_turns * cfg.nbunch * 12 * 8,
                "turns_per_step": e2e_turns, "steps": args.e2e_steps,
                "call": "mbt_track (pinned host beam in, %d turns, stats + beam out)" % e2e_turns},
        "gpu_launches": (4 if bi_info is None else 8) * args.steps,
        "clocks": clk.summary(),
        "finite": ok,
    }
    if bi_info is not None:
        line["beam_ion"] = bi_info
        line["config"]["noise"] = "off"
    if tiles is not None:
        line["config"]["np_per_bunch"] = "proportional to charge, clamped to 2e3..1e5"
        line["config"]["tiles_per_size_class"] = {"np<=4096": tiles[0], "np<=32768": tiles[1], "larger": tiles[2]}
        line["config"]["tiles_chosen_by"] = "mbt_autotune (coordinate descent, 10 device-timed turns per candidate)"
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if args.workload == "uniform" and world == 1 and args.beam_ion_record:
        # the north star's ratio: learned vs Faddeeva field on the beam-ion
        # configuration, measured in the same run as the headline
        line["beam_ion"] = beam_ion_record(args, tmp)
        line["gpu_launches_beam_ion"] = 8 * (args.bi_steps + args.bi_warmup)
    print(json.dumps(line))


def run_reference(args):
    import numpy as np
    rank, world, _ = rank_info()
    if rank != 0:
        return
    import tempfile
    tmp = tempfile.mkdtemp()
    turns = args.warmup + args.steps
    if args.workload.startswith("beam_ion"):
        turns = 3 + min(args.steps, 2)   # about 10 s a turn even on the sample
    per_turn, info = cpu_run(args.workload, turns, tmp)
    if args.workload.startswith("beam_ion"):
        args.warmup, args.steps = 3, turns - 3
    timed = per_turn[args.warmup:]
    t = float(np.sum(timed))
    if info.get("scaled"):
        info["cores"] = 1
    value = info["particles"] * len(timed) / t
    _, _, desc = WORKLOADS[args.workload]
    sample = ("%d warm-up + %d timed turns of the whole ring (%d bunches) split over %d processes, "
              "one per core; time per turn = slowest process" % (args.warmup, args.steps, info["bunches"],
                                                                 info["cores"]))
    if info.get("scaled"):
        sample = ("%d warm-up + %d timed turns of the C restatement (no reference code exists for this stage) "
                  "on one core with 1/%d of the electrons and of the macro-ions, time per turn scaled by %d"
                  % (args.warmup, args.steps, info["scaled"], info["scaled"]))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "bunches": info["bunches"], "macroparticles": info["particles"],
                   "turns_per_step": 1, "parallelism": "%d host processes" % info["cores"]},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": info["cores"], "kind": info["kind"],
                         "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))




def slice_setup(conf):
    """Slice model of a BunchModel = STRONG file: the reference's generated
    bunch, its slicing and bunch offsets (all in libmbt's host code)."""
    from mbtrack_b200 import api
    w, bucket, frac = api.SliceModel.config(conf)
    L = api.lib()
    ib = [L.mbt_bunch_current(w.base, len(bucket), float(f)) * 1e3 for f in frac]
    soa, off = api.SliceModel.reference_beam(w, len(bucket))
    npop, nofe, cm4 = api.SliceModel.slice_beam(w, soa)
    return w, bucket, ib, npop, nofe, api.SliceModel.initial_slices(w, cm4, off)


def slice_cpu(conf, turns):
    """Seconds per turn of the reference's slice model on one core
    (oracle/_ref; the C restatement when that library is absent)."""
    from oracle import binding
    import numpy as np
    if binding.reference_available() or os.path.exists(binding.REF_SO):
        r = binding.ReferenceSlices(conf)
        kind = "reference"
        t0 = time.perf_counter()
        r.run(turns, 100)
    else:
        w, bucket, ib, npop, nofe, s0 = slice_setup(conf)
        r = binding.OracleSlices(w, bucket, ib, npop, nofe)
        r.set_slices(s0)
        kind = "port"
        t0 = time.perf_counter()
        r.run(turns)
    return (time.perf_counter() - t0) / turns, kind, r.nb



def slice_growth_compare(turns):
    """Growth rate of the vertical coupled-bunch motion in the slice model
    and in the per-particle beam-ion stage on one configuration: the
    200-bunch train of tests/confs/beam_ion.conf (same ring, fill and
    charge), CO at the slice model's pressure (2.7e-9 mbar x 5 x 0.15 / 1.3332
    = 1.519 nTorr, fbi_weakstrong.c:20-36) ionised over the whole
    circumference (one interaction point), no wall, no chromaticity (the
    slice model has none), no radiation noise or damping.  The slice model
    runs with the reference's ion kick factor 1e2 and with the thin-lens
    value 1; the per-particle stage with 5e3 macroparticles per bunch."""
    import numpy as np
    import torch
    import tempfile
    from mbtrack_b200 import analysis, api
    from oracle.binding import conf_with
    tmp = tempfile.mkdtemp()
    fill = os.path.join(CONFS, "beam_ion_fill.txt")
    out = {"config": "200-bunch train x 0.5 nC, CO at 1.519 nTorr over the ring, 1 interaction point, no wall, "
                     "no chromaticity, no radiation noise", "turns": turns}

    def envelope(z, zp, par):
        """rms over bunches of the betatron amplitude sqrt(beta J) of the
        vertical centroid (J the Courant-Snyder invariant): free of the
        turn-to-turn betatron phase."""
        g, a, b = par.gamma1[2], par.alpha1[2], par.beta1[2]
        inv = g * z * z + 2.0 * a * z * zp + b * zp * zp
        return np.sqrt((b * inv).mean(axis=1))

    def rate(a):
        wdw = analysis.exponential_window(a)
        return {"window": list(wdw) if wdw else None, "rate_per_turn": analysis.growth_rate(a, wdw) if wdw else None,
                "start": float(np.median(a[:50])), "max": float(a.max()),
                "amplitude_every_100_turns": [float(x) for x in a[::100]]}

    # bunch offsets of 0.1 um rms (slice model): a start below the
    # per-particle stage's sampling noise (0.26 um), as in a linear regime
    sconf = conf_with(os.path.join(CONFS, "slice_fbii.conf"), os.path.join(tmp, "s.conf"), Nslc=23, Np=5000,
                      Iring=84.6875, NrevTot=turns, NrevMon=100, EnableRW_long=0, filling=fill, xxCM_offset=0.0001,
                      xpCM_offset=0.00001, zzCM_offset=0.0001, zpCM_offset=0.00001)
    for kf in (1e2, 1.0):
        w, bucket, ib, npop, nofe, s0 = slice_setup(sconf)
        w.kick_factor = kf
        dev = api.SliceModel(w, bucket, ib, npop, nofe)
        dev.load_slices(s0)
        t0 = time.perf_counter()
        cm = dev.run(turns)[0]
        dev.close()
        r = rate(envelope(cm[:, :, 4], cm[:, :, 5], w.base))
        r["seconds"] = time.perf_counter() - t0
        out["slice_kick_factor_%g" % kf] = r
    pconf = conf_with(os.path.join(CONFS, "beam_ion.conf"), os.path.join(tmp, "p.conf"), NrevTot=turns, Cx=0.0,
                      Cz=0.0, EnableQuantum=0, n_ip=1, pressure_nTorr=0.15 * 5 * 2.7 / 1.3332, filling=fill)
    cfg = api.Config(pconf)
    t = api.Tracker(cfg.params, cfg.bucket, np.full(cfg.nbunch, 5000), cfg.bunch_currents())
    t.generate_beam(3)
    t.enable_beam_ion(cfg.beam_ion())
    t.prepare()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = t.run(turns)
    t.close()
    r = rate(envelope(st[:, :, 2], st[:, :, 8], cfg.params))
    r["seconds"] = time.perf_counter() - t0
    out["per_particle"] = r
    return out

def run_slice_b200(args):
    import numpy as np
    import torch
    from mbtrack_b200 import api
    import tempfile
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    tmp = tempfile.mkdtemp()
    conf = conf_path(args.workload, tmp)
    w, bucket, ib, npop, nofe, s0 = slice_setup(conf)
    nb = len(bucket)
    nion = w.slices * w.ngrid * w.ngrid
    pulls = nb * (nb - 1) // 2 * nion * w.slices
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sec, kind, _ = slice_cpu(conf, 1)
        cpu = {"value": 1.0 / sec, "unit": "turns/s", "cores": 1, "kind": kind,
               "sample": "1 turn of the whole %d-bunch ring on one core (%.1f s)" % (nb, sec)}
    dev = api.SliceModel(w, bucket, ib, npop, nofe)
    dev.load_slices(s0)
    dev.run(args.warmup, outputs=False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        dev.run(args.steps, outputs=False)
    torch.cuda.synchronize()
    t_local = dev.last_ms() / 1e3
    if dist:
        tt = torch.tensor([t_local], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    else:
        t_max = t_local
    value = world * args.steps / t_max
    prof = dev.profile(args.profile_turns)
    # end to end through the public API: slices up from host memory, the
    # per-turn outputs and the slices back down, every step
    e2e_turns = 10
    e2e_t = []
    for _ in range(args.e2e_steps + 1):
        t0 = time.perf_counter()
        dev.load_slices(s0)
        out = dev.run(e2e_turns)
        back = dev.slices()
        e2e_t.append(time.perf_counter() - t0)
    e2e_sec = float(np.mean(e2e_t[1:]))
    if dist:
        tt = torch.tensor([e2e_sec], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_sec = float(tt.item())
        dist.barrier()
        dist.destroy_process_group()
    ok = bool(np.isfinite(back).all() and np.isfinite(out[0]).all())
    dev.close()
    if rank != 0:
        return
    peak = 37.0
    achieved = SLICE_FLOP_PER_PULL * pulls / (prof[2] * 1e-3) / 1e12
    line = {
        "metric": "turns/s", "value": value, "unit": "turns/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][2], "bunches": nb, "slices": w.slices,
                   "macro_ions_per_bunch": nion, "ion_slice_pulls_per_turn": pulls, "turns_per_step": 1,
                   "l2": "state of %.1f MB fits L2; the turn is FP64-bound, not memory-bound"
                         % (nb * nion * 7 * 8 / 1e6),
                   "parallelism": "replicas x%d" % world},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "ws_train (ion train)",
                     "peak_source": "nominal B200 FP64 (no measured FP64 peak); FMA counted as 2",
                     "flop_per_pull": SLICE_FLOP_PER_PULL, "launch_ms": float(prof[2])},
        "kernels_ms_per_turn": {"ws_bunch": float(prof[0]), "ws_optic_rw": float(prof[1]),
                                "ws_train": float(prof[2]), "ws_kick": float(prof[3])},
        "e2e": {"value": world * e2e_turns / e2e_sec, "unit": "turns/s",
                "h2d_bytes_per_step": nb * 6 * w.slices * 8,
                "d2h_bytes_per_step": (e2e_turns * (nb * 8 + w.base.nharm) + nb * 6 * w.slices) * 8,
                "turns_per_step": e2e_turns, "steps": args.e2e_steps,
                "call": "SliceModel.load_slices + run(%d turns, outputs to host) + slices()" % e2e_turns},
        "gpu_launches": 4 * args.steps,
        "clocks": clk.summary(),
        "finite": ok,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if args.growth_turns > 0:
        line["growth_compare"] = slice_growth_compare(args.growth_turns)
    print(json.dumps(line))


def run_slice_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    import tempfile
    tmp = tempfile.mkdtemp()
    conf = conf_path(args.workload, tmp)
    turns = min(args.steps, 2)
    sec, kind, nb = slice_cpu(conf, turns)
    value = 1.0 / sec
    line = {
        "impl": "reference", "metric": "turns/s", "value": value, "unit": "turns/s", "n_gpus": world,
        "steps": turns, "warmup": 0, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][2], "bunches": nb, "turns_per_step": 1,
                   "parallelism": "1 host process"},
        "cpu_baseline": {"value": value, "unit": "turns/s", "cores": 1, "kind": kind,
                         "sample": "%d turns of the whole ring on one core (the ion train runs bunch after "
                                   "bunch in the reference, manager_weakstrong.c:184-233)" % turns},
        "e2e": {"value": value, "unit": "turns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def beam_ion_record(args, tmp):
    """The beam-ion configuration at full size (200-bunch train x 5e4
    macroparticles, CO at 1 nTorr, 20 interaction points, 1000 macro-ions per
    passage per point), one run with the Faddeeva field and one with the
    learned field (trained here): whole-turn device times and the ratio of
    the two macroparticle-turns/s, the beam-ion stage's share, training
    time, the audited field error, the growth-rate comparison."""
    import numpy as np
    import torch
    from mbtrack_b200 import api
    conf = conf_path("beam_ion", tmp)
    cfg = api.Config(conf)
    nb, npb = cfg.nbunch, cfg.params.np_model
    bi0 = cfg.beam_ion()
    evals = bi0.n_ip * (bi0.ions_per_passage * nb * (nb - 1) // 2 + npb * (nb - 1))
    rec = {"workload": "beam-ion weak-strong: 200-bunch train x 5e4 macroparticles, CO at 1 nTorr, 20 interaction "
                       "points, 1000 macro-ions per passage per point; the same turns with the Faddeeva field and with "
                       "the learned field",
           "bunches": nb, "np_per_bunch": npb, "macroparticles": nb * npb,
           "field_evaluations_per_turn": evals, "turns_timed": args.bi_steps, "turns_warmup": args.bi_warmup}
    mlp = api.Mlp(seed=31)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = mlp.train(seed=32, **api.MLP_TRAIN)
    torch.cuda.synchronize()
    rec["training"] = dict(api.MLP_TRAIN, seconds=time.perf_counter() - t0, final_loss=float(hist[-1]),
                           samples_from="the project's Faddeeva field (gauss_field, TOMS 680 w(z))")
    runs = {}
    for name, surr in (("faddeeva", 0), ("learned", 1)):
        bi = cfg.beam_ion()
        bi.surrogate = surr
        trk = api.Tracker.from_config(cfg, seed=1000)
        trk.generate_beam(77)
        trk.enable_beam_ion(bi)
        if surr:
            trk.use_mlp(mlp)
        trk.prepare()
        trk.run(args.bi_warmup, stats=False)
        if surr:
            trk.beam_ion_audit()            # counters from the timed turns only
        torch.cuda.synchronize()
        with ClockSampler(0) as clk:
            st = trk.run(args.bi_steps, stats=True)
        torch.cuda.synchronize()
        turn_ms = float(trk.timing()[0][3]) / args.bi_steps
        r = {"ms_per_turn": turn_ms, "macroparticle_turns_per_s": nb * npb / (turn_ms * 1e-3),
             "clocks": clk.summary(), "finite": bool(np.all(np.isfinite(st)))}
        if surr:
            a = trk.beam_ion_audit()
            r["audit"] = {"audited": int(a[0]), "max_rel_error": float(a[1]), "rms_rel_error": float(a[2]),
                          "faddeeva_fallbacks": int(a[3]), "tensor_failures": int(a[4]),
                          "fallback_fraction": int(a[3]) / float(evals * args.bi_steps),
                          "error": "|F_learned - F_Faddeeva| / |F_Faddeeva| of the field vector, a hashed 1% "
                                   "of the warps each turn"}
        trk.profile(2)
        r["stage_ms_per_turn"] = trk.beam_ion_timing()
        r["kernels_ms_per_turn"] = dict(zip(("frames", "ions", "clouds", "kick"),
                                            [float(v) for v in trk.beam_ion_kernel_times()]))
        r["field_evaluations_per_s"] = evals / (r["stage_ms_per_turn"] * 1e-3)
        trk.close()
        runs[name] = r
    rec.update(runs)
    rec["surrogate_vs_plain"] = runs["faddeeva"]["ms_per_turn"] / runs["learned"]["ms_per_turn"]
    rec["surrogate_vs_plain_meaning"] = ("whole-turn macroparticle-turns/s with the learned field over the same with "
                                         "the Faddeeva field (device time, same beam, ions and seeds)")
    # network arithmetic: 2 x (3x128 + 2x128x128 + 128x2) = 66816 FLOP per evaluation
    rec["learned"]["network_tflops"] = 66816.0 * runs["learned"]["field_evaluations_per_s"] / 1e12
    rec["faddeeva"]["fp64_pipe_active"] = {"value": 0.30, "from": "profiles/beam_ion_faddeeva.md (ncu, small case: "
                                                         "bi_ions 0.313, bi_kick_grouped 0.275, weighted by "
                                                         "their full-size times)"}
    rec["learned"]["xu_pipe_active"] = {"value": 0.72, "from": "profiles/beam_ion_learned_field.md (ncu, small case: "
                                                      "bi_ions_mlp 0.72)"}
    if args.growth_turns_bi > 0:
        rec["growth_check"] = growth_check(cfg, mlp, args.growth_turns_bi)
    mlp.close()
    return rec


def combined_extras(args, cfg, trk, mlp, init_stats, tiles, tmp):
    """The combined workload's comparisons: the same fill, beam and seeds
    with the Faddeeva field (whole-turn time ratio), and, with
    --growth-turns N, N more turns of the learned-field run written through
    the reference's writers (bunch-by-bunch centroid history among them)
    with the transverse growth rates of the coherent motion."""
    import numpy as np
    import torch
    from mbtrack_b200 import analysis, api
    out = {}
    npb = trk.np.copy()
    bi = cfg.beam_ion()
    bi.surrogate = 0
    ref = api.Tracker(cfg.params, cfg.bucket, npb, cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh, seed=1000)
    ref.generate_beam(77)
    ref.enable_beam_ion(bi)
    ref.prepare()
    ref.set_tiles(tiles)
    ref.run(2, stats=False)
    torch.cuda.synchronize()
    ref.run(args.plain_turns, stats=False)
    plain_ms = float(ref.timing()[0][3]) / args.plain_turns
    ref.close()
    learned_ms = float(trk.timing()[0][3]) / args.steps
    out["faddeeva_ms_per_turn"] = plain_ms
    out["learned_ms_per_turn"] = learned_ms
    out["surrogate_vs_plain"] = plain_ms / learned_ms
    if args.growth_turns > 0:
        work = os.path.join(tmp, "combined_work")
        os.makedirs(work, exist_ok=True)
        ocfg, bunch_out = cfg.output()
        wp = cfg.params.copy()
        wp.nrev_tot = args.growth_turns             # the files cover the turns run here
        w = api.Writer(work, wp, ocfg, bunch_out, cfg.bucket, cfg.bunch_currents())
        w.wakes(cfg.Gl, cfg.Gv, cfg.Gh)
        w.begin(init_stats)
        trk.beam_ion_audit()
        st, ai = trk.run_ampinv(args.growth_turns)
        a = trk.beam_ion_audit()
        w.turns(st, ai)
        w.end(trk.get_stats())
        w.close()
        g = {"turns": args.growth_turns, "audit_max_rel_error": float(a[1]), "audit_rms_rel_error": float(a[2]),
             "files": {f: os.path.getsize(os.path.join(work, f)) for f in sorted(os.listdir(work))}}
        for plane in ("HOR", "VER"):
            amp = analysis.centroid_amplitude(st, plane)
            wdw = analysis.exponential_window(amp)
            g[plane] = {"window": list(wdw) if wdw else None,
                        "rate_per_turn": analysis.growth_rate(amp, wdw) if wdw else None,
                        "amplitude_start": float(np.median(amp[:50])), "amplitude_end": float(amp[-1])}
        out["growth"] = g
    return out


def growth_check(cfg, mlp, turns):
    """Growth rate of the vertical coupled-bunch motion with the Faddeeva
    and with the learned field, same train, ions and seeds: the beam-ion
    configuration reduced to 5e3 macroparticles per bunch and 4 interaction
    points at 10 nTorr, so that the instability grows within a few hundred
    turns."""
    import numpy as np
    import torch
    from mbtrack_b200 import analysis, api
    amps, secs = {}, {}
    for surr in (0, 1):
        bi = cfg.beam_ion()
        bi.n_ip, bi.pressure, bi.surrogate = 4, 10e-9, surr
        t = api.Tracker(cfg.params, cfg.bucket, np.full(cfg.nbunch, 5000), cfg.bunch_currents())
        t.generate_beam(3)
        t.enable_beam_ion(bi)
        if surr:
            t.use_mlp(mlp)
        t.prepare()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = t.run(turns)
        torch.cuda.synchronize()
        secs[surr] = time.perf_counter() - t0
        t.close()
        amps[surr] = analysis.centroid_amplitude(st, "VER")
    w = analysis.exponential_window(amps[0])
    out = {"config": "beam-ion train, 5e3 macroparticles per bunch, 4 interaction points, 10 nTorr",
           "turns": turns, "seconds": {"faddeeva": secs[0], "learned": secs[1]}}
    if w is None:
        out["window"] = None
        return out
    k0, k1 = analysis.growth_rate(amps[0], w), analysis.growth_rate(amps[1], w)
    out.update({"window": list(w), "rate_faddeeva": k0, "rate_learned": k1, "rel_diff": abs(k1 - k0) / abs(k0)})
    return out

def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed turns (200; 20 for the beam-ion workloads)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="uniform")
    ap.add_argument("--profile-turns", type=int, default=20)
    ap.add_argument("--e2e-turns", type=int, default=100)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-turns", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--mlp-steps", type=int, default=0,
                    help="training steps of the learned field (0: the library's standard settings)")
    ap.add_argument("--beam-ion-record", type=int, default=1,
                    help="uniform workload at 1 GPU: add the beam-ion record (learned vs Faddeeva field; 0: skip)")
    ap.add_argument("--bi-steps", type=int, default=5, help="timed turns of each beam-ion run of the record")
    ap.add_argument("--bi-warmup", type=int, default=3, help="warm-up turns of each beam-ion run of the record")
    ap.add_argument("--growth-turns-bi", type=int, default=450,
                    help="turns of the growth-rate comparison in the beam-ion record (0: skip)")
    ap.add_argument("--plain-turns", type=int, default=3,
                    help="combined workload: timed turns of the Faddeeva-field comparison run")
    ap.add_argument("--np-per-bunch", type=int, default=0,
                    help="macroparticles per bunch in place of the workload's (small cases for profiling)")
    ap.add_argument("--n-ip", type=int, default=0, help="beam-ion workloads: interaction points (small cases)")
    ap.add_argument("--ions-per-passage", type=int, default=0,
                    help="beam-ion workloads: macro-ions per bunch passage per point (small cases)")
    ap.add_argument("--growth-turns", type=int, default=0,
                    help="beam_ion_mlp: also compare the instability growth rate of the learned and the "
                         "Faddeeva stage over this many turns on a reduced train; slice_fbii: compare the "
                         "slice model's growth rate with the per-particle stage's (0: skip)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.workload.startswith("beam_ion") or args.workload in ("slice_fbii", "combined") else 200
    if args.workload.startswith("beam_ion"):
        args.cpu_turns = min(args.cpu_turns, 2)
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.workload == "slice_fbii":
        (run_slice_reference if args.impl == "reference" else run_slice_b200)(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
