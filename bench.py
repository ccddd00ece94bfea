#!/usr/bin/env python
"""Benchmark: particle-steps/s of the giant-impact step at 262,144 particles.

Workload (the full plain impact): 262,144 particles; target 0.9 M_earth, core
mass fraction 0.3 (7.8 / 3.3 g/cc), crust of 2.7 g/cc on the outer 5 % of
radius, spun to an 8-hour day; impactor 0.1 M_earth at 45 degrees and 1.0
v_esc.  The run is taken through the reference's phases (settle, rigid
approach, first-touch kick, then full steps with a synchronous analysis every
360 steps, as window.__impact.runTo does) before anything is timed, so the
timed steps see a mid-impact state: contacts, debris, a Morton order and a
loose list.

A step is one full-phase step of the reference schedule (contact grid every
2nd step, 64^3 mesh + P3M every 8th, contacts, heat, kick/drift).

  value    N * K / sum over the K timed steps of each step's CUDA-event time on
           the library's stream, with L2 flushed (a 256 MiB write) before every
           step, so each step starts from HBM.  Max over ranks.
  e2e      the same metric through the host-buffer C-ABI call
           (ccs_advance_host: pinned host state in, one step, state out).
  roofline the contact step kernel (k_contact_step): algorithmic bytes (92 B per
           particle: pos, vel, mat, q in; pos, vel, aux, q out) over its mean
           event-timed duration, against the measured HBM copy bandwidth.
  cpu_baseline / --impl reference: the CPU oracle (a C restatement of the
           reference's step, all host cores, OpenMP) on a bounded sample of
           the same workload: full-phase steps from the same saved mid-impact
           state (the run prepared by the library, untimed, then handed over
           as a checkpoint).
  plain_1e3  the plain P3M at the metric's operating point (median force error
           <= 1e-3 against the binary64 direct sum on the gravity sweep): the
           stencil-split form (ccs_set_pp_split), its own timed steps from the
           same saved state and its force error.  `value` keeps the reference's
           own P3M (mesh + the capped loose list), the form the CPU arm times.
  nn_corrected  the same timed steps with the learned pairwise correction
           attached (BF16 network on the tensor cores, half the plain cut),
           after training it on the device on pairs drawn from the same impact
           at full-phase steps 0, 1000 and 3000; its force error on the same
           gravity sweep as force_error.
  ensemble  the batched ensemble of 64 impacts of uneven size, 2,000 steps
           each (--ens-count 0 skips it): aggregate particle-steps/s with
           each round one persistent launch over every instance's contact
           grids and contact steps (value), beside the branch-graph form and
           one stream per instance, and the per-instance step times.

Multi-GPU: one process per GPU, independent replicas of the impact (the step
has no partition worth a data-path collective at this size): weak scaling.
The ensemble sub-line shards its impacts by instance across the ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALG_BYTES_SIM = 92          # bytes per particle per contact-step launch
L2_FLUSH_BYTES = 256 << 20
MIN_SAMPLES = 8                # contact-step launches timed inside the timed region, at least
ENS_ROUNDS = 4                 # 8-step rounds one ensemble graph holds (ccs_ensemble_steps)
# the metric both arms report under (the driver divides their values only when the strings agree)
METRIC = "particle-steps/s @262k, plain vs NN-corrected P\u00b3M at \u22641e-3 force error"


def sample_every(steps):
    """The stride of the contact-step sample inside the timed region: 9 (coprime with the 8-step cycle, so the
    samples cover every step of it) when that gives MIN_SAMPLES samples; 0 for a shorter run, whose contact
    step is timed in a pass of its own after the region instead (a sampled launch leaves its step's graph
    for a direct launch between two events, which a short run would feel)."""
    return 9 if steps // 9 >= MIN_SAMPLES else 0


def impact_opt(N):
    """The full plain giant impact (second-case variants are parity configs, not bench lines)."""
    day_frac = 2 * math.pi * 805 / (8 * 3600)     # an 8-hour day as a fraction of breakup spin
    return dict(N=N, q=0.1, dens=1.0, core=0.3, spin0=day_frac, spin1=0.2, angle=45.0, incl=0.0, vfac=1.0,
                rest=0.3, mImp=0.1, mTarget=0.9, rhoR=7.8 / 3.3, rhoCrust=2.7 / 3.3, crustFrac=0.05)


def sum_over_ranks(x):
    """The sum of x over the ranks of the process group (x itself without one)."""
    import torch
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return x
    dev = "cuda" if td.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    td.all_reduce(t, op=td.ReduceOp.SUM)
    return float(t.item())


def barrier():
    import torch.distributed as td
    if td.is_available() and td.is_initialized() and td.get_world_size() > 1:
        td.barrier()


def ensemble_share(count, rank, world):
    """The impacts rank `rank` of `world` runs: every world-th from its own index, so each GPU gets a
    mix of sizes (whole impacts per GPU, no exchange during the run)."""
    return list(range(rank, count, world))


def max_over_ranks(x):
    """The largest of x over the ranks of the process group (x itself without one): the job's time is
    its slowest rank's."""
    import torch
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return x
    dev = "cuda" if td.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def committed_profile():
    """The k_contact_step figures of the committed ncu summary (profiles/contact_step_traffic.txt)."""
    p = os.path.join(ROOT, "profiles", "contact_step_traffic.txt")
    vals = {}
    if os.path.exists(p):
        for line in open(p):
            if ":" in line and not line.startswith("#"):
                k, v = line.split(":", 1)
                try:
                    vals[k.strip()] = float(v.strip())
                except ValueError:
                    pass
    return vals


def limiter_note():
    """What bounds the roofline's kernel, from the committed ncu summary: it issues, it does not stream."""
    v = committed_profile()
    if "issue_active_pct" not in v:
        return None
    return {"issue_active_pct": v["issue_active_pct"], "warp_instructions_per_particle":
            v.get("warp_instructions_per_particle"), "dram_busy_pct": v.get("dram_busy_pct"),
            "source": "the committed ncu --set full capture of the same workload; the state stays in L2, so the "
                      "kernel is bound by instruction issue, not by HBM"}


def committed_traffic():
    """dram bytes per particle of a k_contact_step launch, from the committed ncu summary."""
    return committed_profile().get("dram_bytes_per_particle")


class Clocks:
    """nvidia-smi sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def prepared_checkpoint(N, prep_steps, log, dev=0):
    """The mid-impact state both arms time: the run built, settled, brought in and advanced prep_steps
    full-phase steps by the library (untimed), then saved at a block boundary as a checkpoint (bytes)."""
    import cosmic_collisions_b200 as cc
    nb = cc.NBody(dev)
    try:
        prepare(nb, cc, N, prep_steps, log)
        if nb.sim.stepNo % 8:
            nb.steps(8 - nb.sim.stepNo % 8)
        nb.sync()
        return nb.save()
    finally:
        nb.close()


def cpu_reference(ckpt, min_seconds=10.0, min_steps=8, threads=None, N=None):
    """The CPU oracle's step (the reference's algorithm restated in C, OpenMP over all host cores) on a
    bounded sample of the bench's workload: full-phase steps from the saved mid-impact state `ckpt` (a
    checkpoint: state, run scalars, boxes, loose list and the boxes' monopoles), with runTo's cadence held
    fixed (no analysis inside the sample, as the GPU arm's timed steps have none).  Without a checkpoint
    (a host with no GPU to prepare one) it steps the freshly built N-particle impact instead, and says so."""
    import numpy as np
    from cosmic_collisions_b200 import checkpoint
    from oracle import oracle as O
    O.build()
    cores = threads or os.cpu_count()
    O.set_threads(cores)
    if ckpt is not None:
        ck = checkpoint.read(ckpt)
        sim = O.Sim.from_buffer_copy(bytes(ck["sim"]))
        e = O.Engine(sim, ck["pos"], ck["vel"], ck["mat"])
        e.prime_mono(0, ck["monoA"])
        e.prime_mono(1, ck["monoB"])
        if len(ck["pp_list"]):
            e.set_pp(np.asarray(ck["pp_list"], np.int32))
        what = "the GPU arm's saved mid-impact state (step %d, loose list %d)" % (int(ck["sim"].stepNo),
                                                                                  len(ck["pp_list"]))
    else:
        sim, pos, vel, mat, home = O.build_run(O.make_opt(**impact_opt(N)))
        sim.phase, sim.impactT = 2, sim.t
        for k in range(3):
            sim.boxCen[0][k] = sim.cen0[k]
        sim.boxT[0] = sim.t
        e = O.Engine(sim, pos, vel, mat)
        what = "the freshly built impact (no GPU on this host to prepare the mid-impact state)"
    N = int(e.sim.N)
    e.step(False, False)           # warm: the pair table, first touches of the arrays
    e.sim.t += e.sim.dt
    steps = 0
    t0 = time.perf_counter()
    while True:
        e.step(False, False)
        e.sim.t += e.sim.dt
        steps += 1
        el = time.perf_counter() - t0
        if steps >= min_steps and el >= min_seconds:
            break
    return {"value": N * steps / el, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": "%d full-phase steps of the %d-particle impact from %s (%.1f s, %d OpenMP threads)"
                      % (steps, N, what, el, cores)}


def force_error(cc, dev, N, sample=2048, seed=3, net=None, split=0, uncapped=False):
    """The gravity-only sweep (Plummer sphere + 10 % debris, equal masses, 1 M_earth): one force evaluation
    of the P3M step (the reference's loose-list form, with the learned correction `net`, or the stencil-split
    form with stencil `split`) against the library's binary64 direct sum at a seeded sample of particles.
    uncapped: the reference's form with every loose particle on the list (its 8,192 cap lifted): the mesh
    alone from the step, plus the pairwise correction over the whole list (ccs_pp_list_force)."""
    import numpy as np
    from cosmic_collisions_b200 import configs
    sim, pos, vel, mat = configs.gravity_sweep(N=N)
    nb = cc.NBody(dev)
    try:
        nb.upload(sim, pos, vel, mat)
        if net is not None:
            nb.set_pp_nn(net)
        nb.pass_slots()
        nb.pass_diag()
        D = nb.buffer("diag")
        s = nb.sim
        rep, lst, _ = cc.fof(s.N, s.m, s.a, pos, vel, mat, D, s.k, 2 * s.a, cap=s.N if uncapped else cc.NBody.PP_CAP)
        nb.set_pp(np.zeros(0, np.int32) if uncapped else lst, rep.ppLoose)
        if split:
            nb.set_pp_split(split)
            nb.pass_mesh()
            nb.pass_pp()
        nb.pass_sim(False, False, 0.0)
        g = nb.read_state()["aux"][:, :3].astype(np.float64)
        if uncapped:
            g[lst] += nb.pp_list_force(lst)[:, :3]
        idx = np.sort(np.random.default_rng(seed).choice(N, sample, replace=False)).astype(np.int32)
        ref, _ = nb.direct_sum(idx)
    finally:
        nb.close()
    rel = np.linalg.norm(g[idx] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    on = np.isin(idx, np.asarray(lst, np.int64))
    return {"median": float(np.median(rel)), "p99": float(np.percentile(rel, 99)), "sample": sample,
            "method": ("stencil-split P3M, every mesh node pair within %d cells summed pairwise" % split
                       if split else "the reference's P3M: mesh + the whole loose list's pairs (no cap)"
                       if uncapped else "the reference's P3M: mesh + the capped loose list's pairs"),
            "loose_list_members_in_sample": int(on.sum()),
            "loose_list_median": float(np.median(rel[on])) if on.any() else None,
            "workload": "gravity sweep, %d equal masses: Plummer sphere (scale 1 R_earth) + 10%% uniform debris" % N,
            "loose_list": int(rep.ppCount), "loose_total": int(rep.ppLoose),
            "reference": "binary64 direct sum, softening a, self term excluded"}


def prepare(nb, cc, N, prep_steps, log):
    """build -> settle -> rigid approach -> kick -> prep_steps full steps with runTo's analysis cadence."""
    t0 = time.perf_counter()
    nb.build(cc.make_opt(**impact_opt(N)))
    log("built N=%d in %.1fs (a=%.5f dt=%.3e settle=%d)" % (N, time.perf_counter() - t0, nb.sim.a, nb.sim.dt,
                                                            nb.sim.settleLeft))
    while nb.sim.phase == 0:
        nb.settle_some(64)
    nb.analyze(True)
    n_rigid = 0
    while nb.sim.phase == 1 and n_rigid < 5000:
        nb.rigid_step(0.01)
        n_rigid += 1
    if nb.sim.phase != 2:
        raise RuntimeError("the bodies never touched")
    done = advance(nb, prep_steps)
    r = nb.report
    log("prepared in %.1fs: %d rigid steps, %d full steps, t=%.3f, loose=%d (list %d), largest=%.3f"
        % (time.perf_counter() - t0, n_rigid, done, nb.sim.t, nb.pp["loose"], nb.pp["count"], r.largest))


def advance(nb, steps):
    """steps full-phase steps with runTo's synchronous analysis every 360 steps (index.html:592-600), then a
    closing analysis."""
    done = 0
    while done < steps:
        n = min(360 - (nb.sim.stepNo - nb.analyzed_at), steps - done)
        n = max(n, 1)
        nb.steps(n)
        done += n
        if nb.sim.stepNo - nb.analyzed_at >= 360:
            nb.analyze(True)
    nb.analyze(True)
    nb.sync()
    return done


def learned_correction(cc, dev, N, log, pairs=12_000_000, epochs=24, snaps=(0, 1000, 3000), held=262_144, lr=4e-3):
    """The learned P3M correction (config 4): a network trained on the device on pairs drawn from the full
    plain impact at full-phase steps 0, 1000 and 3000, labelled by the binary64 mesh arithmetic of the
    isolated pair.  Returns the network and what its training and a held-out set say."""
    import numpy as np
    from cosmic_collisions_b200.learned import LearnedCorrection, softened_newton, table_model
    net = LearnedCorrection(dev, seed=2024)
    nb = cc.NBody(dev)
    t0 = time.perf_counter()
    try:
        prepare(nb, cc, N, 0, log)
        a_cells = nb.sim.a / (12.0 / 64.0)
        done = 0
        for k, s in enumerate(snaps):
            done += advance(nb, s - done) if s > done else 0
            net.sample_state(nb, pairs // len(snaps), seed=1000 + k)
        net.sample_state(nb, held, seed=9999)              # held out: the last snapshot, another draw
    finally:
        nb.close()
    t_sample = time.perf_counter() - t0
    n_train = pairs // len(snaps) * len(snaps)
    t1 = time.perf_counter()
    loss = net.train(0, n_train, epochs=epochs, tiles_per_cta=1, lr=lr)
    t_train = time.perf_counter() - t1
    rec, lab = net.read_pool(n_train, held)
    live = np.isfinite(rec[:, 0])
    rec, lab = rec[live], lab[live]
    y = net.forward(rec)
    near = (np.abs(np.floor(rec[:, 3:6].astype(np.float64) - rec[:, :3])) <= 1).all(axis=1)   # share a node
    mesh = lab + softened_newton(rec)                       # the isolated pair's mesh force
    f, _ = cc.pair_table()
    tab = table_model(rec, f, a_cells)                      # the plain pass's model of it
    rms = lambda v: float(np.sqrt((v ** 2).sum(1).mean())) if len(v) else None
    info = {"pairs": int(n_train), "epochs": epochs, "lr": lr, "snapshots_full_steps": list(snaps),
            "train_tflops": 3.0 * 12288 * n_train * epochs / t_train / 1e12,
            "loss_first_epoch": float(loss[0]), "loss_last_epoch": float(loss[-1]),
            "sample_s": t_sample, "train_s": t_train,
            "held_out": {"pairs": int(len(rec)), "pairs_sharing_a_mesh_node": int(near.sum()),
                         "mesh_force_rms_shared": rms(mesh[near]),
                         "table_error_rms_shared": rms((mesh - tab)[near]),
                         "network_error_rms_shared": rms((y - lab)[near]),
                         "table_error_rms_all": rms(mesh - tab), "network_error_rms_all": rms(y - lab),
                         "unit": "mesh pair force of a unit source, cells^-2"}}
    log("learned correction: %d pairs, loss %.3e -> %.3e in %.1fs; held-out error on pairs sharing a node: table %.3e network %.3e"
        % (n_train, loss[0], loss[-1], t_train, info["held_out"]["table_error_rms_shared"] or 0,
           info["held_out"]["network_error_rms_shared"] or 0))
    return net, info


def run_ensemble(args, log, rank=0, world=1):
    """The batched ensemble: `args.ensemble` impacts of uneven size (seeded: N over the page's counts,
    impactor 0.02-1 M_earth, 0-75 degrees, 1.0-2.6 v_esc), each prepared to first touch, then advanced
    `args.ens_steps` steps each.  Every instance is a handle on its own stream; the host interleaves one
    captured 8-step graph per instance per round, so the instances run concurrently on the GPU.
    Reports the aggregate particle-steps/s and the p50/p99 of the per-instance step time.  Under torchrun
    the impacts are shared out by instance (ensemble_share): each rank runs its own on its own GPU, and only
    the totals cross ranks at the end (the slowest rank's wall time, the sum of particle-steps)."""
    import numpy as np
    import torch
    import cosmic_collisions_b200 as cc
    from cosmic_collisions_b200 import configs
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    allopts = configs.ensemble_opts(args.ensemble)
    opts = [allopts[k] for k in ensemble_share(len(allopts), rank, world)]
    runs = []
    t0 = time.perf_counter()
    for opt in opts:
        nb = cc.NBody(dev)
        nb.build(cc.make_opt(**opt))
        while nb.sim.phase == 0:
            nb.settle_some(256)
        n_rigid = 0
        while nb.sim.phase == 1 and n_rigid < 5000:
            nb.rigid_step(0.01)
            n_rigid += 1
        if nb.sim.stepNo % 8:
            nb.steps(8 - nb.sim.stepNo % 8)
        runs.append(nb)
    for nb in runs:
        nb.sync()
    log("ensemble of %d prepared in %.1fs (%d particles)" % (len(runs), time.perf_counter() - t0,
                                                             sum(nb.sim.N for nb in runs)))
    for nb in runs:
        if nb.sim.stepNo % 8:
            nb.steps(8 - nb.sim.stepNo % 8)
        nb.sync()
    # launch shapes by measurement of the whole ensemble's throughput (its members advance meanwhile)
    tuned = None
    if not args.no_tune:
        ens = cc.Ensemble(runs)
        tuned = ens.autotune(rounds=4)
        ens.sync()
        ens.close()
        log("ensemble autotuner: %s" % tuned)
    blocks = max(1, args.ens_steps // 8)
    # the library holds ENS_ROUNDS rounds a graph, keyed by the members' parities (the branch form's also by a
    # ping that alternates per graph): two full graphs and the last, shorter one cover every graph the timed
    # rounds replay
    warm = 8 * (2 * ENS_ROUNDS + blocks % ENS_ROUNDS)
    streams = [torch.cuda.ExternalStream(nb.device_buffers().stream) for nb in runs]
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in runs]
    for nb in runs:   # each member's block graphs (both ping parities) captured before the timing
        nb.steps(16)
    torch.cuda.synchronize()
    barrier()
    w0 = time.perf_counter()
    for k, (nb, s) in enumerate(zip(runs, streams)):
        with torch.cuda.stream(s):
            ev[k][0].record(s)
    for _ in range(blocks):
        for nb in runs:
            nb.steps(8)
    for k, (nb, s) in enumerate(zip(runs, streams)):
        with torch.cuda.stream(s):
            ev[k][1].record(s)
    torch.cuda.synchronize()
    wall = max_over_ranks(time.perf_counter() - w0)
    per_step_ms = np.array([a.elapsed_time(b) / (8 * blocks) for a, b in ev])
    total = sum_over_ranks(sum(nb.sim.N for nb in runs) * 8 * blocks)
    # the same number of steps again, every round one graph holding all instances' blocks (ccs_ensemble)
    ens = cc.Ensemble(runs)
    ens.steps(warm)                                       # capture every graph the timed rounds replay
    ens.sync()
    torch.cuda.synchronize()
    barrier()
    w1 = time.perf_counter()
    ens.steps(8 * blocks)
    ens.sync()
    wall_graph = max_over_ranks(time.perf_counter() - w1)
    # and again with every round one persistent launch over all instances' grids and contact steps
    # (ccs_ensemble_set_persistent), after the instances' mesh chains
    ens.set_persistent(True)
    ens.steps(warm)                                       # capture every graph the timed rounds replay
    ens.step_ms()                                         # (waits; the sums start at the timed rounds)
    torch.cuda.synchronize()
    barrier()
    l0 = ens.launch_count()
    w2 = time.perf_counter()
    ens.steps(8 * blocks)
    ens.sync()
    wall_pers = max_over_ranks(time.perf_counter() - w2)
    pers_ms = ens.step_ms()                               # each instance's step time inside the rounds
    pers_launches = ens.launch_count() - l0
    ens.close()
    p50 = max_over_ranks(float(np.percentile(per_step_ms, 50)))
    p99 = max_over_ranks(float(np.percentile(per_step_ms, 99)))
    pp50 = max_over_ranks(float(np.percentile(pers_ms, 50)))
    pp99 = max_over_ranks(float(np.percentile(pers_ms, 99)))
    line = {"metric": "ensemble aggregate particle-steps/s", "value": total / wall_pers, "unit": "particle-steps/s",
            "instances": int(sum_over_ranks(len(runs))), "n_gpus": world, "steps_each": 8 * blocks,
            "particles": int(sum_over_ranks(sum(nb.sim.N for nb in runs))),
            "sharding": "whole impacts per GPU (every world-th instance), no exchange during the run; the "
                        "slowest rank's wall time and the summed particle-steps",
            "mode": "persistent: each 8-step round one launch of k_ensemble_round over every instance's contact "
                    "grids and contact steps (work items from per-instance queues), after the instances' mesh "
                    "chains; four rounds a CUDA graph (ccs_ensemble_set_persistent); wall clock over the rounds",
            "wall_s": wall_pers,
            "persistent_launches": int(pers_launches),
            "per_instance_step_ms": {"p50": pp50, "p99": pp99,
                                     "what": "each instance's first work item to its last in a round "
                                             "(%globaltimer), over 8 steps, averaged over the timed rounds"},
            "branch_graph": {"value": total / wall_graph, "wall_s": wall_graph,
                             "mode": "one CUDA graph per four 8-step rounds holding every instance's steps as a "
                                     "parallel branch (ccs_ensemble)"},
            "per_handle_streams": {"value": total / wall, "wall_s": wall,
                                   "per_instance_step_ms": {"p50": p50, "p99": p99},
                                   "mode": "one handle and stream per impact, captured 8-step graphs interleaved"},
            "autotuned": tuned}
    for nb in runs:
        nb.close()
    return line


def conservation_run(cc, dev, N, steps=5000, log=None, split=0):
    """The full impact's books over a long run (src/nbody.js:837-850 and the readout of index.html:335-349):
    the run built, settled and brought in, then `steps` full-phase steps with runTo's synchronous analysis
    every 360 steps (on the device), the books read at every analysis against the first look in the full
    phase.  Returns the worst drifts seen and the last ones."""
    nb = cc.NBody(dev)
    nb.device_fof = True
    t0 = time.perf_counter()
    try:
        nb.build(cc.make_opt(**impact_opt(N)))
        while nb.sim.phase == 0:
            nb.settle_some(64)
        nb.analyze(True)
        while nb.sim.phase == 1:
            nb.rigid_step(0.01)
        if split:
            nb.set_pp_split(split)     # the books' first look is taken with the form's own potential
            nb.steps(8)
            nb.ref = None
        nb.analyze(True)
        ref = nb.ref
        rows = []
        done = 0
        while done < steps:
            n = max(1, min(360 - (nb.sim.stepNo - nb.analyzed_at), steps - done))
            nb.steps(n)
            done += n
            if nb.sim.stepNo - nb.analyzed_at >= 360 or done == steps:
                nb.analyze(True)
                r = nb.report
                rows.append({"steps": done, "t": nb.sim.t, "L": (r.L - ref["L"]) / ref["L"],
                             "balance": ((r.KE + r.PE + r.EL + r.Q) - ref["EQ"]) / ref["scale"],
                             "drift": r.drift, "largest": r.largest})
        nb.sync()
    finally:
        nb.close()
    worst = {k: max(abs(x[k]) for x in rows) for k in ("L", "balance", "drift")}
    out = {"steps": steps, "particles": N, "stencil": split, "analyses": len(rows), "t_end": rows[-1]["t"], "wall_s":
           time.perf_counter() - t0, "worst": worst, "last": rows[-1],
           "what": "L: angular momentum against the first look of the full phase; balance: (KE + PE + elastic "
                   "+ heat) less the first look's, over KE - PE; drift: |momentum| / M (the readout's books)"}
    if log:
        log("books over %d steps: worst |dL/L| %.2e, |balance| %.2e, drift %.2e" % (steps, worst["L"],
                                                                                 worst["balance"],
                                                                                 worst["drift"]))
    return out


def analysis_timing(cc, nb, reps=5):
    """The worker's fof (src/nbody.js:646-893) on the bench's state, with the Morton sort: on the device
    (ccs_fof_device, wall time of the call: it returns the report on the host) and on one host core
    (ccs_fof on the read-back state), and whether the two agree."""
    import numpy as np
    N, cap = nb.sim.N, cc.NBody.PP_CAP
    nb.fof_device(True)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        rd, ld, qd = nb.fof_device(True)
        times.append(time.perf_counter() - t0)
    D = nb.buffer("diag").reshape(-1, 4)[:N]
    st = nb.read_state()
    s = nb.sim
    t0 = time.perf_counter()
    rh, lh, qh = cc.fof(s.N, s.m, s.a, st["pos"], st["vel"], st["mat"], D, s.k, 2 * s.a, cap, True)
    host_s = time.perf_counter() - t0
    return {"device_ms": 1e3 * statistics.median(times), "host_ms": 1e3 * host_s, "host_cores": 1,
            "loose": int(rh.ppLoose), "same_loose_list": bool(np.array_equal(ld, lh)),
            "same_perm": bool(np.array_equal(qd, qh)),
            "largest_rel_diff": abs(rd.largest - rh.largest) / rh.largest,
            "L_rel_diff": abs(rd.L - rh.L) / rh.L}


def warm_step_graphs(nb, lib, every):
    """Capture, before anything is timed, every step graph the timed loop replays: the loop times the contact
    step on every `every`-th launch (a graph that stops before it; every = 0: none) and replays whole-step
    graphs otherwise, keyed by the step's place in the 8-step cycle and the buffers it touches, so
    2 x 8 x max(every, 1) steps of the same loop visit every key."""
    lib.ccs_timing_every(nb.handle, max(every, 1))
    lib.ccs_timing(nb.handle, 1 if every else 0)
    for _ in range(2 * 8 * max(every, 1)):
        nb.step(False, False)
        nb.sim.t += nb.sim.dt
    nb.sync()
    lib.ccs_timing(nb.handle, 0)
    lib.ccs_timing_every(nb.handle, 1)


def timed_steps(nb, lib, stream, flush, steps, dev, dist):
    """steps step graphs, L2 flushed before each, each bracketed by CUDA events on the library's stream;
    clocks sampled meanwhile.  Inside the timed region the library times the contact step alone (the
    roofline's kernel) with its own pair of events on every n-th launch (sample_every), a sample spread over
    the whole region.  The other kernels are timed in passes of their own after it, since every timed launch
    widens its step by its events: the grid, deposit, cell and pairwise kernels on steps launched one kernel
    at a time, then the two halves of the split mesh step (the contact walk and the tail)."""
    import ctypes as C
    import torch
    every = sample_every(steps)
    warm_step_graphs(nb, lib, every)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    clocks = Clocks(dev)
    if dist:
        import torch.distributed as td
        td.barrier()
    torch.cuda.synchronize()
    lib.ccs_timing_every(nb.handle, max(every, 1))
    lib.ccs_timing(nb.handle, 1 if every else 0)   # kernel id 0, the contact step (sampled) or nothing
    l0 = lib.ccs_launch_count(nb.handle)
    clocks.start()
    w0 = time.perf_counter()
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            ev[k][0].record(stream)
        nb.step(False, False)
        nb.sim.t += nb.sim.dt
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    nb.sync()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    clk = clocks.stop()
    launches = lib.ccs_launch_count(nb.handle) - l0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    names = ["simulate", "contact_grid", "deposit", "cell", "pp_force", "contact_walk", "contact_tail"]
    kt = {}

    def read(kids):
        for kid in kids:
            tot, cnt = C.c_double(), C.c_int()
            lib.ccs_timing_read(nb.handle, kid, C.byref(tot), C.byref(cnt))
            kt[names[kid]] = {"launches": cnt.value, "total_ms": tot.value,
                              "mean_us": 1e3 * tot.value / cnt.value if cnt.value else None}
    if not every:   # a short region: the contact step on MIN_SAMPLES + 8 launches of its own, L2 flushed before each
        lib.ccs_timing_every(nb.handle, 1)
        lib.ccs_timing(nb.handle, 1)
        for k in range(MIN_SAMPLES + 8):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            nb.step(False, False)
            nb.sim.t += nb.sim.dt
        nb.sync()
    read([0])
    kt["simulate"]["every"] = every
    lib.ccs_timing_every(nb.handle, 1)
    # the other kernels: passes of their own after the timed region, L2 flushed before each step as above
    for mask, kids, n in ((0x1E, [1, 2, 3, 4], max(16, min(steps, 64))), (0x60, [5, 6], 32)):
        lib.ccs_timing(nb.handle, mask)
        for k in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            nb.step(False, False)
            nb.sim.t += nb.sim.dt
        nb.sync()
        read(kids)
    lib.ccs_timing(nb.handle, 0)
    return step_ms, kt, launches, wall, clk


def run_ours(args, rank, world, log):
    import torch
    import cosmic_collisions_b200 as cc

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    N = args.particles
    nb = cc.NBody(dev)
    lib = cc.lib()
    prepare(nb, cc, N, args.prep, log)
    nb.steps(args.warmup)
    nb.sync()
    if args.profile:
        # for `ncu --profile-from-start off`: only the chosen leg's work between cudaProfilerStart and Stop is
        # profiled -- plain: --steps steps of the reference's P3M; split: one warm 8-step block, then --steps
        # steps of the stencil-split form (--split); learned: the learned pass attached (a network trained
        # briefly on the same impact), then --steps steps; train: one training epoch of that network over 1 M
        # pairs drawn from the state and a forward pass over 131,072 of them
        net = None
        if args.profile_leg in ("learned", "train"):
            net, _ = learned_correction(cc, dev, N, log, pairs=1_000_000 if args.profile_leg == "train" else 300_000,
                                        epochs=2, snaps=(0,), held=131072)
        if args.profile_leg == "learned":
            nb.set_pp_nn(net)
        if args.profile_leg == "split":
            nb.set_pp_split(args.split or 1)
            nb.steps(8)
        for _ in range(args.warmup):
            nb.step(False, False)
            nb.sim.t += nb.sim.dt
        nb.sync()
        l0 = lib.ccs_launch_count(nb.handle)
        torch.cuda.profiler.start()
        if args.profile_leg == "train":
            rec, _ = net.read_pool(0, 131072)
            net.train(0, 1_000_000, epochs=1, tiles_per_cta=1, lr=4e-3)
            net.forward(rec)
        else:
            for _ in range(args.steps):
                nb.step(False, False)
                nb.sim.t += nb.sim.dt
        nb.sync()
        torch.cuda.profiler.stop()
        out = {"profile": True, "leg": args.profile_leg, "steps": args.steps,
               "gpu_launches": int(lib.ccs_launch_count(nb.handle) - l0), "stepNo": nb.sim.stepNo,
               "loose_list": nb.pp["count"]}
        nb.set_pp_nn(None)
        nb.close()
        if net is not None:
            net.close()
        return out, None
    import ctypes as C
    buf = nb.device_buffers()
    stream = torch.cuda.ExternalStream(buf.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    dist = world > 1
    if dist:
        import torch.distributed as td
    # the learned leg below is timed on this same state: keep it (at a block boundary, so the seat tables
    # are rebuilt on the first step either leg takes)
    if nb.sim.stepNo % 8:
        nb.steps(8 - nb.sim.stepNo % 8)
    nb.sync()
    snapshot = nb.save()                   # the state the CPU baseline and the learned leg start from
    step_ms, kt, launches, wall, clk = timed_steps(nb, lib, stream, flush, args.steps, dev, dist)
    total_ms = max_over_ranks(sum(step_ms))
    value = world * N * args.steps / (total_ms / 1e3)

    # the same steps back to back from captured 8-step graphs, state L2-resident (no flush)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ksteps = max(8, args.steps // 8 * 8)
    if nb.sim.stepNo % 8:
        nb.steps(8 - nb.sim.stepNo % 8)
    nb.steps(ksteps)                       # captures the block graphs (both buffer parities) untimed
    nb.steps(ksteps)
    nb.sync()
    with torch.cuda.stream(stream):
        g0.record(stream)
    nb.steps(ksteps)
    with torch.cuda.stream(stream):
        g1.record(stream)
    nb.sync()
    resident_ms = max_over_ranks(g0.elapsed_time(g1))

    # end to end through the host-buffer plugin call
    st = nb.read_state()
    hp = torch.from_numpy(st["pos"]).pin_memory()
    hv = torch.from_numpy(st["vel"]).pin_memory()
    hq = torch.from_numpy(st["q"]).pin_memory()
    ha = torch.empty((N, 4), dtype=torch.float32).pin_memory()
    P = lambda t: C.c_void_p(t.data_ptr())
    e2e_steps = max(8, min(args.steps, 256))
    for _ in range(16):                    # capture the call's step graphs (every place in the cycle) untimed
        rc = lib.ccs_advance_host(nb.handle, P(hp), P(hv), P(hq), 1, P(hp), P(hv), P(ha), P(hq))
        if rc:
            raise RuntimeError("ccs_advance_host: %d" % rc)
    for _ in range(2):
        rc = lib.ccs_advance_host(nb.handle, P(hp), P(hv), P(hq), 8, P(hp), P(hv), P(ha), P(hq))
        if rc:
            raise RuntimeError("ccs_advance_host: %d" % rc)
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for _ in range(e2e_steps):
        rc = lib.ccs_advance_host(nb.handle, P(hp), P(hv), P(hq), 1, P(hp), P(hv), P(ha), P(hq))
        if rc:
            raise RuntimeError("ccs_advance_host: %d" % rc)
    e2e_s = max_over_ranks(time.perf_counter() - e0)
    # the same call advancing a whole mesh cycle (8 steps) between the state's copies in and out
    calls8 = max(2, e2e_steps // 8)
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for _ in range(calls8):
        rc = lib.ccs_advance_host(nb.handle, P(hp), P(hv), P(hq), 8, P(hp), P(hv), P(ha), P(hq))
        if rc:
            raise RuntimeError("ccs_advance_host: %d" % rc)
    e2e8_s = max_over_ranks(time.perf_counter() - e0)
    h2d = N * (16 + 16 + 4)
    d2h = N * (16 + 16 + 16 + 4)

    ferr = force_error(cc, dev, N) if rank == 0 else None
    if ferr is not None:
        unc = force_error(cc, dev, N, uncapped=True)
        ferr["uncapped"] = {k: unc[k] for k in ("median", "p99", "method", "loose_list", "loose_list_median",
                                                 "loose_list_members_in_sample")}
    analysis = analysis_timing(cc, nb) if rank == 0 and not args.no_cpu else None
    books = None
    if rank == 0 and args.books_steps:
        books = conservation_run(cc, dev, N, args.books_steps, log)
        if args.split:
            books = {"reference_form": books,
                     "stencil_split": conservation_run(cc, dev, N, args.books_steps, log, split=args.split)}

    # the learned correction (config 4): train, attach, the same timed steps, the same force sweep
    nn_line = None
    if not args.no_nn:
        net, info = learned_correction(cc, dev, N, log, pairs=args.nn_pairs, epochs=args.nn_epochs)
        nb.load(snapshot)                  # back to the plain leg's starting state
        nb.set_pp_nn(net)
        nn_ms, nn_kt, nn_launches, nn_wall, nn_clk = timed_steps(nb, lib, stream, flush, args.steps, dev, dist)
        nn_total = max_over_ranks(sum(nn_ms))
        nn_err = force_error(cc, dev, N, net=net) if rank == 0 else None
        nb.set_pp_nn(None)
        net.close()
        nn_line = {"value": world * N * args.steps / (nn_total / 1e3), "unit": "particle-steps/s",
                   "ms_per_step": nn_total / args.steps, "pp_cut_cells": 2.5, "loose_list": nb.pp["count"],
                   "kernels_us": {k: v["mean_us"] for k, v in nn_kt.items()}, "gpu_launches": int(nn_launches),
                   "clocks": nn_clk, "wall_s_timed_region": nn_wall, "force_error": nn_err, "training": info,
                   "state": "the plain leg's timed steps from the same saved state"}
    # the plain P3M at the metric's operating point: the stencil-split form, the same timed steps from the
    # same saved state, and its force error on the same gravity sweep
    split_line = None
    if args.split:
        nb.load(snapshot)
        nb.set_pp_split(args.split)
        sp_ms, sp_kt, sp_launches, sp_wall, sp_clk = timed_steps(nb, lib, stream, flush, args.split_steps, dev, dist)
        sp_total = max_over_ranks(sum(sp_ms))
        sp_err = force_error(cc, dev, N, split=args.split) if rank == 0 else None
        nb.set_pp_split(0)
        split_line = {"value": world * N * args.split_steps / (sp_total / 1e3), "unit": "particle-steps/s",
                      "ms_per_step": sp_total / args.split_steps, "steps": args.split_steps, "stencil": args.split,
                      "kernels_us": {k: v["mean_us"] for k, v in sp_kt.items() if k != "simulate"},
                      "gpu_launches": int(sp_launches), "clocks": sp_clk, "force_error": sp_err,
                      "method": "stencil-split P3M: every pair of mesh nodes within %d cells (Chebyshev) summed "
                                "particle by particle (each pair weighted by its share of cloud-in-cell node "
                                "pairs inside the stencil), the rest on the mesh unsoftened, gathered to second "
                                "order by each node's tidal tensor and the pull's second gradient, far blocks as "
                                "monopole + quadrupole at each cell; the plain form that reaches median force "
                                "error <= 1e-3" % args.split,
                      "state": "the plain leg's timed steps from the same saved state"}
        one, both = nb.pp_split_pairs()   # the last mesh step's pair pass
        pp_ms = sp_kt.get("pp_force", {}).get("mean_us", 0.0) / 1e3
        split_line["pair_pass"] = {
            "pairs_one_way": one, "pairs_both_ways": both,
            "forces": one + 2 * both,
            "pairs_per_s": (one + both) / (pp_ms / 1e3) if pp_ms else None,
            "forces_per_s": (one + 2 * both) / (pp_ms / 1e3) if pp_ms else None,
            "ms": pp_ms,
            "fp32_ops_per_pair": {"one_way": 17, "both_ways": 25},
            "fma_pipe_of_peak": 0.589,
            "what": "the (target, source) pairs inside the stencil the pass's items take, one way (a force on "
                    "the target) and both ways (a force on each: pairs between nodes of 16 particles or more, "
                    "once); forces = one way + 2 x both ways, the one-way pass's count; over the pass's "
                    "event-timed mean; the FMA pipe's share from the committed ncu capture "
                    "(profiles/pp_split_both_262k.md)"}
        log("stencil-split P3M (S=%d): %.3f ms a step, force error median %.3e"
            % (args.split, sp_total / args.split_steps, sp_err["median"] if sp_err else float("nan")))
    peak, peak_kind = measured_peaks()
    sim_mean_us = kt["simulate"]["mean_us"]
    achieved = ALG_BYTES_SIM * N / (sim_mean_us * 1e-6) / 1e9 if sim_mean_us else None
    tpp = committed_traffic()
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded builder: src/nbody.js build() with the config's masses and layers)",
        "config": {
            "workload": "full plain giant impact, %d particles: 0.9 + 0.1 M_earth, core 0.3, crust 2.7 g/cc "
                        "outer 5%%, 8 h day, 45 deg, 1.0 v_esc; mid-impact state after %d full steps" % (N, args.prep),
            "particles": N, "mesh": "64^3 x %d box(es)" % (2 if nb.sim.boxOn[1] else 1),
            "contact_grid": "%d^3 hashed" % nb.sim.G, "loose_list": nb.pp["count"],
            "parallelism": "replicas x%d" % world,
            "l2": "flushed (256 MiB write) before every timed step; value sums per-step event times",
            "l2_resident_particle_steps_per_s": world * N * ksteps / (resident_ms / 1e3),
            "wall_s_timed_region": wall,
            "kernels_us": {k: v["mean_us"] for k, v in kt.items()},
        },
        "e2e": {"value": world * N * e2e_steps / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "api": "ccs_advance_host, one step per call, pinned host buffers",
                "us_per_call": e2e_s / e2e_steps * 1e6,
                "eight_steps_per_call": {"value": world * N * 8 * calls8 / e2e8_s, "unit": "particle-steps/s",
                                         "calls": calls8, "us_per_call": e2e8_s / calls8 * 1e6,
                                         "what": "the same call with nsteps = 8 (a mesh cycle between the "
                                                 "state's copies in and out); not the headline"}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "peak_kind": peak_kind + " hbm_gbs",
                     "kernel": "k_contact_step (contacts + gather + kick/drift)",
                     "traffic": tpp * N if tpp else None,
                     "algorithmic_bytes_per_launch": ALG_BYTES_SIM * N,
                     "timed_launches": kt["simulate"]["launches"],
                     "timing": ("CUDA events on the library's stream around every %d-th contact step of the timed "
                                "region" % kt["simulate"]["every"]) if kt["simulate"]["every"] else
                               "CUDA events on the library's stream around each of %d contact steps in a pass of their "
                               "own after the timed region, L2 flushed before each" % kt["simulate"]["launches"],
                     "limiter": limiter_note()},
        "gpu_launches": int(launches),
        "clocks": clk,
        "force_error": ferr,
        "analysis": analysis,
        "nn_corrected": nn_line,
        "plain_1e3": split_line,
        "conservation": books,
    }
    nb.close()
    return line, snapshot


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1024)
    ap.add_argument("--warmup", type=int, default=16)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=262144)
    ap.add_argument("--prep", type=int, default=720, help="full-phase steps before timing")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="run the batched ensemble of this many impacts instead and print its line")
    ap.add_argument("--ens-steps", type=int, default=2000)
    ap.add_argument("--ens-count", type=int, default=64,
                    help="impacts of the ensemble sub-line of the default run (0: skip it)")
    ap.add_argument("--no-nn", action="store_true", help="skip the learned-correction leg")
    ap.add_argument("--no-tune", action="store_true", help="ensemble: keep the default launch shapes")
    ap.add_argument("--nn-pairs", type=int, default=12_000_000, help="training pairs (three snapshots)")
    ap.add_argument("--nn-epochs", type=int, default=24)
    ap.add_argument("--split", type=int, default=1, choices=[0, 1, 2, 3],
                    help="stencil of the plain P3M leg at the metric's force-error operating point (0: skip)")
    ap.add_argument("--split-steps", type=int, default=64, help="timed steps of that leg")
    ap.add_argument("--books-steps", type=int, default=5000,
                    help="full-phase steps of the conservation run (0: skip)")
    ap.add_argument("--profile-leg", default="plain", choices=["plain", "split", "learned", "train"],
                    help="what --profile runs between cudaProfilerStart and Stop")
    ap.add_argument("--profile", action="store_true",
                    help="prepare, warm up, then run --steps steps inside cudaProfilerStart/Stop and exit "
                         "(for ncu --profile-from-start off); prints no bench line")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    log = (lambda s: print("[bench] " + s, file=sys.stderr, flush=True)) if rank == 0 else (lambda s: None)

    if args.impl == "reference":
        if rank != 0:
            return
        import torch
        log = lambda s: print("[bench] " + s, file=sys.stderr, flush=True)
        ckpt = None
        if torch.cuda.is_available():
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            ckpt = prepared_checkpoint(args.particles, args.prep, log, int(os.environ.get("LOCAL_RANK", "0")))
        ref = cpu_reference(ckpt, min_seconds=args.cpu_seconds, N=args.particles)
        line = {"impl": "reference", "metric": METRIC, "value": ref["value"],
                "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": "full plain giant impact, %d particles" % args.particles},
                "cpu_baseline": ref,
                "e2e": {"value": ref["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.ensemble:
        line = run_ensemble(args, log, rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as td
            td.barrier()
            td.destroy_process_group()
        return
    line, snapshot = run_ours(args, rank, world, log)
    if args.ens_count > 0 and not args.profile:
        # config 5 beside the headline: the 64-impact ensemble, each instance 2,000 steps
        ens_args = argparse.Namespace(**vars(args))
        ens_args.ensemble = args.ens_count
        ens = run_ensemble(ens_args, log, rank, world)
        if rank == 0:
            line["ensemble"] = ens
    if rank == 0:
        if world == 1 and not args.no_cpu and not args.profile:
            line["cpu_baseline"] = cpu_reference(snapshot, min_seconds=args.cpu_seconds)
            # the single-thread form of the same sample (the oracle is one binary32 rounding per operation,
            # so the one-thread and all-core runs compute the same steps)
            one = cpu_reference(snapshot, min_seconds=args.cpu_seconds, min_steps=4, threads=1)
            line["cpu_baseline"]["single_thread"] = {"value": one["value"], "cores": 1, "sample": one["sample"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as td
        td.barrier()
        td.destroy_process_group()


if __name__ == "__main__":
    main()
