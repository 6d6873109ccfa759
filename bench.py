#!/usr/bin/env python
"""Benchmark of the B200 v2 encoder on the headline workload.

Headline workload (the 1080p configuration the metric is quoted on):
1920x1080 4:2:0, GOP4 hierarchical B-frames, CQP QP 32, preset MEDIUM,
profile 1 (two searched references: the reference encoder's reachable form
of "4 references"), deblocking + SAO.  Source: seeded synthetic sinusoid
texture + 16 moving noise rectangles + 1-px high-contrast lines over 5% of
the area (tcodec_b200.synth 'rects_lines').

Batched form (the headline): --streams independent 1080p streams per GPU
(default 16; stream s encodes clip frames s, s+1, ...) advance together and
share every CTU-engine launch (tcb_batch_encode).  A step = one input frame
for every stream; frames/s counts packets emitted in the timed region (GOP4
emits one packet per input in steady state).  Every step reads fresh input
frames of a device-resident clip.

  value      frames/s of the batch with inputs already in HBM
  e2e        the same through host (pinned) buffers: host->device copies and
             packet / reconstruction read-back inside the timed region
  plain_gpu  one stream alone through the same kernels

Two more forms run at N=1 (section "forms" of the JSON line):

  mixed_batch  64 independent P-only streams, resolutions uniform over
               {320x240, 640x360, 1280x720, 1920x1080}, QP uniform over
               {22, 27, 32, 37}, 32 frames each, all in one batch; against
               the plain one-stream-at-a-time GPU path on the same mix
               (per-resolution seconds/frame measured on a sample).
  served       Poisson arrivals (200 sessions/s) of 8..64-frame P-only
               sessions of the same mix, admitted under an HBM budget
               (tcb_server); per-frame latency p50/p99 and aggregate
               frames/s.
  Both check every stream / session against the reference encoder's
  digests (tests/golden/mixed_streams.json).

--impl reference times the reference C encoder (oracle/_ref, built from the
reference sources) on all host cores: one encoder process per core, each
on its own segment of the clip, one input frame per process per step.

Multi-GPU: one process per GPU (torchrun); every rank encodes its own
independent streams (replicas, weak scaling, no collective on the data
path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, QP, PRESET, PROFILE = 1920, 1080, 32, 2, 1
METRIC = "1080p v2 encode frames/s (bit-exact), batched/served vs plain GPU; p50/p99 latency"
UNIT = "frames/s"
GOLDEN = os.path.join(ROOT, "tests", "golden", "bench_1080p_gop4b.json")
GRAPHS = False   # --graphs: batched / served steps replayed as CUDA graphs
PIPELINE = True   # batched steps entropy-code the previous step during the device step (--no-pipeline: off)
TRAFFIC = os.path.join(ROOT, "profiles", "ctu_engine_traffic.txt")
OPS = os.path.join(ROOT, "profiles", "ctu_engine_ops.txt")   # work counts per frame (profiling build)   # JSON body
MIXED_GOLDEN = os.path.join(ROOT, "tests", "golden", "mixed_streams.json")
SERVED_BUDGET = 150 * 10**9          # HBM budget of the served form (bytes)


def make_clip(n):
    from tcodec_b200 import synth
    return synth.workload("rects_lines", frames=n)


def make_cfg(lib):
    from tcodec_b200 import api
    return api.make_config(lib, W, H, qp=QP, preset=PRESET, profile=PROFILE, keyframe_interval=1000,
                           b_frames=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- reference arm
def _ref_worker(args):
    seg, frames_needed, barrier, q, steps, warmup = args
    from oracle import tcref
    from tcodec_b200 import api
    lib = tcref.ref_lib()
    frames = make_clip(frames_needed)[seg:]
    enc = api.Encoder(lib, make_cfg(lib))
    i = 0
    for _ in range(warmup):
        enc.encode(*frames[i % len(frames)])
        i += 1
    barrier.wait()
    t0 = time.perf_counter()
    n = 0
    for _ in range(steps):
        if enc.encode(*frames[i % len(frames)]) is not None:
            n += 1
        i += 1
    t1 = time.perf_counter()
    barrier.wait()
    enc.close()
    q.put((n, t0, t1))


def run_reference(steps, warmup, procs):
    """Reference encoder on `procs` host processes; returns (frames/s,
    frames, seconds)."""
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    q = ctx.Queue()
    need = warmup + steps + procs
    ps = [ctx.Process(target=_ref_worker, args=((k, need, barrier, q, steps, warmup),)) for k in range(procs)]
    for p in ps:
        p.start()
    res = [q.get() for _ in ps]
    for p in ps:
        p.join()
    frames = sum(r[0] for r in res)
    t0 = min(r[1] for r in res)
    t1 = max(r[2] for r in res)
    return frames / (t1 - t0), frames, t1 - t0


CPU_WARMUP, CPU_STEPS = 5, 3   # bounded cpu_baseline sample: per process, untimed / timed inputs


def cpu_baseline(procs):
    """Bounded sample of the reference arm: `procs` reference encoder
    processes (one per host core), each on its own segment of the workload,
    past the key frame and the first GOP (CPU_WARMUP inputs, untimed) and
    then timed over CPU_STEPS steady GOP4-B inputs, wall clock from the
    first process's start to the last one's end."""
    t0 = time.perf_counter()
    fps, frames, secs = run_reference(CPU_STEPS, CPU_WARMUP, procs)
    wall = time.perf_counter() - t0
    return {"value": fps, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{procs} reference encoder processes (oracle/_ref, the reference C built -O3, scalar), one "
                      f"per host core, each past {CPU_WARMUP} untimed inputs (key frame and first GOP) then "
                      f"{CPU_STEPS} timed steady GOP4-B inputs of the 1920x1080 workload: {frames} packets in "
                      f"{secs:.1f} s ({wall:.1f} s wall with warm-up)"}


# ---------------------------------------------------------------- mixed workloads
def _render_stream(spec):
    from tcodec_b200 import synth
    return synth.stream_clip(spec)


def render_streams(specs, procs):
    """Frames of every stream spec, rendered on `procs` spawned processes
    (before any CUDA work in this process)."""
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(_render_stream, specs, chunksize=1)


def stream_digest(packets):
    h = hashlib.sha256()
    for p in packets:
        h.update(len(p).to_bytes(4, "little") + p)
    return h.hexdigest()


def run_mixed_batch(lib, specs, clips):
    """All streams in one batch, host (pinned) inputs; returns device time,
    frames and every stream's packets."""
    import torch
    from tcodec_b200 import api
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=PRESET, profile=PROFILE,
                            keyframe_interval=1000) for s in specs]
    pinned = [[tuple(torch.from_numpy(np.ascontiguousarray(p)).pin_memory().numpy() for p in f) for f in c]
              for c in clips]
    batch = api.BatchEncoder(lib, cfgs)
    batch.set_graphs(GRAPHS)
    if PIPELINE:
        batch.set_pipelined(True)
    lib.tcb_batch_set_timing(batch.h, 1)
    n = len(specs)
    nf = max(len(c) for c in clips)
    got = [[] for _ in range(n)]
    stream = torch.cuda.ExternalStream(lib.tcb_batch_stream(batch.h))
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    for t in range(nf):
        pk = batch.encode([pinned[i][t] if t < len(pinned[i]) else None for i in range(n)], on_device=False)
        for i, p in enumerate(pk):
            if p is not None:
                got[i].append(p)
    tail = batch.flush()
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    st = (ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64())
    lib.tcb_batch_get_timing(batch.h, *[ctypes.byref(x) for x in st])
    batch.close()
    for i in range(n):
        got[i].extend(tail[i])
    return dict(ms=ev0.elapsed_time(ev1), wall=wall, frames=sum(len(g) for g in got), packets=got,
                ctu_ms=st[0].value, launches=st[4].value)


def plain_seconds_per_frame(lib, w, h, qp, frames):
    """One stream alone (device inputs, tcb_encoder_encode_device): seconds
    per frame over `frames` after 2 warm-up frames."""
    import torch
    from tcodec_b200 import api
    enc = api.Encoder(lib, api.make_config(lib, w, h, qp=qp, preset=PRESET, profile=PROFILE,
                                           keyframe_interval=1000))
    lib.tcb_encoder_set_recon_readback(enc.h, 0)
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f) for f in frames]
    stream = torch.cuda.ExternalStream(lib.tcb_encoder_stream(enc.h))

    def one(f):
        pkt = api.Packet()
        r = lib.tcb_encoder_encode_device(enc.h, f[0].data_ptr(), w, f[1].data_ptr(), w // 2, f[2].data_ptr(),
                                          w // 2, ctypes.byref(pkt))
        if r != api.TC_OK:
            raise RuntimeError(f"plain encode -> {r}")

    for f in dev[:2]:
        one(f)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for f in dev[2:]:
        one(f)
    ev1.record(stream)
    torch.cuda.synchronize()
    enc.close()
    return ev0.elapsed_time(ev1) / 1000.0 / max(1, len(dev) - 2)


def run_forms(lib, mixed_specs, mixed_clips, served_specs, served_clips):
    from tcodec_b200 import serving, synth
    golden = json.load(open(MIXED_GOLDEN)) if os.path.exists(MIXED_GOLDEN) else None
    out = {}
    # ---- batched, 64-stream mix ------------------------------------------
    mb = run_mixed_batch(lib, mixed_specs, mixed_clips)
    exact = None
    if golden:
        exact = all(stream_digest(mb["packets"][i]) == golden["batch"][i]["digest"]
                    for i in range(len(mixed_specs)))
    # plain path on the same mix: seconds per frame for every (resolution,
    # QP) pair of the mix, measured on the first stream of the mix with that
    # pair (its own frames 0..7: 2 warm-up + 6 timed), summed over the mix's
    # frames
    spf = {}
    for spec, c in zip(mixed_specs, mixed_clips):
        key = (spec["w"], spec["h"], spec["qp"])
        if key not in spf:
            spf[key] = plain_seconds_per_frame(lib, spec["w"], spec["h"], spec["qp"], c[:8])
    plain_s = sum(len(c) * spf[(s["w"], s["h"], s["qp"])] for s, c in zip(mixed_specs, mixed_clips))
    mixed_frames = sum(len(c) for c in mixed_clips)
    batched_fps = mb["frames"] / (mb["ms"] / 1000.0)
    plain_fps = mixed_frames / plain_s
    pix = sum(s["w"] * s["h"] * len(c) for s, c in zip(mixed_specs, mixed_clips))
    out["mixed_batch"] = {
        "streams": len(mixed_specs), "frames": mb["frames"], "value": batched_fps, "unit": UNIT,
        "pixels_per_s": pix / (mb["ms"] / 1000.0), "plain_gpu_fps": plain_fps,
        "batched_over_plain": batched_fps / plain_fps, "bit_exact_all_streams": exact,
        "plain_s_per_frame": {f"{w}x{h}@qp{q}": v for (w, h, q), v in sorted(spf.items())},
        "what": "64 P-only streams (mixed resolution and QP, 32 frames) in one tcb_batch, host inputs and packets "
                "inside the timed region; plain = the same frames encoded one stream at a time, s/frame of "
                "every (resolution, QP) pair of the mix measured on that pair's first stream (6 timed frames "
                "after 2 warm-up frames)"}
    # ---- served -------------------------------------------------------------
    out["served"] = run_served(lib, served_specs, served_clips, golden)
    return out


def run_served(lib, served_specs, served_clips, golden):
    """The served form over `served_specs` (a prefix of the Poisson schedule)
    replayed in real time through tcb_server under the HBM budget; every
    session with a reference digest on file (the first sessions, and the
    seeded sample of tests/golden/mixed_streams.json) is checked."""
    import torch
    from tcodec_b200 import serving
    free, total = torch.cuda.mem_get_info()
    budget = min(SERVED_BUDGET, int(free * 0.9))
    sv = serving.serve(lib, served_specs, served_clips, budget, max_active=256, preset=PRESET, profile=PROFILE,
                       graphs=GRAPHS)
    want = {}
    if golden:
        want.update({j: r["digest"] for j, r in enumerate(golden.get("served", []))})
        want.update({int(k): r["digest"] for k, r in golden.get("served_sample", {}).items()})
    checked = [j for j in range(len(served_specs)) if j in want]
    exact = (all(stream_digest(sv["packets"][j]) == want[j] for j in checked) if checked else None)
    lat = sorted(sv["latencies"])
    lat_a = sorted(sv["latencies_admitted"])
    start = sorted(sv["first_packet_s"])
    def pct(v, q):   # q-quantile in ms, None for no samples
        return 1000 * v[min(len(v) - 1, int(q * len(v)))] if v else None
    pix_s = sum(s["w"] * s["h"] * s["frames"] for s in served_specs)
    # saturated window: steps taken while sessions waited for admission
    sat = [e for e in sv["step_log"] if e[3] > 0]
    sat_fps = None
    if len(sat) > 1:
        sat_fps = sum(e[1] for e in sat[1:]) / max(1e-9, sat[-1][0] - sat[0][0])
    tm = sv["timing"]
    return {
        "sessions": len(served_specs), "frames": sv["frames"], "value": sv["frames"] / sv["makespan"],
        "unit": UNIT, "pixels_per_s": pix_s / sv["makespan"], "makespan_s": sv["makespan"],
        "saturated_fps": sat_fps,
        "saturated_what": "frames/s over the steps taken while sessions were waiting for admission "
                          "(arrivals outpace the encoder; slots and budget bind)",
        "latency_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99),
                       "what": "per frame: push to the server until its packet returns (frames pushed while "
                               "their session waited for admission included)"},
        "latency_admitted_ms": {"p50": pct(lat_a, 0.5), "p99": pct(lat_a, 0.99),
                                "frames": len(lat_a),
                                "what": "per frame pushed after its session was admitted: push until its packet"},
        "session_start_ms": {"p50": pct(start, 0.5), "p99": pct(start, 0.99),
                             "what": "per session: arrival until its first packet (admission queueing included)"},
        "admission": {"host_ms": tm["admit_ms"], "sessions_admitted": tm["admitted"],
                      "ms_per_session": tm["admit_ms"] / max(1, tm["admitted"]),
                      "share_of_step_time": tm["admit_ms"] / max(1e-9, tm["step_ms"]),
                      "what": "host time inside tcb_server_step admitting sessions (encoder set-up in the "
                              "budget's arena), against the whole steps' host time"},
        "hbm_budget_bytes": sv["budget"], "peak_bytes_in_use": sv["peak_bytes"],
        "peak_active_sessions": sv["peak_active"], "steps": sv["steps"],
        "bit_exact_sessions_checked": len(checked), "bit_exact_checked_sessions": exact,
        "bit_exact_all_sessions": exact if len(checked) == len(served_specs) else None,
        "what": f"first {len(served_specs)} sessions of the Poisson schedule (200 sessions/s, 8..64 frames, "
                "P-only, mixed resolution/QP), replayed in real time through tcb_server (at most 256 admitted); "
                "makespan from the first arrival to the last packet"}


# ---------------------------------------------------------------- standalone kernels
def run_standalone_kernels(lib, peak, iters=8, frames=64):
    """HBM roofline of the standalone frame kernels on `frames` 1920x1080
    frames per call (inputs + outputs far larger than L2; L2 flushed
    before every timed call): deblocking (3 bytes per pixel of full CTUs),
    SAO (4 B/px: source + reconstruction read, reconstruction written) and
    motion compensation (3 B/px: luma + chroma read and written) with a
    uniform fractional vector (+2.5, +0.75) px and with random vectors."""
    import torch
    from tcodec_b200 import api
    W_, H_, N = 1920, 1080, frames
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    y = torch.randint(0, 256, (N, H_, W_), dtype=torch.uint8, device="cuda", generator=g)
    src = (y.int() + torch.randint(-5, 6, (N, H_, W_), device="cuda", generator=g)).clamp(0, 255).to(torch.uint8)
    cb = torch.randint(0, 256, (N, H_ // 2, W_ // 2), dtype=torch.uint8, device="cuda", generator=g)
    cr = torch.randint(0, 256, (N, H_ // 2, W_ // 2), dtype=torch.uint8, device="cuda", generator=g)
    py, pcb, pcr = torch.empty_like(y), torch.empty_like(cb), torch.empty_like(cr)
    nctu = ((W_ + 63) // 64) * ((H_ + 63) // 64)
    par = torch.zeros(N, nctu * 3, dtype=torch.int16, device="cuda")
    gw, gh = (W_ + 7) // 8, (H_ + 7) // 8
    mv_glob = torch.tensor([10, 3], dtype=torch.int16, device="cuda").repeat(N, gh * gw, 1).contiguous()
    mv_rand = torch.randint(-96, 97, (N, gh * gw, 2), dtype=torch.int16, device="cuda", generator=g)
    ff = (api.FilterFrame * N)()
    for i, f in enumerate(ff):
        f.width, f.height, f.stride_y, f.stride_c, f.stride_src, f.qp = W_, H_, W_, W_ // 2, W_, 32
        f.y, f.cb, f.cr = y[i].data_ptr(), cb[i].data_ptr(), cr[i].data_ptr()
        f.src_y, f.sao_params = src[i].data_ptr(), par[i].data_ptr()

    def mc_frames(mv):
        m = (api.McFrame * N)()
        for i, f in enumerate(m):
            f.width, f.height, f.stride_y, f.stride_c = W_, H_, W_, W_ // 2
            f.ref_y, f.ref_cb, f.ref_cr = src[i].data_ptr(), cb[i].data_ptr(), cr[i].data_ptr()
            f.pred_y, f.pred_cb, f.pred_cr = py[i].data_ptr(), pcb[i].data_ptr(), pcr[i].data_ptr()
            f.mv = mv[i].data_ptr()
        return m

    st = torch.cuda.current_stream()
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device="cuda")
    # Tile shape (threads per CTA) of each kernel from the autotuner, timed
    # on 32 scratch 1080p frames; the kernels below then run that variant.
    torch.cuda.synchronize()
    if lib.tcb_autotune_frame_kernels(W_, H_, 32) != 0:
        raise RuntimeError("tcb_autotune_frame_kernels failed")
    tuned = {k: lib.tcb_autotune_threads(v, W_, H_) for k, v in
             (("tcb_deblock_frames", api.KERNEL_DEBLOCK), ("tcb_sao_frames", api.KERNEL_SAO),
              ("tcb_mc_frames", api.KERNEL_MC))}
    out = {}
    cases = (("tcb_deblock_frames", lib.tcb_deblock_frames, ff, 3.0 * W_ * (H_ // 64 * 64)),
             ("tcb_sao_frames", lib.tcb_sao_frames, ff, 4.0 * W_ * H_),
             ("tcb_mc_frames (uniform fractional vector)", lib.tcb_mc_frames, mc_frames(mv_glob), 3.0 * W_ * H_),
             ("tcb_mc_frames (random vectors)", lib.tcb_mc_frames, mc_frames(mv_rand), 3.0 * W_ * H_))
    for name, fn, arg, per_frame in cases:
        ts = []
        for _ in range(iters):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            if fn(arg, N, st.cuda_stream) != 0:
                raise RuntimeError(f"{name} failed")
            e1.record(st)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        t = sorted(ts[2:])[len(ts[2:]) // 2] / 1000.0
        achieved = per_frame * N / t / 1e9
        out[name] = {"frames_per_call": N, "ms": t * 1000.0, "algorithmic_bytes": per_frame * N,
                     "achieved_gbs": achieved, "frac_of_hbm": achieved / peak,
                     "threads_per_cta": tuned[name.split(" ")[0]]}
    return out


# ---------------------------------------------------------------- engine phase profile
PHASES = ["refs/mvp", "ME", "MC", "resid jobs", "skip chk", "scan", "CfL", "replay", "decide(total)",
          "write pass", "deblock+sao", "me0:int", "me0:subpel"]


def run_phase_profile(streams, steps, ops_out=None):
    """Counters of the CTU engine on the batched 1080p GOP4-B workload, read
    from the profiling build (`make -C tcodec_b200 prof`: the same kernels
    compiled with -DTCB_PHASE_PROFILE):

    * per-phase cycles of each CTU (thread 0's clock64 deltas summed over CTUs);
    * each CTA's residency and the cycles it waited for a left or above
      neighbour's publish flag;
    * work counts: integer-search SAD pixel differences, quarter-sample SAD
      pixels, and 8x8 / 4x4 transform units coded.  The encode is
      deterministic, so these counts hold for the production build too.

    The counters slow the engine: its timings are for shares, not for
    throughput."""
    from tcodec_b200 import api, synth
    lib = api.load_library(os.path.join(ROOT, "tcodec_b200", "libtcodec_b200_prof.so"))
    lib = api.bind_b200(lib)
    lib.tcb_debug_phase_cycles.argtypes = [ctypes.c_void_p]
    lib.tcb_debug_op_counts.argtypes = [ctypes.c_void_p]
    S = streams
    clip = synth.workload("rects_lines", frames=12)
    batch = api.BatchEncoder(lib, [make_cfg(lib) for _ in range(S)])
    cyc, ops = (ctypes.c_ulonglong * 64)(), (ctypes.c_ulonglong * 4)()
    tot, steady = [0, 0, 0, 0], 0
    for t in range(steps):
        t0 = time.time()
        pk = batch.encode([clip[(t + s) % len(clip)] for s in range(S)])
        dt = time.time() - t0
        lib.tcb_debug_phase_cycles(cyc)
        lib.tcb_debug_op_counts(ops)
        coded = sum(p is not None for p in pk)
        enc = cyc[8] + cyc[9] + cyc[10]
        print(f"step {t} {dt * 1000:.0f} ms, {coded} frames: residency {cyc[14] / 1e9:.2f} Gcyc, encode "
              f"{100 * enc / max(1, cyc[14]):.1f} %, neighbour wait {100 * cyc[13] / max(1, cyc[14]):.1f} %; "
              f"int SAD px {ops[0] / 1e9:.3f} G, qpel SAD px {ops[1] / 1e9:.3f} G, "
              f"TU8 {ops[2] / 1e6:.2f} M, TU4 {ops[3] / 1e6:.2f} M")
        if t == steps - 1:
            for i, n in enumerate(PHASES):
                print(f"   {n:14s} {cyc[i] / 1e6:10.1f} Mcyc  {100 * cyc[i] / max(1, enc):5.1f} %")
            # per quadtree depth: leaf decisions, their phases (share of the
            # encode) and group 0's search split
            print("   depth  leaves/CTU  kcyc/leaf  " + "  ".join(f"{n[:8]:>8s}" for n in PHASES[:8])
                  + "   me:int  me:qpel")
            nctu = S * ((1920 + 63) // 64) * ((1080 + 63) // 64)
            for d in range(4):
                n = cyc[48 + d]
                tot_d = sum(cyc[16 + 8 * d + k] for k in range(8))
                row = "  ".join(f"{100 * cyc[16 + 8 * d + k] / max(1, enc):7.1f}%" for k in range(8))
                print(f"   {d:5d}  {n / nctu:10.1f}  {tot_d / max(1, n) / 1e3:9.1f}  {row}  "
                      f"{100 * cyc[52 + 2 * d] / max(1, enc):6.1f}%  {100 * cyc[53 + 2 * d] / max(1, enc):6.1f}%")
            print("   inside residual jobs (thread 0, all leaves): " + ", ".join(
                f"{n} {100 * cyc[k] / max(1, enc):.1f}%" for k, n in
                ((60, "setup+residual"), (61, "8x8 transform chain"), (62, "recon+sums"), (63, "intra fill"))))
        if t >= 4 and coded == S:          # steady GOP4-B steps (after the first anchor)
            steady += 1
            for i in range(4):
                tot[i] += ops[i]
    batch.close()
    per_frame = {k: tot[i] / max(1, steady * S) for i, k in enumerate(("int_sad_px", "qpel_sad_px", "tu8", "tu4"))}
    print("per frame:", json.dumps(per_frame))
    if ops_out:
        out = {"workload": f"1920x1080 GOP4-B, CQP 32, preset medium, profile 1, {S} streams, "
                           f"mean over {steady} steady steps",
               "per_frame": per_frame,
               "int32_lanes_per_sm_clock": 64,
               "peak_note": "integer peak taken as 64 INT32 lane operations per SM per clock (half the 128 "
                            "FP32 lanes), an assumption; a packed SAD (vsadu4) counts 4 byte differences",
               "command": "python bench.py --phase-profile --streams %d --steps %d --ops-out <file>" % (S, steps)}
        with open(ops_out, "w") as f:
            f.write(json.dumps(out, indent=1) + "\n")


# ---------------------------------------------------------------- B200 arm
def run_b200(args, rank, world):
    """Batched pass (device-resident and host inputs) and a plain
    single-stream pass.  Stream s of the batch encodes clip frames s, s+1, ..."""
    import torch
    from tcodec_b200 import api
    lib = api.bind_b200(api.load_library())
    dev = torch.device("cuda", torch.cuda.current_device())
    K, Wm, S = args.steps, args.warmup, args.streams
    clip = make_clip(S + Wm + K)
    dplanes = [tuple(torch.from_numpy(np.ascontiguousarray(p)).to(dev) for p in f) for f in clip]
    torch.cuda.synchronize()
    tuned = None
    if not args.no_tune:
        # the engine's knobs for this frame size, timed on this workload's own
        # frames (one GOP per combination after the key frame and first GOP)
        from tcodec_b200 import tuning
        tuned = tuning.describe(tuning.tune_engine(lib, make_cfg(lib), clip, streams=S, steps=4, warmup=5))

    def timed(stream_ptr, fn_step, after_warmup=None, finish=None):
        # finish (pipelined batches): the packets still pending after the
        # last step, coded inside the timed region, so the region holds
        # exactly the device steps and the entropy coding of its frames
        stream = torch.cuda.ExternalStream(stream_ptr)
        for t in range(Wm):
            fn_step(t)
        if after_warmup:
            after_warmup()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        frames, nbytes, lat = 0, 0, []
        for t in range(Wm, Wm + K):
            t0 = time.perf_counter()
            n, b = fn_step(t)
            lat.append(time.perf_counter() - t0)
            frames += n
            nbytes += b
        if finish:
            n, b = finish()
            frames += n
            nbytes += b
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        return ev0.elapsed_time(ev1), frames, nbytes, lat

    def batch_pass(on_device):
        batch = api.BatchEncoder(lib, [make_cfg(lib) for _ in range(S)])
        batch.set_graphs(GRAPHS)
        if PIPELINE:
            batch.set_pipelined(True)
        lib.tcb_batch_set_timing(batch.h, 1)
        pinned = None
        if not on_device:
            pinned = [tuple(torch.from_numpy(np.ascontiguousarray(p)).pin_memory().numpy() for p in f) for f in clip]
        per = [[] for _ in range(S)]   # every stream's packets, coding order

        def keep(pk):
            for i, p in enumerate(pk):
                if p is not None:
                    per[i].append(p)

        def step(t):
            if on_device:
                planes = [tuple((dplanes[s + t][k].data_ptr(), dplanes[s + t][k].shape[1]) for k in range(3))
                          for s in range(S)]
            else:
                planes = [pinned[s + t] for s in range(S)]
            pk = batch.encode(planes, on_device=on_device)
            keep(pk)
            got = [p for p in pk if p is not None]
            return len(got), sum(len(p) for p in got)

        st = (ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64())
        hs = (ctypes.c_double(), ctypes.c_double(), ctypes.c_double())

        def reset():
            lib.tcb_batch_get_timing(batch.h, *[ctypes.byref(x) for x in st])
            lib.tcb_batch_get_host_timing(batch.h, *[ctypes.byref(x) for x in hs])

        def drain():
            pk = batch.drain()
            keep(pk)
            got = [p for p in pk if p is not None]
            return len(got), sum(len(p) for p in got)

        def after_warmup():
            if PIPELINE:       # nothing pending when the timed region starts
                keep(batch.drain())
            reset()

        res = timed(lib.tcb_batch_stream(batch.h), step, after_warmup, drain if PIPELINE else None)
        reset()
        tail = batch.flush()
        batch.close()
        ms, frames, nbytes, lat = res
        for i in range(S):
            per[i].extend(tail[i])
        return dict(ms=ms, frames=frames, bytes=nbytes, lat=lat, packets=per[0], streams=per, ctu_ms=st[0].value,
                    ctu_launches=st[1].value, ctu_count=st[2].value, steps=st[3].value, launches=st[4].value,
                    host=[x.value for x in hs])

    def plain_pass():
        enc = api.Encoder(lib, make_cfg(lib))

        def step(t):
            y, cb, cr = dplanes[t]
            pkt = api.Packet()
            r = lib.tcb_encoder_encode_device(enc.h, y.data_ptr(), W, cb.data_ptr(), W // 2, cr.data_ptr(), W // 2,
                                              ctypes.byref(pkt))
            if r == api.TC_ERR_NEED_MORE:
                return 0, 0
            if r != api.TC_OK:
                raise RuntimeError(f"encode -> {r}")
            return 1, pkt.size

        ms, frames, nbytes, lat = timed(lib.tcb_encoder_stream(enc.h), step)
        enc.close()
        return dict(ms=ms, frames=frames)

    clocks = ClockSampler(torch.cuda.current_device())
    with clocks:
        dev_run = batch_pass(True)
    e2e_run = batch_pass(False)
    plain = plain_pass() if not args.no_plain else None
    return dev_run, e2e_run, plain, clocks.summary(), tuned


def check_bit_exact(dev_run, e2e_run, args):
    """(bit_exact, what): every stream's whole packet sequence against the
    reference digests of tests/golden/bench_1080p_gop4b.json when this run
    fed the streams the same number of inputs, else the first packets of
    stream 0; None when no answer on file covers the run."""
    if not os.path.exists(GOLDEN):
        return None, None
    g = json.load(open(GOLDEN))
    st = g.get("streams")
    n_in = args.warmup + args.steps
    if st and st["inputs"] == n_in and args.streams <= st["count"]:
        ok = all(stream_digest(run["streams"][i]) == st["digests"][i]
                 for run in (dev_run, e2e_run) for i in range(args.streams))
        return ok, (f"all {args.streams} streams, every packet of {n_in} inputs + flush, device-resident and "
                    f"host-input runs, against the reference encoder's digests")
    if g["inputs"] <= n_in:
        want = g["packets"]
        got = [hashlib.sha256(p).hexdigest() for p in dev_run["packets"][:len(want)]]
        same_e2e = [hashlib.sha256(p).hexdigest() for p in e2e_run["packets"][:len(want)]] == got
        return bool(got == want and same_e2e), f"stream 0, first {len(want)} packets"
    return None, None


def api_lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


def _reduce(x, world, op):
    if world <= 1:
        return x
    import torch
    dev = "cuda" if torch.distributed.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world):
    """Slowest rank's time: the job's time."""
    import torch
    return _reduce(x, world, torch.distributed.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(x, world):
    """All ranks' frames: the job's work."""
    import torch
    return _reduce(x, world, torch.distributed.ReduceOp.SUM if world > 1 else None)


def job_throughput(frames_per_rank, ms_per_rank, world):
    """Whole-job frames/s: every rank's frames over the slowest rank's
    device time (ranks encode independent streams; weak scaling)."""
    return sum_over_ranks(frames_per_rank, world) / (max_over_ranks(ms_per_rank, world) / 1000.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--streams", type=int, default=32, help="1080p streams per GPU in the batched form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed-batch and served forms")
    ap.add_argument("--served-sessions", type=int, default=64)
    ap.add_argument("--served-only", action="store_true",
                    help="only the served form over --served-sessions sessions of the Poisson schedule, with its "
                         "sampled bit-exact check (one JSON line)")
    ap.add_argument("--no-kernels", action="store_true", help="skip the standalone-kernel roofline section")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the engine's default knobs instead of timing every combination first "
                         "(tcodec_b200.tuning)")
    ap.add_argument("--no-pipeline", action="store_true",
                    help="unpipelined batch steps (default: each call entropy-codes the previous call's frames "
                         "during its own device step)")
    ap.add_argument("--graphs", action="store_true",
                    help="replay every batched / served step's device work as one CUDA graph")
    ap.add_argument("--phase-profile", action="store_true",
                    help="per-phase cycle split and work counts of the CTU engine from the profiling build "
                         "(make -C tcodec_b200 prof); --ops-out writes the work counts")
    ap.add_argument("--ops-out", default=None)
    ap.add_argument("--kernels-only", action="store_true",
                    help="only time the standalone frame kernels (deblock, SAO, motion compensation)")
    args = ap.parse_args()
    global GRAPHS, PIPELINE
    GRAPHS = args.graphs
    PIPELINE = not args.no_pipeline
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    config = {"workload": "1920x1080 4:2:0, GOP4 hierarchical B, CQP QP32, preset medium, profile 1 (2 searched "
                          "refs), deblock+SAO, synthetic source (sinusoids + 16 moving noise rectangles + "
                          "1-px lines over 5% area)",
              "streams_per_gpu": args.streams, "frames_per_step": f"one per stream ({args.streams})",
              "l2": "fresh input frames every step from a device-resident clip (no reuse across steps)",
              "parallelism": f"replicas x{args.gpus}: every GPU encodes its own {args.streams} streams"}

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import tcref
        if not tcref.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference build) is missing"}))
            return
        procs = max(1, os.cpu_count() or 1)
        fps, frames, secs = run_reference(args.steps, args.warmup, procs)
        line = {"metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000 * secs / max(1, args.steps), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic",
                "config": config, "impl": "reference",
                "cpu_baseline": {"value": fps, "unit": UNIT, "cores": procs, "kind": "reference",
                                 "sample": f"{procs} reference encoder processes, one input frame each per step, "
                                           f"{frames} frames in {secs:.1f} s"},
                "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if args.served_only:
        from tcodec_b200 import synth
        specs = synth.served_sessions()[:args.served_sessions]
        clips = render_streams(specs, max(1, os.cpu_count() or 1))
        import torch
        golden = json.load(open(MIXED_GOLDEN)) if os.path.exists(MIXED_GOLDEN) else None
        clocks = ClockSampler(torch.cuda.current_device())
        with clocks:
            res = run_served(api_lib(), specs, clips, golden)
        print(json.dumps({"metric": METRIC, "form": "served", "served": res, "clocks": clocks.summary()}))
        return
    if args.phase_profile:
        run_phase_profile(args.streams, max(args.steps, 6), args.ops_out)
        return
    if args.kernels_only:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]) \
            if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
        print(json.dumps(run_standalone_kernels(api_lib(), peak, iters=max(3, args.steps))))
        return
    forms = not args.no_forms and world == 1
    if forms:
        from tcodec_b200 import synth
        procs = max(1, min(32, os.cpu_count() or 1))
        mixed_specs = synth.mixed_streams()
        served_specs = synth.served_sessions()[:args.served_sessions]
        rendered = render_streams(mixed_specs + served_specs, procs)
        mixed_clips, served_clips = rendered[:len(mixed_specs)], rendered[len(mixed_specs):]
    import torch
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev_run, e2e_run, plain, clocks, tuned = run_b200(args, rank, world)
    # Bit-exactness against the reference's committed answers for this
    # workload, on every rank (each rank encodes the same streams), both
    # runs (device-resident and host inputs).
    exact, exact_what = check_bit_exact(dev_run, e2e_run, args)
    if exact is not None and world > 1:
        import torch
        exact = _reduce(1.0 if exact else 0.0, world, torch.distributed.ReduceOp.MIN) > 0.5
    bit_exact = exact
    ms = max_over_ranks(dev_run["ms"], world)
    frames = sum_over_ranks(dev_run["frames"], world)
    ms_e2e = max_over_ranks(e2e_run["ms"], world)
    frames_e2e = sum_over_ranks(e2e_run["frames"], world)
    if world > 1:
        torch.distributed.barrier()
    if rank != 0:
        torch.distributed.destroy_process_group()
        return

    value = frames / (ms / 1000.0)
    e2e = frames_e2e / (ms_e2e / 1000.0)
    # Roofline of the dominant kernel (the CTU engine).  Algorithmic bytes
    # per frame: the stages it fuses at their standalone minimum traffic,
    # MC 3WH + deblock 3WH + SAO 4WH = 10*W*H bytes.
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    steps = max(1, dev_run["steps"])
    launches = max(1, dev_run["ctu_launches"])
    per_launch_s = max(1e-9, dev_run["ctu_ms"] / 1000.0 / launches)
    # frames the timed launches encoded (all CTUs of every stream per step)
    nctu_frame = ((W + 63) // 64) * ((H + 63) // 64)
    frames_in_launches = dev_run["ctu_count"] / nctu_frame
    alg_bytes_per_launch = 10.0 * W * H * frames_in_launches / launches
    achieved = alg_bytes_per_launch / per_launch_s / 1e9
    traffic = None
    if os.path.exists(TRAFFIC):
        # DRAM bytes of a captured launch, scaled by the CTUs of this run's
        # launches (each CTU writes its records, spills and reconstruction once)
        t = json.load(open(TRAFFIC))["measured"]
        per_ctu = (t["dram_read_bytes"] + t["dram_write_bytes"]) / t["ctus"]
        traffic = per_ctu * dev_run["ctu_count"] / launches
    # Integer work of the engine (the bound the byte roofline does not show):
    # the profiling build's per-frame counts of integer-search SAD pixel
    # differences and coded transform units, which are the same in this
    # build (the encode is deterministic), over this run's engine time.
    integer_work = None
    if os.path.exists(OPS):
        o = json.load(open(OPS))
        pf = o["per_frame"]
        fr_s = frames_in_launches / (dev_run["ctu_ms"] / 1000.0)          # frames per engine-second
        sad = pf["int_sad_px"] * fr_s
        macs = (2048.0 * pf["tu8"] + 256.0 * pf["tu4"]) * fr_s
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        clk = (clocks.get("sm_mhz") or 1965.0) * 1e6
        lane_peak = sms * o["int32_lanes_per_sm_clock"] * clk
        integer_work = {
            "sad_pixel_diffs_per_s": sad, "transform_macs_per_s": macs,
            "int32_lane_peak_ops_per_s": lane_peak,
            "sad_frac_of_packed_peak": sad / (4.0 * lane_peak),   # four byte differences per lane op (vsadu4)
            "transform_mac_frac": macs / lane_peak,
            "counts": os.path.relpath(OPS, ROOT), "peak_note": o["peak_note"]}
    lat = sorted(dev_run["lat"])
    p50 = lat[len(lat) // 2] * 1000 if lat else None
    p99 = lat[min(len(lat) - 1, int(0.99 * len(lat)))] * 1000 if lat else None
    nctu = ((W + 63) // 64) * ((H + 63) // 64)
    S = args.streams
    import_rec = 1.5 * W * H * S
    rec_bytes = (13504 * nctu + 1.5 * W * H) * S
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic", "config": config,
        "bit_exact": bit_exact, "bit_exact_what": exact_what, "frames_timed": int(frames),
        "latency_ms": {"p50": p50, "p99": p99, "what": "per-step batch call latency (one frame of every stream), "
                       "device-resident input"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "ctu_persistent_kernel (CTU RDO engine)",
                     "peak_source": peak_src,
                     "note": "algorithmic bytes 10*W*H per frame (MC 3WH + deblock 3WH + SAO 4WH) over the "
                             "step's persistent launch; the engine is latency / integer-pipe bound, not HBM bound"},
        "ctu_engine": {"ms_per_step": dev_run["ctu_ms"] / steps, "launches_per_step": launches / steps,
                       "ctus_per_launch": dev_run["ctu_count"] / launches, "integer_work": integer_work},
        "host_ms_per_step": {k: v / steps for k, v in zip(("plan_launch", "wait_device", "entropy"),
                                                          dev_run["host"])},
        "batch": {"streams_per_gpu": args.streams, "form": "batched: every stream's CTUs in one persistent "
                  "wavefront launch per step (tcb_batch_encode)", "cuda_graphs": GRAPHS, "pipelined": PIPELINE},
        "plain_gpu": (None if plain is None else {"value": plain["frames"] / (plain["ms"] / 1000.0), "unit": UNIT,
                      "what": "one stream alone through the same kernels (tcb_encoder_encode_device)"}),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(import_rec),
                "d2h_bytes_per_step": int(rec_bytes + e2e_run["bytes"] / max(1, args.steps))},
        "gpu_launches": int(dev_run["launches"]),
        "engine_tuning": tuned if tuned else {"search_window": 4, "queue_order": "diagonal",
                                              "what": "defaults (--no-tune)"},
        "clocks": clocks,
    }
    if forms:
        line["forms"] = run_forms(api_lib(), mixed_specs, mixed_clips, served_specs, served_clips)
    if not args.no_kernels and world == 1:
        line["standalone_kernels"] = run_standalone_kernels(api_lib(), peak)
    if not args.no_cpu_baseline:
        try:
            from oracle import tcref
            if tcref.available():
                line["cpu_baseline"] = cpu_baseline(max(1, os.cpu_count() or 1))
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": f"failed: {e}"}
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
