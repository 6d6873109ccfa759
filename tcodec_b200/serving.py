"""Request loop of the served form: encode sessions arrive over time, are
opened on a tcb_server (admission by HBM footprint, FIFO), are fed their
frames as the server's per-session queue frees up, and are advanced
together one frame per step (continuous batching).

`serve(lib, sessions, clips, ...)` replays an arrival schedule in real time
(session i becomes visible `arrival_s` seconds after the start) and
measures, per frame, the time from the frame being handed to the server
(`push`) to its packet coming back from a step.
"""
from __future__ import annotations

import time
from typing import Dict, List

from . import api


def serve(lib, sessions: List[dict], clips: List[list], hbm_budget_bytes: int, max_active: int = 64,
          preset: int = api.PRESET_MEDIUM, profile: int = 1, on_step=None, graphs: bool = False) -> Dict:
    """Run every session to completion.  sessions[i] has arrival_s, w, h, qp;
    clips[i] is its list of (y, cb, cr) frames.  Returns packets per
    session, per-frame latencies (s), makespan (s) and step statistics."""
    n = len(sessions)
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=preset, profile=profile,
                            keyframe_interval=1000) for s in sessions]
    srv = api.Server(lib, hbm_budget_bytes, max_active)
    srv.set_graphs(graphs)
    sid: Dict[int, int] = {}
    inv: Dict[int, int] = {}
    fed = [0] * n
    push_t: List[List[float]] = [[] for _ in range(n)]
    push_active: List[List[bool]] = [[] for _ in range(n)]   # session admitted when the frame was pushed
    packets: List[List[bytes]] = [[] for _ in range(n)]
    done = [False] * n
    lat: List[float] = []
    lat_admitted: List[float] = []          # frames pushed after their session was admitted
    first_pkt: List[float] = [0.0] * n      # arrival -> first packet of each session (s)
    step_log: List[tuple] = []              # (end of step s, packets, active, waiting)
    steps = 0
    peak_active = 0
    peak_bytes = 0
    nxt = 0
    t0 = time.perf_counter()
    try:
        while not all(done):
            now = time.perf_counter() - t0
            while nxt < n and sessions[nxt]["arrival_s"] <= now:
                s = srv.open(cfgs[nxt])
                sid[nxt], inv[s] = s, nxt
                nxt += 1
            for i, s in sid.items():
                if done[i]:
                    continue
                active = srv.state(s) == api.SESSION_ACTIVE
                while fed[i] < len(clips[i]) and srv.push(s, clips[i][fed[i]]):
                    push_t[i].append(time.perf_counter())
                    push_active[i].append(active)
                    fed[i] += 1
                    if fed[i] == len(clips[i]):
                        srv.finish(s)
            out = srv.step()
            t = time.perf_counter()
            steps += 1
            for s, status, pkt in out:
                if status not in (api.TC_OK, api.TC_ERR_NEED_MORE):
                    raise RuntimeError(f"session {inv[s]} failed: {status}")
                if pkt is not None:
                    i = inv[s]
                    k = len(packets[i])
                    lat.append(t - push_t[i][k])
                    if push_active[i][k]:
                        lat_admitted.append(t - push_t[i][k])
                    if not packets[i]:
                        first_pkt[i] = t - t0 - sessions[i]["arrival_s"]
                    packets[i].append(pkt)
            st = srv.stats()
            step_log.append((t - t0, sum(1 for o in out if o[2] is not None), st["active"], st["waiting"]))
            peak_active = max(peak_active, st["active"])
            peak_bytes = max(peak_bytes, st["bytes_in_use"])
            for i, s in sid.items():
                if not done[i] and srv.state(s) == api.SESSION_DONE:
                    done[i] = True
            if on_step:
                on_step(steps, st)
            if not out and nxt < n and st["active"] == 0:
                # idle until the next arrival
                time.sleep(max(0.0, sessions[nxt]["arrival_s"] - (time.perf_counter() - t0)))
        makespan = time.perf_counter() - t0
        budget = srv.stats()["bytes_budget"]
        timing = srv.timing()
    finally:
        srv.close()
    return dict(packets=packets, latencies=lat, makespan=makespan, steps=steps, peak_active=peak_active,
                peak_bytes=peak_bytes, budget=budget, frames=sum(len(p) for p in packets), timing=timing,
                latencies_admitted=lat_admitted,
                first_packet_s=first_pkt, step_log=step_log)
