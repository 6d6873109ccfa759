"""Served form (tcb_server_*): sessions of different sizes arrive while
others are running, wait for budget when HBM is short, are admitted as
earlier sessions retire, and share every step's CTU-engine launch.  Each
session's packets must equal encoding that session alone (bit-exact), and
device memory in use must never exceed the budget."""
import pytest

pytestmark = pytest.mark.gpu


def test_served_sessions_match_alone_and_respect_budget():
    from tcodec_b200 import api, synth
    lib = api.load_library()
    specs = [  # (w, h, qp, preset, profile, frames, b_frames, arrival step)
        (160, 96, 32, 2, 1, 5, False, 0),
        (128, 72, 22, 2, 0, 4, False, 0),
        (192, 128, 37, 1, 1, 6, False, 1),
        (96, 80, 27, 2, 1, 6, True, 2),
        (320, 240, 32, 2, 1, 3, False, 3),
        (128, 128, 27, 2, 1, 4, False, 6),
    ]
    clips = [synth.stream_clip(dict(w=w, h=h, seed=300 + i, frames=n))
             for i, (w, h, _, _, _, n, _, _) in enumerate(specs)]
    cfgs = [api.make_config(lib, w, h, qp=qp, preset=pr, profile=pf, keyframe_interval=1000, b_frames=b)
            for (w, h, qp, pr, pf, _, b, _) in specs]

    srv = api.Server(lib, hbm_budget_bytes=1, max_active=3)   # probe footprints first
    sizes = [srv.session_bytes(c) for c in cfgs]
    srv.close()
    # The 320x240 session fits only once at most the smallest other session
    # is still admitted, so it has to wait for earlier sessions to retire.
    budget = sizes[4] + min(sizes)
    assert sizes[4] + sizes[0] > budget and sizes[0] + sizes[1] <= budget
    srv = api.Server(lib, hbm_budget_bytes=budget, max_active=3)
    sid = {}
    fed = [0] * len(specs)
    got = {i: [] for i in range(len(specs))}
    saw_waiting = False
    step = 0
    while True:
        for i, spec in enumerate(specs):
            if i not in sid and spec[7] <= step:
                sid[i] = srv.open(cfgs[i])
        for i, s in sid.items():
            while fed[i] < len(clips[i]) and srv.push(s, clips[i][fed[i]]):
                fed[i] += 1
                if fed[i] == len(clips[i]):
                    srv.finish(s)
        out = srv.step()
        st = srv.stats()
        assert st["bytes_in_use"] <= budget
        saw_waiting |= st["waiting"] > 0 and st["active"] > 0
        inv = {v: k for k, v in sid.items()}
        for s, status, pkt in out:
            assert status in (api.TC_OK, api.TC_ERR_NEED_MORE), (s, status)
            if pkt is not None:
                got[inv[s]].append(pkt)
        step += 1
        if len(sid) == len(specs) and all(srv.state(s) == api.SESSION_DONE for s in sid.values()):
            break
        assert step < 200, "served sessions did not drain"
    assert saw_waiting, "budget never made a session wait"
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()
    for i in range(len(specs)):
        want = api.encode_sequence(lib, cfgs[i], clips[i])
        assert got[i] == want, i


def test_failed_admission_is_retried():
    """A session whose admission fails (its first device allocation fails,
    injected on the host) stays queued and is admitted at a later step; no
    session is lost and packets stay bit-exact."""
    from tcodec_b200 import api, synth
    lib = api.bind_b200(api.load_library())
    specs = [(128, 72, 30), (96, 80, 34)]
    clips = [synth.stream_clip(dict(w=w, h=h, seed=700 + i, frames=4)) for i, (w, h, _) in enumerate(specs)]
    cfgs = [api.make_config(lib, w, h, qp=q, preset=2, profile=1, keyframe_interval=1000) for w, h, q in specs]
    srv = api.Server(lib, hbm_budget_bytes=1 << 30, max_active=4)
    sids = [srv.open(c) for c in cfgs]
    fed = [0, 0]
    got = [[], []]
    try:
        for step in range(40):
            for i, s in enumerate(sids):
                while fed[i] < len(clips[i]) and srv.push(s, clips[i][fed[i]]):
                    fed[i] += 1
                    if fed[i] == len(clips[i]):
                        srv.finish(s)
            if step == 0:
                assert lib.tcb_debug_fail_allocations_after(0) < 0
            out = srv.step()
            if step == 0:
                assert lib.tcb_debug_fail_allocations_after(-1) < 0   # the failure fired
                st = srv.stats()
                assert st["waiting"] == 2 and st["active"] == 0 and st["bytes_in_use"] == 0
            for s, status, pkt in out:
                assert status in (api.TC_OK, api.TC_ERR_NEED_MORE), (s, status)
                if pkt is not None:
                    got[sids.index(s)].append(pkt)
            if all(srv.state(s) == api.SESSION_DONE for s in sids):
                break
        else:
            raise AssertionError("sessions did not drain")
    finally:
        lib.tcb_debug_fail_allocations_after(-1)
        srv.close()
    for i in range(2):
        assert got[i] == api.encode_sequence(lib, cfgs[i], clips[i]), i
