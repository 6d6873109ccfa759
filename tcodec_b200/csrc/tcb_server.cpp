// tcb_server.cpp — served form of the v2 encoder: continuous batching of
// encode sessions that arrive and leave at any time.
//
// * Admission: sessions queue FIFO at tcb_server_open.  At each step the
//   head of the queue is admitted while a batch slot is free and the
//   session's device footprint (EncImpl::device_footprint: DPB pool,
//   input, MV grids, decision records, flags, B reorder buffers at their
//   cap) fits in what is left of the HBM budget.  The budget is one
//   device allocation made at creation (DeviceArena); sessions are carved
//   out of it and returned to it, so admission never calls cudaMalloc and
//   never synchronises the device.
// * Residency: an admitted session's reference frames, MV grids and rate /
//   QP state stay on the device (its tc_encoder_t) until it finishes.
// * Stepping: every step advances each admitted session that has an input
//   frame (or a B-frame tail to drain) by one frame, all of them in one
//   shared persistent CTU-engine launch (the batched form); a session that
//   joins mid-stream simply appears in the next step's queue.  Per-session
//   output is bit-identical to encoding the session alone.
#include <string.h>

#include <chrono>
#include <deque>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec_b200.h"
#include "tcb_arena.h"
#include "tcb_batch.h"
#include "tcb_encoder.h"

using namespace tcb;

namespace {

enum SessionState { WAITING = 0, ACTIVE = 1, DONE = 2 };

struct HostFrame {
    std::vector<uint8_t> y, cb, cr;
};

struct Session {
    tc_config_t cfg{};
    size_t footprint = 0;
    int state = WAITING;
    int slot = -1;
    bool finishing = false;
    std::deque<HostFrame> queue;
    tc_error_t error = TC_OK;
};

}  // namespace

struct tcb_server {
    tcb_batch *batch = nullptr;
    DeviceArena arena;
    int max_active = 0;
    std::vector<Session> sessions;
    std::deque<int> waiting;
    std::vector<int> slot_session;       // batch slot -> session id (-1 free)
    std::vector<tc_packet_t> pkts;
    std::vector<int> status;
    int device = 0;
    // host time inside admission (encoder set-up on the arena) and inside
    // whole steps, milliseconds since creation; sessions admitted
    double admit_ms = 0.0, step_ms = 0.0;
    long long admitted = 0;
};

namespace {

bool config_ok(const tc_config_t &c) {
    return c.use_v2 && c.width > 0 && c.height > 0 && !(c.width & 1) && !(c.height & 1) &&
           c.width <= TC_MAX_WIDTH && c.height <= TC_MAX_HEIGHT;
}

void retire(tcb_server *s, int id) {
    Session &ss = s->sessions[id];
    if (ss.slot >= 0) {
        batch_detach(s->batch, ss.slot);   // frees the session's arena blocks
        s->slot_session[ss.slot] = -1;
        ss.slot = -1;
    }
    ss.queue.clear();
    ss.state = DONE;
}

// FIFO admission: stop at the first session that does not fit.
void admit(tcb_server *s) {
    while (!s->waiting.empty()) {
        const int id = s->waiting.front();
        Session &ss = s->sessions[id];
        int free_slot = -1;
        for (int k = 0; k < s->max_active && free_slot < 0; ++k)
            if (s->slot_session[k] < 0) free_slot = k;
        if (free_slot < 0 || ss.footprint > s->arena.capacity() - s->arena.used()) return;
        tc_encoder_t *e = encoder_create(&ss.cfg, &s->arena);
        if (!e) return;                    // fragmented: retry after others leave
        e->impl->recon_readback = false;   // served sessions return packets only
        const int slot = batch_attach(s->batch, e);
        if (slot < 0) { tc_encoder_destroy(e); return; }
        s->slot_session[slot] = id;
        ss.slot = slot;
        ss.state = ACTIVE;
        s->waiting.pop_front();
        ++s->admitted;
    }
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

size_t tcb_server_session_bytes(const tc_config_t *cfg) {
    if (!cfg || !config_ok(*cfg)) return 0;
    return EncImpl::device_footprint(*cfg);
}

tcb_server_t *tcb_server_create(size_t hbm_budget_bytes, int max_active) {
    if (hbm_budget_bytes == 0 || max_active <= 0 || max_active > MAX_STREAMS) return nullptr;
    tcb_server *s = new (std::nothrow) tcb_server();
    if (!s) return nullptr;
    if (cudaGetDevice(&s->device) != cudaSuccess || s->arena.init(hbm_budget_bytes) != cudaSuccess) {
        delete s;
        return nullptr;
    }
    s->batch = batch_new(max_active);
    if (!s->batch) { s->arena.destroy(); delete s; return nullptr; }
    s->max_active = max_active;
    s->slot_session.assign(max_active, -1);
    s->pkts.resize(max_active);
    s->status.resize(max_active);
    return s;
}

void tcb_server_destroy(tcb_server_t *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    for (int id = 0; id < (int)s->sessions.size(); ++id)
        if (s->sessions[id].state == ACTIVE) retire(s, id);
    batch_free(s->batch);
    s->arena.destroy();
    delete s;
}

int tcb_server_open(tcb_server_t *s, const tc_config_t *cfg) {
    if (!s || !cfg || !config_ok(*cfg)) return TC_ERR_PARAM;
    Session ss;
    ss.cfg = *cfg;
    ss.footprint = EncImpl::device_footprint(*cfg);
    if (ss.footprint > s->arena.capacity()) return TC_ERR_MEMORY;   // could never be admitted
    s->sessions.push_back(std::move(ss));
    const int id = (int)s->sessions.size() - 1;
    s->waiting.push_back(id);
    return id;
}

tc_error_t tcb_server_push(tcb_server_t *s, int id, const tc_pixel_t *y, int sy, const tc_pixel_t *cb, int scb,
                           const tc_pixel_t *cr, int scr) {
    if (!s || id < 0 || id >= (int)s->sessions.size() || !y || !cb || !cr) return TC_ERR_PARAM;
    Session &ss = s->sessions[id];
    if (ss.state == DONE || ss.finishing) return TC_ERR_PARAM;
    const int W = ss.cfg.width, H = ss.cfg.height;
    if (sy < W || scb < W / 2 || scr < W / 2) return TC_ERR_PARAM;
    if ((int)ss.queue.size() >= TCB_SERVER_QUEUE) return TC_ERR_NEED_MORE;
    HostFrame f;
    f.y.resize((size_t)W * H);
    f.cb.resize((size_t)(W / 2) * (H / 2));
    f.cr.resize((size_t)(W / 2) * (H / 2));
    for (int r = 0; r < H; ++r) memcpy(&f.y[(size_t)r * W], y + (size_t)r * sy, W);
    for (int r = 0; r < H / 2; ++r) {
        memcpy(&f.cb[(size_t)r * (W / 2)], cb + (size_t)r * scb, W / 2);
        memcpy(&f.cr[(size_t)r * (W / 2)], cr + (size_t)r * scr, W / 2);
    }
    ss.queue.push_back(std::move(f));
    return TC_OK;
}

tc_error_t tcb_server_finish(tcb_server_t *s, int id) {
    if (!s || id < 0 || id >= (int)s->sessions.size()) return TC_ERR_PARAM;
    Session &ss = s->sessions[id];
    if (ss.state == DONE) return TC_OK;
    ss.finishing = true;
    return TC_OK;
}

int tcb_server_session_state(tcb_server_t *s, int id) {
    if (!s || id < 0 || id >= (int)s->sessions.size()) return TC_ERR_PARAM;
    return s->sessions[id].state;
}

static int server_step(tcb_server_t *s, tcb_server_packet_t *out);

int tcb_server_step(tcb_server_t *s, tcb_server_packet_t *out, int cap) {
    if (!s || !out || cap < s->max_active) return TC_ERR_PARAM;
    if (cudaSetDevice(s->device) != cudaSuccess) return TC_ERR_INTERNAL;
    const auto t0 = std::chrono::steady_clock::now();
    admit(s);
    s->admit_ms += ms_since(t0);
    const int r = server_step(s, out);
    s->step_ms += ms_since(t0);
    return r;
}

void tcb_server_get_timing(tcb_server_t *s, double *admit_ms, double *step_ms, long long *admitted) {
    if (!s) return;
    if (admit_ms) *admit_ms = s->admit_ms;
    if (step_ms) *step_ms = s->step_ms;
    if (admitted) *admitted = s->admitted;
}

// The encoding part of a step: every admitted session with input (or a
// B-frame tail) advances one frame.
static int server_step(tcb_server_t *s, tcb_server_packet_t *out) {
    std::vector<int> part;
    for (int slot = 0; slot < s->max_active; ++slot) {
        const int id = s->slot_session[slot];
        if (id < 0) continue;
        Session &ss = s->sessions[id];
        EncImpl &e = *batch_slot(s->batch, slot)->impl;
        s->status[slot] = TC_ERR_NEED_MORE;
        memset(&s->pkts[slot], 0, sizeof(tc_packet_t));
        tc_error_t r;
        if (!ss.queue.empty()) {
            const HostFrame &f = ss.queue.front();
            const int W = ss.cfg.width;
            if (!e.upload(f.y.data(), W, f.cb.data(), W / 2, f.cr.data(), W / 2, e.cur)) return TC_ERR_INTERNAL;
            ss.queue.pop_front();
            r = e.plan_input();
        } else if (ss.finishing) {
            r = e.plan_flush();
            if (r == TC_ERR_EOF) { retire(s, id); continue; }
        } else {
            continue;
        }
        if (r == TC_OK) part.push_back(slot);
        else if (r != TC_ERR_NEED_MORE) { ss.error = r; retire(s, id); }
    }
    if (part.empty()) return 0;
    // Per-slot status tells which sessions failed; a failed session is
    // retired and reports its error in its entry.
    batch_run(s->batch, part, s->pkts.data(), s->status.data());
    int n = 0;
    for (int slot : part) {
        const int id = s->slot_session[slot];
        out[n].session = id;
        out[n].status = s->status[slot];
        out[n].packet = s->pkts[slot];
        ++n;
        if (s->status[slot] != TC_OK && s->status[slot] != TC_ERR_NEED_MORE) {
            s->sessions[id].error = (tc_error_t)s->status[slot];
            retire(s, id);
        }
    }
    return n;
}

void tcb_server_set_graphs(tcb_server_t *s, int enabled) {
    if (s) batch_set_graphs(s->batch, enabled != 0);
}

void tcb_server_stats(tcb_server_t *s, int *waiting, int *active, int *done, size_t *bytes_in_use,
                      size_t *bytes_budget) {
    if (!s) return;
    int w = 0, a = 0, d = 0;
    for (const Session &ss : s->sessions) {
        w += ss.state == WAITING;
        a += ss.state == ACTIVE;
        d += ss.state == DONE;
    }
    if (waiting) *waiting = w;
    if (active) *active = a;
    if (done) *done = d;
    if (bytes_in_use) *bytes_in_use = s->arena.used();
    if (bytes_budget) *bytes_budget = s->arena.capacity();
}

}  // extern "C"
