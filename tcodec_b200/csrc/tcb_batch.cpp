// tcb_batch.cpp — batched form of the v2 encoder: N independent streams
// (any mix of resolutions, QPs, presets) advance one frame per call and
// share one CTU-engine launch per call: a persistent kernel drains a queue
// holding every participating stream's CTUs in anti-diagonal order, so a
// 1080p stream's at most 9 CTUs per diagonal are joined by everyone else's
// and the 148 SMs fill up.  Per-stream entropy coding runs on host
// threads in parallel; all device work is ordered on the batch's CUDA
// stream, optionally replayed as a CUDA graph, and optionally pipelined
// (each call entropy-codes the previous call's frames during its own
// device step).
#include <string.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec_b200.h"
#include "tcb_batch.h"
#include "tcb_encoder.h"
#include "tcb_launch.h"

using namespace tcb;

struct tcb_batch {
    std::vector<tc_encoder_t *> encs;        // slot -> stream (NULL: free slot)
    cudaStream_t st = nullptr;
    FrameParams *d_params = nullptr;         // [n] contiguous for the kernel
    int *d_items = nullptr;
    int *d_ctrl = nullptr;
    int num_sms = 148;
    size_t items_cap = 0;
    std::vector<int> h_items;
    std::vector<std::vector<std::vector<int>>> stream_diag;   // [s][d] item words
    int max_diag = 0;
    bool timing = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double ctu_ms = 0.0;
    long long ctu_launches = 0, ctu_count = 0, steps = 0, kernel_launches = 0;
    double host_plan_ms = 0.0, host_wait_ms = 0.0, host_entropy_ms = 0.0;   // wall-clock split of steps
    int device = 0;
    int *h_items_pin = nullptr;              // pinned staging of h_items (the upload is capturable)
    size_t h_items_pin_cap = 0;
    // CUDA-graph replay of the step's device work: executable graphs keyed
    // by the captured node sequence (P and B steps differ in topology).
    bool graphs = false;
    // Pipelined steps (tcb_batch_set_pipelined): the streams whose frames
    // await entropy coding from the previous step.
    bool pipelined = false;
    std::vector<int> prev_part;
    struct GraphSlot {
        uint64_t sig;
        cudaGraph_t tmpl;                    // the graph exec was instantiated from
        cudaGraphExec_t exec;
        std::vector<cudaGraphNode_t> nodes;  // tmpl's nodes, in cudaGraphGetNodes order
    };
    std::vector<GraphSlot> gcache;
    long long graph_launches = 0, graph_builds = 0;
    int graph_update_fail = 0;               // 1000 * (node type + 1) + position of the last refused node
};

namespace {

void release(tcb_batch *b) {
    if (b->st) cudaStreamSynchronize(b->st);
    for (tc_encoder_t *e : b->encs) {
        if (e && e->impl) e->impl->st = e->impl->own_st;
        if (e) tc_encoder_destroy(e);
    }
    for (auto &g : b->gcache) {
        cudaGraphExecDestroy(g.exec);
        cudaGraphDestroy(g.tmpl);
    }
    cudaFree(b->d_params);
    cudaFree(b->d_items);
    cudaFree(b->d_ctrl);
    cudaFreeHost(b->h_items_pin);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

std::vector<cudaGraphNode_t> graph_nodes(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return {};
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return {};
    return nodes;
}

// FNV-1a over the node types and kernel functions of a captured graph.
uint64_t graph_signature(const std::vector<cudaGraphNode_t> &nodes) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
    mix(nodes.size());
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) return 0;
        mix((uint64_t)t);
        if (t == cudaGraphNodeTypeKernel) {
            cudaKernelNodeParams kp;
            if (cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess) return 0;
            mix((uint64_t)(uintptr_t)kp.func);
        }
    }
    return h;
}

// Copy every node's parameters from a new capture of the same shape into
// the executable graph (node i of the capture onto node i of the
// template).  Returns 0, or 1000 * (node type + 1) + i for the first node
// the runtime refused.
int update_exec(tcb_batch::GraphSlot &slot, const std::vector<cudaGraphNode_t> &nodes) {
    if (nodes.size() != slot.nodes.size()) return 1;
    for (size_t i = 0; i < nodes.size(); ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) != cudaSuccess) return 2;
        cudaError_t e = cudaErrorNotSupported;
        if (t == cudaGraphNodeTypeKernel) {
            cudaKernelNodeParams p;
            e = cudaGraphKernelNodeGetParams(nodes[i], &p);
            if (e == cudaSuccess) e = cudaGraphExecKernelNodeSetParams(slot.exec, slot.nodes[i], &p);
        } else if (t == cudaGraphNodeTypeMemcpy) {
            cudaMemcpy3DParms p;
            e = cudaGraphMemcpyNodeGetParams(nodes[i], &p);
            if (e == cudaSuccess) e = cudaGraphExecMemcpyNodeSetParams(slot.exec, slot.nodes[i], &p);
        } else if (t == cudaGraphNodeTypeMemset) {
            cudaMemsetParams p;
            e = cudaGraphMemsetNodeGetParams(nodes[i], &p);
            if (e == cudaSuccess) e = cudaGraphExecMemsetNodeSetParams(slot.exec, slot.nodes[i], &p);
        } else if (t == cudaGraphNodeTypeEventRecord) {
            cudaEvent_t ev;
            e = cudaGraphEventRecordNodeGetEvent(nodes[i], &ev);
            if (e == cudaSuccess) e = cudaGraphExecEventRecordNodeSetEvent(slot.exec, slot.nodes[i], ev);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            return 1000 * ((int)t + 1) + (int)i;
        }
    }
    return 0;
}

// Launch a captured step: update the cached executable graph of the same
// shape in place (new pointers and sizes), or instantiate one.  Takes
// ownership of g.
tc_error_t launch_graph(tcb_batch *b, cudaGraph_t g) {
    const std::vector<cudaGraphNode_t> nodes = graph_nodes(g);
    const uint64_t sig = graph_signature(nodes);
    tcb_batch::GraphSlot *hit = nullptr;
    for (auto &slot : b->gcache)
        if (slot.sig == sig) { hit = &slot; break; }
    if (hit) {
        const int r = update_exec(*hit, nodes);
        if (r == 0) {
            cudaGraphDestroy(g);
        } else {                                   // refused: rebuild this shape's executable graph
            b->graph_update_fail = r;
            cudaGraphExecDestroy(hit->exec);
            cudaGraphDestroy(hit->tmpl);
            hit->tmpl = g;
            hit->nodes = nodes;
            hit->exec = nullptr;
            if (cudaGraphInstantiate(&hit->exec, g, 0) != cudaSuccess) return TC_ERR_INTERNAL;
            ++b->graph_builds;
        }
    } else {
        if (b->gcache.size() >= 8) {              // bounded cache: drop the oldest shape
            cudaGraphExecDestroy(b->gcache.front().exec);
            cudaGraphDestroy(b->gcache.front().tmpl);
            b->gcache.erase(b->gcache.begin());
        }
        cudaGraphExec_t exec = nullptr;
        if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            return TC_ERR_INTERNAL;
        }
        ++b->graph_builds;
        b->gcache.push_back({sig, g, exec, nodes});
        hit = &b->gcache.back();
    }
    if (cudaGraphLaunch(hit->exec, b->st) != cudaSuccess) return TC_ERR_INTERNAL;
    ++b->graph_launches;
    return TC_OK;
}

// Device work of one step (parameter uploads, global-motion walks, work
// queue, CTU engine, copy-back), enqueued on the batch stream.  Host
// sources are pinned, so the whole sequence can be captured.
tc_error_t enqueue_step(tcb_batch *b, const std::vector<int> &part, const std::vector<int> &off,
                        const std::vector<int> &cnt) {
    for (int s : part) {
        EncImpl &e = *b->encs[s]->impl;
        const tc_error_t r = e.stage_b();
        if (r != TC_OK) return r;
        if (cudaMemcpyAsync(b->d_params + s, e.d_params, sizeof(FrameParams), cudaMemcpyDeviceToDevice, b->st) !=
            cudaSuccess)
            return TC_ERR_INTERNAL;
    }
    // Global-motion walks of all P streams, one CTA each, written into the
    // batch's parameter copies.
    std::vector<GlobJob> jobs;
    for (int s : part) {
        EncImpl &e = *b->encs[s]->impl;
        if (e.pend.glob) jobs.push_back({e.cur.y, e.pend.glob_ref, e.W, e.H, e.sy, b->d_params + s});
    }
    if (!jobs.empty()) {
        if (launch_glob_mv_multi(jobs.data(), (int)jobs.size(), b->st) != cudaSuccess) return TC_ERR_INTERNAL;
        b->kernel_launches += ((int)jobs.size() + GlobJobs::MAX - 1) / GlobJobs::MAX;
    }
    if (cudaMemcpyAsync(b->d_items, b->h_items_pin, sizeof(int) * b->h_items.size(), cudaMemcpyHostToDevice,
                        b->st) != cudaSuccess)
        return TC_ERR_INTERNAL;
    // One persistent launch drains the merged queue (per-stream publish
    // flags keep every stream's wavefront order).  Inside a captured graph
    // the timing events become external event-record nodes.
    const unsigned evf = b->graphs ? cudaEventRecordExternal : cudaEventRecordDefault;
    if (b->timing && cudaEventRecordWithFlags(b->ev0, b->st, evf) != cudaSuccess) return TC_ERR_INTERNAL;
    const bool persistent = b->encs[part[0]]->impl->persistent;
    if (persistent) {
        if (cudaMemsetAsync(b->d_ctrl, 0, 2 * sizeof(int), b->st) != cudaSuccess ||
            launch_ctu_persistent(b->d_params, b->d_items, (int)b->h_items.size(), b->d_ctrl, b->num_sms, b->st) !=
                cudaSuccess)
            return TC_ERR_INTERNAL;
        b->kernel_launches += 1;
    } else {
        for (size_t d = 0; d < off.size(); ++d)
            if (cnt[d] && launch_ctu_items(b->d_params, b->d_items + off[d], cnt[d], b->st) != cudaSuccess)
                return TC_ERR_INTERNAL;
        for (size_t d = 0; d < off.size(); ++d) b->kernel_launches += cnt[d] ? 1 : 0;
    }
    if (b->timing && cudaEventRecordWithFlags(b->ev1, b->st, evf) != cudaSuccess) return TC_ERR_INTERNAL;
    for (int s : part) {
        // Host reconstruction copies are 2D copies of padded planes, which
        // an executable graph cannot take new addresses for: in graph mode
        // they follow the graph launch as ordinary stream copies.
        const tc_error_t r = b->encs[s]->impl->stage_c(!b->graphs);
        if (r != TC_OK) return r;
        // the queue's error word is the batch's
        if (persistent && cudaMemcpyAsync(b->encs[s]->impl->h_ctrl, b->d_ctrl, 2 * sizeof(int),
                                          cudaMemcpyDeviceToHost, b->st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    }
    return TC_OK;
}

// Entropy coding of the committed frames of `part`, one host thread per
// stream; status[s] is the stream's result.
tc_error_t entropy_code(tcb_batch *b, const std::vector<int> &part, tc_packet_t *pkts, int *status) {
    const int n = (int)b->encs.size();
    std::vector<std::thread> th;
    std::vector<tc_error_t> rs(n, TC_OK);
    for (int s : part)
        th.emplace_back([&, s]() { rs[s] = b->encs[s]->impl->stage_d(&pkts[s]); });
    for (auto &t : th) t.join();
    tc_error_t worst = TC_OK;
    for (int s : part) {
        status[s] = rs[s];
        if (rs[s] != TC_OK) worst = rs[s];
    }
    return worst;
}

// Run stage_a..stage_d for the streams whose plan produced a frame (in a
// pipelined batch, stage_d of the previous step's frames).
tc_error_t run_step(tcb_batch *b, const std::vector<int> &part, tc_packet_t *pkts, int *status) {
    auto t0 = std::chrono::steady_clock::now();
    for (int s : part) {
        EncImpl &e = *b->encs[s]->impl;
        const tc_error_t r = e.stage_a(e.pend.poc, e.pend.qp_off);
        if (r != TC_OK) return r;
    }
    bool need_sync = false;
    for (int s : part) need_sync |= b->encs[s]->impl->pend.need_hist != 0;
    if (need_sync && cudaStreamSynchronize(b->st) != cudaSuccess) return TC_ERR_INTERNAL;
    // Merged anti-diagonal item lists of the participating streams (the
    // queue order), staged in pinned memory.  Merged slot m holds diagonal
    // m - lag of every stream, where lag is 0 (TCB_QUEUE_DIAGONAL) or the
    // stream's rank in the step (TCB_QUEUE_STAGGERED), as tuned for the
    // step's largest frame size.  Either way each stream's diagonals stay in
    // order and one slot never holds two CTUs of one stream, so every CTU's
    // neighbours come earlier in the queue (the persistent wavefront's
    // condition) and a slot's CTUs are independent.
    int big = part[0];
    for (int s : part) {
        const EncImpl &e = *b->encs[s]->impl, &eb = *b->encs[big]->impl;
        if ((long long)e.W * e.H > (long long)eb.W * eb.H) big = s;
    }
    const bool stagger =
        engine_tuning(b->encs[big]->impl->W, b->encs[big]->impl->H).queue_order == TCB_QUEUE_STAGGERED;
    int nslots = 0;
    for (size_t r = 0; r < part.size(); ++r)
        nslots = std::max(nslots, (stagger ? (int)r : 0) + (int)b->stream_diag[part[r]].size());
    std::vector<int> off(nslots), cnt(nslots);
    b->h_items.clear();
    for (int m = 0; m < nslots; ++m) {
        off[m] = (int)b->h_items.size();
        for (size_t r = 0; r < part.size(); ++r) {
            const auto &sd = b->stream_diag[part[r]];
            const int d = m - (stagger ? (int)r : 0);
            if (d >= 0 && d < (int)sd.size()) b->h_items.insert(b->h_items.end(), sd[d].begin(), sd[d].end());
        }
        cnt[m] = (int)b->h_items.size() - off[m];
    }
    if (b->h_items.size() > b->items_cap) {
        cudaFree(b->d_items);
        b->d_items = nullptr;
        b->items_cap = 0;
        if (tcb::dev_alloc(&b->d_items, sizeof(int) * b->h_items.size()) != cudaSuccess) return TC_ERR_MEMORY;
        b->items_cap = b->h_items.size();
    }
    if (b->h_items.size() > b->h_items_pin_cap) {
        cudaFreeHost(b->h_items_pin);
        b->h_items_pin = nullptr;
        b->h_items_pin_cap = 0;
        if (tcb::pinned_alloc(&b->h_items_pin, sizeof(int) * b->h_items.size()) != cudaSuccess) return TC_ERR_MEMORY;
        b->h_items_pin_cap = b->h_items.size();
    }
    memcpy(b->h_items_pin, b->h_items.data(), sizeof(int) * b->h_items.size());
    if (b->graphs) {
        if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return TC_ERR_INTERNAL;
        const tc_error_t r = enqueue_step(b, part, off, cnt);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->st, &g);   // ends the capture on every path
        if (r != TC_OK || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return r != TC_OK ? r : TC_ERR_INTERNAL;
        }
        const tc_error_t lr = launch_graph(b, g);
        if (lr != TC_OK) return lr;
        for (int s : part) {
            const tc_error_t rr = b->encs[s]->impl->readback_recon();
            if (rr != TC_OK) return rr;
        }
    } else {
        const tc_error_t r = enqueue_step(b, part, off, cnt);
        if (r != TC_OK) return r;
    }
    const bool persistent = b->encs[part[0]]->impl->persistent;
    if (b->timing) { b->host_plan_ms += ms_since(t0); t0 = std::chrono::steady_clock::now(); }
    tc_error_t worst = TC_OK;
    // Pipelined: the previous step's frames are entropy coded now, while this
    // step runs on the device; their packets are this call's result.
    if (b->pipelined && !b->prev_part.empty()) {
        const tc_error_t r = entropy_code(b, b->prev_part, pkts, status);
        if (r != TC_OK) worst = r;
        if (b->timing) { b->host_entropy_ms += ms_since(t0); t0 = std::chrono::steady_clock::now(); }
    }
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return TC_ERR_INTERNAL;
    if (b->timing) { b->host_wait_ms += ms_since(t0); t0 = std::chrono::steady_clock::now(); }
    if (b->timing) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        b->ctu_ms += ms;
        b->ctu_launches += persistent ? 1 : b->max_diag;
        b->steps++;
        b->ctu_count += (long long)b->h_items.size();
    }
    for (int s : part) {
        const tc_error_t r = b->encs[s]->impl->commit_frame();
        if (r != TC_OK) { status[s] = r; return r; }
        b->kernel_launches += b->encs[s]->impl->kernel_launches;
        b->encs[s]->impl->kernel_launches = 0;
    }
    if (b->pipelined) {
        b->prev_part = part;
        return worst;
    }
    const tc_error_t r = entropy_code(b, part, pkts, status);
    if (b->timing) b->host_entropy_ms += ms_since(t0);
    return r;
}

// A call without a device step: a pipelined batch codes the frames still
// awaiting entropy coding and returns their packets (TC_OK); otherwise
// `none` (TC_OK from encode, TC_ERR_EOF from flush).
tc_error_t drain(tcb_batch *b, tc_packet_t *pkts, int *status, tc_error_t none) {
    if (b->prev_part.empty()) return none;
    const std::vector<int> part = b->prev_part;
    b->prev_part.clear();
    return entropy_code(b, part, pkts, status);
}

}  // namespace

tcb_batch *tcb::batch_new(int cap) {
    if (cap <= 0 || cap > MAX_STREAMS) return nullptr;
    tcb_batch *b = new (std::nothrow) tcb_batch();
    if (!b) return nullptr;
    if (cudaGetDevice(&b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        tcb::dev_alloc(&b->d_params, sizeof(FrameParams) * cap) != cudaSuccess ||
        tcb::dev_alloc(&b->d_ctrl, 2 * sizeof(int)) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess) {
        release(b);
        return nullptr;
    }
    b->encs.assign(cap, nullptr);
    b->stream_diag.assign(cap, {});
    return b;
}

int tcb::batch_attach(tcb_batch *b, tc_encoder_t *e) {
    int s = 0;
    while (s < (int)b->encs.size() && b->encs[s]) ++s;
    if (s == (int)b->encs.size()) return -1;
    b->encs[s] = e;
    EncImpl &im = *e->impl;
    im.st = b->st;                          // all device work on the batch stream
    im.defer_glob = true;
    im.entropy_threads = 1;                 // the batch codes its streams in parallel
    std::vector<std::vector<int>> diags(im.diag_off.size());
    for (int d = 0; d < (int)im.diag_off.size(); ++d)
        for (int r = 0; r < im.ctu_rows; ++r) {
            const int c = d - r;
            if (c >= 0 && c < im.ctu_cols) diags[d].push_back((s << 20) | (r << 10) | c);
        }
    b->stream_diag[s] = std::move(diags);
    b->max_diag = 0;
    for (auto &sd : b->stream_diag) b->max_diag = std::max(b->max_diag, (int)sd.size());
    return s;
}

void tcb::batch_detach(tcb_batch *b, int s) {
    if (s < 0 || s >= (int)b->encs.size() || !b->encs[s]) return;
    cudaStreamSynchronize(b->st);
    tc_encoder_t *e = b->encs[s];
    e->impl->st = e->impl->own_st;
    tc_encoder_destroy(e);
    b->encs[s] = nullptr;
    b->stream_diag[s].clear();
    b->max_diag = 0;
    for (auto &sd : b->stream_diag) b->max_diag = std::max(b->max_diag, (int)sd.size());
}

tc_encoder_t *tcb::batch_slot(tcb_batch *b, int s) {
    return (s >= 0 && s < (int)b->encs.size()) ? b->encs[s] : nullptr;
}

cudaStream_t tcb::batch_stream(tcb_batch *b) { return b->st; }

void tcb::batch_set_graphs(tcb_batch *b, bool on) {
    if (b) b->graphs = on;
}

tc_error_t tcb::batch_run(tcb_batch *b, const std::vector<int> &part, tc_packet_t *pkts, int *status) {
    if (part.empty()) return TC_OK;
    if (cudaSetDevice(b->device) != cudaSuccess) return TC_ERR_INTERNAL;
    return run_step(b, part, pkts, status);
}

void tcb::batch_free(tcb_batch *b) { if (b) release(b); }

extern "C" {

tcb_batch_t *tcb_batch_create(const tc_config_t *configs, int n) {
    if (!configs || n <= 0 || n > MAX_STREAMS) return nullptr;
    tcb_batch *b = batch_new(n);
    if (!b) return nullptr;
    for (int s = 0; s < n; ++s)
        if (!configs[s].use_v2) { release(b); return nullptr; }   // batches run the v2 CTU engine
    for (int s = 0; s < n; ++s) {
        tc_encoder_t *e = tc_encoder_create(&configs[s]);
        if (!e || batch_attach(b, e) != s) {
            if (e) tc_encoder_destroy(e);
            release(b);
            return nullptr;
        }
    }
    return b;
}

void tcb_batch_destroy(tcb_batch_t *b) {
    if (b) release(b);
}

int tcb_batch_size(tcb_batch_t *b) { return b ? (int)b->encs.size() : 0; }

tc_encoder_t *tcb_batch_encoder(tcb_batch_t *b, int i) {
    return (b && i >= 0 && i < (int)b->encs.size()) ? b->encs[i] : nullptr;
}

void *tcb_batch_stream(tcb_batch_t *b) { return b ? (void *)b->st : nullptr; }

tc_error_t tcb_batch_encode(tcb_batch_t *b, const tc_pixel_t *const *y, const int *stride_y,
                            const tc_pixel_t *const *cb, const int *stride_cb, const tc_pixel_t *const *cr,
                            const int *stride_cr, int on_device, tc_packet_t *packets, int *status) {
    if (!b || !y || !cb || !cr || !stride_y || !stride_cb || !stride_cr || !packets || !status) return TC_ERR_PARAM;
    if (cudaSetDevice(b->device) != cudaSuccess) return TC_ERR_INTERNAL;
    const int n = (int)b->encs.size();
    std::vector<int> part;
    for (int s = 0; s < n; ++s) {
        status[s] = TC_ERR_NEED_MORE;
        memset(&packets[s], 0, sizeof(tc_packet_t));
        if (!y[s] || !cb[s] || !cr[s]) continue;
        EncImpl &e = *b->encs[s]->impl;
        if (!e.upload(y[s], stride_y[s], cb[s], stride_cb[s], cr[s], stride_cr[s], e.cur,
                      on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice))
            return TC_ERR_INTERNAL;
        const tc_error_t r = e.plan_input();
        if (r == TC_OK) part.push_back(s);
        else if (r != TC_ERR_NEED_MORE) { status[s] = r; return r; }
    }
    if (part.empty()) return drain(b, packets, status, TC_OK);
    return run_step(b, part, packets, status);
}

tc_error_t tcb_batch_flush(tcb_batch_t *b, tc_packet_t *packets, int *status) {
    if (!b || !packets || !status) return TC_ERR_PARAM;
    if (cudaSetDevice(b->device) != cudaSuccess) return TC_ERR_INTERNAL;
    const int n = (int)b->encs.size();
    std::vector<int> part;
    for (int s = 0; s < n; ++s) {
        status[s] = TC_ERR_EOF;
        memset(&packets[s], 0, sizeof(tc_packet_t));
        const tc_error_t r = b->encs[s]->impl->plan_flush();
        if (r == TC_OK) part.push_back(s);
        else if (r != TC_ERR_EOF) { status[s] = r; return r; }
    }
    if (part.empty()) return drain(b, packets, status, TC_ERR_EOF);
    return run_step(b, part, packets, status);
}

tc_error_t tcb_batch_drain(tcb_batch_t *b, tc_packet_t *packets, int *status) {
    if (!b || !packets || !status) return TC_ERR_PARAM;
    for (size_t s = 0; s < b->encs.size(); ++s) {
        status[s] = TC_ERR_NEED_MORE;
        memset(&packets[s], 0, sizeof(tc_packet_t));
    }
    return drain(b, packets, status, TC_ERR_EOF);
}

tc_error_t tcb_batch_set_pipelined(tcb_batch_t *b, int enabled) {
    if (!b) return TC_ERR_PARAM;
    if (!b->prev_part.empty()) return TC_ERR_PARAM;   // frames still await entropy coding
    for (tc_encoder_t *e : b->encs)
        if (e && !e->impl->set_pipelined(enabled != 0)) {
            for (tc_encoder_t *f : b->encs)
                if (f) f->impl->set_pipelined(false);
            b->pipelined = false;
            return TC_ERR_PARAM;
        }
    b->pipelined = enabled != 0;
    return TC_OK;
}

void tcb_batch_set_timing(tcb_batch_t *b, int enabled) {
    if (b) b->timing = enabled != 0;
}

void tcb_batch_set_graphs(tcb_batch_t *b, int enabled) { tcb::batch_set_graphs(b, enabled != 0); }

int tcb_batch_get_graph_stats(tcb_batch_t *b, int64_t *graph_launches, int64_t *graph_builds) {
    if (!b) return 0;
    if (graph_launches) *graph_launches = b->graph_launches;
    if (graph_builds) *graph_builds = b->graph_builds;
    const int r = b->graph_update_fail;
    b->graph_launches = b->graph_builds = 0;
    b->graph_update_fail = 0;
    return r;
}

void tcb_batch_get_host_timing(tcb_batch_t *b, double *plan_ms, double *wait_ms, double *entropy_ms) {
    if (!b) return;
    if (plan_ms) *plan_ms = b->host_plan_ms;
    if (wait_ms) *wait_ms = b->host_wait_ms;
    if (entropy_ms) *entropy_ms = b->host_entropy_ms;
    b->host_plan_ms = b->host_wait_ms = b->host_entropy_ms = 0.0;
}

void tcb_batch_get_timing(tcb_batch_t *b, double *ctu_ms, int64_t *ctu_launches, int64_t *ctu_count,
                          int64_t *steps, int64_t *kernel_launches) {
    if (!b) return;
    if (ctu_ms) *ctu_ms = b->ctu_ms;
    if (ctu_launches) *ctu_launches = b->ctu_launches;
    if (ctu_count) *ctu_count = b->ctu_count;
    if (steps) *steps = b->steps;
    if (kernel_launches) *kernel_launches = b->kernel_launches;
    b->ctu_ms = 0.0; b->ctu_launches = 0; b->ctu_count = 0; b->steps = 0; b->kernel_launches = 0;
}

}  // extern "C"
