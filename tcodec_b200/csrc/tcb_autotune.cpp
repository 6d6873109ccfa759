// tcb_autotune.cpp — autotuner of the frame kernels' tile shape.
//
// The standalone frame kernels (deblocking, SAO, motion compensation) come
// in several CTA sizes.  Which is fastest depends on the frame size (how
// many CTAs a launch has against the 148 SMs) and on the kernel's balance
// of shared-memory, register and issue limits, so it is measured rather
// than fixed: tcb_autotune_frame_kernels times every variant on scratch
// frames of the size asked for and records the fastest in a process-wide
// table that the kernels' C entry points consult on every call.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec_b200.h"
#include "tcb_encoder.h"
#include "tcb_filters.h"

namespace tcb {

namespace {

std::mutex g_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;   // (kernel, width, height) -> threads per CTA

__global__ void fill_bytes(uint8_t *p, size_t n, uint32_t seed) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)i * 2654435761u ^ seed;
        x ^= x >> 15; x *= 2246822519u; x ^= x >> 13;
        p[i] = (uint8_t)(x >> 24);
    }
}

// Quarter-sample vectors within +-24 samples (random), or one fractional
// vector (+2.5, +0.75) samples for every block (coherent motion, where
// blocks of a warp share their phase).  The two load the MC kernel
// differently, so the scratch frames alternate between them.
__global__ void fill_mv(int16_t *mv, int n, uint32_t seed, int coherent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)i * 2654435761u ^ seed;
        x ^= x >> 15; x *= 2246822519u; x ^= x >> 13;
        mv[i] = coherent ? (int16_t)((i & 1) ? 3 : 10) : (int16_t)((int)(x % 193u) - 96);
    }
}

struct Scratch {
    std::vector<void *> bufs;
    ~Scratch() {
        for (void *p : bufs) cudaFree(p);
    }
    template <class T>
    T *alloc(size_t n) {
        void *p = nullptr;
        if (dev_alloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
        bufs.push_back(p);
        return (T *)p;
    }
};

// Median over `reps` samples of the time of `inner` back-to-back calls of
// fn, after one warm-up call.  A single call of a 32-frame launch lasts
// about 50 us, too short against event-timing noise to separate variants
// that differ by 10 %; several calls per sample are not.
template <class F>
float time_ms(F fn, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, int reps, int inner, bool *ok) {
    std::vector<float> t;
    if (fn() != cudaSuccess) { *ok = false; return 0.f; }
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0, st);
        for (int i = 0; i < inner; ++i)
            if (fn() != cudaSuccess) { *ok = false; return 0.f; }
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) { *ok = false; return 0.f; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        t.push_back(ms);
    }
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

}  // namespace

int tuned_threads(int kernel, int width, int height) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_tuned.find({kernel, width, height});
    return it == g_tuned.end() ? 0 : it->second;
}

void set_tuned_threads(int kernel, int width, int height, int threads) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (threads) g_tuned[{kernel, width, height}] = threads;
    else g_tuned.erase({kernel, width, height});
}

// Engine knobs per frame size (tcb_engine_set_tuning): neither changes any
// output, only the time a step takes.
namespace {
std::map<std::pair<int, int>, EngineTuning> g_engine;
}

EngineTuning engine_tuning(int width, int height) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_engine.find({width, height});
    return it == g_engine.end() ? EngineTuning{} : it->second;
}

void set_engine_tuning(int width, int height, const EngineTuning *t) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (t) g_engine[{width, height}] = *t;
    else g_engine.erase({width, height});
}

}  // namespace tcb

extern "C" {

tc_error_t tcb_autotune_frame_kernels(int width, int height, int frames) {
    using namespace tcb;
    if (width <= 0 || height <= 0 || (width & 1) || (height & 1) || width > TC_MAX_WIDTH ||
        height > TC_MAX_HEIGHT || frames < 1 || frames > 32)
        return TC_ERR_PARAM;
    const int sy = (width + 63) & ~63, sc = ((width / 2) + 63) & ~63, hc = height / 2;
    const int gw = (width + 7) >> 3, gh = (height + 7) >> 3;
    const int nctu = ((width + 63) >> 6) * ((height + 63) >> 6);
    Scratch S;
    std::vector<DeblockFrame> db(frames);
    std::vector<SaoFrame> sao(frames);
    std::vector<tcb_mc_frame_t> mc(frames);
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return TC_ERR_INTERNAL;
    tc_error_t r = TC_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) r = TC_ERR_INTERNAL;
    for (int f = 0; f < frames && r == TC_OK; ++f) {
        uint8_t *y = S.alloc<uint8_t>((size_t)sy * height), *cb = S.alloc<uint8_t>((size_t)sc * hc),
                *cr = S.alloc<uint8_t>((size_t)sc * hc), *src = S.alloc<uint8_t>((size_t)sy * height),
                *py = S.alloc<uint8_t>((size_t)sy * height), *pcb = S.alloc<uint8_t>((size_t)sc * hc),
                *pcr = S.alloc<uint8_t>((size_t)sc * hc);
        int16_t *mv = S.alloc<int16_t>((size_t)gw * gh * 2), *params = S.alloc<int16_t>((size_t)nctu * 3);
        if (!y || !cb || !cr || !src || !py || !pcb || !pcr || !mv || !params) { r = TC_ERR_MEMORY; break; }
        fill_bytes<<<256, 256, 0, st>>>(y, (size_t)sy * height, 17u * f + 1);
        fill_bytes<<<256, 256, 0, st>>>(cb, (size_t)sc * hc, 17u * f + 2);
        fill_bytes<<<256, 256, 0, st>>>(cr, (size_t)sc * hc, 17u * f + 3);
        fill_bytes<<<256, 256, 0, st>>>(src, (size_t)sy * height, 17u * f + 4);
        fill_mv<<<64, 256, 0, st>>>(mv, gw * gh * 2, 17u * f + 5, f & 1);
        db[f] = {y, cb, cr, width, height, sy, sc, 32};
        sao[f] = {y, src, width, height, sy, sy, (int)tc_lambda_host(32), params};
        mc[f].width = width; mc[f].height = height; mc[f].stride_y = sy; mc[f].stride_c = sc;
        mc[f].ref_y = y; mc[f].ref_cb = cb; mc[f].ref_cr = cr;
        mc[f].pred_y = py; mc[f].pred_cb = pcb; mc[f].pred_cr = pcr;
        mc[f].mv = mv;
    }
    if (r == TC_OK && cudaStreamSynchronize(st) != cudaSuccess) r = TC_ERR_INTERNAL;
    if (r == TC_OK) {
        // Deblocking and SAO filter the scratch planes in place on every
        // call; the content stays random, which is what is timed.
        struct Variant { int kernel; std::vector<int> threads; };
        const int T = TCB_STAGING_TMA;
        const Variant vs[3] = {{TCB_KERNEL_DEBLOCK, {64, 128, 256, 64 | T, 128 | T, 256 | T}},
                               {TCB_KERNEL_SAO, {64, 128}}, {TCB_KERNEL_MC, {64, 128, 256}}};
        for (const Variant &v : vs) {
            int best = 0;
            float best_ms = 0.f;
            for (int th : v.threads) {
                bool ok = true;
                const float ms = time_ms(
                    [&]() {
                        if (v.kernel == TCB_KERNEL_DEBLOCK) return launch_deblock_frames(db.data(), frames, st, th);
                        if (v.kernel == TCB_KERNEL_SAO) return launch_sao_frames(sao.data(), frames, st, th);
                        return launch_mc_frames(mc.data(), frames, st, th);
                    },
                    st, e0, e1, 7, 4, &ok);
                if (!ok) { r = TC_ERR_INTERNAL; break; }
                if (!best || ms < best_ms) { best = th; best_ms = ms; }
            }
            if (r != TC_OK) break;
            set_tuned_threads(v.kernel, width, height, best);
        }
    }
    cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    return r;
}

int tcb_autotune_threads(int kernel, int width, int height) { return tcb::tuned_threads(kernel, width, height); }

tc_error_t tcb_autotune_set_threads(int kernel, int width, int height, int threads) {
    const int th = kernel == TCB_KERNEL_DEBLOCK ? (threads & ~TCB_STAGING_TMA) : threads;
    const bool ok = threads == 0 || th == 128 || th == 64 ||
                    (th == 256 && (kernel == TCB_KERNEL_DEBLOCK || kernel == TCB_KERNEL_MC));
    if (kernel < TCB_KERNEL_DEBLOCK || kernel > TCB_KERNEL_MC || width <= 0 || height <= 0 || !ok)
        return TC_ERR_PARAM;
    tcb::set_tuned_threads(kernel, width, height, threads);
    return TC_OK;
}

tc_error_t tcb_engine_set_tuning(int width, int height, int search_window, int queue_order) {
    if (width <= 0 || height <= 0) return TC_ERR_PARAM;
    if (search_window == 0 && queue_order == 0) {        // back to the defaults
        tcb::set_engine_tuning(width, height, nullptr);
        return TC_OK;
    }
    if (search_window < TCB_SEARCH_WINDOW_MIN || search_window > TCB_SEARCH_WINDOW_MAX ||
        (queue_order != TCB_QUEUE_DIAGONAL && queue_order != TCB_QUEUE_STAGGERED))
        return TC_ERR_PARAM;
    const tcb::EngineTuning t{search_window, queue_order};
    tcb::set_engine_tuning(width, height, &t);
    return TC_OK;
}

tc_error_t tcb_engine_get_tuning(int width, int height, int *search_window, int *queue_order) {
    if (width <= 0 || height <= 0 || !search_window || !queue_order) return TC_ERR_PARAM;
    const tcb::EngineTuning t = tcb::engine_tuning(width, height);
    *search_window = t.search_window;
    *queue_order = t.queue_order;
    return TC_OK;
}

unsigned int tcb_frame_kernels_errors(void) {
    cudaDeviceSynchronize();
    return tcb::tma_waits_expired();
}

}  // extern "C"
