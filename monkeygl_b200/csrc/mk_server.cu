// mk_server.cu -- continuous batching of ray-casting and reslice requests
// over several resident volumes on one device.
//
// No counterpart in MonkeyGL: its demo server (server.py) renders one request
// at a time through a process-wide singleton that holds one volume
// (core/DataManager.cpp:46-54).  Here:
//
//  * Volumes are mk_volume handles admitted against an HBM budget that also
//    covers the fixed per-slot buffers; a volume that does not fit is refused.
//  * A request takes a slot: its LUTs go to the slot's 1D float4 texture
//    arrays (same filtering as mk_volume_set_transfer_function), its label
//    parameters and kernel parameters to the slot's descriptor, and the
//    brick visibility / MIP bounds of its volume under its tables are built
//    into the slot's maps -- the same kernel and inputs mk_render_vr uses, so
//    the image equals mk_render_vr's for the same request.
//  * Every step, the worker thread lists up to tiles_per_step 32x8 tiles of
//    the requests in flight (admission order), copies the list to a device
//    queue and launches a CUDA graph holding one persistent kernel: one block
//    per resident slot of the device, each pulling tiles with an atomic
//    counter until the list is exhausted (no waiting on other blocks or on
//    the host).  A request spans steps when it has more tiles than a step
//    takes; requests admitted meanwhile join the next step.  Steps alternate
//    between two streams, so the next step's tiles fill the tail of the one
//    before (a step ends with its slowest tile); up to four are in flight.
//    Finished images go back on a copy stream behind the steps that hold
//    their tiles.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "host_encode.h"
#include "mk_internal.h"
#include "mk_math.h"
#include "mk_raycast_impl.cuh"
#include "mk_reslice_impl.cuh"

namespace mk {

// Device descriptor of the request held by a slot.
struct SlotDesc {
    int kind;                    // 0 ray casting, 1 plane
    int mode;                    // RayMode, or mk_mpr_type
    int track;                   // Track (ray casting)
    int pad;
    RayParams rp;
    PlaneParams pp;
    cudaTextureObject_t vol, mask, plane_tex;
    LabelTable lt;
    BrickView bv;
    void *out;
};

struct TileItem {
    unsigned short slot, tx, ty, pad;
};

// queue layout: int count, int pad, TileItem items[count]
__global__ void __launch_bounds__(256, 3) k_serve(const SlotDesc *__restrict__ slots, const int *__restrict__ queue,
                                               int *__restrict__ next) {
    __shared__ LabelSmem S;
    __shared__ RayParams s_rp;
    __shared__ BrickView s_bv;
    __shared__ float s_acc[kMaxTrackedLabels][256];
    __shared__ CoopSample s_coop[256];
    __shared__ uint8_t s_px[8][32 * 3];
    __shared__ unsigned long long s_count;
    __shared__ int s_item, s_slot;
    const int tid = threadIdx.x;
    if (tid == 0) s_slot = -1;
    const int count = queue[0];
    const TileItem *items = reinterpret_cast<const TileItem *>(queue + 2);
    for (;;) {
        __syncthreads();                       // the previous tile is done with shared memory
        if (tid == 0) s_item = atomicAdd(next, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= count) break;
        const TileItem t = items[it];
        const SlotDesc &D = slots[t.slot];
        const int mode = D.mode;
        if (D.kind == 0) {
            const int track = D.track;
            if (s_slot != (int)t.slot) {       // uniform: shared value and tile item
                load_label_smem(S, D.lt, track);
                if (tid == 0) {
                    s_rp = D.rp;
                    s_bv = D.bv;
                    s_count = 0;
                }
                __syncthreads();
                if (tid == 0) s_slot = t.slot;
            }
            const cudaTextureObject_t vol = D.vol, mask = D.mask;
            if (mode == kModeVR) {
                if (track == kTrackNone)
                    raycast_tile<kModeVR, kTrackNone, false>(s_rp, vol, mask, S, s_bv, s_acc, s_coop, s_px, &s_count, t.tx, t.ty);
                else if (track == kTrackShared)
                    raycast_tile<kModeVR, kTrackShared, false>(s_rp, vol, mask, S, s_bv, s_acc, s_coop, s_px, &s_count, t.tx,
                                                               t.ty);
                else
                    raycast_tile<kModeVR, kTrackLocal, false>(s_rp, vol, mask, S, s_bv, s_acc, s_coop, s_px, &s_count, t.tx,
                                                              t.ty);
            } else if (mode == kModeMIP) {
                raycast_tile<kModeMIP, kTrackNone, false>(s_rp, vol, mask, S, s_bv, s_acc, s_coop, s_px, &s_count, t.tx, t.ty);
            } else {
                raycast_tile<kModeSurface, kTrackNone, false>(s_rp, vol, mask, S, s_bv, s_acc, s_coop, s_px, &s_count, t.tx,
                                                              t.ty);
            }
        } else {
            const PlaneParams P = D.pp;
            if (mode == MK_MPR_AVERAGE) plane_tile<MK_MPR_AVERAGE, false>(P, D.plane_tex, D.out, t.tx, t.ty);
            else if (mode == MK_MPR_MIP) plane_tile<MK_MPR_MIP, false>(P, D.plane_tex, D.out, t.tx, t.ty);
            else plane_tile<MK_MPR_MINIP, false>(P, D.plane_tex, D.out, t.tx, t.ty);
        }
    }
}

namespace {

using Clock = std::chrono::steady_clock;

struct Slot {
    cudaArray_t tf_array[MK_MAX_LABELS] = {};
    cudaTextureObject_t tf_tex[MK_MAX_LABELS] = {};
    float *d_alpha = nullptr;           // max_labels * lut_len alpha columns
    uint32_t *d_vis = nullptr;
    float *d_tmax = nullptr;
    void *d_out = nullptr;
    void *h_stage = nullptr;            // pinned output staging
    float *h_lut = nullptr;             // pinned LUT staging (max_labels * lut_len * 4)
    float *h_alpha = nullptr;           // pinned alpha staging (max_labels * lut_len)
    float *d_fy = nullptr;              // ray parameter table of the request (grown on demand)
    int fy_cap = 0;
    uint64_t ticket = 0;                // 0 = free
};

struct ServerVolume {
    mk_volume vol = nullptr;            // nullptr while evicted (or being uploaded)
    size_t bytes = 0;                   // device bytes while resident; evicted: those of its last upload (the estimate if none)
    int users = 0;                      // requests queued or in flight
    int in_slots = 0;                   // requests admitted into slots: they pin the volume
    bool loading = false;               // queued for, or in, an upload by the loader thread
    uint64_t last_use = 0;              // admission clock of the latest request
    int dims[3] = {0, 0, 0};
    // host copies for reloads (evict_idle only)
    std::shared_ptr<const std::vector<int16_t>> host_vox;
    std::shared_ptr<const std::vector<uint8_t>> host_lab;
};

struct Req {
    mk_request r;
    std::vector<float> luts, params;
    int slot = -1;
    int tiles_x = 0, tiles_total = 0, tiles_issued = 0;
    std::shared_ptr<const std::vector<int>> order;   // tile order (ray casting: centre first)
    size_t out_bytes = 0;
    bool direct = false;
    int enc_w = 0, enc_h = 0, enc_ch = 0;   // encoded form: PNG geometry (enc_ch 0: none)
    size_t enc_len = 0;
    bool done = false;
    int status = MK_OK;
    double t_submit = 0, t_start = -1, t_done = 0;
};

struct Step {
    cudaEvent_t kernel_done = nullptr, copies_done = nullptr;
    std::vector<uint64_t> finishing;
};

}  // namespace
}  // namespace mk

using namespace mk;

struct mk_server_s {
    mk_server_config cfg;
    int blocks = 0;
    cudaStream_t stream = nullptr;                 // admissions: tables, descriptors, brick visibility
    cudaStream_t step_stream[2] = {};              // steps alternate, so one fills the other's tail
    cudaStream_t copy_stream = nullptr;            // finished images to the host
    cudaEvent_t uploaded = nullptr;                // after the latest admissions
    bool uploads_pending = false;
    cudaEvent_t last_kernel[2] = {};               // latest step kernel on each step stream
    std::vector<Slot> slots;
    SlotDesc *d_slots = nullptr, *h_slots = nullptr;
    int *d_queue[2] = {}, *h_queue[2] = {}, *d_next[2] = {};
    cudaGraph_t graph[2] = {};
    cudaGraphExec_t graph_exec[2] = {};
    cudaEvent_t queue_free[2] = {};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> event_pool;
    int max_items = 0;
    size_t vis_words = 0;
    size_t slot_bytes = 0, resident = 0, budget = 0;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<int, ServerVolume> volumes;
    int next_volume = 1;
    std::map<uint64_t, Req> reqs;
    std::map<std::array<int, 4>, std::shared_ptr<const std::vector<int>>> orders;   // centre-first tile orders
    std::deque<uint64_t> pending;
    std::vector<uint64_t> active;       // in slots, admission order
    std::deque<Step> inflight;
    uint64_t next_ticket = 1, step_count = 0, use_clock = 0;
    // evict_idle: volumes waiting for an upload, and the thread that does it
    std::deque<int> load_queue;
    std::condition_variable cv_load;
    std::thread loader;
    // requests whose image waits for its PNG + Base64 form
    std::deque<uint64_t> enc_queue;
    std::condition_variable cv_enc;
    std::thread encoder;
    mk_server_stats stats;
    bool stop = false;
    int fatal = MK_OK;
    std::string fatal_msg;
    std::thread worker;
    Clock::time_point t0;

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

void release(mk_server_s *s) {
    for (int b = 0; b < 2; ++b) {
        if (s->graph_exec[b]) cudaGraphExecDestroy(s->graph_exec[b]);
        if (s->graph[b]) cudaGraphDestroy(s->graph[b]);
        if (s->d_queue[b]) cudaFree(s->d_queue[b]);
        if (s->h_queue[b]) cudaFreeHost(s->h_queue[b]);
        if (s->d_next[b]) cudaFree(s->d_next[b]);
        if (s->queue_free[b]) cudaEventDestroy(s->queue_free[b]);
        if (s->last_kernel[b]) cudaEventDestroy(s->last_kernel[b]);
    }
    for (auto &e : s->event_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    for (auto &sl : s->slots) {
        for (int l = 0; l < MK_MAX_LABELS; ++l) {
            if (sl.tf_tex[l]) cudaDestroyTextureObject(sl.tf_tex[l]);
            if (sl.tf_array[l]) cudaFreeArray(sl.tf_array[l]);
        }
        cudaFree(sl.d_alpha);
        cudaFree(sl.d_vis);
        cudaFree(sl.d_tmax);
        cudaFree(sl.d_out);
        cudaFree(sl.d_fy);
        cudaFreeHost(sl.h_stage);
        cudaFreeHost(sl.h_lut);
        cudaFreeHost(sl.h_alpha);
    }
    if (s->d_slots) cudaFree(s->d_slots);
    if (s->h_slots) cudaFreeHost(s->h_slots);
    for (auto &kv : s->volumes) mk_volume_destroy(kv.second.vol);
    if (s->uploaded) cudaEventDestroy(s->uploaded);
    if (s->stream) cudaStreamDestroy(s->stream);
    for (int b = 0; b < 2; ++b)
        if (s->step_stream[b]) cudaStreamDestroy(s->step_stream[b]);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
}

// Mark every unfinished request failed (called with the lock held).
void fail_all(mk_server_s *s, int status, const std::string &msg) {
    s->fatal = status;
    s->fatal_msg = msg;
    for (auto &kv : s->reqs) {
        if (!kv.second.done) {
            kv.second.done = true;
            kv.second.status = status;
            kv.second.t_done = s->now_ms();
        }
    }
    s->pending.clear();
    s->active.clear();
    s->inflight.clear();
    for (auto &sl : s->slots) sl.ticket = 0;
    s->cv_done.notify_all();
}

// Upload a request's tables and descriptor into its slot (lock held).
int admit(mk_server_s *s, uint64_t ticket, int slot_index) {
    Req &q = s->reqs[ticket];
    Slot &sl = s->slots[slot_index];
    ServerVolume &V = s->volumes[q.r.volume];
    VolumeState &vs = V.vol->st;
    const int L = s->cfg.lut_len;
    SlotDesc &D = s->h_slots[slot_index];
    memset(&D, 0, sizeof(D));
    if (q.r.kind == MK_REQUEST_MPR) {
        D.kind = 1;
        D.mode = q.r.plane.mpr_type;
        fill_plane_params(vs, &q.r.plane, D.pp);
        D.plane_tex = q.r.plane.sampling == MK_SAMPLE_NEAREST ? vs.tex_point : vs.tex_linear;
        D.out = sl.d_out;
    } else {
        mk_vr_params vp = q.r.vr;
        vp.render_type = q.r.kind;
        D.kind = 0;
        D.mode = q.r.kind;
        fill_ray_params(vs, &vp, D.rp);
        D.rp.out = static_cast<uint8_t *>(sl.d_out);
        // the slot's own table, built on the admission stream like its brick
        // maps (the slot's previous request, and with it every kernel that
        // read the old table, has finished)
        if (sl.fy_cap < vs.accu_len) {
            cudaFree(sl.d_fy);
            sl.d_fy = nullptr;
            sl.fy_cap = 0;
            MK_CUDA_TRY(cudaMalloc(&sl.d_fy, (size_t)vs.accu_len * sizeof(float)));
            sl.fy_cap = vs.accu_len;
        }
        int trc = launch_fy_table(vs, D.rp.scale, sl.d_fy, s->stream);
        if (trc != MK_OK) return trc;
        D.rp.fy_tab = sl.d_fy;
        float params[MK_MAX_LABELS][3];
        for (int l = 0; l < MK_MAX_LABELS; ++l) {
            const bool has = l < q.r.n_luts;
            params[l][0] = has ? q.params[3 * l + 0] : 0.0f;
            params[l][1] = has ? q.params[3 * l + 1] : 1.0f;
            params[l][2] = has ? q.params[3 * l + 2] : 0.0f;
            D.lt.tf[l] = has ? sl.tf_tex[l] : 0;
            D.lt.alpha[l] = params[l][0];
            D.lt.ww[l] = params[l][1];
            D.lt.wl[l] = params[l][2];
        }
        D.track = tracking_mode_for(vs.present_labels, params);
        if (q.r.kind == MK_REQUEST_MIP) set_mip_window(D.rp, vs.present_labels, params);
        D.vol = vs.tex_linear;
        D.mask = vs.tex_mask;
        const float *alpha_ptr[MK_MAX_LABELS];
        int lens[MK_MAX_LABELS];
        const int n = q.r.n_luts;
        if (n > 0) {
            memcpy(sl.h_lut, q.luts.data(), (size_t)n * L * 4 * sizeof(float));
            for (int l = 0; l < n; ++l) {
                for (int i = 0; i < L; ++i) sl.h_alpha[(size_t)l * L + i] = q.luts[((size_t)l * L + i) * 4 + 3];
                MK_CUDA_TRY(cudaMemcpy2DToArrayAsync(sl.tf_array[l], 0, 0, sl.h_lut + (size_t)l * L * 4,
                                                     L * sizeof(float4), L * sizeof(float4), 1,
                                                     cudaMemcpyHostToDevice, s->stream));
            }
            MK_CUDA_TRY(cudaMemcpyAsync(sl.d_alpha, sl.h_alpha, (size_t)n * L * sizeof(float),
                                        cudaMemcpyHostToDevice, s->stream));
        }
        for (int l = 0; l < MK_MAX_LABELS; ++l) {
            alpha_ptr[l] = l < n ? sl.d_alpha + (size_t)l * L : nullptr;
            lens[l] = l < n ? L : 0;
        }
        int rc = launch_brick_visibility(&vs, alpha_ptr, lens, params, sl.d_vis, sl.d_tmax, s->stream);
        if (rc != MK_OK) return rc;
        D.bv.visible_bits = sl.d_vis;
        D.bv.mip_tmax = sl.d_tmax;
        D.bv.minmax = vs.d_minmax;
        D.bv.nbx = vs.nb[0];
        D.bv.nby = vs.nb[1];
        D.bv.nbz = vs.nb[2];
    }
    MK_CUDA_TRY(cudaMemcpyAsync(s->d_slots + slot_index, &D, sizeof(SlotDesc), cudaMemcpyHostToDevice, s->stream));
    s->uploads_pending = true;
    sl.ticket = ticket;
    q.slot = slot_index;
    return MK_OK;
}

// List the next tiles, launch the step graph and queue the copies of the
// images it finishes (lock held).
int issue_step(mk_server_s *s) {
    const int b = (int)(s->step_count & 1);
    MK_CUDA_TRY(cudaEventSynchronize(s->queue_free[b]));   // the copy of this list two steps ago is done
    TileItem *items = reinterpret_cast<TileItem *>(s->h_queue[b] + 2);
    int n = 0;
    Step st;
    const double now = s->now_ms();
    for (uint64_t t : s->active) {
        Req &q = s->reqs[t];
        if (q.tiles_issued >= q.tiles_total) continue;
        if (n >= s->max_items) break;
        if (q.t_start < 0) q.t_start = now;
        while (q.tiles_issued < q.tiles_total && n < s->max_items) {
            const int k = q.tiles_issued++;
            items[n].slot = (unsigned short)q.slot;
            const int t = q.order ? (*q.order)[k] : k;
            items[n].tx = (unsigned short)(t % q.tiles_x);
            items[n].ty = (unsigned short)(t / q.tiles_x);
            items[n].pad = 0;
            ++n;
        }
        if (q.tiles_issued == q.tiles_total) st.finishing.push_back(t);
    }
    if (n == 0) return MK_OK;
    s->h_queue[b][0] = n;
    s->h_queue[b][1] = 0;
    cudaStream_t ss = s->step_stream[b];
    if (s->uploads_pending) {                              // descriptors and maps of new requests first
        MK_CUDA_TRY(cudaEventRecord(s->uploaded, s->stream));
        s->uploads_pending = false;
    }
    MK_CUDA_TRY(cudaStreamWaitEvent(ss, s->uploaded, 0));
    MK_CUDA_TRY(cudaMemcpyAsync(s->d_queue[b], s->h_queue[b], 8 + (size_t)n * sizeof(TileItem),
                                cudaMemcpyHostToDevice, ss));
    MK_CUDA_TRY(cudaEventRecord(s->queue_free[b], ss));
    MK_CUDA_TRY(cudaGraphLaunch(s->graph_exec[b], ss));
    const auto ev = s->event_pool[s->step_count % s->event_pool.size()];
    st.kernel_done = ev.first;
    st.copies_done = ev.second;
    MK_CUDA_TRY(cudaEventRecord(st.kernel_done, ss));
    // A finishing request's earlier tiles are in earlier steps: those on this
    // stream are ordered before this one, the other stream's latest may still run.
    MK_CUDA_TRY(cudaStreamWaitEvent(s->copy_stream, st.kernel_done, 0));
    MK_CUDA_TRY(cudaStreamWaitEvent(s->copy_stream, s->last_kernel[b ^ 1], 0));
    MK_CUDA_TRY(cudaEventRecord(s->last_kernel[b], ss));
    for (uint64_t t : st.finishing) {
        Req &q = s->reqs[t];
        Slot &sl = s->slots[q.slot];
        void *dst = q.direct ? q.r.out : sl.h_stage;
        MK_CUDA_TRY(cudaMemcpyAsync(dst, sl.d_out, q.out_bytes, cudaMemcpyDeviceToHost, s->copy_stream));
    }
    MK_CUDA_TRY(cudaEventRecord(st.copies_done, s->copy_stream));
    s->inflight.push_back(std::move(st));
    ++s->step_count;
    s->stats.steps++;
    s->stats.tiles += (uint64_t)n;
    return MK_OK;
}

void worker_loop(mk_server_s *s) {
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->stop && s->pending.empty() && s->active.empty() && s->inflight.empty()) break;
        if (s->fatal != MK_OK) {
            if (s->stop) break;
            s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        bool progressed = false;
        int rc = MK_OK;
        // 1. retire finished steps, oldest first
        while (!s->inflight.empty()) {
            const cudaError_t e = cudaEventQuery(s->inflight.front().copies_done);
            if (e == cudaErrorNotReady) break;
            if (e != cudaSuccess) {
                rc = MK_ERR_CUDA;
                set_last_error(std::string("mk_server: ") + cudaGetErrorString(e));
                break;
            }
            Step st = std::move(s->inflight.front());
            s->inflight.pop_front();
            std::vector<std::pair<void *, std::pair<const void *, size_t>>> copies;
            for (uint64_t t : st.finishing) {
                Req &q = s->reqs[t];
                if (!q.direct) copies.push_back({q.r.out, {s->slots[q.slot].h_stage, q.out_bytes}});
            }
            lk.unlock();
            for (auto &c : copies) memcpy(c.first, c.second.first, c.second.second);
            lk.lock();
            const double now = s->now_ms();
            for (uint64_t t : st.finishing) {
                Req &q = s->reqs[t];
                if (q.enc_ch) {
                    s->enc_queue.push_back(t);        // done once the encoder has written its form
                    s->cv_enc.notify_one();
                } else {
                    q.done = true;
                    q.t_done = now;
                }
                s->slots[q.slot].ticket = 0;
                s->active.erase(std::find(s->active.begin(), s->active.end(), t));
                auto it = s->volumes.find(q.r.volume);
                if (it != s->volumes.end()) {
                    it->second.users--;
                    it->second.in_slots--;
                }
                s->stats.completed++;
            }
            s->cv_done.notify_all();
            if (!s->load_queue.empty()) s->cv_load.notify_one();   // volumes may be evictable now
            progressed = true;
        }
        // 2. admit waiting requests into free slots, in arrival order; a
        //    request whose volume is not resident waits for the loader
        //    thread (which it wakes) and does not hold up later requests
        for (auto pit = s->pending.begin(); rc == MK_OK && pit != s->pending.end();) {
            int free_slot = -1;
            for (int i = 0; i < (int)s->slots.size(); ++i)
                if (s->slots[i].ticket == 0) {
                    free_slot = i;
                    break;
                }
            if (free_slot < 0) break;
            const uint64_t t = *pit;
            ServerVolume &V = s->volumes[s->reqs[t].r.volume];
            if (!V.vol || V.loading) {
                if (!V.loading) {
                    V.loading = true;
                    s->load_queue.push_back(s->reqs[t].r.volume);
                    s->cv_load.notify_one();
                }
                ++pit;
                continue;
            }
            pit = s->pending.erase(pit);
            rc = admit(s, t, free_slot);
            V.in_slots++;
            V.last_use = ++s->use_clock;
            s->active.push_back(t);
            progressed = true;
        }
        // 3. keep up to four steps in flight
        if (rc == MK_OK && s->inflight.size() < 4) {
            bool work = false;
            for (uint64_t t : s->active) {
                const Req &q = s->reqs[t];
                if (q.tiles_issued < q.tiles_total) {
                    work = true;
                    break;
                }
            }
            if (work) {
                rc = issue_step(s);
                progressed = true;
            }
        }
        if (rc != MK_OK) {
            fail_all(s, rc, "mk_server: CUDA failure in the worker");
            continue;
        }
        if (!progressed) {
            if (!s->inflight.empty()) {
                lk.unlock();
                std::this_thread::yield();
                lk.lock();
            } else {
                s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
    }
}

// Writes the PNG + Base64 form of finished requests that asked for it (the
// image is already in the request's host buffer), one request at a time with
// the encoder's parallel bands, while the worker runs later steps.
void encoder_loop(mk_server_s *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->enc_queue.empty()) {
            if (s->stop && s->pending.empty() && s->active.empty() && s->inflight.empty()) break;
            s->cv_enc.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        const uint64_t t = s->enc_queue.front();
        s->enc_queue.pop_front();
        auto it = s->reqs.find(t);
        if (it == s->reqs.end() || it->second.done) continue;   // failed meanwhile
        const Req &q = it->second;
        const uint8_t *img = static_cast<const uint8_t *>(q.r.out);
        const int w = q.enc_w, h = q.enc_h, ch = q.enc_ch;
        char *dst = q.r.encoded;
        const size_t cap = q.r.encoded_capacity;
        lk.unlock();
        const std::vector<uint8_t> png = encode_png(img, w, h, ch);
        size_t n = 0;
        int st = MK_OK;
        if (png.empty() || ((png.size() + 2) / 3) * 4 + 1 > cap) {
            st = MK_ERR_OUT_OF_MEMORY;
        } else {
            n = base64_encode(png.data(), png.size(), dst);
            dst[n] = '\0';
        }
        lk.lock();
        auto jt = s->reqs.find(t);          // a failure meanwhile may have completed (and freed) it
        if (jt == s->reqs.end() || jt->second.done) continue;
        jt->second.enc_len = n;
        jt->second.status = st;
        jt->second.done = true;
        jt->second.t_done = s->now_ms();
        s->cv_done.notify_all();
    }
}

// Resident volumes that may be evicted to make room for `need` more bytes:
// those no admitted request uses, least recently used first, volumes with
// no queued request before those with one.  Empty if they are not enough
// (lock held).
std::vector<int> eviction_victims(mk_server_s *s, int keep, size_t need) {
    std::vector<std::pair<std::pair<int, uint64_t>, int>> cand;
    for (auto &kv : s->volumes) {
        const ServerVolume &V = kv.second;
        if (kv.first == keep || !V.vol || V.loading || V.in_slots > 0) continue;
        cand.push_back({{V.users > 0 ? 1 : 0, V.last_use}, kv.first});
    }
    std::sort(cand.begin(), cand.end());
    std::vector<int> out;
    size_t freed = 0;
    for (auto &c : cand) {
        if (s->resident + need <= s->budget + freed) break;
        out.push_back(c.second);
        freed += s->volumes[c.second].bytes;
    }
    if (s->resident + need > s->budget + freed) out.clear();
    return out;
}

// Upload of one volume from its host copy (evict_idle); the caller reserved
// `est` bytes of the budget.  Returns the handle or nullptr (status in rc).
mk_volume upload_volume(const mk_server_s *s, const ServerVolume &V, int &rc) {
    mk_volume v = nullptr;
    rc = mk_volume_create(&v, V.host_vox->data(), V.dims[0], V.dims[1], V.dims[2], s->cfg.device);
    if (rc == MK_OK && V.host_lab) rc = mk_volume_set_mask(v, V.host_lab->data());
    if (rc == MK_OK) rc = mk_volume_synchronize(v, nullptr);
    if (rc != MK_OK && v) {
        mk_volume_destroy(v);
        v = nullptr;
    }
    return v;
}

size_t volume_estimate(int dx, int dy, int dz, bool labels);

// evict_idle: uploads evicted volumes that requests wait for, evicting idle
// ones to make room.  Runs beside the worker, so steps of requests for
// resident volumes continue during an upload.
void loader_loop(mk_server_s *s) {
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->stop) break;
        if (s->load_queue.empty()) {
            s->cv_load.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        const int id = s->load_queue.front();
        auto it = s->volumes.find(id);
        if (it == s->volumes.end() || it->second.vol) {
            if (it != s->volumes.end()) it->second.loading = false;
            s->load_queue.pop_front();
            continue;
        }
        ServerVolume &V = it->second;
        // the device bytes of its previous upload (an evicted volume keeps
        // them), or the estimate for one never uploaded: an estimate above
        // the real size would make two volumes that fit the budget together
        // look as if they did not, and every switch between them an eviction
        const size_t est = V.bytes;
        std::vector<int> victims = eviction_victims(s, id, est);
        if (s->resident + est > s->budget && victims.empty()) {
            // every resident volume is in use: wait for requests to retire
            s->cv_load.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        s->load_queue.pop_front();
        std::vector<mk_volume> dead;
        for (int vid : victims) {
            ServerVolume &E = s->volumes[vid];
            dead.push_back(E.vol);
            E.vol = nullptr;
            s->resident -= E.bytes;             // E.bytes stays: the size of its next upload
            s->stats.evictions++;
        }
        s->resident += est;                     // reserved while uploading
        lk.unlock();
        for (mk_volume d : dead) mk_volume_destroy(d);
        int rc = MK_OK;
        mk_volume v = upload_volume(s, V, rc);  // V stays in the map: only this thread erases loading volumes
        size_t bytes = 0;
        if (v) mk_volume_device_bytes(v, &bytes);
        lk.lock();
        s->resident -= est;
        V.loading = false;
        if (v) {
            V.vol = v;
            V.bytes = bytes;
            s->resident += bytes;
            s->stats.loads++;
        } else {
            // the requests waiting for this volume fail with the upload's status
            const std::string msg = "mk_server: upload of an evicted volume failed";
            for (auto pit = s->pending.begin(); pit != s->pending.end();) {
                Req &q = s->reqs[*pit];
                if (q.r.volume != id) {
                    ++pit;
                    continue;
                }
                q.done = true;
                q.status = rc;
                q.t_done = s->now_ms();
                V.users--;
                pit = s->pending.erase(pit);
            }
            set_last_error(msg);
            s->cv_done.notify_all();
        }
        s->cv_work.notify_all();
    }
}

// Device allocations of a server go through here.  MK_SERVER_FAIL_ALLOC=n in
// the environment makes the n-th one (counting from 1, per mk_server_create)
// report cudaErrorMemoryAllocation without calling cudaMalloc, so that the
// clean-up after a failed allocation can be tested without exhausting HBM.
struct AllocInjector {
    long fail_at = -1, count = 0;
    AllocInjector() {
        const char *e = getenv("MK_SERVER_FAIL_ALLOC");
        if (e && *e) fail_at = atol(e);
    }
    cudaError_t operator()(void **p, size_t bytes) {
        if (++count == fail_at) return cudaErrorMemoryAllocation;
        return cudaMalloc(p, bytes);
    }
};

size_t volume_estimate(int dx, int dy, int dz, bool labels) {
    const size_t nvox = (size_t)dx * dy * dz;
    const size_t nb = (size_t)((dx + 7) / 8) * ((dy + 7) / 8) * ((dz + 7) / 8);
    return nvox * 2 + (labels ? nvox : 0) + nb * 20 + (nb / 32 + 2) * 4 + (size_t)(1.74 * dz + 16) * 4;
}

}  // namespace

extern "C" int mk_server_create(const mk_server_config *config, mk_server *out) {
    if (!config || !out) {
        set_last_error("mk_server_create: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    mk_server_config c = *config;
    if (c.max_bricks == 0) c.max_bricks = 64 * 64 * 256;
    if (c.tiles_per_step == 0) c.tiles_per_step = 8192;
    if (c.max_slots < 1 || c.max_slots > 256 || c.max_pending < 1 || c.max_pixels < 1 || c.lut_len < 2 ||
        c.lut_len > 4096 || c.max_labels < 1 || c.max_labels > MK_MAX_LABELS || c.max_bricks < 1 ||
        c.tiles_per_step < 1 || c.tiles_per_step > (1 << 20)) {
        set_last_error("mk_server_create: bad configuration (1 <= max_slots <= 256, max_pending >= 1, "
                       "max_pixels >= 1, 2 <= lut_len <= 4096, 1 <= max_labels <= 65, tiles_per_step <= 2^20)");
        return MK_ERR_INVALID_ARGUMENT;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("mk_server_create: no CUDA device");
        return MK_ERR_NO_DEVICE;
    }
    if (c.device < 0 || c.device >= ndev) {
        set_last_error("mk_server_create: device index out of range");
        return MK_ERR_INVALID_ARGUMENT;
    }
    MK_CUDA_TRY(cudaSetDevice(c.device));
    size_t free_b = 0, total_b = 0;
    MK_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    mk_server_s *s = new mk_server_s();
    s->cfg = c;
    s->budget = c.hbm_budget_bytes ? c.hbm_budget_bytes : (size_t)(0.9 * (double)free_b);
    s->vis_words = (size_t)c.max_bricks / 32 + 2;
    s->max_items = c.tiles_per_step;
    const size_t L = (size_t)c.lut_len;
    s->slot_bytes = (size_t)c.max_slots * ((size_t)c.max_labels * L * 20 + s->vis_words * 4 +
                                           (size_t)c.max_bricks * 4 + (size_t)c.max_pixels * 4 + sizeof(SlotDesc)) +
                    2 * (8 + (size_t)s->max_items * sizeof(TileItem));
    if (s->slot_bytes > s->budget) {
        set_last_error("mk_server_create: the slot buffers alone exceed the HBM budget");
        delete s;
        return MK_ERR_BUDGET;
    }
    s->resident = s->slot_bytes;
    memset(&s->stats, 0, sizeof(s->stats));
    int rc = MK_OK;
    cudaError_t e = cudaSuccess;
    AllocInjector dev_alloc;
    do {
        if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) break;
        if ((e = cudaStreamCreateWithFlags(&s->step_stream[0], cudaStreamNonBlocking)) != cudaSuccess) break;
        if ((e = cudaStreamCreateWithFlags(&s->step_stream[1], cudaStreamNonBlocking)) != cudaSuccess) break;
        if ((e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) break;
        if ((e = cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming)) != cudaSuccess) break;
        if ((e = cudaEventRecord(s->uploaded, s->stream)) != cudaSuccess) break;
        s->slots.resize(c.max_slots);
        cudaChannelFormatDesc cd = cudaCreateChannelDesc<float4>();
        for (auto &sl : s->slots) {
            for (int l = 0; l < c.max_labels && e == cudaSuccess; ++l) {
                if ((e = cudaMallocArray(&sl.tf_array[l], &cd, c.lut_len, 1)) != cudaSuccess) break;
                cudaResourceDesc rd;
                memset(&rd, 0, sizeof(rd));
                rd.resType = cudaResourceTypeArray;
                rd.res.array.array = sl.tf_array[l];
                cudaTextureDesc td;
                memset(&td, 0, sizeof(td));
                td.normalizedCoords = 1;
                td.filterMode = cudaFilterModeLinear;
                td.addressMode[0] = cudaAddressModeClamp;
                td.readMode = cudaReadModeElementType;
                e = cudaCreateTextureObject(&sl.tf_tex[l], &rd, &td, nullptr);
            }
            if (e != cudaSuccess) break;
            if ((e = dev_alloc((void **)&sl.d_alpha, (size_t)c.max_labels * L * sizeof(float))) != cudaSuccess) break;
            if ((e = dev_alloc((void **)&sl.d_vis, s->vis_words * sizeof(uint32_t))) != cudaSuccess) break;
            if ((e = dev_alloc((void **)&sl.d_tmax, (size_t)c.max_bricks * sizeof(float))) != cudaSuccess) break;
            if ((e = dev_alloc((void **)&sl.d_out, (size_t)c.max_pixels * 4)) != cudaSuccess) break;
            if ((e = cudaMallocHost(&sl.h_stage, (size_t)c.max_pixels * 4)) != cudaSuccess) break;
            if ((e = cudaMallocHost(&sl.h_lut, (size_t)c.max_labels * L * 4 * sizeof(float))) != cudaSuccess) break;
            if ((e = cudaMallocHost(&sl.h_alpha, (size_t)c.max_labels * L * sizeof(float))) != cudaSuccess) break;
        }
        if (e != cudaSuccess) break;
        if ((e = dev_alloc((void **)&s->d_slots, c.max_slots * sizeof(SlotDesc))) != cudaSuccess) break;
        if ((e = cudaMallocHost(&s->h_slots, c.max_slots * sizeof(SlotDesc))) != cudaSuccess) break;
        const size_t qbytes = 8 + (size_t)s->max_items * sizeof(TileItem);
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            if ((e = dev_alloc((void **)&s->d_queue[b], qbytes)) != cudaSuccess) break;
            if ((e = cudaMallocHost(&s->h_queue[b], qbytes)) != cudaSuccess) break;
            if ((e = dev_alloc((void **)&s->d_next[b], sizeof(int))) != cudaSuccess) break;
            if ((e = cudaEventCreateWithFlags(&s->queue_free[b], cudaEventDisableTiming)) != cudaSuccess) break;
            if ((e = cudaEventRecord(s->queue_free[b], s->step_stream[b])) != cudaSuccess) break;
            if ((e = cudaEventCreateWithFlags(&s->last_kernel[b], cudaEventDisableTiming)) != cudaSuccess) break;
            e = cudaEventRecord(s->last_kernel[b], s->step_stream[b]);
        }
        if (e != cudaSuccess) break;
        for (int i = 0; i < 8 && e == cudaSuccess; ++i) {
            cudaEvent_t a = nullptr, b2 = nullptr;
            if ((e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming)) != cudaSuccess) break;
            if ((e = cudaEventCreateWithFlags(&b2, cudaEventDisableTiming)) != cudaSuccess) {
                cudaEventDestroy(a);
                break;
            }
            s->event_pool.push_back({a, b2});
        }
        if (e != cudaSuccess) break;
        int per_sm = 0, sms = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_serve, 256, 0)) != cudaSuccess) break;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device)) != cudaSuccess) break;
        s->blocks = std::max(1, per_sm) * sms;
        // one graph per queue buffer: reset the tile counter, run the persistent kernel
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            cudaStream_t cap = nullptr;
            if ((e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) != cudaSuccess) break;
            e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaMemsetAsync(s->d_next[b], 0, sizeof(int), cap);
                k_serve<<<s->blocks, 256, 0, cap>>>(s->d_slots, s->d_queue[b], s->d_next[b]);
                e = cudaStreamEndCapture(cap, &s->graph[b]);
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&s->graph_exec[b], s->graph[b], 0);
            cudaStreamDestroy(cap);
        }
        if (e != cudaSuccess) break;
        e = cudaStreamSynchronize(s->stream);
    } while (0);
    if (e != cudaSuccess) {
        set_last_error(std::string("mk_server_create: ") + cudaGetErrorString(e));
        rc = e == cudaErrorMemoryAllocation ? MK_ERR_OUT_OF_MEMORY : MK_ERR_CUDA;
        cudaGetLastError();
        release(s);
        delete s;
        return rc;
    }
    s->stats.budget_bytes = s->budget;
    s->t0 = Clock::now();
    s->worker = std::thread(worker_loop, s);
    s->encoder = std::thread(encoder_loop, s);
    if (c.evict_idle) s->loader = std::thread(loader_loop, s);
    *out = s;
    return MK_OK;
}

extern "C" int mk_server_destroy(mk_server s) {
    if (!s) return MK_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    s->cv_load.notify_all();
    if (s->loader.joinable()) s->loader.join();
    s->cv_enc.notify_all();
    if (s->encoder.joinable()) s->encoder.join();
    cudaSetDevice(s->cfg.device);
    cudaStreamSynchronize(s->stream);
    cudaStreamSynchronize(s->step_stream[0]);
    cudaStreamSynchronize(s->step_stream[1]);
    cudaStreamSynchronize(s->copy_stream);
    release(s);
    delete s;
    return MK_OK;
}

extern "C" int mk_server_add_volume(mk_server s, const int16_t *voxels, int dim_x, int dim_y, int dim_z,
                                    const uint8_t *labels, int *volume_id) {
    if (!s || !voxels || !volume_id || dim_x <= 0 || dim_y <= 0 || dim_z <= 0) {
        set_last_error("mk_server_add_volume: null pointer or non-positive dimension");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const size_t nb = (size_t)((dim_x + 7) / 8) * ((dim_y + 7) / 8) * ((dim_z + 7) / 8);
    if (nb > (size_t)s->cfg.max_bricks) {
        set_last_error("mk_server_add_volume: the volume has more bricks than the server's max_bricks");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const size_t est = volume_estimate(dim_x, dim_y, dim_z, labels != nullptr);
    const size_t nvox = (size_t)dim_x * dim_y * dim_z;
    ServerVolume sv;
    sv.dims[0] = dim_x;
    sv.dims[1] = dim_y;
    sv.dims[2] = dim_z;
    if (s->cfg.evict_idle) {
        if (est + s->slot_bytes > s->budget) {
            set_last_error("mk_server_add_volume: the volume alone exceeds the HBM budget");
            return MK_ERR_BUDGET;
        }
        sv.host_vox = std::make_shared<const std::vector<int16_t>>(voxels, voxels + nvox);
        if (labels) sv.host_lab = std::make_shared<const std::vector<uint8_t>>(labels, labels + nvox);
    }
    std::vector<mk_volume> dead;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->resident + est > s->budget) {
            std::vector<int> victims;
            if (s->cfg.evict_idle) victims = eviction_victims(s, -1, est);
            if (victims.empty()) {
                if (!s->cfg.evict_idle) {
                    set_last_error("mk_server_add_volume: the volume does not fit the HBM budget");
                    return MK_ERR_BUDGET;
                }
                // registered evicted: uploaded for its first request
                const int id = s->next_volume++;
                sv.bytes = est;
                s->volumes[id] = sv;
                *volume_id = id;
                return MK_OK;
            }
            for (int vid : victims) {
                ServerVolume &E = s->volumes[vid];
                dead.push_back(E.vol);
                E.vol = nullptr;
                s->resident -= E.bytes;         // E.bytes stays: the size of its next upload
                s->stats.evictions++;
            }
        }
        s->resident += est;                      // reserved while uploading
    }
    for (mk_volume d : dead) mk_volume_destroy(d);
    mk_volume v = nullptr;
    int rc = mk_volume_create(&v, voxels, dim_x, dim_y, dim_z, s->cfg.device);
    if (rc == MK_OK && labels) rc = mk_volume_set_mask(v, labels);
    if (rc == MK_OK) rc = mk_volume_synchronize(v, nullptr);
    size_t bytes = 0;
    if (rc == MK_OK) rc = mk_volume_device_bytes(v, &bytes);
    std::lock_guard<std::mutex> lk(s->mu);
    s->resident -= est;
    if (rc != MK_OK) {
        if (v) mk_volume_destroy(v);
        return rc;
    }
    const int id = s->next_volume++;
    sv.vol = v;
    sv.bytes = bytes;
    sv.last_use = ++s->use_clock;
    s->volumes[id] = sv;
    s->resident += bytes;
    *volume_id = id;
    return MK_OK;
}

extern "C" int mk_server_remove_volume(mk_server s, int volume_id) {
    if (!s) return MK_ERR_INVALID_ARGUMENT;
    mk_volume v = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->volumes.find(volume_id);
        if (it == s->volumes.end()) {
            set_last_error("mk_server_remove_volume: unknown volume");
            return MK_ERR_INVALID_ARGUMENT;
        }
        if (it->second.users > 0 || it->second.loading) {
            set_last_error("mk_server_remove_volume: requests for the volume are queued or in flight, "
                           "or it is being uploaded");
            return MK_ERR_NOT_READY;
        }
        v = it->second.vol;
        if (v) s->resident -= it->second.bytes;
        s->volumes.erase(it);
    }
    return v ? mk_volume_destroy(v) : MK_OK;
}

extern "C" int mk_server_submit(mk_server s, const mk_request *req, uint64_t *ticket) {
    if (!s || !req || !ticket || !req->out) {
        set_last_error("mk_server_submit: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->fatal != MK_OK) {
        set_last_error(s->fatal_msg);
        return s->fatal;
    }
    auto vit = s->volumes.find(req->volume);
    if (vit == s->volumes.end()) {
        set_last_error("mk_server_submit: unknown volume");
        return MK_ERR_INVALID_ARGUMENT;
    }
    // parameters are validated against the volume's dims (an evicted
    // volume has no device state; a stand-in carries its dims)
    VolumeState dims_only;
    for (int k = 0; k < 3; ++k) dims_only.dims[k] = vit->second.dims[k];
    const VolumeState &vs = vit->second.vol ? vit->second.vol->st : dims_only;
    Req q;
    q.r = *req;
    const int L = s->cfg.lut_len;
    if (req->kind == MK_REQUEST_MPR) {
        PlaneParams P;
        const int rc = fill_plane_params(vs, &req->plane, P);
        if (rc != MK_OK) return rc;
        if ((size_t)P.W * P.H > (size_t)s->cfg.max_pixels) {
            set_last_error("mk_server_submit: the plane exceeds max_pixels");
            return MK_ERR_INVALID_ARGUMENT;
        }
        q.tiles_x = (P.W + 31) / 32;
        q.tiles_total = q.tiles_x * ((P.H + 7) / 8);
        q.out_bytes = (size_t)P.W * P.H * sizeof(int16_t);
        if (req->encoded) {
            if (P.W % 2) {
                set_last_error("mk_server_submit: an encoded plane needs an even width");
                return MK_ERR_INVALID_ARGUMENT;
            }
            q.enc_w = P.W / 2;                // MonkeyGL's packing: 2 int16 per RGBA pixel
            q.enc_h = P.H;
            q.enc_ch = 4;
        }
    } else if (req->kind >= MK_REQUEST_VR && req->kind <= MK_REQUEST_SURFACE) {
        mk_vr_params vp = req->vr;
        vp.render_type = req->kind;
        RayParams P;
        const int rc = fill_ray_params(vs, &vp, P);
        if (rc != MK_OK) return rc;
        if ((size_t)P.W * P.H > (size_t)s->cfg.max_pixels) {
            set_last_error("mk_server_submit: the image exceeds max_pixels");
            return MK_ERR_INVALID_ARGUMENT;
        }
        if (req->n_luts < 0 || req->n_luts > s->cfg.max_labels || (req->n_luts > 0 && (!req->luts || !req->label_params))) {
            set_last_error("mk_server_submit: 0 <= n_luts <= max_labels, with luts and label_params");
            return MK_ERR_INVALID_ARGUMENT;
        }
        for (int l = 0; l < req->n_luts; ++l) {
            if (!(req->label_params[3 * l + 1] > 0.0f)) {
                set_last_error("mk_server_submit: window width must be > 0");
                return MK_ERR_INVALID_ARGUMENT;
            }
        }
        q.luts.assign(req->luts, req->luts + (size_t)req->n_luts * L * 4);
        q.params.assign(req->label_params, req->label_params + (size_t)req->n_luts * 3);
        q.tiles_x = (P.W + 31) / 32;
        q.tiles_total = q.tiles_x * ((P.H + 7) / 8);
        q.out_bytes = (size_t)P.W * P.H * (P.rgba ? 4 : 3);
        if (req->encoded) {
            q.enc_w = P.W;
            q.enc_h = P.H;
            q.enc_ch = P.rgba ? 4 : 3;
        }
        const std::array<int, 4> key = {P.W, P.H, (int)lrintf(P.xT), (int)lrintf(P.yT)};
        auto oit = s->orders.find(key);
        if (oit == s->orders.end()) {
            if (s->orders.size() >= 64) s->orders.clear();
            oit = s->orders.emplace(key, std::make_shared<const std::vector<int>>(
                                             centre_first_tiles(P.W, P.H, key[2], key[3]))).first;
        }
        q.order = oit->second;
    } else {
        set_last_error("mk_server_submit: unknown request kind");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (q.enc_ch && req->encoded_capacity < encoded_capacity(q.enc_w, q.enc_h, q.enc_ch)) {
        set_last_error("mk_server_submit: encoded_capacity below mk_encoded_capacity of the image");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if ((int)s->pending.size() >= s->cfg.max_pending) {
        s->stats.rejected++;
        set_last_error("mk_server_submit: the queue is full");
        return MK_ERR_QUEUE_FULL;
    }
    q.r.luts = nullptr;
    q.r.label_params = nullptr;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, req->out) == cudaSuccess) q.direct = attr.type == cudaMemoryTypeHost;
    else cudaGetLastError();
    q.t_submit = s->now_ms();
    const uint64_t t = s->next_ticket++;
    s->reqs.emplace(t, std::move(q));
    s->pending.push_back(t);
    vit->second.users++;
    s->stats.submitted++;
    *ticket = t;
    lk.unlock();
    s->cv_work.notify_one();
    return MK_OK;
}

extern "C" int mk_server_wait(mk_server s, uint64_t ticket, int timeout_ms, mk_request_times *times) {
    if (!s) return MK_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) {
        set_last_error("mk_server_wait: unknown ticket");
        return MK_ERR_INVALID_ARGUMENT;
    }
    auto done = [&] { return s->reqs[ticket].done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return MK_ERR_TIMEOUT;
    Req &q = s->reqs[ticket];
    if (times) {
        times->submitted_ms = q.t_submit;
        times->started_ms = q.t_start;
        times->completed_ms = q.t_done;
        times->encoded_length = q.enc_len;
    }
    const int st = q.status;
    if (st != MK_OK) set_last_error(s->fatal_msg);
    s->reqs.erase(ticket);
    return st;
}

extern "C" int mk_server_get_stats(mk_server s, mk_server_stats *out) {
    if (!s || !out) return MK_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->resident_bytes = s->resident;
    out->budget_bytes = s->budget;
    out->volumes = (int)s->volumes.size();
    out->pending = (int)s->pending.size();
    int busy = 0;
    for (auto &sl : s->slots) busy += sl.ticket != 0;
    out->slots_busy = busy;
    return MK_OK;
}
