// server.cu - request server: admission by device-memory budget, continuous
// batching of DiTO fits, concurrent builds (include/obvh_server.h).
//
// One scheduler thread owns every CUDA call after creation.  Each round it
//   1. retires finished work (an event query per fit round and build lane):
//      fit results are copied out of the round's pinned buffer, scratch and
//      copied-in inputs go back to the arena;
//   2. admits pending requests in arrival order while their blocks fit in the
//      arena (a request that alone exceeds the budget fails at once; a build
//      waiting only for a free lane lets later fits pass);
//   3. launches all admitted fits as one batched persistent kernel on a free
//      fit round (two rounds alternate, so the next batch's copies overlap the
//      running one), the admitted builds of up to 16,384 triangles as one
//      launch of the one-CTA-per-mesh build kernel on the batch round's
//      stream, and each larger build on a free lane's stream (the whole-GPU
//      chain).
// Callers' threads only touch host-side state under the mutex.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "dito_batch_host.h"
#include "mesh_batch_host.h"
#include "obvh_build.h"
#include "obvh_server.h"
#include "pipeline_host.h"
#include "runtime.h"

namespace obvh {
namespace server {

using Clock = std::chrono::steady_clock;

constexpr size_t kAlign = 768;  // 256-byte aligned and a whole number of 12-byte points

// First-fit allocator over one device allocation (host-side bookkeeping).
class Arena {
public:
    void init(size_t size) {
        size_ = size;
        free_.clear();
        if (size) free_[0] = size;
        used_ = peak_ = 0;
    }
    bool alloc(size_t bytes, size_t* off) {
        bytes = round(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes, at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = round(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    static size_t round(size_t b) { return (std::max<size_t>(b, 1) + kAlign - 1) / kAlign * kAlign; }
    size_t size() const { return size_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

private:
    size_t size_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

struct Block {
    size_t off = 0, bytes = 0;
    bool live = false;
};

enum class Kind { Fit, Build };
enum class State { Pending, Admitted, Running, Done, Failed };

struct Request {
    uint64_t id = 0;
    Kind kind = Kind::Fit;
    State state = State::Pending;
    kr_error error = nullptr;
    bool device_input = false;
    const kr_vec3* points = nullptr;
    uint64_t count = 0;
    kr_obb3 obb{};
    const kr_vec3* verts = nullptr;
    uint64_t nverts = 0;
    const kr_uvec4* faces = nullptr;
    uint32_t nfaces = 0;
    uint32_t flags = 0;
    float ci = 0.f, ct = 0.f;
    obvh_server_build_view view{};
    Block input, output, scratch;
    Clock::time_point t_submit, t_done;
};

struct FitRound {
    dito_batch::Batch* batch = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    DeviceBuffer out;
    PinnedBuffer host_out;
    PinnedBuffer word;  // the batch's device error word
    std::vector<Request*> reqs;
    bool busy = false;
};

// The small builds admitted together, built by one launch of the
// one-CTA-per-mesh kernel (mesh_batch_host.h) into their own arena blocks.
struct BuildBatchRound {
    meshbatch::Runner* runner = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    PinnedBuffer words;  // the run's status: error, job counter, each mesh's primitive slots
    std::vector<Request*> reqs;
    bool busy = false;
};
constexpr uint32_t kSmallBuildsPerRound = 1024;

struct BuildLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    PinnedBuffer words;  // error, slots, lbvh error
    Request* req = nullptr;
};

// Bytes of the outputs of a build of n triangles with `flags`.
struct BuildOutputs {
    size_t nodes, parents, counts, costs, bounds, obbs, xfs, collapsed, prims, total;
};
BuildOutputs build_outputs(uint32_t n, uint32_t flags) {
    const size_t nn = 2ull * n - 1;
    BuildOutputs o;
    size_t p = 0;
    auto take = [&](size_t b) {
        const size_t at = p;
        p += (b + 255) / 256 * 256;
        return at;
    };
    o.nodes = take(36 * nn);
    o.parents = take(4 * nn);
    o.counts = take(4 * nn);
    o.costs = take(4 * nn);
    o.bounds = take(2 * sizeof(kr_aabb3));
    o.obbs = (flags & OBVH_BUILD_OBBS) ? take(sizeof(kr_obb3) * nn) : 0;
    o.xfs = (flags & OBVH_BUILD_OBBS) ? take(sizeof(kr_mat4) * nn) : 0;
    o.collapsed = (flags & OBVH_BUILD_COLLAPSE) ? take(36 * nn) : 0;
    o.prims = (flags & OBVH_BUILD_COLLAPSE) ? take(4ull * n) : 0;
    o.total = p;
    return o;
}

class Server {
public:
    obvh_server_config cfg{};
    int device = 0;
    char* base = nullptr;
    Arena arena;
    std::mutex m;
    std::condition_variable wake;  // the scheduler
    std::condition_variable done;  // waiting callers
    std::deque<Request*> pending;
    std::vector<Request*> admitted_fits;
    std::vector<Request*> admitted_builds;
    std::vector<Request*> admitted_small;  // builds of 2..runner_max_faces() triangles, for a batch round
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    uint64_t next_id = 1;
    std::vector<FitRound> rounds;
    std::vector<BuildLane> lanes;
    BuildBatchRound brd;
    std::thread worker;
    bool stop = false;
    bool kick = false;       // a submit or a release since the scheduler last looked
    uint64_t in_flight = 0;  // submitted, not yet done or failed
    // statistics
    uint64_t submitted = 0, completed = 0, failed = 0, fits = 0, builds = 0, fit_batches = 0, build_batches = 0;
    std::vector<float> latencies;
    Clock::time_point first_submit{}, last_done{};
    kr_error fatal = nullptr;

    ~Server() {
        {
            std::lock_guard<std::mutex> lock(m);
            stop = true;
        }
        wake.notify_all();
        if (worker.joinable()) worker.join();
        for (FitRound& r : rounds) {
            if (r.batch) dito_batch::free_batch(r.batch);
            if (r.done) cudaEventDestroy(r.done);
            if (r.stream) cudaStreamDestroy(r.stream);
            r.out.release();
            r.host_out.release();
            r.word.release();
        }
        for (BuildLane& l : lanes) {
            if (l.done) cudaEventDestroy(l.done);
            if (l.stream) cudaStreamDestroy(l.stream);
            l.words.release();
        }
        if (brd.runner) meshbatch::free_runner(brd.runner);
        if (brd.done) cudaEventDestroy(brd.done);
        if (brd.stream) cudaStreamDestroy(brd.stream);
        brd.words.release();
        if (base) cudaFree(base);
    }

    kr_error start() {
        OBVH_TRY_CUDA(cudaGetDevice(&device));
        OBVH_TRY_CUDA(cudaMalloc(&base, cfg.hbm_budget_bytes));
        arena.init(cfg.hbm_budget_bytes);
        rounds.resize(2);
        for (FitRound& r : rounds) {
            OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
            OBVH_TRY_CUDA(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
            r.batch = dito_batch::make_batch(cfg.fit_flags, nullptr);
            if (!r.batch) return "obvh_server: out of host memory";
            OBVH_TRY(r.out.reserve(sizeof(kr_obb3) * cfg.max_batch_sets));
            OBVH_TRY(r.host_out.reserve(sizeof(kr_obb3) * cfg.max_batch_sets));
            OBVH_TRY(r.word.reserve(16));
        }
        lanes.resize(cfg.build_lanes);
        for (BuildLane& l : lanes) {
            OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking));
            OBVH_TRY_CUDA(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming));
            OBVH_TRY(l.words.reserve(16));
        }
        OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&brd.stream, cudaStreamNonBlocking));
        OBVH_TRY_CUDA(cudaEventCreateWithFlags(&brd.done, cudaEventDisableTiming));
        OBVH_TRY(meshbatch::make_runner(kSmallBuildsPerRound, &brd.runner));
        OBVH_TRY(brd.words.reserve(4ull * (2 + kSmallBuildsPerRound)));
        worker = std::thread([this] { loop(); });
        return kr_success;
    }

    // ---- submission (callers' threads) ----
    kr_error submit(std::unique_ptr<Request> r, uint64_t* id) {
        std::lock_guard<std::mutex> lock(m);
        if (stop) return "obvh_server: shutting down";
        if (fatal) return fatal;
        r->id = next_id++;
        r->t_submit = Clock::now();
        if (submitted == 0) first_submit = r->t_submit;
        ++submitted;
        ++in_flight;
        if (r->kind == Kind::Fit) ++fits; else ++builds;
        *id = r->id;
        pending.push_back(r.get());
        all.emplace(r->id, std::move(r));
        kick = true;
        wake.notify_one();
        return kr_success;
    }

    // ---- scheduler ----
    size_t fit_input_bytes(const Request& r) const { return r.device_input ? 0 : 12 * r.count; }

    void finish(Request* r, kr_error e) {  // under the lock
        r->t_done = Clock::now();
        last_done = r->t_done;
        r->error = e;
        r->state = e ? State::Failed : State::Done;
        if (e) {
            ++failed;
        } else {
            ++completed;
            latencies.push_back(std::chrono::duration<float, std::milli>(r->t_done - r->t_submit).count());
        }
        --in_flight;
    }

    void free_block(Block& b) {  // under the lock
        if (b.live) arena.release(b.off, b.bytes);
        b.live = false;
    }

    bool take_block(Block& b, size_t bytes) {  // under the lock
        if (bytes == 0) return true;
        size_t off = 0;
        if (!arena.alloc(bytes, &off)) return false;
        b.off = off;
        b.bytes = bytes;
        b.live = true;
        return true;
    }

    // Admission in arrival order (under the lock).
    void admit() {
        size_t free_lanes = 0;
        for (const BuildLane& l : lanes) free_lanes += l.req == nullptr;
        free_lanes = free_lanes > admitted_builds.size() ? free_lanes - admitted_builds.size() : 0;
        for (auto it = pending.begin(); it != pending.end();) {
            Request* r = *it;
            if (r->kind == Kind::Fit) {
                const size_t need = Arena::round(fit_input_bytes(*r));
                if (need > arena.size()) {
                    finish(r, "obvh_server: the fit needs more device memory than the budget");
                    it = pending.erase(it);
                    continue;
                }
                if (!take_block(r->input, fit_input_bytes(*r))) break;  // wait for memory
                r->state = State::Admitted;
                admitted_fits.push_back(r);
                it = pending.erase(it);
                continue;
            }
            // build
            const BuildOutputs o = build_outputs(r->nfaces, r->flags);
            const size_t in_bytes = r->device_input ? 0 : (12 * r->nverts + 255) / 256 * 256 + 16ull * r->nfaces;
            const size_t ws = obvh_build_workspace_bytes(r->nfaces);
            if (Arena::round(in_bytes) + Arena::round(o.total) + Arena::round(ws) > arena.size()) {
                finish(r, "obvh_server: the build needs more device memory than the budget");
                it = pending.erase(it);
                continue;
            }
            if (r->nfaces >= 2 && r->nfaces <= meshbatch::runner_max_faces()) {
                // a small build: the next batch round builds it, with the
                // round's own scratch
                Block in, out;
                if (!take_block(in, in_bytes)) break;
                if (!take_block(out, o.total)) {
                    free_block(in);
                    break;
                }
                r->input = in;
                r->output = out;
                r->state = State::Admitted;
                admitted_small.push_back(r);
                it = pending.erase(it);
                continue;
            }
            if (free_lanes == 0) {  // memory may be there; let fits behind pass
                ++it;
                continue;
            }
            Block in, out, scratch;
            if (!take_block(in, in_bytes)) break;
            if (!take_block(out, o.total)) {
                free_block(in);
                break;
            }
            if (!take_block(scratch, ws)) {
                free_block(in);
                free_block(out);
                break;
            }
            r->input = in;
            r->output = out;
            r->scratch = scratch;
            r->state = State::Admitted;
            admitted_builds.push_back(r);
            --free_lanes;
            it = pending.erase(it);
        }
    }

    // Retire finished rounds and lanes (under the lock).
    void retire() {
        if (brd.busy && cudaEventQuery(brd.done) != cudaErrorNotReady) {
            const cudaError_t e = cudaEventQuery(brd.done);
            const uint32_t* w = static_cast<const uint32_t*>(brd.words.ptr);
            const kr_error ke = e != cudaSuccess ? cuda_error(e) : (w[0] ? "obvh_server: device error in a build" : nullptr);
            for (size_t i = 0; i < brd.reqs.size(); ++i) {
                Request* r = brd.reqs[i];
                r->view.primitive_slots = w[2 + i];
                free_block(r->input);
                if (ke) free_block(r->output);
                finish(r, ke);
            }
            brd.reqs.clear();
            brd.busy = false;
        }
        for (FitRound& rd : rounds) {
            if (!rd.busy || cudaEventQuery(rd.done) == cudaErrorNotReady) continue;
            const cudaError_t e = cudaEventQuery(rd.done);
            const kr_obb3* res = static_cast<const kr_obb3*>(rd.host_out.ptr);
            const uint32_t dev_err = *static_cast<const uint32_t*>(rd.word.ptr);
            const kr_error ke = e != cudaSuccess ? cuda_error(e)
                                : (dev_err ? "obvh_server: device error in a fit batch (wait timed out or input not finite)"
                                           : kr_success);
            for (size_t i = 0; i < rd.reqs.size(); ++i) {
                Request* r = rd.reqs[i];
                r->obb = res[i];
                free_block(r->input);
                finish(r, ke);
            }
            rd.reqs.clear();
            rd.busy = false;
        }
        for (BuildLane& l : lanes) {
            if (!l.req || cudaEventQuery(l.done) == cudaErrorNotReady) continue;
            const cudaError_t e = cudaEventQuery(l.done);
            Request* r = l.req;
            const uint32_t* w = static_cast<const uint32_t*>(l.words.ptr);
            r->view.primitive_slots = w[1];
            free_block(r->input);
            free_block(r->scratch);
            kr_error ke = e != cudaSuccess ? cuda_error(e) : ((w[0] | w[2]) ? "obvh_server: device error in a build" : nullptr);
            if (ke) free_block(r->output);
            finish(r, ke);
            l.req = nullptr;
        }
    }

    // Launch what was admitted (CUDA calls; the lock is not held).
    void launch_fits(FitRound& rd, std::vector<Request*>& batch) {
        const float* fbase = reinterpret_cast<const float*>(base);
        std::vector<int64_t> first(batch.size());
        std::vector<uint64_t> count(batch.size());
        kr_error e = kr_success;
        for (size_t i = 0; i < batch.size() && !e; ++i) {
            Request* r = batch[i];
            const float* src;
            if (r->device_input) {
                src = reinterpret_cast<const float*>(r->points);
            } else {
                src = reinterpret_cast<const float*>(base + r->input.off);
                if (r->count) {
                    const cudaError_t ce = cudaMemcpyAsync(base + r->input.off, r->points, 12 * r->count,
                                                           cudaMemcpyHostToDevice, rd.stream);
                    if (ce != cudaSuccess) e = cuda_error(ce);
                }
            }
            first[i] = static_cast<int64_t>(src - fbase);
            count[i] = r->count;
        }
        if (!e) e = dito_batch::replan(*rd.batch, first.data(), count.data(), batch.size(), rd.stream);
        if (!e) e = dito_batch::enqueue(*rd.batch, reinterpret_cast<const kr_vec3*>(base),
                                        static_cast<kr_obb3*>(rd.out.ptr), rd.stream);
        if (!e) {
            const cudaError_t ce = cudaMemcpyAsync(rd.host_out.ptr, rd.out.ptr, sizeof(kr_obb3) * batch.size(),
                                                   cudaMemcpyDeviceToHost, rd.stream);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        if (!e) e = dito_batch::enqueue_status(*rd.batch, static_cast<uint32_t*>(rd.word.ptr), rd.stream);
        if (!e) {
            const cudaError_t ce = cudaEventRecord(rd.done, rd.stream);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        std::lock_guard<std::mutex> lock(m);
        ++fit_batches;
        if (e) {
            // nothing was queued that reads the inputs beyond this point; wait for what was
            cudaStreamSynchronize(rd.stream);
            for (Request* r : batch) {
                free_block(r->input);
                finish(r, e);
            }
            rd.busy = false;
            done.notify_all();
            return;
        }
        rd.reqs = batch;
        for (Request* r : batch) r->state = State::Running;
    }

    // A build's inputs on the device (copied in on `s` from host memory) and
    // its output view over its output block.
    kr_error stage_build(Request* r, cudaStream_t s, const kr_vec3** dv, const kr_uvec4** df) {
        const BuildOutputs o = build_outputs(r->nfaces, r->flags);
        char* out = base + r->output.off;
        *dv = r->verts;
        *df = r->faces;
        kr_error e = kr_success;
        if (!r->device_input) {
            char* in = base + r->input.off;
            kr_vec3* v = reinterpret_cast<kr_vec3*>(in);
            kr_uvec4* f = reinterpret_cast<kr_uvec4*>(in + (12 * r->nverts + 255) / 256 * 256);
            cudaError_t ce = cudaMemcpyAsync(v, r->verts, 12 * r->nverts, cudaMemcpyHostToDevice, s);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(f, r->faces, 16ull * r->nfaces, cudaMemcpyHostToDevice, s);
            if (ce != cudaSuccess) e = cuda_error(ce);
            *dv = v;
            *df = f;
        }
        obvh_server_build_view& vw = r->view;
        vw.nodes = reinterpret_cast<kr_bvh_node*>(out + o.nodes);
        vw.parents = reinterpret_cast<kr_u32*>(out + o.parents);
        vw.primitive_counts = reinterpret_cast<kr_u32*>(out + o.counts);
        vw.costs = reinterpret_cast<kr_scalar*>(out + o.costs);
        vw.bounds = reinterpret_cast<kr_aabb3*>(out + o.bounds);
        vw.obbs = (r->flags & OBVH_BUILD_OBBS) ? reinterpret_cast<kr_obb3*>(out + o.obbs) : nullptr;
        vw.transforms = (r->flags & OBVH_BUILD_OBBS) ? reinterpret_cast<kr_mat4*>(out + o.xfs) : nullptr;
        vw.collapsed = (r->flags & OBVH_BUILD_COLLAPSE) ? reinterpret_cast<kr_bvh_node*>(out + o.collapsed) : nullptr;
        vw.primitives = (r->flags & OBVH_BUILD_COLLAPSE) ? reinterpret_cast<kr_u32*>(out + o.prims) : nullptr;
        vw.face_count = r->nfaces;
        return e;
    }

    // The small builds of a batch round, one launch for all of them.
    void launch_small_builds(std::vector<Request*>& batch) {
        std::vector<meshbatch::JobBases> bases(batch.size());
        std::vector<uint32_t> faces(batch.size());
        kr_error e = kr_success;
        for (size_t i = 0; i < batch.size() && !e; ++i) {
            Request* r = batch[i];
            const kr_vec3* dv = nullptr;
            const kr_uvec4* df = nullptr;
            e = stage_build(r, brd.stream, &dv, &df);
            const obvh_server_build_view& vw = r->view;
            bases[i] = meshbatch::JobBases{dv, reinterpret_cast<const uint4*>(df), vw.nodes, vw.parents,
                                           vw.primitive_counts, vw.costs, vw.bounds, vw.obbs, vw.transforms,
                                           vw.collapsed, vw.primitives, r->ci, r->ct};
            faces[i] = r->nfaces;
        }
        const uint32_t k = static_cast<uint32_t>(batch.size());
        if (!e) e = meshbatch::run(*brd.runner, bases.data(), faces.data(), k, brd.stream);
        if (!e) {
            cudaError_t ce = cudaMemcpyAsync(brd.words.ptr, meshbatch::status(*brd.runner), 4ull * (2 + k),
                                             cudaMemcpyDeviceToHost, brd.stream);
            if (ce == cudaSuccess) ce = cudaEventRecord(brd.done, brd.stream);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        std::lock_guard<std::mutex> lock(m);
        ++build_batches;
        if (e) {
            cudaStreamSynchronize(brd.stream);
            for (Request* r : batch) {
                free_block(r->input);
                free_block(r->output);
                finish(r, e);
            }
            brd.busy = false;
            done.notify_all();
            return;
        }
        brd.reqs = batch;
        for (Request* r : batch) r->state = State::Running;
    }

    void launch_build(BuildLane& l, Request* r) {
        const kr_vec3* dv = nullptr;
        const kr_uvec4* df = nullptr;
        kr_error e = stage_build(r, l.stream, &dv, &df);
        obvh_server_build_view& vw = r->view;
        void* ws = base + r->scratch.off;
        if (!e) e = obvh_build_workspace_init(ws, r->nfaces, l.stream);
        if (!e)
            e = obvh_build_async(dv, df, r->nfaces, r->flags, r->ci, r->ct, vw.nodes, vw.parents, vw.primitive_counts,
                                 vw.costs, vw.bounds, vw.obbs, vw.transforms, vw.collapsed, vw.primitives, ws, l.stream);
        if (!e) {
            const pipeline::StatusWords sw = pipeline::status_words(r->nfaces);
            uint32_t* w = static_cast<uint32_t*>(l.words.ptr);
            const char* wsb = static_cast<const char*>(ws);
            cudaError_t ce = cudaMemcpyAsync(w + 0, wsb + sw.error, 4, cudaMemcpyDeviceToHost, l.stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(w + 1, wsb + sw.slots, 4, cudaMemcpyDeviceToHost, l.stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(w + 2, wsb + sw.lbvh_error, 4, cudaMemcpyDeviceToHost, l.stream);
            if (ce == cudaSuccess) ce = cudaEventRecord(l.done, l.stream);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        std::lock_guard<std::mutex> lock(m);
        if (e) {
            cudaStreamSynchronize(l.stream);
            free_block(r->input);
            free_block(r->scratch);
            free_block(r->output);
            finish(r, e);
            l.req = nullptr;
            done.notify_all();
            return;
        }
        r->state = State::Running;
    }

    void loop() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lock(m);
        for (;;) {
            kick = false;
            retire();
            if (!stop) admit();
            done.notify_all();
            // pick work to launch
            FitRound* rd = nullptr;
            std::vector<Request*> batch;
            if (!admitted_fits.empty()) {
                for (FitRound& r : rounds)
                    if (!r.busy) {
                        rd = &r;
                        break;
                    }
                if (rd) {
                    const size_t k = std::min<size_t>(admitted_fits.size(), cfg.max_batch_sets);
                    batch.assign(admitted_fits.begin(), admitted_fits.begin() + k);
                    admitted_fits.erase(admitted_fits.begin(), admitted_fits.begin() + k);
                    rd->busy = true;
                }
            }
            std::vector<Request*> small;
            if (!brd.busy && !admitted_small.empty()) {
                const size_t k = std::min<size_t>(admitted_small.size(), kSmallBuildsPerRound);
                small.insert(small.end(), admitted_small.begin(), admitted_small.begin() + k);
                admitted_small.erase(admitted_small.begin(), admitted_small.begin() + k);
                brd.busy = true;
            }
            std::vector<std::pair<BuildLane*, Request*>> starts;
            for (BuildLane& l : lanes) {
                if (admitted_builds.empty()) break;
                if (l.req) continue;
                l.req = admitted_builds.front();
                admitted_builds.erase(admitted_builds.begin());
                starts.emplace_back(&l, l.req);
            }
            const bool busy = std::any_of(rounds.begin(), rounds.end(), [](const FitRound& r) { return r.busy; }) ||
                              std::any_of(lanes.begin(), lanes.end(), [](const BuildLane& l) { return l.req; }) ||
                              brd.busy;
            if (rd || !starts.empty() || !small.empty()) {
                lock.unlock();
                if (rd) launch_fits(*rd, batch);
                if (!small.empty()) launch_small_builds(small);
                for (auto& sl : starts) launch_build(*sl.first, sl.second);
                lock.lock();
                continue;
            }
            if (stop) {  // nothing new is admitted once stopping: fail what still waits
                for (Request* r : pending) finish(r, "obvh_server: shut down before the request was admitted");
                pending.clear();
                done.notify_all();
                if (!busy && admitted_fits.empty() && admitted_builds.empty() && admitted_small.empty()) break;
            }
            if (busy) {
                wake.wait_for(lock, std::chrono::microseconds(20));
            } else {
                // nothing runs and nothing more can be admitted until a submit,
                // a release or a stop (the wait releases the lock)
                wake.wait(lock, [&] { return stop || kick; });
            }
        }
    }

    Request* find(uint64_t id) {
        auto it = all.find(id);
        return it == all.end() ? nullptr : it->second.get();
    }
};

}  // namespace server
}  // namespace obvh

using obvh::server::Kind;
using obvh::server::Request;
using obvh::server::Server;
using obvh::server::State;

struct obvh_server_s {
    Server s;
};

namespace {
kr_error fail(kr_error e) {
    obvh::set_last_error(e);
    return e;
}
}  // namespace

extern "C" kr_error obvh_server_create(const obvh_server_config* config, obvh_server* out) {
    if (!out) return fail("obvh_server_create: null output handle");
    *out = nullptr;
    obvh_server_s* h = new (std::nothrow) obvh_server_s();
    if (!h) return fail("obvh_server_create: out of host memory");
    obvh_server_config c{};
    if (config) c = *config;
    if (c.hbm_budget_bytes == 0) c.hbm_budget_bytes = 120ull << 30;
    if (c.build_lanes == 0) c.build_lanes = 4;
    if (c.max_batch_sets == 0) c.max_batch_sets = 8192;
    if (c.build_lanes > 64) return fail("obvh_server_create: at most 64 build lanes");
    h->s.cfg = c;
    kr_error e = h->s.start();
    if (e) {
        delete h;
        return fail(e);
    }
    *out = h;
    return kr_success;
}

extern "C" kr_error obvh_server_destroy(obvh_server server) {
    delete server;
    return kr_success;
}

extern "C" kr_error obvh_server_submit_fit(obvh_server server, const kr_vec3* points, kr_size count, kr_u64* id) {
    if (!server || !id || (count && !points)) return fail("obvh_server_submit_fit: null argument");
    if (count >= (1ull << 32) - 4) return fail("obvh_server_submit_fit: 2^32 points or more");
    auto r = std::make_unique<Request>();
    r->kind = Kind::Fit;
    r->points = points;
    r->count = count;
    kr_error e = server->s.submit(std::move(r), id);
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_server_submit_fit_device(obvh_server server, const kr_vec3* d_points, kr_size count,
                                                  kr_u64* id) {
    if (!server || !id || (count && !d_points)) return fail("obvh_server_submit_fit_device: null argument");
    if (reinterpret_cast<uintptr_t>(d_points) & 3u) return fail("obvh_server_submit_fit_device: points not 4-byte aligned");
    if (count >= (1ull << 32) - 4) return fail("obvh_server_submit_fit_device: 2^32 points or more");
    auto r = std::make_unique<Request>();
    r->kind = Kind::Fit;
    r->device_input = true;
    r->points = d_points;
    r->count = count;
    kr_error e = server->s.submit(std::move(r), id);
    return e ? fail(e) : kr_success;
}

namespace {
kr_error submit_build(obvh_server server, const kr_vec3* v, kr_size nv, const kr_uvec4* f, kr_u32 nf, kr_u32 flags,
                      kr_scalar ci, kr_scalar ct, bool device, kr_u64* id) {
    if (!server || !id || !v || !f) return fail("obvh_server_submit_build: null argument");
    if (nf == 0) return fail("obvh_server_submit_build: no faces");
    if (nf > (1u << 30)) return fail("obvh_server_submit_build: more than 2^30 faces");
    if (!device)
        for (kr_u32 i = 0; i < nf; ++i)
            for (int k = 0; k < 3; ++k)
                if (f[i].v[k] >= nv) return fail("obvh_server_submit_build: a face indexes past the vertex array");
    auto r = std::make_unique<Request>();
    r->kind = Kind::Build;
    r->device_input = device;
    r->verts = v;
    r->nverts = nv;
    r->faces = f;
    r->nfaces = nf;
    r->flags = flags & (OBVH_BUILD_OBBS | OBVH_BUILD_COLLAPSE);
    r->ci = ci;
    r->ct = ct;
    kr_error e = server->s.submit(std::move(r), id);
    return e ? fail(e) : kr_success;
}
}  // namespace

extern "C" kr_error obvh_server_submit_build(obvh_server server, const kr_vec3* vertices, kr_size vertex_count,
                                             const kr_uvec4* faces, kr_u32 face_count, kr_u32 flags, kr_scalar ci,
                                             kr_scalar ct, kr_u64* id) {
    return submit_build(server, vertices, vertex_count, faces, face_count, flags, ci, ct, false, id);
}

extern "C" kr_error obvh_server_submit_build_device(obvh_server server, const kr_vec3* d_vertices,
                                                    kr_size vertex_count, const kr_uvec4* d_faces, kr_u32 face_count,
                                                    kr_u32 flags, kr_scalar ci, kr_scalar ct, kr_u64* id) {
    return submit_build(server, d_vertices, vertex_count, d_faces, face_count, flags, ci, ct, true, id);
}

extern "C" kr_error obvh_server_wait(obvh_server server, kr_u64 id, kr_u32 timeout_ms, kr_u32* done) {
    if (!server || !done) return fail("obvh_server_wait: null argument");
    Server& s = server->s;
    std::unique_lock<std::mutex> lock(s.m);
    Request* r = s.find(id);
    if (!r) return fail("obvh_server_wait: unknown request");
    auto ready = [&] { return r->state == State::Done || r->state == State::Failed; };
    if (timeout_ms) s.done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready);
    *done = ready() ? 1u : 0u;
    if (r->state == State::Failed) return fail(r->error);
    return kr_success;
}

extern "C" kr_error obvh_server_drain(obvh_server server, kr_u32 timeout_ms, kr_u32* done) {
    if (!server || !done) return fail("obvh_server_drain: null argument");
    Server& s = server->s;
    std::unique_lock<std::mutex> lock(s.m);
    *done = s.done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return s.in_flight == 0; }) ? 1u : 0u;
    return kr_success;
}

extern "C" kr_error obvh_server_fit_result(obvh_server server, kr_u64 id, kr_obb3* obb) {
    if (!server || !obb) return fail("obvh_server_fit_result: null argument");
    Server& s = server->s;
    std::lock_guard<std::mutex> lock(s.m);
    Request* r = s.find(id);
    if (!r || r->kind != Kind::Fit) return fail("obvh_server_fit_result: unknown fit request");
    if (r->state == State::Failed) return fail(r->error);
    if (r->state != State::Done) return fail("obvh_server_fit_result: not done yet");
    *obb = r->obb;
    return kr_success;
}

extern "C" kr_error obvh_server_build_result(obvh_server server, kr_u64 id, obvh_server_build_view* view) {
    if (!server || !view) return fail("obvh_server_build_result: null argument");
    Server& s = server->s;
    std::lock_guard<std::mutex> lock(s.m);
    Request* r = s.find(id);
    if (!r || r->kind != Kind::Build) return fail("obvh_server_build_result: unknown build request");
    if (r->state == State::Failed) return fail(r->error);
    if (r->state != State::Done) return fail("obvh_server_build_result: not done yet");
    *view = r->view;
    return kr_success;
}

extern "C" kr_error obvh_server_latency(obvh_server server, kr_u64 id, kr_scalar* ms) {
    if (!server || !ms) return fail("obvh_server_latency: null argument");
    Server& s = server->s;
    std::lock_guard<std::mutex> lock(s.m);
    Request* r = s.find(id);
    if (!r) return fail("obvh_server_latency: unknown request");
    if (r->state != State::Done) return fail("obvh_server_latency: not done");
    *ms = std::chrono::duration<float, std::milli>(r->t_done - r->t_submit).count();
    return kr_success;
}

extern "C" kr_error obvh_server_release(obvh_server server, kr_u64 id) {
    if (!server) return fail("obvh_server_release: null server");
    Server& s = server->s;
    std::lock_guard<std::mutex> lock(s.m);
    Request* r = s.find(id);
    if (!r) return fail("obvh_server_release: unknown request");
    if (r->state != State::Done && r->state != State::Failed) return fail("obvh_server_release: still in flight");
    s.free_block(r->input);
    s.free_block(r->output);
    s.free_block(r->scratch);
    s.all.erase(id);
    s.kick = true;
    s.wake.notify_one();  // memory came back: admission may proceed
    return kr_success;
}

extern "C" kr_error obvh_server_get_stats(obvh_server server, obvh_server_stats* st) {
    if (!server || !st) return fail("obvh_server_get_stats: null argument");
    Server& s = server->s;
    std::lock_guard<std::mutex> lock(s.m);
    obvh_server_stats o{};
    o.submitted = s.submitted;
    o.completed = s.completed;
    o.failed = s.failed;
    o.fits = s.fits;
    o.builds = s.builds;
    o.fit_batches = s.fit_batches;
    o.build_batches = s.build_batches;
    std::vector<float> l = s.latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const size_t k = static_cast<size_t>(q * (l.size() - 1) + 0.5);
            return l[std::min(k, l.size() - 1)];
        };
        o.p50_ms = pct(0.50);
        o.p99_ms = pct(0.99);
        double sum = 0;
        for (float x : l) sum += x;
        o.mean_ms = static_cast<kr_scalar>(sum / l.size());
        o.max_ms = l.back();
    }
    o.arena_bytes = s.arena.size();
    o.peak_bytes = s.arena.peak();
    o.in_use_bytes = s.arena.used();
    if (s.completed + s.failed > 0)
        o.span_s = std::chrono::duration<float>(s.last_done - s.first_submit).count();
    *st = o;
    return kr_success;
}
