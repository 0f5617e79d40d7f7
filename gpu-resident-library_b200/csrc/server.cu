// Continuous-batching server (server.hpp) and its extern "C" entry points
// (gpufhe_server_*, include/gpufhe_b200.h). The reference has no serving
// loop: its multi-ciphertext driver runs independent chains on separate
// streams (bench/bench_batch.cpp:95-105).
#include "server.hpp"

#include <algorithm>
#include <stdexcept>
#include <string>
#include <thread>

#include "gpufhe_b200.h"

namespace srv {

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr size_t GRANULE = 256;
size_t round_up(size_t x) { return (x + GRANULE - 1) & ~(GRANULE - 1); }

// SplitMix64 (Steele, Lea, Flood: "Fast splittable pseudorandom number
// generators", OOPSLA 2014): the output of a counter-indexed stream.
__host__ __device__ inline uint64_t splitmix64(uint64_t seed, uint64_t ctr) {
    uint64_t z = seed + (ctr + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Seeded residues: word i of tower t of component c is
// floor(splitmix64(seed, c<<40 | t<<24 | i) * q_t / 2^64), a value in [0, q_t)
// that depends only on (seed, c, t, i), not on what else runs.
__global__ void k_seed_fill(u64* __restrict__ c0, u64* __restrict__ c1, const ModC* __restrict__ mod, uint32_t L,
                            uint32_t n, uint64_t seed) {
    const size_t total = (size_t)2 * L * n;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const uint32_t comp = (uint32_t)(k / ((size_t)L * n));
        const size_t rem = k - (size_t)comp * L * n;
        const uint32_t t = (uint32_t)(rem / n), i = (uint32_t)(rem - (size_t)t * n);
        const uint64_t x = splitmix64(seed, ((uint64_t)comp << 40) | ((uint64_t)t << 24) | i);
        (comp ? c1 : c0)[rem] = __umul64hi(x, mod[t].q);
    }
}

}  // namespace

// ---------------------------------------------------------------- Arena

Arena::Arena(size_t bytes) {
    cap_ = bytes & ~(GRANULE - 1);
    if (cap_ == 0) throw std::invalid_argument("server arena: budget leaves no room for requests");
    void* p = nullptr;
    if (cudaMalloc(&p, cap_) != cudaSuccess) {
        cudaGetLastError();
        throw std::length_error("server arena: cudaMalloc of " + std::to_string(cap_) + " bytes failed");
    }
    base_ = static_cast<u64*>(p);
    free_[0] = cap_;
}

Arena::~Arena() {
    if (base_) cudaFree(base_);
}

bool Arena::alloc(size_t bytes, size_t& off) {
    bytes = round_up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < bytes) continue;
        off = it->first;
        const size_t left = it->second - bytes;
        free_.erase(it);
        if (left) free_[off + bytes] = left;
        used_ += bytes;
        return true;
    }
    return false;
}

void Arena::release(size_t off, size_t bytes) {
    bytes = round_up(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        free_.erase(nx);
    }
    if (it != free_.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            free_.erase(it);
        }
    }
}

// ---------------------------------------------------------------- Server

Server::Server(const std::vector<gfx::Context*>& ctxs, size_t budget_bytes, uint32_t max_active, uint32_t batch_cap,
               bool plain)
    : ctxs_(ctxs), max_active_(max_active), batch_cap_(batch_cap), plain_(plain) {
    if (ctxs_.empty()) throw std::invalid_argument("server: no contexts");
    device_ = ctxs_[0]->device();
    size_t resident = 0;
    for (auto* c : ctxs_) {
        if (!c) throw std::invalid_argument("server: null context");
        if (c->device() != device_) throw std::invalid_argument("server: contexts on different devices");
        if (!pl::supported_logn((int)c->logn())) throw std::invalid_argument("server: ring size outside 2^10..2^16");
        resident += c->resident_bytes();
    }
    ck(cudaSetDevice(device_), "cudaSetDevice");
    st_.resident_bytes = resident;
    if (budget_bytes <= resident) throw std::invalid_argument("server: HBM budget below the resident tables and keys");
    arena_ = std::make_unique<Arena>(budget_bytes - resident);
    st_.arena_bytes = arena_->capacity();
    streams_.resize(ctxs_.size());
    for (auto& s : streams_) ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    for (size_t i = 0; i < 2 * ctxs_.size(); ++i) {
        plans_.push_back(std::make_unique<pl::Plan>());
        plans_.back()->concurrent = true;   // the rings' steps run side by side on their streams
    }
    ck(cudaEventCreate(&epoch_ev_), "cudaEventCreate");
    epoch_ = std::chrono::steady_clock::now();
    for (auto* c : ctxs_) c->hold();       // the contexts outlive the server
}

Server::~Server() {
    cudaSetDevice(device_);
    for (auto s : streams_) cudaStreamSynchronize(s);
    for (auto& f : inflight_)
        for (auto e : f.ev) cudaEventDestroy(e);
    for (auto e : ev_pool_) cudaEventDestroy(e);
    if (epoch_ev_) cudaEventDestroy(epoch_ev_);
    plans_.clear();
    for (auto s : streams_) cudaStreamDestroy(s);
    for (auto* c : ctxs_) gfx::Context::drop(c);
}

uint32_t Server::final_level(uint32_t level, const std::vector<ReqOp>& ops) {
    for (const auto& o : ops)
        if (o.mode == pl::EMR) --level;
    return level;
}

size_t Server::request_bytes(uint32_t ctx, uint32_t level) const {
    const gfx::Context& c = *ctxs_.at(ctx);
    return round_up((size_t)4 * level * c.n() * 8) + round_up(pl::op_workspace_words(c, level) * 8);
}

uint64_t Server::submit(uint32_t ctx, uint32_t level, const std::vector<ReqOp>& ops, double arrival_s, uint64_t seed,
                        const u64* h_in, u64* h_out) {
    if (ctx >= ctxs_.size()) throw std::invalid_argument("submit: context index");
    const gfx::Context& c = *ctxs_[ctx];
    if (level < 1 || level > c.fullQ()) throw std::invalid_argument("submit: level out of range");
    if (ops.empty()) throw std::invalid_argument("submit: empty request");
    uint32_t L = level;
    for (const auto& o : ops) {
        if (o.mode == pl::EMR) {
            if (L < 2) throw std::invalid_argument("submit: EvalMult+Rescale below level 2");
            if (!c.key(0)) throw std::invalid_argument("submit: no relinearisation key");
            --L;
        } else if (o.mode == pl::ROT) {
            if (o.galois % 2 == 0 || o.galois >= 2ull * c.n()) throw std::invalid_argument("submit: bad Galois element");
            if (!c.key(o.galois)) throw std::invalid_argument("submit: no rotation key for this Galois element");
        } else {
            throw std::invalid_argument("submit: request operations are EvalMult+Rescale or rotation");
        }
    }
    if (request_bytes(ctx, level) > arena_->capacity())
        throw std::length_error("submit: request larger than the whole arena");
    auto r = std::make_unique<Request>();
    r->id = next_id_++;
    r->ctx = ctx;
    r->level = r->start_level = level;
    r->seed = seed;
    r->ops = ops;
    r->h_in = h_in;
    r->h_out = h_out;
    r->t_arrival = arrival_s;
    auto pos = std::upper_bound(queue_.begin(), queue_.end(), arrival_s,
                                [](double t, const std::unique_ptr<Request>& q) { return t < q->t_arrival; });
    const uint64_t id = r->id;
    queue_.insert(pos, std::move(r));
    return id;
}

int Server::tune(uint32_t max_batch) {
    ck(cudaSetDevice(device_), "cudaSetDevice");
    if (!inflight_.empty() || !active_.empty())
        throw std::invalid_argument("tune: the server must be idle");
    int tuned = 0;
    for (size_t c = 0; c < ctxs_.size(); ++c) {
        const gfx::Context& ctx = *ctxs_[c];
        cudaStream_t s = streams_[c];
        // batches of EvalMult+Rescale over levels 2..fullQ, one per batch-size class
        for (uint32_t nops = 1; nops <= max_batch; nops *= 2) {
            std::vector<pl::Op> ops(nops);
            std::vector<u64*> ws(nops);
            std::vector<std::pair<size_t, size_t>> held;
            bool fits = true;
            for (uint32_t k = 0; k < nops && fits; ++k) {
                const uint32_t L = 2 + (uint32_t)(((uint64_t)k * 7919u) % (ctx.fullQ() - 1));
                const size_t bytes = request_bytes((uint32_t)c, L);
                size_t off = 0;
                if (!arena_->alloc(bytes, off)) { fits = false; break; }
                held.push_back({off, bytes});
                u64* base = arena_->base() + off / 8;
                const size_t ctw = (size_t)L * ctx.n();
                ck(cudaMemsetAsync(base, 0, 2 * ctw * 8, s), "tune inputs");
                pl::Op& op = ops[k];
                op.L = L;
                op.mode = pl::EMR;
                op.in[0] = op.in[2] = base;
                op.in[1] = op.in[3] = base + ctw;
                op.out[0] = base + 2 * ctw;
                op.out[1] = base + 3 * ctw;
                ws[k] = base + round_up(4 * ctw * 8) / 8;
            }
            if (fits && ctx.key(0)) {
                pl::Plan& plan = *plans_[2 * c];
                pl::build_plan_into(plan, ctx, ops, ws, s);
                pl::tune(plan, s, true);
                ck(cudaStreamSynchronize(s), "tune");
                ++tuned;
            }
            for (auto& h : held) arena_->release(h.first, h.second);
            if (!fits) break;
        }
    }
    return tuned;
}

void Server::start() {
    cudaSetDevice(device_);
    ck(cudaEventRecord(epoch_ev_, streams_[0]), "cudaEventRecord");
    ck(cudaEventSynchronize(epoch_ev_), "cudaEventSynchronize");
    epoch_ = std::chrono::steady_clock::now();
    started_ = true;
}

double Server::now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - epoch_).count();
}

cudaEvent_t Server::get_event() {
    if (!ev_pool_.empty()) {
        cudaEvent_t e = ev_pool_.back();
        ev_pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    ck(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

bool Server::admit(Request& r) {
    const gfx::Context& c = *ctxs_[r.ctx];
    const size_t bytes = request_bytes(r.ctx, r.start_level);
    size_t off = 0;
    if (!arena_->alloc(bytes, off)) return false;
    r.arena_off = off;
    r.arena_bytes = bytes;
    const size_t ctw = (size_t)r.start_level * c.n();
    u64* base = arena_->base() + off / 8;
    r.ct[0][0] = base;
    r.ct[0][1] = base + ctw;
    r.ct[1][0] = base + 2 * ctw;
    r.ct[1][1] = base + 3 * ctw;
    r.ws = base + round_up(4 * ctw * 8) / 8;
    r.cur = 0;
    cudaStream_t s = streams_[r.ctx];
    if (r.h_in) {
        ck(cudaMemcpyAsync(r.ct[0][0], r.h_in, 2 * ctw * 8, cudaMemcpyHostToDevice, s), "request upload");
    } else {
        const unsigned blocks = (unsigned)std::min<size_t>((2 * ctw + 255) / 256, 4 * 148);
        k_seed_fill<<<blocks, 256, 0, s>>>(r.ct[0][0], r.ct[0][1], c.dev().mod, r.start_level, c.n(), r.seed);
        ck(cudaGetLastError(), "seed fill");
    }
    r.t_admit = now();
    if (first_admit_ < 0) first_admit_ = r.t_admit;
    st_.peak_bytes = std::max(st_.peak_bytes, arena_->in_use());
    return true;
}

void Server::retire_oldest() {
    InFlight f = std::move(inflight_.front());
    inflight_.pop_front();
    std::vector<double> t(f.ev.size());
    const auto w0 = std::chrono::steady_clock::now();
    for (size_t k = 0; k < f.ev.size(); ++k) ck(cudaEventSynchronize(f.ev[k]), "step wait");
    st_.host_wait_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    for (size_t k = 0; k < f.ev.size(); ++k) {
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, epoch_ev_, f.ev[k]), "cudaEventElapsedTime");
        t[k] = ms * 1e-3;
    }
    for (Request* r : f.finishing) {
        for (size_t k = 0; k < f.ctxs.size(); ++k)
            if (f.ctxs[k] == (int)r->ctx) r->t_finish = t[k];
        last_finish_ = std::max(last_finish_, r->t_finish);
        arena_->release(r->arena_off, r->arena_bytes);
        ++st_.completed;
    }
    for (auto e : f.ev) ev_pool_.push_back(e);
    // move the finished requests from active_ to done_, keeping order
    if (!f.finishing.empty()) {
        std::vector<std::unique_ptr<Request>> keep;
        keep.reserve(active_.size());
        for (auto& r : active_) {
            if (r->t_finish >= 0) done_.push_back(std::move(r));
            else keep.push_back(std::move(r));
        }
        active_.swap(keep);
    }
    if (first_admit_ >= 0 && last_finish_ >= 0) st_.busy_s = last_finish_ - first_admit_;
}

int Server::step() {
    ck(cudaSetDevice(device_), "cudaSetDevice");
    if (!started_) start();
    // retire what has completed; keep at most one step in flight while building the next
    while (!inflight_.empty()) {
        bool ready = inflight_.size() >= 2;
        if (!ready) {
            ready = true;
            for (auto e : inflight_.front().ev) {
                const cudaError_t q = cudaEventQuery(e);
                if (q == cudaErrorNotReady) { ready = false; break; }
                ck(q, "cudaEventQuery");
            }
        }
        if (!ready) break;
        retire_oldest();
    }
    // FIFO admission of arrived requests while memory (and the active cap) allows
    const double t = now();
    while (!queue_.empty() && queue_.front()->t_arrival <= t) {
        size_t live = 0;
        for (auto& r : active_) live += r->t_finish < 0;
        if (plain_ && (live || !inflight_.empty())) break;
        if (max_active_ && live >= max_active_) break;
        if (!admit(*queue_.front())) break;
        active_.push_back(std::move(queue_.front()));
        queue_.pop_front();
        st_.peak_active = std::max<uint64_t>(st_.peak_active, live + 1);
    }
    // next operation of every admitted request, grouped by context
    const size_t nctx = ctxs_.size();
    std::vector<std::vector<pl::Op>> ops(nctx);
    std::vector<std::vector<u64*>> ws(nctx);
    std::vector<std::vector<Request*>> who(nctx);
    for (auto& rp : active_) {
        Request& r = *rp;
        if (r.next_op >= r.ops.size()) continue;   // all issued, waiting to retire
        if (batch_cap_ && ops[r.ctx].size() >= batch_cap_) continue;
        const ReqOp& ro = r.ops[r.next_op];
        pl::Op op;
        op.L = r.level;
        op.mode = ro.mode;
        const int nx = r.cur ^ 1;
        if (ro.mode == pl::EMR) {
            op.key_id = 0;
            op.in[0] = r.ct[r.cur][0];
            op.in[1] = r.ct[r.cur][1];
            op.in[2] = r.ct[r.cur][0];
            op.in[3] = r.ct[r.cur][1];
        } else {
            op.key_id = ro.galois;
            op.galois = ro.galois;
            op.in[0] = r.ct[r.cur][0];
            op.in[1] = r.ct[r.cur][1];
        }
        op.out[0] = r.ct[nx][0];
        op.out[1] = r.ct[nx][1];
        ops[r.ctx].push_back(op);
        ws[r.ctx].push_back(r.ws);
        who[r.ctx].push_back(&r);
    }
    InFlight f;
    int queued = 0;
    const int slot = (int)(step_no_ & 1);
    const auto b0 = std::chrono::steady_clock::now();
    for (size_t c = 0; c < nctx; ++c) {
        if (ops[c].empty()) continue;
        cudaStream_t s = streams_[c];
        pl::Plan& plan = *plans_[2 * c + slot];
        pl::build_plan_into(plan, *ctxs_[c], ops[c], ws[c], s);
        pl::tune(plan, s, false);   // cached schedule or the default: no timing runs on the serving path
        ck(pl::launch(plan, s), "pipeline launch");
        for (size_t k = 0; k < who[c].size(); ++k) {
            Request& r = *who[c][k];
            const bool emr = ops[c][k].mode == pl::EMR;
            if (emr) { --r.level; ++st_.emr_ops; }
            r.cur ^= 1;
            ++r.next_op;
            if (r.next_op == r.ops.size()) {
                if (r.h_out) {
                    const size_t w = (size_t)r.level * ctxs_[c]->n();
                    ck(cudaMemcpyAsync(r.h_out, r.ct[r.cur][0], w * 8, cudaMemcpyDeviceToHost, s), "result download");
                    ck(cudaMemcpyAsync(r.h_out + w, r.ct[r.cur][1], w * 8, cudaMemcpyDeviceToHost, s),
                       "result download");
                }
                f.finishing.push_back(&r);
            }
        }
        cudaEvent_t e = get_event();
        ck(cudaEventRecord(e, s), "cudaEventRecord");
        f.ctxs.push_back((int)c);
        f.ev.push_back(e);
        queued += (int)ops[c].size();
        st_.max_batch = std::max<uint64_t>(st_.max_batch, ops[c].size());
    }
    st_.host_build_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - b0).count();
    if (queued) {
        inflight_.push_back(std::move(f));
        ++step_no_;
        ++st_.steps;
        st_.ops += queued;
    }
    return queued;
}

bool Server::drain(double max_seconds) {
    if (!started_) start();
    const double t_end = now() + max_seconds;
    while (true) {
        if (now() > t_end) return false;
        if (step() > 0) continue;
        if (!inflight_.empty()) {
            retire_oldest();
            continue;
        }
        if (queue_.empty() && active_.empty()) return true;
        if (!queue_.empty()) {
            const double wait = queue_.front()->t_arrival - now();
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 2e-4)));
        }
    }
}

}  // namespace srv

// ---------------------------------------------------------------- C ABI

gfx::Context* gpufhe_impl(gpufhe_ctx* h);

struct gpufhe_server {
    std::unique_ptr<srv::Server> s;
};

#define GPUFHE_TRY(...)                                                  \
    try { __VA_ARGS__ } catch (const std::invalid_argument& e) {         \
        gfx::set_error(e.what()); return GPUFHE_EINVAL;                  \
    } catch (const std::length_error& e) {                               \
        gfx::set_error(e.what()); return GPUFHE_ENOMEM;                  \
    } catch (const std::exception& e) {                                  \
        gfx::set_error(e.what()); return GPUFHE_ECUDA;                   \
    }

extern "C" {

int gpufhe_server_create(gpufhe_ctx* const* ctxs, uint32_t nctx, uint64_t budget_bytes, uint32_t max_active,
                         uint32_t batch_cap, int plain, gpufhe_server** out) {
    if (!ctxs || !out || !nctx) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        std::vector<gfx::Context*> v(nctx);
        for (uint32_t i = 0; i < nctx; ++i) v[i] = gpufhe_impl(ctxs[i]);
        *out = new gpufhe_server{std::make_unique<srv::Server>(v, budget_bytes, max_active, batch_cap, plain != 0)};
        return GPUFHE_OK;
    })
}

void gpufhe_server_destroy(gpufhe_server* h) { delete h; }

uint64_t gpufhe_server_request_bytes(gpufhe_server* h, uint32_t ctx, uint32_t level) {
    if (!h) return 0;
    try { return h->s->request_bytes(ctx, level); } catch (...) { return 0; }
}

int gpufhe_server_submit(gpufhe_server* h, uint32_t ctx, uint32_t level, const gpufhe_req_op* ops, uint32_t nops,
                         double arrival_s, uint64_t seed, const uint64_t* h_in, uint64_t* h_out, uint64_t* id) {
    if (!h || !ops) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    GPUFHE_TRY({
        std::vector<srv::ReqOp> v(nops);
        for (uint32_t i = 0; i < nops; ++i) v[i] = {ops[i].mode, ops[i].galois};
        const uint64_t r = h->s->submit(ctx, level, v, arrival_s, seed, h_in, h_out);
        if (id) *id = r;
        return GPUFHE_OK;
    })
}

int gpufhe_server_tune(gpufhe_server* h, uint32_t max_batch, uint32_t* tuned) {
    if (!h) return GPUFHE_EINVAL;
    GPUFHE_TRY({
        const int t = h->s->tune(max_batch ? max_batch : 256);
        if (tuned) *tuned = (uint32_t)t;
        return GPUFHE_OK;
    })
}

int gpufhe_server_start(gpufhe_server* h) {
    if (!h) return GPUFHE_EINVAL;
    GPUFHE_TRY({
        h->s->start();
        return GPUFHE_OK;
    })
}

int gpufhe_server_step(gpufhe_server* h, uint32_t* queued) {
    if (!h) return GPUFHE_EINVAL;
    GPUFHE_TRY({
        const int q = h->s->step();
        if (queued) *queued = (uint32_t)q;
        return GPUFHE_OK;
    })
}

int gpufhe_server_drain(gpufhe_server* h, double max_seconds) {
    if (!h) return GPUFHE_EINVAL;
    GPUFHE_TRY({
        if (!h->s->drain(max_seconds)) {
            gfx::set_error("gpufhe_server_drain: requests still pending at the time limit");
            return GPUFHE_ETIMEOUT;
        }
        return GPUFHE_OK;
    })
}

uint64_t gpufhe_server_pending(gpufhe_server* h) { return h ? h->s->pending() : 0; }

int gpufhe_server_get_stats(gpufhe_server* h, gpufhe_server_stats* out) {
    if (!h || !out) return GPUFHE_EINVAL;
    const srv::Stats& s = h->s->stats();
    out->steps = s.steps;
    out->ops = s.ops;
    out->emr_ops = s.emr_ops;
    out->completed = s.completed;
    out->peak_active = s.peak_active;
    out->max_batch = s.max_batch;
    out->peak_bytes = s.peak_bytes;
    out->arena_bytes = s.arena_bytes;
    out->resident_bytes = s.resident_bytes;
    out->busy_s = s.busy_s;
    out->host_build_s = s.host_build_s;
    out->host_wait_s = s.host_wait_s;
    return GPUFHE_OK;
}

int gpufhe_server_records(gpufhe_server* h, gpufhe_request_record* out, uint32_t cap, uint32_t* count) {
    if (!h || !count) return GPUFHE_EINVAL;
    const auto& d = h->s->finished();
    const uint32_t m = (uint32_t)std::min<size_t>(cap, d.size());
    for (uint32_t i = 0; out && i < m; ++i) {
        const srv::Request& r = *d[i];
        out[i].id = r.id;
        out[i].ctx = r.ctx;
        out[i].start_level = r.start_level;
        out[i].final_level = r.level;
        out[i].nops = (uint32_t)r.ops.size();
        out[i].t_arrival = r.t_arrival;
        out[i].t_admit = r.t_admit;
        out[i].t_finish = r.t_finish;
    }
    *count = (uint32_t)d.size();
    return GPUFHE_OK;
}

}  // extern "C"
