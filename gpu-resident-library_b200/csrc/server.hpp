// Continuous-batching server for encrypted requests of mixed ring size and
// level. A request is a chain of operations (EvalMult+Rescale of its
// ciphertext with itself, or a rotation) on one resident ciphertext. Every
// step takes the next operation of every admitted request, groups them by
// context (ring size), and launches one batched plan per context on that
// context's stream. Two steps stay in flight: the host builds and queues step
// s+1 while the GPU runs step s (a request's next operation follows its
// previous one on the same stream), so a request that arrives while others
// run is admitted as soon as arena memory frees up and joins the next step.
//
// Memory for a request (two ping-pong ciphertexts at its start level plus its
// pipeline workspace) comes from one device arena sized by the HBM budget
// minus every resident byte of the contexts (tables and keys); admission is
// FIFO and stops at the first arrived request that does not fit. The memory
// of a finished request returns to the arena only after the step that
// finished it has completed on the GPU.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "context.hpp"
#include "pipeline.hpp"

namespace srv {

struct ReqOp {
    uint32_t mode;     // pl::EMR or pl::ROT
    uint64_t galois;   // ROT: Galois element, also the rotation key's id
};

struct Request {
    uint64_t id = 0;
    uint32_t ctx = 0;
    uint32_t level = 0;          // level after the operations issued so far
    uint32_t start_level = 0;
    uint64_t seed = 0;
    std::vector<ReqOp> ops;
    const u64* h_in = nullptr;   // host input [2][start_level][n], or null: seeded fill on the device
    u64* h_out = nullptr;        // host result [2][final level][n], or null
    // seconds since the server epoch; t_finish is the device time at which
    // the step holding the request's last operation completed
    double t_arrival = 0, t_admit = -1, t_finish = -1;
    size_t arena_off = 0, arena_bytes = 0;
    u64* ct[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [buffer][component]
    u64* ws = nullptr;
    int cur = 0;                 // buffer holding the current ciphertext
    uint32_t next_op = 0;        // operations issued so far
};

// First-fit sub-allocator (256-byte granules) over one device allocation.
class Arena {
public:
    explicit Arena(size_t bytes);
    ~Arena();
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;
    bool alloc(size_t bytes, size_t& off);
    void release(size_t off, size_t bytes);
    u64* base() const { return base_; }
    size_t capacity() const { return cap_; }
    size_t in_use() const { return used_; }
private:
    u64* base_ = nullptr;
    size_t cap_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;   // offset -> size, coalesced
};

struct Stats {
    uint64_t steps = 0;          // steps that launched work
    uint64_t ops = 0;            // operations executed
    uint64_t emr_ops = 0;        // of which EvalMult+Rescale
    uint64_t completed = 0;      // requests finished
    uint64_t peak_active = 0;    // most requests admitted at once
    uint64_t max_batch = 0;      // most operations in one plan
    size_t peak_bytes = 0;       // most arena bytes in use
    size_t arena_bytes = 0;      // arena capacity
    size_t resident_bytes = 0;   // tables + keys of every context
    double busy_s = 0;           // first admission to last completion
    double host_build_s = 0;     // host time building and launching steps
    double host_wait_s = 0;      // host time blocked on a step still running on the GPU
};

class Server {
public:
    // Contexts are borrowed and must outlive the server. budget_bytes is the
    // HBM budget for everything the server keeps resident (context tables and
    // keys included); max_active caps the admitted requests (0 = budget
    // only); batch_cap caps the operations of one plan (0 = no cap); plain
    // runs one request at a time (the plain one-chain-at-a-time form).
    Server(const std::vector<gfx::Context*>& ctxs, size_t budget_bytes, uint32_t max_active, uint32_t batch_cap,
           bool plain);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Queues a request arriving arrival_s seconds after the epoch; returns its id.
    uint64_t submit(uint32_t ctx, uint32_t level, const std::vector<ReqOp>& ops, double arrival_s, uint64_t seed,
                    const u64* h_in, u64* h_out);
    // Runs the autotuner for every context on EvalMult+Rescale batches of
    // 1, 2, 4, ... max_batch operations (zero-filled buffers from the arena:
    // timing does not depend on the residues), so that steps find their
    // schedule in the cache; the server must be idle. Returns the number of
    // batch shapes tuned.
    int tune(uint32_t max_batch);
    // Resets the epoch to now (arrival times count from here).
    void start();
    // One scheduling step: retire completed steps, admit arrived requests,
    // queue the next operation of every admitted request. Returns the number
    // of operations queued (0 when there was nothing to queue).
    int step();
    // Steps until every submitted request finished; false on timeout.
    bool drain(double max_seconds);
    double now() const;
    size_t pending() const { return queue_.size() + active_.size(); }
    const std::vector<std::unique_ptr<Request>>& finished() const { return done_; }
    const Stats& stats() const { return st_; }
    size_t request_bytes(uint32_t ctx, uint32_t level) const;
    static uint32_t final_level(uint32_t level, const std::vector<ReqOp>& ops);

private:
    struct InFlight {
        std::vector<int> ctxs;                  // contexts that launched
        std::vector<cudaEvent_t> ev;            // one per launched context
        std::vector<Request*> finishing;        // requests whose last op is in this step
    };
    std::vector<gfx::Context*> ctxs_;
    std::unique_ptr<Arena> arena_;
    uint32_t max_active_, batch_cap_;
    bool plain_;
    bool started_ = false;
    std::deque<std::unique_ptr<Request>> queue_;      // submitted, ordered by arrival
    std::vector<std::unique_ptr<Request>> active_;    // admitted, in admission order
    std::vector<std::unique_ptr<Request>> done_;
    std::vector<cudaStream_t> streams_;
    std::vector<std::unique_ptr<pl::Plan>> plans_;    // [ctx][2]: one per in-flight step
    std::vector<cudaEvent_t> ev_pool_;
    std::deque<InFlight> inflight_;
    uint64_t step_no_ = 0;
    std::chrono::steady_clock::time_point epoch_;
    cudaEvent_t epoch_ev_ = nullptr;
    double first_admit_ = -1, last_finish_ = -1;
    uint64_t next_id_ = 1;
    Stats st_;
    int device_ = 0;

    bool admit(Request& r);
    void retire_oldest();
    cudaEvent_t get_event();
};

}  // namespace srv
