// Host interface of the batched pipeline (pipeline.cu).
#pragma once
#include <memory>
#include <vector>

#include "context.hpp"
#include "pipeline.cuh"

namespace pl {

// One operation of a batch; see Mode for the meaning of in/out.
struct Op {
    uint32_t L = 0;
    uint32_t mode = EMR;
    uint64_t key_id = 0;      // context key (0 = relinearisation)
    uint64_t galois = 0;      // ROT: Galois element
    const u64* in[4] = {nullptr, nullptr, nullptr, nullptr};
    u64* out[2] = {nullptr, nullptr};
};

struct HostTables;

struct Plan {
    Plan();
    DevCtx dc{};
    uint32_t logn = 0, nops = 0;
    PairDesc* d_pairs = nullptr;
    uint2* d_jobs = nullptr;
    // [phase (index NPHASE: the second P7 launch)][integer jobs, FP64 jobs, both interleaved]
    size_t job_off[NPHASE + 1][3] = {};
    uint32_t job_cnt[NPHASE + 1][3] = {};
    uint4* d_mac_jobs = nullptr;
    uint32_t* d_plist = nullptr;
    u64* ws = nullptr;
    size_t ws_words = 0;
    bool own_ws = false;
    std::vector<Op> ops;      // host copy (device pointers and levels)
    std::vector<PairDesc> pairs_host;
    // launch schedule (chosen by tune() or the context's tuning cache)
    int p5_form = 0;                   // P5_REG128, P5_ASYNC or P5_REG256
    bool p5_fp = false;                // P5 key rows of 50-bit Q towers on the FP64 pipe (p5_mac_fp)
    int p5_fp_form = 0;                // 0: 4 digits in flight, 4 CTAs per SM; 1: 2 digits, 5 CTAs;
                                       // 2, 3: TMA ring of three or two stages
    bool p5_split = false;             // FP64 and integer P5 rows on two streams at once (fork / join)
    // the second stream and its fork / join events, made on first use
    mutable cudaStream_t side = nullptr;
    mutable cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    unsigned mix = 0x1ff;              // bit k: phase k+1 as one launch over its interleaved job list
    int p3_form = 0;                   // 0 plain P3; 1, 2 warp-specialised (128 x 2 CTAs, 256 x 1 CTA)
    bool tuned = false;
    // The plan's launches share the GPU with other streams' steps (the
    // server's rings run side by side): the autotuner, which times each
    // candidate alone, then leaves out the TMA form of the FP64 P5 rows,
    // whose ring holds about 197 KB of shared memory per SM and keeps the
    // other streams' kernels off those SMs.
    bool concurrent = false;
    const gfx::Context* ctx = nullptr;
    std::vector<uint64_t> key_pins;    // keys this plan holds resident (Context::acquire)
    void* d_blob = nullptr;            // device tables (pairs, jobs, P5 groups, pair lists)
    void* h_blob = nullptr;            // pinned host mirror of d_blob
    size_t blob_cap = 0;
    // pinned mirrors outgrown by a rebuild: freeing one (cudaFreeHost) would
    // synchronize the device under a running step, so they are kept until the
    // plan is destroyed (at most the sum of a doubling series: < 2x h_blob)
    std::vector<void*> old_h_blobs;
    std::unique_ptr<HostTables> staging;
    ~Plan();
    Plan(const Plan&) = delete;                  // owns device memory and a hold on ctx
    Plan& operator=(const Plan&) = delete;
};

bool supported_logn(int logn);
// Makes the plan's second stream and fork / join events on the current
// device (once); false when they cannot be made.
bool ensure_side(const Plan& p);
size_t op_workspace_words(const gfx::Context& c, uint32_t L);
void validate(const gfx::Context& c, const Op& op);
// ws == nullptr: the plan allocates (and owns) its workspace.
std::unique_ptr<Plan> build_plan(const gfx::Context& c, const std::vector<Op>& ops, u64* ws, size_t ws_words);
// Rebuilds `p` in place for a new batch (one workspace pointer per op),
// reusing its buffers when large enough; the tables are uploaded with one
// cudaMemcpyAsync on `s` from the plan's pinned mirror, so the host must not
// rebuild `p` again before work queued on `s` has consumed them.
void build_plan_into(Plan& p, const gfx::Context& c, const std::vector<Op>& ops, const std::vector<u64*>& ws_ptrs,
                     cudaStream_t s);
// mask selects phases P1..P9 (bit k = phase k+1); 0x1ff runs the whole batch.
cudaError_t launch(const Plan& p, cudaStream_t s, unsigned mask = 0x1ff);
// Picks the launch schedule of `p` (P5 form; integer and FP64 transform
// jobs as two launches or one interleaved launch): from the context's tuning cache when it holds
// this shape (ring size, digits, batch-size class), else by timing every
// candidate with CUDA events on `s` (one dimension at a time on the phases it
// changes; two interleaved passes, best of three launches each; a candidate
// wins only if 1.5% faster) and caching the winner. Timing re-runs the batch, so it is skipped (defaults
// kept) when `measure` is false, while `s` is capturing a graph, or when an
// operation writes over its own input (in-place rescale).
void tune(Plan& p, cudaStream_t s, bool measure = true);
constexpr int MAC_MAX_DNUM = 16;
// P5 forms: register prefetch with 128 threads x 4 words, the cp.async
// pipelined form, register prefetch with 256 threads x 2 words, the TMA
// (bulk copy + mbarrier) ring.
constexpr int P5_REG128 = 0, P5_ASYNC = 1, P5_REG256 = 2, P5_TMA = 3;
inline int mac_smem(uint32_t dnum) { return (int)(dnum * 2 * MAC_TILE * sizeof(u64)); }
// The pipelined P5 runs when two CTAs' key tiles and staging buffers fit in one SM.
constexpr int MAC_ASYNC_SMEM_MAX = 113 * 1024;
inline bool mac_async_ok(uint32_t dnum) { return maca_smem((int)dnum) <= MAC_ASYNC_SMEM_MAX; }
// The TMA form needs its key tile and stage ring in one CTA's shared memory.
constexpr int MAC_TMA_SMEM_MAX = 200 * 1024;
inline bool mac_tma_ok(uint32_t dnum) { return p5t_smem((int)dnum) <= MAC_TMA_SMEM_MAX; }
static_assert(MAC_MAX_DNUM * 2 * MAC_TILE * 8 <= 227 * 1024, "register P5 forms at the largest dnum");
int input_count(uint32_t mode);
// Rebinds operation `idx` of a built plan to new buffers / mode (same level
// and job shape) by a one-thread kernel on `s`: no allocation and no host
// transfer, so it can be recorded in a CUDA graph together with launch().
// KS and ROT plans share one job shape, so a keyswitch plan also serves
// rotations at the same level.
void rebind(Plan& p, uint32_t idx, const Op& op, const gfx::Context& c, cudaStream_t s);
uint32_t output_towers(const Op& op);

}  // namespace pl
