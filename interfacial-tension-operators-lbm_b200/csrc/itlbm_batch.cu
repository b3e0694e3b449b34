// itlbm_batch.cu -- many cases stepped together (include/itlbm.h, itlbm_batch_*).
//
// The reference runs one process per case (rodar_lote.py:231-243, a thread pool of subprocesses at
// :300-318).  Here every admitted case keeps its double-buffered state on the device and all of them
// advance together:
//   * a slot table of per-case descriptors (CaseDev) lives in device memory; each descriptor carries
//     the case's buffer parity and the number of sub-steps it runs in the current replay;
//   * tile work tables list the TX x TY tiles of every active case, one per storage form (FP64, FP32,
//     FP32 fold), with their lengths in device memory;
//   * one replay is a CUDA graph of `chunk` sub-steps: each non-empty table is a chain of launches on
//     its own stream between a fork and a join, one CTA per table entry (the grid is the table length
//     rounded up to a bucket); a case whose chunk is shorter skips its tiles in the remaining
//     sub-steps.  The graph is re-captured only when a table's bucket or storage changes;
//   * case state comes from a stream-ordered memory pool, and the initial profiles of a round's
//     admissions are filled by host threads into mapped pinned memory that the init kernel reads.
// Each case stops at its next diagnostic step (every diag_every steps and its last step, as
// Imm_OPS.cpp:293), is measured there by the same device diagnostics as a single case, and retires at
// its step count or when the stop rule of Imm_OPS.cpp:346-352 / Imm_INCL.cpp:428-433 fires.
#include "itlbm_site.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <thread>
#include <vector>

namespace itlbm {
void fill_params(CaseDev &c, const itlbm_operador &op, double tau, double A_fact, double beta,
                 double rho0);
void fill_shift(CaseDev &c, double rho0, double u0x);
}  // namespace itlbm

using namespace itlbm;

namespace {

struct Pending {
    itlbm_case_desc desc;
    int n_steps;
    long long tag;
    double t_submit;
    std::string snapshot;  // restore from this file instead of the initial state
    long long start = 0;   // its step count
};

struct Active {
    itlbm_case_desc desc{};
    int n_steps = 0;
    long long tag = 0;
    double t_submit = 0;
    int slot = -1;
    void *mem = nullptr;
    double *aux = nullptr;
    size_t bytes = 0;
    int next_step = 0;  // index of the next step to run
    int parity = 0;     // buffer holding the state at next_step
    int chunk_len = 0;
    bool diag_at_end = false;
    bool measured = false;  // its last advance ended at one of its diagnostic steps (aux kept there)
    bool held = false;      // retired, state kept for itlbm_batch_read_fields until released
};

size_t case_bytes(const itlbm_case_desc &d, bool &need_aux) {
    const size_t elem = elem_of(d.precision);
    need_aux = d.op.tipo >= ITLBM_OP_F1 || d.geometry == ITLBM_GEOM_STRIP;
    return (size_t)2 * buf_elems_of(d.nx, d.ny, d.precision) * elem +
           (need_aux ? (size_t)4 * aux_elems_of(d.nx, d.ny) * 8 : 0);
}

// the work tables, per storage form: [0] FP64, [1] FP32, [2] FP32 fold
// ... and one per tile shape within each: table p holds storage form p / NSHAPE, shape p % NSHAPE
constexpr int NPREC = 3;
constexpr int NTAB = NPREC * NSHAPE;
int table_of(int prec) { return prec == ITLBM_PREC_F64 ? 0 : (prec == ITLBM_PREC_F32 ? 1 : 2); }
int prec_of_table(int p) {
    p /= NSHAPE;
    return p == 0 ? ITLBM_PREC_F64 : (p == 1 ? ITLBM_PREC_F32 : ITLBM_PREC_F32_FOLD);
}
int shape_of_table(int p) { return p % NSHAPE; }

const double U_LIMITE = 0.4;  // Imm_OPS.cpp:45

}  // namespace

struct itlbm_batch {
    itlbm_batch_config cfg{};
    int device = 0, sms = 0;
    cudaStream_t stream = nullptr;
    // case state comes from a stream-ordered pool that keeps up to the HBM budget reserved:
    // admissions and retirements neither map nor unmap device memory nor synchronise the device
    cudaMemPool_t pool = nullptr;
    // initial profiles of the cases admitted in one round, in mapped pinned host memory that the
    // init kernel reads directly (no device staging buffer to allocate and free per case)
    double *stage = nullptr, *stage_dev = nullptr;
    size_t stage_cap = 0, stage_used = 0;
    struct InitJob {
        int slot;
        itlbm_case_desc d;
        CaseDev h;
        size_t off;  // of its profile in the staging buffer
    };
    std::vector<InitJob> inits;  // admitted this round, initial state not yet launched
    std::vector<int> dev_inits;  // admitted this round, initial state formed on the device, not yet launched
    int desc_lo = INT_MAX, desc_hi = -1;  // slots whose descriptors are not yet on the device
    std::deque<Pending> pending;
    std::vector<Active *> slots;
    std::vector<int> free_slots;
    std::vector<CaseDev> h_cases;
    CaseDev *d_cases = nullptr;
    TileRef *d_tiles[NTAB] = {};  // per storage form and tile shape
    int tiles_cap[NTAB] = {};
    int *d_ntiles = nullptr;
    bool tables_dirty = true;
    int grid[NTAB] = {};
    int ntab[NTAB] = {};  // current table lengths
    int occ[NTAB] = {};   // resident CTAs per SM of each table's step kernel
    // launch shape: -1 = one CTA per table entry, 0 = persistent CTAs at the occupancy limit, k > 0 =
    // k persistent CTAs per SM; with ctas_per_sm = 0 the first full replay times -1 against 0
    int mode = -1;
    bool tuning = false;
    // a partial last tile column of a case in narrow tiles (16 x 16, 8 x 32) instead of 32 x 8; with
    // ctas_per_sm = 0 the first full replay times both tilings and keeps the faster (on the measured
    // mixes 32 x 8 throughout, which is also the tiling without autotuning)
    bool narrow = false;
    bool tile_fixed = false;  // the tiling was set by the caller, not timed
    cudaEvent_t tev[2] = {};
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // one chain of step launches per non-empty table, each on its own stream between a fork and a
    // join on `stream`: the tables hold different cases, so their steps need no order between them
    cudaStream_t side[NPREC] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[NPREC] = {};
    // within one storage form, the narrow-tile tables run on streams of their own beside the 32 x 8
    // table, each sub-step after every shape's previous sub-step (events shape_ev)
    cudaStream_t shape_st[NPREC][NSHAPE] = {};
    cudaEvent_t shape_ev[NPREC][NSHAPE] = {}, shape_fork[NPREC] = {};
    // diagnostics: the cases that fall due in an advance are measured together, drops and strips each
    // by one sequence of launches over a table of jobs, their scratch in per-case segments of one
    // block (grown on demand, up to DIAG_SCRATCH_LIMIT or the largest single case; more due cases than
    // that are measured in groups)
    void *dscratch = nullptr;
    size_t dscratch_cap = 0;
    DiagJob *d_jobs = nullptr, *h_jobs = nullptr;  // one per slot at most in an advance (pinned host)
    int *d_blk = nullptr, *h_blk = nullptr;        // block -> job maps of the full-field passes
    size_t blk_cap = 0;
    itlbm_drop_diag *d_drop = nullptr, *h_drop = nullptr;  // per slot (pinned host)
    itlbm_strip_diag *d_strip = nullptr, *h_strip = nullptr;
    std::deque<itlbm_batch_event> events;
    std::chrono::steady_clock::time_point t0;
    size_t hbm_used = 0;
    bool hold = false;  // retired cases are held until itlbm_batch_release
    int nheld = 0;
    long long node_updates = 0;
    double device_ms = 0, diag_ms = 0, advance_ms = 0, admit_ms = 0, capture_ms = 0;
    int replays = 0, finished = 0, captures = 0;
    cudaEvent_t ev2 = nullptr;  // end of the diagnostics

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// Grid of a table of n tiles: n rounded up to m x 2^e with m < 32 (at most 1/16 more CTAs, which
// exit at once), so that admissions and retirements change the grid -- and re-capture the graph --
// only when the table crosses a bucket.
int grid_bucket(int n) {
    if (n <= 32) return n;
    int e = 0;
    while ((n >> e) >= 32) e++;
    return ((n + (1 << e) - 1) >> e) << e;
}

// Grids of the current launch shape: empty tables launch nothing; one CTA per entry rounds the
// table up to its bucket; persistent CTAs stride over the table.
void set_grids(itlbm_batch *b) {
    for (int p = 0; p < NTAB; p++) {
        if (b->ntab[p] == 0) b->grid[p] = 0;
        else if (b->mode < 0) b->grid[p] = grid_bucket(b->ntab[p]);
        else b->grid[p] = (b->mode > 0 ? b->mode : std::max(1, b->occ[p])) * b->sms;
    }
}

int upload_tables(itlbm_batch *b) {
    std::vector<TileRef> t[NTAB];
    for (Active *a : b->slots) {
        if (!a || a->held) continue;
        const CaseDev &c = b->h_cases[a->slot];
        case_tiles(c, b->narrow, a->slot, &t[table_of(a->desc.precision) * NSHAPE]);
    }
    int n[NTAB];
    for (int p = 0; p < NTAB; p++) {
        n[p] = (int)t[p].size();
        if (n[p] > b->tiles_cap[p]) {
            if (b->d_tiles[p]) cudaFree(b->d_tiles[p]);
            b->tiles_cap[p] = std::max(n[p], 2 * b->tiles_cap[p]);
            cudaError_t e = cudaMalloc(&b->d_tiles[p], sizeof(TileRef) * b->tiles_cap[p]);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(work table)");
        }
        if (n[p]) {
            cudaError_t e = cudaMemcpyAsync(b->d_tiles[p], t[p].data(), sizeof(TileRef) * n[p],
                                            cudaMemcpyHostToDevice, b->stream);
            if (e != cudaSuccess) return cuda_fail(e, "work table upload");
        }
    }
    for (int p = 0; p < NTAB; p++) b->ntab[p] = n[p];
    set_grids(b);
    // the graph reads the table pointers it was captured with: keep them, or re-capture
    cudaError_t e = cudaMemcpyAsync(b->d_ntiles, n, sizeof(int) * NTAB, cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "work table length");
    return cudaStreamSynchronize(b->stream) == cudaSuccess ? ITLBM_OK : cuda_fail(cudaGetLastError(), "sync");
}

// Sub-steps [k0, k1) of the tables of storage form pi, from stream st.  The tables of one storage form
// (one per tile shape) hold tiles of the same cases: sub-step k of every tile of a case must end before
// any tile of it starts sub-step k + 1 (which reads what k wrote and overwrites what k read).  A
// single table runs in line on st; several run side by side, the 32 x 8 table on st and each narrow
// table on a stream of its own, every launch of sub-step k > k0 waiting for the other shapes'
// launches of sub-step k - 1, so that the small narrow-tile launches overlap the large one.
cudaError_t enqueue_chain(itlbm_batch *b, int pi, int k0, int k1, cudaStream_t st) {
    int shapes[NSHAPE], n = 0;
    for (int sh = 0; sh < NSHAPE; sh++)
        if (b->grid[pi * NSHAPE + sh] > 0) shapes[n++] = sh;
    auto launch = [&](int sh, int k, cudaStream_t on) {
        const int p = pi * NSHAPE + sh;
        return launch_step(b->d_cases, b->d_tiles[p], 0, b->d_ntiles + p, b->grid[p], k, -1, prec_of_table(p),
                           sh, on);
    };
    cudaError_t e = cudaSuccess;
    if (n == 1) {
        for (int k = k0; k < k1 && e == cudaSuccess; k++) e = launch(shapes[0], k, st);
        return e;
    }
    auto stream_of = [&](int sh) { return sh == SHAPE_32x8 ? st : b->shape_st[pi][sh]; };
    if ((e = cudaEventRecord(b->shape_fork[pi], st)) != cudaSuccess) return e;
    for (int j = 0; j < n; j++)
        if (shapes[j] != SHAPE_32x8 && (e = cudaStreamWaitEvent(stream_of(shapes[j]), b->shape_fork[pi], 0)) != cudaSuccess)
            return e;
    for (int k = k0; k < k1; k++) {
        if (k > k0)  // every wait of sub-step k first: each names the other shapes' records of k - 1
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++)
                    if (i != j && (e = cudaStreamWaitEvent(stream_of(shapes[j]), b->shape_ev[pi][shapes[i]], 0)) !=
                                      cudaSuccess)
                        return e;
        for (int j = 0; j < n; j++) {
            if ((e = launch(shapes[j], k, stream_of(shapes[j]))) != cudaSuccess) return e;
            if ((e = cudaEventRecord(b->shape_ev[pi][shapes[j]], stream_of(shapes[j]))) != cudaSuccess) return e;
        }
    }
    for (int j = 0; j < n; j++)
        if (shapes[j] != SHAPE_32x8 && (e = cudaStreamWaitEvent(st, b->shape_ev[pi][shapes[j]], 0)) != cudaSuccess)
            return e;
    return e;
}

// Sub-steps [k0, k1) of every table on the batch stream: the storage forms hold different cases, so
// one form runs in line and several run as parallel chains (fork, one chain per form on its own
// stream, join), in a capture or directly.
cudaError_t enqueue_steps(itlbm_batch *b, int k0, int k1) {
    bool busy[NPREC] = {};
    int used = 0;
    for (int pi = 0; pi < NPREC; pi++) {
        for (int sh = 0; sh < NSHAPE; sh++) busy[pi] = busy[pi] || b->grid[pi * NSHAPE + sh] > 0;
        used += busy[pi];
    }
    cudaError_t e = cudaSuccess;
    if (used <= 1) {
        for (int pi = 0; pi < NPREC && e == cudaSuccess; pi++)
            if (busy[pi]) e = enqueue_chain(b, pi, k0, k1, b->stream);
        return e;
    }
    if ((e = cudaEventRecord(b->ev_fork, b->stream)) != cudaSuccess) return e;
    for (int pi = 0; pi < NPREC; pi++) {
        if (!busy[pi]) continue;
        if ((e = cudaStreamWaitEvent(b->side[pi], b->ev_fork, 0)) != cudaSuccess) return e;
        if ((e = enqueue_chain(b, pi, k0, k1, b->side[pi])) != cudaSuccess) return e;
        if ((e = cudaEventRecord(b->ev_join[pi], b->side[pi])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(b->stream, b->ev_join[pi], 0)) != cudaSuccess) return e;
    }
    return e;
}

// Adds the host wall time of its scope to a counter of the batch, in ms.
struct ScopeTimer {
    const itlbm_batch *b;
    double &acc;
    double t;
    ScopeTimer(const itlbm_batch *b_, double &acc_) : b(b_), acc(acc_), t(b_->now()) {}
    ~ScopeTimer() { acc += (b->now() - t) * 1e3; }
};

int capture_graph(itlbm_batch *b) {
    ScopeTimer timer(b, b->capture_ms);
    b->captures++;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "begin capture");
    const cudaError_t el = enqueue_steps(b, 0, b->cfg.chunk);
    e = cudaStreamEndCapture(b->stream, &g);
    if (el != cudaSuccess) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return cuda_fail(el, "captured step launches");
    }
    if (e != cudaSuccess) return cuda_fail(e, "end capture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "graph instantiate");
}

// Node updates of sub-steps [k0, k1) of this replay.
long long updates_in(const itlbm_batch *b, int k0, int k1) {
    long long u = 0;
    for (const Active *a : b->slots)
        if (a && !a->held) u += (long long)std::max(0, std::min(a->chunk_len, k1) - k0) * a->desc.nx * a->desc.ny;
    return u;
}

// Autotuning on the first full replay of at least 18 sub-steps, in timed windows of
// M = max(6, K / 16) sub-steps (CUDA events, rate per node update): the tiling -- narrow tiles at the partial last tile column of a case against
// 32 x 8 tiles throughout -- with one CTA per table entry, then persistent CTAs at the occupancy limit
// with the better tiling.  The faster of each runs the rest of the replay and is captured into the
// graph.  Every choice runs the same arithmetic on every node, so the results do not depend on it.
constexpr int TUNE_MIN_WINDOW = 6;  // shorter windows were noisy enough to pick a 30 % slower tiling
int tune_and_run(itlbm_batch *b, int K) {
    const int M = std::max(TUNE_MIN_WINDOW, K / 16);
    int k0 = 0;
    auto window = [&](int mode, bool narrow, double &rate) -> int {
        if (narrow != b->narrow) {
            b->narrow = narrow;
            const int r = upload_tables(b);
            if (r) return r;
        }
        b->mode = mode;
        set_grids(b);
        cudaEventRecord(b->tev[0], b->stream);
        cudaError_t e = enqueue_steps(b, k0, k0 + M);
        cudaEventRecord(b->tev[1], b->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b->tev[1]);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->tev[0], b->tev[1]);
        if (e != cudaSuccess) return cuda_fail(e, "autotuning window");
        rate = ms > 0 ? (double)updates_in(b, k0, k0 + M) / ms : 0.0;
        k0 += M;
        return ITLBM_OK;
    };
    double r_narrow = 0, r_uniform = 0, r_persist = 0;
    int r;
    bool narrow = b->narrow;
    if (!b->tile_fixed) {
        if ((r = window(-1, true, r_narrow)) != ITLBM_OK || (r = window(-1, false, r_uniform)) != ITLBM_OK)
            return r;
        narrow = r_narrow >= r_uniform;
    } else {
        if ((r = window(-1, narrow, r_narrow)) != ITLBM_OK) return r;
        r_uniform = r_narrow;
    }
    if ((r = window(0, narrow, r_persist)) != ITLBM_OK) return r;
    // persistent CTAs only when clearly faster (the two are within noise on small tables)
    const int mode = r_persist > 1.02 * std::max(r_narrow, r_uniform) ? 0 : -1;
    if (b->narrow != narrow) {
        b->narrow = narrow;
        if ((r = upload_tables(b)) != ITLBM_OK) return r;
    }
    b->mode = mode;
    b->tuning = false;
    set_grids(b);
    cudaError_t e;
    if ((e = enqueue_steps(b, k0, K)) != cudaSuccess) return cuda_fail(e, "step launches");
    return capture_graph(b);
}

// A retired case leaves the work table; with hold on it keeps its state until itlbm_batch_release.
void retire(itlbm_batch *b, Active *a) {
    b->tables_dirty = true;
    b->finished++;
    if (b->hold) {
        a->held = true;
        a->chunk_len = 0;
        b->h_cases[a->slot].chunk_len = 0;
        b->nheld++;
        return;
    }
    cudaFreeAsync(a->mem, b->stream);
    if (a->aux) cudaFreeAsync(a->aux, b->stream);
    b->hbm_used -= a->bytes;
    b->slots[a->slot] = nullptr;
    b->free_slots.push_back(a->slot);
    b->h_cases[a->slot] = CaseDev{};
    delete a;
}

// Room for `len` profile values in the staging buffer: wait for the round's earlier initial states
// when it is full, grow it when one profile does not fit.
cudaError_t stage_reserve(itlbm_batch *b, size_t len) {
    if (b->stage_used + len <= b->stage_cap) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (b->stage_used > 0 && (e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return e;
    b->stage_used = 0;
    if (len <= b->stage_cap) return cudaSuccess;
    if (b->stage) cudaFreeHost(b->stage);
    b->stage = b->stage_dev = nullptr;
    b->stage_cap = 0;
    const size_t cap = std::max<size_t>(len, (size_t)1 << 20);
    if ((e = cudaHostAlloc((void **)&b->stage, sizeof(double) * cap, cudaHostAllocMapped | cudaHostAllocPortable)) !=
        cudaSuccess)
        return e;
    if ((e = cudaHostGetDevicePointer((void **)&b->stage_dev, b->stage, 0)) != cudaSuccess) return e;
    b->stage_cap = cap;
    return cudaSuccess;
}

// The initial profiles of the cases admitted so far in this round, filled by host threads that take
// chunks of about 16 K nodes from all of them at once (most boxes are too small to split alone), then
// their initial-state launches, in admission order.
// The descriptors of the slots admitted since the last upload, in one copy on the batch stream (the
// init kernels read them from the device).
cudaError_t upload_descs(itlbm_batch *b) {
    if (b->desc_hi < b->desc_lo) return cudaSuccess;
    const int lo = b->desc_lo, hi = b->desc_hi;
    b->desc_lo = INT_MAX;
    b->desc_hi = -1;
    return cudaMemcpyAsync(b->d_cases + lo, b->h_cases.data() + lo, sizeof(CaseDev) * (size_t)(hi - lo + 1),
                           cudaMemcpyHostToDevice, b->stream);
}

cudaError_t flush_inits(itlbm_batch *b) {
    if (b->inits.empty()) return cudaSuccess;
    struct Chunk {
        int job, ya, yb;
    };
    std::vector<Chunk> chunks;
    for (int j = 0; j < (int)b->inits.size(); j++) {
        const auto &w = b->inits[j];
        if (w.d.geometry != ITLBM_GEOM_DROP) {
            chunks.push_back({j, 0, 1});
            continue;
        }
        const int rows = std::max(1, 16384 / std::max(1, w.h.nx));
        for (int y = 0; y < w.h.ny; y += rows) chunks.push_back({j, y, std::min(w.h.ny, y + rows)});
    }
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < chunks.size();) {
            const auto &w = b->inits[chunks[k].job];
            init_profile_rows(w.h, w.d, b->stage + w.off, chunks[k].ya, chunks[k].yb);
        }
    };
    const int nthr = (int)std::min<size_t>(chunks.size(),
                                           std::min(16u, std::max(1u, std::thread::hardware_concurrency())));
    std::vector<std::thread> pool;
    for (int t = 1; t < nthr; t++) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    cudaError_t e = upload_descs(b);
    for (const auto &w : b->inits)
        if (e == cudaSuccess) e = launch_init_from(w.h, b->d_cases + w.slot, w.d, b->stage_dev + w.off, b->stream);
    b->inits.clear();
    return e;
}

int admit_cases(itlbm_batch *b) {
    b->stage_used = 0;  // the previous round's initial states are complete (advance ends synchronised)
    while (!b->pending.empty() && !b->free_slots.empty()) {
        const Pending &p = b->pending.front();
        bool need_aux;
        const size_t bytes = case_bytes(p.desc, need_aux);
        if (b->hbm_used + bytes > b->cfg.hbm_budget) break;  // first in, first admitted
        Active *a = new Active();
        a->desc = p.desc;
        a->n_steps = p.n_steps;
        a->tag = p.tag;
        a->t_submit = p.t_submit;
        a->bytes = bytes;
        const itlbm_case_desc &d = p.desc;
        CaseDev h{};
        case_layout(h, d.nx, d.ny, d.precision);
        fill_params(h, d.op, d.tau, d.A_fact, d.beta, d.rho_B > 0 ? d.rho_B : 1.0);
        fill_shift(h, h.rho0, d.geometry == ITLBM_GEOM_DROP ? d.v0 : 0.0);
        const size_t elem = elem_of(d.precision);
        const size_t per_buf = (size_t)h.buf_elems * elem;
        cudaError_t e = cudaMallocFromPoolAsync(&a->mem, 2 * per_buf, b->pool, b->stream);
        if (e == cudaSuccess && need_aux)
            e = cudaMallocFromPoolAsync(&a->aux, sizeof(double) * 4 * (size_t)h.aux_stride, b->pool, b->stream);
        if (e != cudaSuccess) {
            if (a->mem) cudaFreeAsync(a->mem, b->stream);
            delete a;
            cudaGetLastError();
            return ITLBM_OK;  // the device is fuller than the budget says: try again next round
        }
        if ((e = case_bind(h, a->mem, per_buf)) != cudaSuccess) {
            cudaFreeAsync(a->mem, b->stream);
            if (a->aux) cudaFreeAsync(a->aux, b->stream);
            delete a;
            return cuda_fail(e, "state buffers");
        }
        h.aux = a->aux;
        h.parity0 = 0;
        h.chunk_len = 0;
        const int slot = b->free_slots.back();
        b->free_slots.pop_back();
        a->slot = slot;
        b->slots[slot] = a;
        b->h_cases[slot] = h;
        // the descriptor goes up with the round's others, in one copy on the batch stream (which is
        // not ordered after the legacy stream's copies) before any init kernel reads it
        b->desc_lo = std::min(b->desc_lo, slot);
        b->desc_hi = std::max(b->desc_hi, slot);
        if (p.snapshot.empty() && profile_on_device(d)) {
            b->dev_inits.push_back(slot);
        } else if (p.snapshot.empty()) {
            const size_t len = profile_len(h, d);
            // a full staging buffer is reused only after the profiles queued in it are launched
            if (e == cudaSuccess && b->stage_used + len > b->stage_cap) e = flush_inits(b);
            if (e == cudaSuccess) e = stage_reserve(b, len);
            if (e == cudaSuccess) {
                b->inits.push_back(itlbm_batch::InitJob{slot, d, h, b->stage_used});
                b->stage_used += len;
            }
            if (e != cudaSuccess) return cuda_fail(e, "admission");
        } else {
            e = upload_descs(b);
            if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
            if (e != cudaSuccess) return cuda_fail(e, "admission");
            const int r = snap_read_state(p.snapshot.c_str(), h, h.buf[0]);
            if (r) return r;
            a->next_step = (int)p.start;
        }
        b->hbm_used += bytes;
        b->tables_dirty = true;
        b->pending.pop_front();
    }
    return ITLBM_OK;
}

int admit(itlbm_batch *b) {
    const int r = admit_cases(b);
    // the descriptors first, then the init kernels that form their states on the device
    cudaError_t e = upload_descs(b);
    for (const int slot : b->dev_inits) {
        const Active *a = b->slots[slot];
        if (e == cudaSuccess && a) e = launch_init_from(b->h_cases[slot], b->d_cases + slot, a->desc, nullptr, b->stream);
    }
    b->dev_inits.clear();
    if (e == cudaSuccess) e = flush_inits(b);
    if (r) return r;
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "initial states");
}

// Scratch of the diagnostics measured together: room for every due case, up to this many bytes (or
// the largest single case); beyond it the due cases are measured in groups.
constexpr size_t DIAG_SCRATCH_LIMIT = (size_t)4 << 30;

// The diagnostics of the cases in `due` (their last sub-step of this replay is a diagnostic step),
// enqueued on the batch stream: for each group of cases whose scratch fits, one table of drop jobs
// and one of strip jobs, each measured by one sequence of launches.  Each job has its own scratch
// segment and keeps the reduction order of the case alone.
int run_diagnostics(itlbm_batch *b, const std::vector<Active *> &due) {
    if (due.empty()) return ITLBM_OK;
    size_t total = 0, largest = 0;
    long long blocks = 0;
    for (const Active *a : due) {
        const size_t need = diag_job_bytes(a->desc.nx, a->desc.ny, a->desc.geometry);
        total += need;
        largest = std::max(largest, need);
        blocks += diag_nblocks((long long)a->desc.nx * a->desc.ny);
    }
    cudaError_t e = cudaSuccess;
    const size_t want = std::max(largest, std::min(total, DIAG_SCRATCH_LIMIT));
    if (b->dscratch_cap < want) {
        // grow (a device-wide synchronisation, rare: the first rounds of diagnostics); when the device
        // has no room for all due cases, fall back to the largest single one
        if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return cuda_fail(e, "synchronize");
        void *p = nullptr;
        for (size_t sz : {want, largest}) {
            if (sz <= b->dscratch_cap) break;
            if (cudaMalloc(&p, sz) == cudaSuccess) {
                if (b->dscratch) cudaFree(b->dscratch);
                b->dscratch = p;
                b->dscratch_cap = sz;
                break;
            }
            cudaGetLastError();
        }
        if (b->dscratch_cap < largest) return fail(ITLBM_E_OOM, "diagnostic scratch");
    }
    if ((size_t)blocks > b->blk_cap) {
        if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return cuda_fail(e, "synchronize");
        const size_t cap = std::max<size_t>((size_t)blocks, 2 * b->blk_cap);
        if (b->d_blk) cudaFree(b->d_blk);
        if (b->h_blk) cudaFreeHost(b->h_blk);
        b->d_blk = nullptr;
        b->h_blk = nullptr;
        b->blk_cap = 0;
        if ((e = cudaMalloc(&b->d_blk, sizeof(int) * cap)) != cudaSuccess ||
            (e = cudaHostAlloc((void **)&b->h_blk, sizeof(int) * cap, cudaHostAllocDefault)) != cudaSuccess)
            return cuda_fail(e, "diagnostic block map");
        b->blk_cap = cap;
    }
    // the host tables of this advance are written once and copied in order; a group's copies are
    // queued before its launches, and no later group reuses its part of the tables
    int job_at = 0;
    size_t blk_at = 0;
    size_t k = 0;
    while (k < due.size()) {
        size_t used = 0, k1 = k;
        while (k1 < due.size()) {
            const Active *a = due[k1];
            const size_t need = diag_job_bytes(a->desc.nx, a->desc.ny, a->desc.geometry);
            if (used + need > b->dscratch_cap) break;
            used += need;
            k1++;
        }
        // this group: jobs [k, k1), scratch segments in order, drops then strips
        size_t off = 0;
        for (int geom : {ITLBM_GEOM_DROP, ITLBM_GEOM_STRIP}) {
            const int j0 = job_at;
            const size_t b0 = blk_at;
            int nblk = 0;
            size_t seg = 0;
            for (size_t i = k; i < k1; i++) {
                const Active *a = due[i];
                const size_t need = diag_job_bytes(a->desc.nx, a->desc.ny, a->desc.geometry);
                if (a->desc.geometry != geom) {
                    seg += need;
                    continue;
                }
                DiagJob &J = b->h_jobs[job_at];
                J = DiagJob{};
                diag_job_layout(J, (char *)b->dscratch + off + seg, a->desc.nx, a->desc.ny, geom);
                seg += need;
                J.c = b->d_cases + a->slot;
                J.out = geom == ITLBM_GEOM_DROP ? (void *)(b->d_drop + a->slot) : (void *)(b->d_strip + a->slot);
                J.cur = a->parity ^ (a->chunk_len & 1);
                J.step = a->next_step + a->chunk_len - 1;
                J.v0 = a->desc.v0;
                J.x_ini = a->desc.nx / 2;
                J.y_ini = a->desc.ny / 2;
                J.use_force = a->desc.op.tipo >= ITLBM_OP_F1 ? 1 : 0;
                J.p = a->desc.p;
                J.q = a->desc.q;
                J.block0 = nblk;
                for (int q = 0; q < J.nblocks; q++) b->h_blk[blk_at + nblk + q] = job_at - j0;
                nblk += J.nblocks;
                job_at++;
            }
            const int nj = job_at - j0;
            if (nj == 0) continue;
            blk_at += nblk;
            if ((e = cudaMemcpyAsync(b->d_jobs + j0, b->h_jobs + j0, sizeof(DiagJob) * nj, cudaMemcpyHostToDevice,
                                     b->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(b->d_blk + b0, b->h_blk + b0, sizeof(int) * nblk, cudaMemcpyHostToDevice,
                                     b->stream)) != cudaSuccess ||
                (e = launch_diag_jobs(b->d_jobs + j0, nj, b->d_blk + b0, nblk, geom, b->stream)) != cudaSuccess)
                return cuda_fail(e, "diagnostics");
        }
        // the next group reuses the scratch: stream order keeps its launches after this group's
        k = k1;
    }
    return ITLBM_OK;
}

}  // namespace

extern "C" {

int itlbm_batch_create(const itlbm_batch_config *cfg, itlbm_batch **out) {
    if (!out) return fail(ITLBM_E_ARG, "NULL argument");
    *out = nullptr;
    itlbm_batch *b = new itlbm_batch();
    if (cfg) b->cfg = *cfg;
    if (b->cfg.max_cases <= 0) b->cfg.max_cases = 4096;
    if (b->cfg.chunk <= 0) b->cfg.chunk = 500;
    if (b->cfg.diag_every <= 0) b->cfg.diag_every = 500;
    cudaError_t e = cudaGetDevice(&b->device);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "cudaGetDevice");
    }
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (b->cfg.hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        b->cfg.hbm_budget = (size_t)(0.9 * (double)fr);
    }
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = b->device;
        if ((e = cudaMemPoolCreate(&b->pool, &props)) != cudaSuccess) {
            delete b;
            return cuda_fail(e, "case memory pool");
        }
        cuuint64_t keep = b->cfg.hbm_budget;
        cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    // launch shape: ctas_per_sm < 0, one CTA per entry of the work table (the grid follows the table
    // and the graph is re-captured when it changes); > 0, that many persistent CTAs per SM striding
    // over it; 0, whichever of the two (persistent at the occupancy limit) the first full replay
    // measures faster
    b->mode = b->cfg.ctas_per_sm > 0 ? b->cfg.ctas_per_sm : -1;
    b->tuning = b->cfg.ctas_per_sm == 0;
    // ITLBM_BATCH_TILING=narrow | uniform fixes the tiling instead of timing it
    if (const char *v = getenv("ITLBM_BATCH_TILING")) {
        if (!strcmp(v, "narrow") || !strcmp(v, "uniform")) {
            b->narrow = !strcmp(v, "narrow");
            b->tile_fixed = true;
        }
    }
    for (int p = 0; p < NTAB; p++) b->occ[p] = step_occupancy(prec_of_table(p));
    const int M = b->cfg.max_cases;
    b->slots.assign(M, nullptr);
    for (int s = M - 1; s >= 0; s--) b->free_slots.push_back(s);
    b->h_cases.assign(M, CaseDev{});
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_cases, sizeof(CaseDev) * M)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_ntiles, sizeof(int) * NTAB)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_drop, sizeof(itlbm_drop_diag) * M)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_strip, sizeof(itlbm_strip_diag) * M)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_jobs, sizeof(DiagJob) * M)) != cudaSuccess ||
        (e = cudaHostAlloc((void **)&b->h_jobs, sizeof(DiagJob) * M, cudaHostAllocDefault)) != cudaSuccess ||
        (e = cudaHostAlloc((void **)&b->h_drop, sizeof(itlbm_drop_diag) * M, cudaHostAllocDefault)) != cudaSuccess ||
        (e = cudaHostAlloc((void **)&b->h_strip, sizeof(itlbm_strip_diag) * M, cudaHostAllocDefault)) != cudaSuccess) {
        itlbm_batch_destroy(b);
        return cuda_fail(e, "batch allocation");
    }
    cudaMemsetAsync(b->d_cases, 0, sizeof(CaseDev) * M, b->stream);
    cudaMemsetAsync(b->d_ntiles, 0, sizeof(int) * NTAB, b->stream);
    cudaStreamSynchronize(b->stream);
    // work tables with room for a first batch, so the graph can be captured with their addresses
    for (int p = 0; p < NTAB; p++) {
        b->tiles_cap[p] = 1 << 16;
        if ((e = cudaMalloc(&b->d_tiles[p], sizeof(TileRef) * b->tiles_cap[p])) != cudaSuccess) {
            itlbm_batch_destroy(b);
            return cuda_fail(e, "work table");
        }
    }
    cudaEventCreate(&b->ev0);
    cudaEventCreate(&b->ev1);
    cudaEventCreate(&b->ev2);
    for (int t = 0; t < 2; t++) cudaEventCreate(&b->tev[t]);
    if ((e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming)) != cudaSuccess) {
        itlbm_batch_destroy(b);
        return cuda_fail(e, "batch events");
    }
    for (int p = 0; p < NPREC; p++) {
        for (int sh = 0; sh < NSHAPE; sh++)
            if ((sh != SHAPE_32x8 &&
                 (e = cudaStreamCreateWithFlags(&b->shape_st[p][sh], cudaStreamNonBlocking)) != cudaSuccess) ||
                (e = cudaEventCreateWithFlags(&b->shape_ev[p][sh], cudaEventDisableTiming)) != cudaSuccess) {
                itlbm_batch_destroy(b);
                return cuda_fail(e, "batch streams");
            }
        if ((e = cudaEventCreateWithFlags(&b->shape_fork[p], cudaEventDisableTiming)) != cudaSuccess) {
            itlbm_batch_destroy(b);
            return cuda_fail(e, "batch streams");
        }
    }
    for (int p = 0; p < NPREC; p++)
        if ((e = cudaStreamCreateWithFlags(&b->side[p], cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&b->ev_join[p], cudaEventDisableTiming)) != cudaSuccess) {
            itlbm_batch_destroy(b);
            return cuda_fail(e, "batch streams");
        }
    b->t0 = std::chrono::steady_clock::now();
    int r = capture_graph(b);
    if (r) {
        itlbm_batch_destroy(b);
        return r;
    }
    *out = b;
    return ITLBM_OK;
}

void itlbm_batch_destroy(itlbm_batch *b) {
    if (!b) return;
    if (use_device(b->device) != ITLBM_OK) return;  // the device is gone: nothing left to free on it
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (Active *a : b->slots)
        if (a) {
            cudaFreeAsync(a->mem, b->stream);
            if (a->aux) cudaFreeAsync(a->aux, b->stream);
            delete a;
        }
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->d_cases) cudaFree(b->d_cases);
    for (int p = 0; p < NTAB; p++)
        if (b->d_tiles[p]) cudaFree(b->d_tiles[p]);
    if (b->d_ntiles) cudaFree(b->d_ntiles);
    if (b->d_drop) cudaFree(b->d_drop);
    if (b->d_strip) cudaFree(b->d_strip);
    if (b->d_jobs) cudaFree(b->d_jobs);
    if (b->d_blk) cudaFree(b->d_blk);
    if (b->dscratch) cudaFree(b->dscratch);
    if (b->h_jobs) cudaFreeHost(b->h_jobs);
    if (b->h_blk) cudaFreeHost(b->h_blk);
    if (b->h_drop) cudaFreeHost(b->h_drop);
    if (b->h_strip) cudaFreeHost(b->h_strip);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->ev2) cudaEventDestroy(b->ev2);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    for (int t = 0; t < 2; t++)
        if (b->tev[t]) cudaEventDestroy(b->tev[t]);
    for (int p = 0; p < NPREC; p++) {
        if (b->ev_join[p]) cudaEventDestroy(b->ev_join[p]);
        if (b->side[p]) cudaStreamDestroy(b->side[p]);
        if (b->shape_fork[p]) cudaEventDestroy(b->shape_fork[p]);
        for (int sh = 0; sh < NSHAPE; sh++) {
            if (b->shape_ev[p][sh]) cudaEventDestroy(b->shape_ev[p][sh]);
            if (b->shape_st[p][sh]) cudaStreamDestroy(b->shape_st[p][sh]);
        }
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->pool) cudaMemPoolDestroy(b->pool);
    if (b->stage) cudaFreeHost(b->stage);
    delete b;
}

int itlbm_batch_submit_saved(itlbm_batch *b, const char *path, int n_steps, long long tag) {
    if (!b || !path) return fail(ITLBM_E_ARG, "bad argument");
    SnapHeader hd;
    int r = snap_read_header(path, hd);
    if (r) return r;
    if (n_steps <= hd.steps) return fail(ITLBM_E_ARG, "the snapshot is already at or past n_steps");
    if ((r = itlbm_batch_submit(b, &hd.desc, n_steps, tag)) != ITLBM_OK) return r;
    b->pending.back().snapshot = path;
    b->pending.back().start = hd.steps;
    return ITLBM_OK;
}

int itlbm_batch_save(itlbm_batch *b, long long tag, const char *path) {
    if (!b || !path) return fail(ITLBM_E_ARG, "bad argument");
    if (int rd = use_device(b->device)) return rd;
    for (Active *a : b->slots) {
        if (!a || a->held || a->tag != tag) continue;
        cudaError_t e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return cuda_fail(e, "synchronize");
        const CaseDev &h = b->h_cases[a->slot];
        return snap_write(path, a->desc, a->next_step, h, h.buf[a->parity]);
    }
    return fail(ITLBM_E_ARG, "no active case with this tag");
}

int itlbm_batch_submit(itlbm_batch *b, const itlbm_case_desc *d, int n_steps, long long tag) {
    if (!b || !d || n_steps < 1) return fail(ITLBM_E_ARG, "bad argument");
    if (d->nx < 1 || d->ny < 1 || !box_tileable(d->nx, d->ny) || !(d->tau > 0.0) ||
        !prec_valid(d->precision) ||
        (d->geometry != ITLBM_GEOM_DROP && d->geometry != ITLBM_GEOM_STRIP) ||
        (d->geometry == ITLBM_GEOM_STRIP && (d->nx != d->ny || (d->p == 0 && d->q == 0))))
        return fail(ITLBM_E_ARG, "invalid case description");
    bool need_aux;
    if (case_bytes(*d, need_aux) > b->cfg.hbm_budget)
        return fail(ITLBM_E_ADMISSION, "case larger than the batch's HBM budget");
    b->pending.push_back(Pending{*d, n_steps, tag, b->now(), std::string(), 0});
    return ITLBM_OK;
}

int itlbm_batch_advance(itlbm_batch *b, void *stream) {
    (void)stream;  // the batch runs on its own stream (graphs cannot be captured on the legacy one)
    if (!b) return fail(ITLBM_E_ARG, "NULL batch");
    ScopeTimer timer(b, b->advance_ms);
    if (int rd = use_device(b->device)) return rd;
    int r;
    {
        ScopeTimer t_admit(b, b->admit_ms);
        r = admit(b);
    }
    if (r) return r;
    // plan: every case runs to its next diagnostic step, at most `chunk` steps
    const int de = b->cfg.diag_every;
    int K = 0, hi = -1;
    long long updates = 0;
    for (Active *a : b->slots) {
        if (!a || a->held) continue;
        hi = std::max(hi, a->slot);
        int d = ((a->next_step + de - 1) / de) * de;  // next multiple of diag_every >= next_step
        if (d > a->n_steps - 1) d = a->n_steps - 1;
        a->chunk_len = std::min(d - a->next_step + 1, b->cfg.chunk);
        a->diag_at_end = (a->next_step + a->chunk_len - 1 == d);
        CaseDev &h = b->h_cases[a->slot];
        h.parity0 = a->parity;
        h.chunk_len = a->chunk_len;
        h.aux_at_end = (a->diag_at_end && a->aux) ? 1 : 0;
        K = std::max(K, a->chunk_len);
        updates += (long long)a->chunk_len * a->desc.nx * a->desc.ny;
    }
    if (K == 0) return (int)b->events.size();
    // the descriptors up to the highest slot in use (the step kernels read no other)
    cudaError_t e = cudaMemcpyAsync(b->d_cases, b->h_cases.data(), sizeof(CaseDev) * (size_t)(hi + 1),
                                    cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "case table upload");
    if (b->tables_dirty) {
        TileRef *old[NTAB];
        int g[NTAB];
        for (int p = 0; p < NTAB; p++) {
            old[p] = b->d_tiles[p];
            g[p] = b->grid[p];
        }
        r = upload_tables(b);
        if (r) return r;
        bool changed = false;
        for (int p = 0; p < NTAB; p++) changed = changed || old[p] != b->d_tiles[p] || g[p] != b->grid[p];
        if (changed) {
            r = capture_graph(b);
            if (r) return r;
        }
        b->tables_dirty = false;
    }
    cudaEventRecord(b->ev0, b->stream);
    if (b->tuning && K == b->cfg.chunk && K >= 3 * TUNE_MIN_WINDOW) {
        r = tune_and_run(b, K);
        if (r) return r;
    } else if (K == b->cfg.chunk) {
        e = cudaGraphLaunch(b->graph, b->stream);
        if (e != cudaSuccess) return cuda_fail(e, "graph launch");
    } else {
        if ((e = enqueue_steps(b, 0, K)) != cudaSuccess) return cuda_fail(e, "step launches");
    }
    cudaEventRecord(b->ev1, b->stream);
    b->replays++;
    b->node_updates += updates;
    // diagnostics that fell due, all of them together
    std::vector<Active *> measured;
    for (Active *a : b->slots)
        if (a && !a->held && a->diag_at_end) measured.push_back(a);
    if ((r = run_diagnostics(b, measured)) != ITLBM_OK) return r;
    cudaEventRecord(b->ev2, b->stream);
    if (!measured.empty()) {
        int lo = INT_MAX, hi = -1;
        for (Active *a : measured) {
            lo = std::min(lo, a->slot);
            hi = std::max(hi, a->slot);
        }
        e = cudaMemcpyAsync(b->h_drop + lo, b->d_drop + lo, sizeof(itlbm_drop_diag) * (hi - lo + 1),
                            cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->h_strip + lo, b->d_strip + lo, sizeof(itlbm_strip_diag) * (hi - lo + 1),
                                cudaMemcpyDeviceToHost, b->stream);
        if (e != cudaSuccess) return cuda_fail(e, "diagnostic copy");
    }
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return cuda_fail(e, "replay");
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->device_ms += ms;
    if (!measured.empty() && cudaEventElapsedTime(&ms, b->ev1, b->ev2) == cudaSuccess) b->diag_ms += ms;
    const double t = b->now();
    std::vector<Active *> gone;
    for (Active *a : measured) {
        itlbm_batch_event ev{};
        ev.tag = a->tag;
        ev.kind = ITLBM_EV_DIAG;
        ev.geometry = a->desc.geometry;
        ev.step = a->next_step + a->chunk_len - 1;
        ev.t_submit = a->t_submit;
        ev.t_event = t;
        bool unstable;
        if (a->desc.geometry == ITLBM_GEOM_DROP) {
            ev.drop = b->h_drop[a->slot];
            ev.drop.step = ev.step;
            unstable = !ev.drop.ok || ev.drop.n_ruim > 0 || ev.drop.u_max > U_LIMITE;
        } else {
            ev.strip = b->h_strip[a->slot];
            ev.strip.step = ev.step;
            unstable = !ev.strip.ok || ev.strip.u_max > U_LIMITE;
        }
        b->events.push_back(ev);
        if (unstable || ev.step == a->n_steps - 1) {
            itlbm_batch_event fin = ev;
            fin.kind = unstable ? ITLBM_EV_UNSTABLE : ITLBM_EV_DONE;
            fin.step = unstable ? ev.step : a->n_steps;
            b->events.push_back(fin);
            gone.push_back(a);
        }
    }
    for (Active *a : b->slots) {
        if (!a || a->held) continue;
        a->next_step += a->chunk_len;
        a->parity ^= (a->chunk_len & 1);
        a->measured = a->diag_at_end;
    }
    for (Active *a : gone) retire(b, a);
    return (int)b->events.size();
}

int itlbm_batch_hold_finished(itlbm_batch *b, int on) {
    if (!b) return fail(ITLBM_E_ARG, "NULL batch");
    b->hold = on != 0;
    return ITLBM_OK;
}

namespace {
Active *find_tag(itlbm_batch *b, long long tag) {
    for (Active *a : b->slots)
        if (a && a->tag == tag) return a;
    return nullptr;
}
}  // namespace

int itlbm_batch_read_fields(itlbm_batch *b, long long tag, int form, double *rho_R, double *rho_B,
                            double *ux, double *uy, double *uz) {
    if (!b || (form != ITLBM_FIELDS_VTK && form != ITLBM_FIELDS_PROFILE)) return fail(ITLBM_E_ARG, "bad argument");
    Active *a = find_tag(b, tag);
    if (!a) return fail(ITLBM_E_ARG, "no active or held case with this tag");
    const bool force = a->desc.op.tipo >= ITLBM_OP_F1;
    if (a->next_step < 1 || (force && !a->measured))
        return fail(ITLBM_E_STATE, "the case's last step was not a measured one (class F needs its force)");
    if (int rd = use_device(b->device)) return rd;
    const size_t n = (size_t)a->desc.nx * a->desc.ny;
    double *t = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&t, sizeof(double) * 5 * n, b->pool, b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "field staging");
    // the post-collision populations of the last step sit in the buffer of the next step's state
    e = launch_fields(b->d_cases + a->slot, b->h_cases[a->slot], a->parity, force, form, t, t + n, t + 2 * n,
                      t + 3 * n, t + 4 * n, b->stream);
    double *outs[5] = {rho_R, rho_B, ux, uy, uz};
    for (int k = 0; k < 5 && e == cudaSuccess; k++)
        if (outs[k]) e = cudaMemcpyAsync(outs[k], t + k * n, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream);
    cudaFreeAsync(t, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "read_fields");
}

int itlbm_batch_release(itlbm_batch *b, long long tag) {
    if (!b) return fail(ITLBM_E_ARG, "NULL batch");
    Active *a = find_tag(b, tag);
    if (!a || !a->held) return fail(ITLBM_E_ARG, "no held case with this tag");
    if (int rd = use_device(b->device)) return rd;
    a->held = false;
    b->nheld--;
    const bool hold = b->hold;
    b->hold = false;
    b->finished--;  // retire() counts it again
    retire(b, a);
    b->hold = hold;
    return ITLBM_OK;
}

int itlbm_batch_poll(itlbm_batch *b, itlbm_batch_event *ev, int max) {
    if (!b || (max > 0 && !ev)) return fail(ITLBM_E_ARG, "bad argument");
    int n = 0;
    while (n < max && !b->events.empty()) {
        ev[n++] = b->events.front();
        b->events.pop_front();
    }
    return n;
}

int itlbm_batch_stats_get(const itlbm_batch *b, itlbm_batch_stats *out) {
    if (!b || !out) return fail(ITLBM_E_ARG, "bad argument");
    out->active = 0;
    for (Active *a : b->slots) out->active += (a && !a->held) ? 1 : 0;
    out->held = b->nheld;
    out->narrow_edges = b->narrow ? 1 : 0;
    out->pending = (int)b->pending.size();
    out->finished = b->finished;
    out->node_updates = b->node_updates;
    out->device_ms = b->device_ms;
    out->hbm_used = b->hbm_used;
    out->replays = b->replays;
    out->captures = b->captures;
    out->diag_ms = b->diag_ms;
    out->advance_ms = b->advance_ms;
    out->admit_ms = b->admit_ms;
    out->capture_ms = b->capture_ms;
    out->launch_mode = b->mode;
    return ITLBM_OK;
}

}  // extern "C"
