// engine.cu — host runtime behind include/mr_cuda.h.
//
// Owns devices buffers (a per-context caching pool), request validation,
// window computation, batch packing, the window-then-full-board retry and the
// result objects.  Nothing here searches on the CPU: every path and field is
// computed by the kernels in relax.cu, and any device failure is returned as a
// status so the caller can take its own CPU fallback (the contract of
// crates/mr-cpu/src/negotiated.rs:539-553).
#include <cuda.h>  // CUtensorMap and its encoder's types (the encoder is reached through the runtime)
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "kernels.h"
#include "mr_cuda.h"

using namespace mrc;

namespace {

thread_local std::string g_err;

mrc_status fail(mrc_status s, std::string msg) {
    g_err = std::move(msg);
    return s;
}

#define MRC_CUDA(call, what)                                                                        \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? MRC_ERR_OUT_OF_MEMORY : MRC_ERR_BACKEND_UNAVAILABLE, \
                        std::string(what) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

#define MRC_TRY(expr)                 \
    do {                              \
        mrc_status s_ = (expr);       \
        if (s_ != MRC_OK) return s_;  \
    } while (0)

// Grow-and-reuse device allocator; callers hold the context mutex.
class Pool {
   public:
    ~Pool() { trim(); }
    // Sizes above 1 MiB are rounded up to quarter-octave classes (2^k x 1,
    // 1.25, 1.5, 1.75), so blocks freed by one batch fit the next batches of
    // similar size and steady serving does not keep calling cudaMalloc (which
    // can synchronise the device) or cudaFree.
    static size_t size_class(size_t bytes) {
        bytes = std::max<size_t>((bytes + 255) & ~(size_t)255, 256);
        if (bytes <= (1u << 20)) return bytes;
        size_t p = 1u << 20;
        while (p * 2 <= bytes) p *= 2;
        const size_t q = p / 4;
        return (bytes + q - 1) / q * q;
    }
    cudaError_t alloc(size_t bytes, void **out) {
        bytes = size_class(bytes);
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes + (8u << 20)) {
            *out = it->second;
            used_[it->second] = it->first;
            cached_ -= it->first;
            free_.erase(it);
            return cudaSuccess;
        }
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            trim();
            e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) {
                (void)cudaGetLastError();
                return e;
            }
        }
        used_[p] = bytes;
        *out = p;
        return cudaSuccess;
    }
    void release(void *p) {
        if (!p) return;
        auto it = used_.find(p);
        if (it == used_.end()) return;
        free_.emplace(it->second, p);
        cached_ += it->second;
        used_.erase(it);
    }
    void trim() {
        for (auto &kv : free_) cudaFree(kv.second);
        free_.clear();
        cached_ = 0;
    }
    // bytes held in free blocks (device memory the pool can hand out again)
    size_t cached() const { return cached_; }

   private:
    std::multimap<size_t, void *> free_;
    std::unordered_map<void *, size_t> used_;
    size_t cached_ = 0;
};

}  // namespace

namespace {

// Phase trace: with MRC_TRACE set in the environment, the instance and batch
// calls print the host time of each phase to stderr.  The stream is
// synchronised at every mark so device work is charged to the phase that
// queued it (tracing therefore removes the overlap it measures around).
struct Trace {
    const char *call;
    cudaStream_t stream;
    std::chrono::steady_clock::time_point t0, t;
    static bool enabled() {
        static const bool on = std::getenv("MRC_TRACE") != nullptr;
        return on;
    }
    Trace(const char *c, cudaStream_t s) : call(c), stream(s), t0(std::chrono::steady_clock::now()), t(t0) {}
    void mark(const char *phase) {
        cudaStreamSynchronize(stream);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "mrc trace %s %-14s %8.3f ms (at %8.3f)\n", call, phase,
                     std::chrono::duration<double, std::milli>(now - t).count(),
                     std::chrono::duration<double, std::milli>(now - t0).count());
        t = now;
    }
};
thread_local Trace *g_trace = nullptr;
void trace_mark(const char *phase) {
    if (g_trace) g_trace->mark(phase);
}
struct TraceScope {
    std::unique_ptr<Trace> tr;
    TraceScope(const char *call, cudaStream_t s) {
        if (Trace::enabled()) {
            tr.reset(new Trace(call, s));
            g_trace = tr.get();
        }
    }
    ~TraceScope() {
        if (tr) g_trace = nullptr;
    }
};

// Pinned host staging reused across calls: host inputs are gathered here by
// several threads and reach HBM with full-rate asynchronous copies.
struct HostStage {
    void *p = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;  // the last copy out of the stage
    ~HostStage() {
        if (p) cudaFreeHost(p);
        if (done) cudaEventDestroy(done);
    }
    cudaError_t reserve(size_t n) {
        if (!done) {
            cudaError_t e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        cudaError_t e = cudaEventSynchronize(done);  // no copy may still read the old contents
        if (e != cudaSuccess) return e;
        if (n <= bytes) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t want = std::max(n + n / 4, (size_t)64 << 20);
        e = cudaHostAlloc(&p, want, cudaHostAllocMapped);
        if (e != cudaSuccess) return e;
        bytes = want;
        return cudaSuccess;
    }
};

}  // namespace

struct mrc_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    Pool pool;
    HostStage stage;
    int sms = 148;
    size_t smem_optin = 0;
    // autotuned relax configuration per (layers, directed): tile height, CTA
    // width, schedule (0 = bulk-synchronous rounds, 1 = asynchronous queue)
    std::map<uint32_t, std::array<uint32_t, 3>> tuned;
    uint32_t default_schedule = 1;  // for batches without a tuned configuration
    // board bytes moved to HBM since creation: through the pinned stage or a
    // pageable copy, and straight from the caller's page-locked arrays
    uint64_t staged_bytes = 0, in_place_bytes = 0;
};

namespace {

// RAII handle on a pool block.
struct DBuf {
    mrc_context *ctx = nullptr;
    void *p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { reset(); }
    void reset() {
        if (ctx && p) ctx->pool.release(p);
        p = nullptr;
        bytes = 0;
    }
    mrc_status get(mrc_context *c, size_t n, const char *what) {
        reset();
        ctx = c;
        bytes = n;
        MRC_CUDA(c->pool.alloc(n, &p), what);
        return MRC_OK;
    }
    template <class T>
    T *as() const {
        return reinterpret_cast<T *>(p);
    }
};

struct GridView {
    uint32_t w = 0, h = 0, layers = 0;
    uint64_t n = 0;
    const uint32_t *cost = nullptr;
    const uint8_t *board = nullptr;
    const uint8_t *via_forbidden = nullptr;
    bool obstacle(uint32_t c) const { return cost[c] == kMax; }
    bool board_forbidden(uint32_t c) const { return board && (board[c] & kTraceNode); }
};

mrc_status view_grid(const mrc_grid *g, GridView *v) {
    if (!g) return fail(MRC_ERR_INVALID_ARGUMENT, "grid is NULL");
    v->w = g->w;
    v->h = g->h;
    v->layers = g->layers == 0 ? 1 : g->layers;  // Dims::with_layers clamps to >= 1
    v->n = (uint64_t)v->w * v->h * v->layers;
    if (v->n > 0xFFFFFFFFull) return fail(MRC_ERR_MALFORMED_GRID, "grid exceeds the 32-bit CellIdx domain");
    if (v->n && !g->cost) return fail(MRC_ERR_MALFORMED_GRID, "grid cost is NULL");
    if (v->layers > 32) return fail(MRC_ERR_LIMIT, "more than 32 layers");
    v->cost = g->cost;
    v->board = g->board_constraint;
    v->via_forbidden = g->via_forbidden;
    return MRC_OK;
}

struct NetCopy {
    uint32_t src, dst;
    std::vector<uint32_t> pads, vpads;  // sorted, unique
    uint32_t board = 0;                 // index into the batch's boards
    uint32_t over_off = 0, n_over = 0;  // directed-price overrides on the board (negotiation with clearance)
};

bool sorted_contains(const std::vector<uint32_t> &v, uint32_t c) { return std::binary_search(v.begin(), v.end(), c); }

// Endpoint/pad validation: metal/src/lib.rs:446-467 and negotiated.rs:1392-1407,
// plus the board trace-node rule of route_variant (negotiated.rs:1483-1492).
mrc_status validate_nets(const GridView &g, const mrc_net *nets, uint32_t n, std::vector<NetCopy> *out) {
    if (n && !nets) return fail(MRC_ERR_INVALID_ARGUMENT, "nets is NULL");
    out->resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        const mrc_net &nt = nets[i];
        NetCopy &c = (*out)[i];
        c.src = nt.src;
        c.dst = nt.dst;
        if ((nt.n_passable_pads && !nt.passable_pads) || (nt.n_via_passable_pads && !nt.via_passable_pads))
            return fail(MRC_ERR_INVALID_ARGUMENT, "net " + std::to_string(i) + ": pad list pointer is NULL");
        c.pads.assign(nt.passable_pads, nt.passable_pads + nt.n_passable_pads);
        c.vpads.assign(nt.via_passable_pads, nt.via_passable_pads + nt.n_via_passable_pads);
        std::sort(c.pads.begin(), c.pads.end());
        c.pads.erase(std::unique(c.pads.begin(), c.pads.end()), c.pads.end());
        std::sort(c.vpads.begin(), c.vpads.end());
        c.vpads.erase(std::unique(c.vpads.begin(), c.vpads.end()), c.vpads.end());
        auto bad = [&](const char *why) {
            return fail(MRC_ERR_INVALID_ENDPOINT, "net " + std::to_string(i) + ": " + why);
        };
        for (uint32_t p : c.pads)
            if (p >= g.n) return bad("passable pad out of bounds");
        for (uint32_t p : c.vpads)
            if (p >= g.n || !sorted_contains(c.pads, p)) return bad("via pad out of bounds or not an own pad");
        if (c.src >= g.n || c.dst >= g.n) return bad("endpoint out of bounds");
        if (g.board_forbidden(c.src) || g.board_forbidden(c.dst)) return bad("endpoint outside the board outline");
        if (g.obstacle(c.src) && !sorted_contains(c.pads, c.src)) return bad("source on a foreign obstacle");
        if (g.obstacle(c.dst) && !sorted_contains(c.pads, c.dst)) return bad("target on a foreign obstacle");
    }
    return MRC_OK;
}

mrc_window full_window(uint32_t w, uint32_t h) { return mrc_window{0, 0, w ? w - 1 : 0, h ? h - 1 : 0}; }

// net_window, crates/mr-cpu/src/negotiated.rs:568-594.
mrc_window net_window(uint32_t w, uint32_t h, const NetCopy &n) {
    const uint32_t plane = w * h;
    auto xy = [&](uint32_t c, uint32_t *x, uint32_t *y) {
        const uint32_t r = c % plane;
        *x = r % w;
        *y = r / w;
    };
    uint32_t sx, sy, dx, dy;
    xy(n.src, &sx, &sy);
    xy(n.dst, &dx, &dy);
    uint32_t x0 = std::min(sx, dx), y0 = std::min(sy, dy), x1 = std::max(sx, dx), y1 = std::max(sy, dy);
    for (uint32_t p : n.pads) {
        uint32_t px, py;
        xy(p, &px, &py);
        x0 = std::min(x0, px);
        y0 = std::min(y0, py);
        x1 = std::max(x1, px);
        y1 = std::max(y1, py);
    }
    const uint32_t span = std::max(x1 - x0, y1 - y0);
    const uint32_t margin = std::max<uint32_t>(16, (3 * span + 9) / 10);
    mrc_window win;
    win.x0 = x0 > margin ? x0 - margin : 0;
    win.y0 = y0 > margin ? y0 - margin : 0;
    win.x1 = std::min<uint64_t>((uint64_t)x1 + margin, w ? w - 1 : 0);
    win.y1 = std::min<uint64_t>((uint64_t)y1 + margin, h ? h - 1 : 0);
    return win;
}

bool window_valid(const mrc_window &win, uint32_t w, uint32_t h) {
    return w > 0 && h > 0 && win.x0 <= win.x1 && win.y0 <= win.y1 && win.x1 < w && win.y1 < h;
}

bool is_full(const mrc_window &win, uint32_t w, uint32_t h) {
    return win.x0 == 0 && win.y0 == 0 && win.x1 + 1 == w && win.y1 + 1 == h;
}

}  // namespace

// ---------------------------------------------------------------------------
// Boards

struct mrc_board {
    mrc_context *ctx = nullptr;
    GridView view;                 // points into the host copies below
    std::vector<uint32_t> cost;    // host copy for endpoint validation
    std::vector<uint8_t> board;    // host copy of the board mask (may be empty)
    std::vector<uint8_t> viaf;     // host copy of the static via mask (may be empty)
    bool directed = false;
    DBuf d_cost, d_flags, d_x, d_y, d_via, d_dir;
    DevBoard dev{};
};

namespace {

// The device-readable address of page-locked, mapped host memory; null for
// pageable memory.
const void *mapped_host(const void *p) {
    if (!p) return nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

mrc_status upload(mrc_context *ctx, DBuf &buf, const void *src, size_t bytes, const char *what) {
    MRC_TRY(buf.get(ctx, std::max<size_t>(bytes, 4), what));
    if (bytes) MRC_CUDA(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream), what);
    return MRC_OK;
}

// Upload the board and its edge prices; `keep_host` keeps the validation copies.
mrc_status board_build(mrc_context *ctx, const mrc_grid *grid, const mrc_edges *edges, bool keep_host,
                       mrc_board *b) {
    MRC_TRY(view_grid(grid, &b->view));
    GridView &g = b->view;
    if (!edges) return fail(MRC_ERR_INVALID_ARGUMENT, "edges is NULL");
    const uint32_t ex = g.w ? g.w - 1 : 0, ey = g.h ? g.h - 1 : 0, ev = g.layers - 1;
    if (edges->n_x_edge_costs != ex || edges->n_y_edge_costs != ey || edges->n_via_edge_costs != ev)
        return fail(MRC_ERR_INVALID_ARGUMENT, "isolated batch shape does not match grid/nets");
    if ((ex && !edges->x_edge_costs) || (ey && !edges->y_edge_costs) ||
        (ev && (!edges->via_edge_costs || !edges->via_allowed)))
        return fail(MRC_ERR_INVALID_ARGUMENT, "edge price pointer is NULL");
    b->ctx = ctx;
    b->directed = edges->directed_in_costs != nullptr;
    // uploads read the caller's arrays (page-locked ones at full link rate)
    const uint32_t *src_cost = g.cost;
    const uint8_t *src_board = g.board, *src_viaf = g.via_forbidden;
    if (keep_host) {
        b->cost.assign(g.cost, g.cost + g.n);
        if (g.board) b->board.assign(g.board, g.board + g.n);
        if (g.via_forbidden) b->viaf.assign(g.via_forbidden, g.via_forbidden + g.n);
        g.cost = b->cost.data();
        g.board = g.board ? b->board.data() : nullptr;
        g.via_forbidden = g.via_forbidden ? b->viaf.data() : nullptr;
    }
    const size_t n = (size_t)g.n;
    {
        const size_t big = n * 4 + ((g.board || g.via_forbidden) ? n : 0) + (b->directed ? n * 16 : 0);
        const bool pinned = mapped_host(src_cost) && (!src_board || mapped_host(src_board)) &&
                            (!src_viaf || mapped_host(src_viaf)) &&
                            (!b->directed || mapped_host(edges->directed_in_costs));
        (pinned ? ctx->in_place_bytes : ctx->staged_bytes) += big;
    }
    MRC_TRY(upload(ctx, b->d_cost, src_cost, n * 4, "upload cost"));
    const bool has_flags = g.board || g.via_forbidden;
    if (has_flags) {
        if (g.board) {
            MRC_TRY(upload(ctx, b->d_flags, src_board, n, "upload board mask"));
        } else {
            MRC_TRY(b->d_flags.get(ctx, std::max<size_t>(n, 4), "board flags"));
            MRC_CUDA(cudaMemsetAsync(b->d_flags.p, 0, n, ctx->stream), "clear flags");
        }
        if (g.via_forbidden) {
            DBuf tmp;
            MRC_TRY(upload(ctx, tmp, src_viaf, n, "upload via mask"));
            MRC_CUDA(combine_flags_launch(b->d_flags.as<uint8_t>(), tmp.as<uint8_t>(), n, ctx->stream), "combine masks");
            MRC_CUDA(cudaStreamSynchronize(ctx->stream), "combine masks");
        }
    }
    std::vector<uint32_t> vias(std::max<uint32_t>(ev, 1), 0);
    uint32_t via_mask = 0;
    for (uint32_t k = 0; k < ev; ++k) {
        vias[k] = edges->via_edge_costs[k];
        if (edges->via_allowed[k]) via_mask |= 1u << k;
    }
    MRC_TRY(upload(ctx, b->d_x, edges->x_edge_costs, (size_t)ex * 4, "upload x edges"));
    MRC_TRY(upload(ctx, b->d_y, edges->y_edge_costs, (size_t)ey * 4, "upload y edges"));
    MRC_TRY(upload(ctx, b->d_via, vias.data(), vias.size() * 4, "upload via edges"));
    if (b->directed) MRC_TRY(upload(ctx, b->d_dir, edges->directed_in_costs, n * 16, "upload directed prices"));
    b->dev.w = g.w;
    b->dev.h = g.h;
    b->dev.layers = g.layers;
    b->dev.via_mask = via_mask;
    b->dev.cost = b->d_cost.as<uint32_t>();
    b->dev.flags = has_flags ? b->d_flags.as<uint8_t>() : nullptr;
    b->dev.x_edge = b->d_x.as<uint32_t>();
    b->dev.y_edge = b->d_y.as<uint32_t>();
    b->dev.via_edge = b->d_via.as<uint32_t>();
    b->dev.directed = b->directed ? b->d_dir.as<uint4>() : nullptr;
    return MRC_OK;
}

}  // namespace

namespace {

// Boards of many instances uploaded with one copy: each board's device arrays
// are 256-byte-aligned slices of one pool block.  The boards keep no host copy;
// their views point at the caller's arrays for the duration of the call.
struct BoardPack {
    DBuf data;
    DBuf spans;  // gather list of the page-locked upload
    std::vector<std::unique_ptr<mrc_board>> boards;
};

struct PackOff {
    size_t cost, flags, x, y, via, dir;
};

void pack_views(BoardPack *pk, const std::vector<PackOff> &offs) {
    unsigned char *base = pk->data.as<unsigned char>();
    for (size_t k = 0; k < offs.size(); ++k) {
        mrc_board &b = *pk->boards[k];
        const PackOff &o = offs[k];
        b.dev.w = b.view.w;
        b.dev.h = b.view.h;
        b.dev.layers = b.view.layers;
        b.dev.cost = reinterpret_cast<const uint32_t *>(base + o.cost);
        b.dev.flags = o.flags != SIZE_MAX ? base + o.flags : nullptr;
        b.dev.x_edge = reinterpret_cast<const uint32_t *>(base + o.x);
        b.dev.y_edge = reinterpret_cast<const uint32_t *>(base + o.y);
        b.dev.via_edge = reinterpret_cast<const uint32_t *>(base + o.via);
        b.dev.directed = o.dir != SIZE_MAX ? reinterpret_cast<const uint4 *>(base + o.dir) : nullptr;
    }
}

// Page-locked instances: the cost, mask and directed arrays are read in place by
// one gather launch; only the small edge vectors and the gather list pass
// through the stage.  `src[k]` holds the mapped addresses of instance k's cost,
// board mask, via mask and directed prices.
mrc_status board_pack_direct(mrc_context *ctx, const mrc_isolated_request *inst, uint32_t n, BoardPack *pk,
                             const std::vector<PackOff> &offs, size_t total,
                             const std::vector<std::array<const void *, 4>> &src) {
    MRC_TRY(pk->data.get(ctx, std::max<size_t>(total, 256), "instance boards"));
    auto up16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
    // stage layout: per instance the device bytes from o.x to the end of the via
    // prices (same padding as on the device), then the spans, then chunk starts
    std::vector<size_t> small(n);
    size_t sb = 0;
    for (uint32_t k = 0; k < n; ++k) {
        small[k] = sb;
        sb += up16(offs[k].via + (size_t)std::max(inst[k].edges.n_via_edge_costs, 1u) * 4 - offs[k].x);
    }
    const size_t max_spans = (size_t)4 * n;
    const size_t o_spans = sb, o_chunks = up16(o_spans + max_spans * sizeof(HostSpan));
    const size_t stage_bytes = o_chunks + max_spans * 8;
    MRC_CUDA(ctx->stage.reserve(stage_bytes), "pinned staging buffer");
    unsigned char *host = static_cast<unsigned char *>(ctx->stage.p);
    const unsigned char *host_dev = static_cast<const unsigned char *>(mapped_host(host));
    if (!host_dev) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "pinned staging buffer is not mapped into the device");
    HostSpan *spans = reinterpret_cast<HostSpan *>(host + o_spans);
    uint64_t *chunk = reinterpret_cast<uint64_t *>(host + o_chunks);
    unsigned char *base = pk->data.as<unsigned char>();
    uint32_t ns = 0;
    uint64_t nc = 0;
    auto add = [&](const void *a, const void *b, size_t off, size_t bytes, uint32_t kind) {
        if (!bytes) return;
        spans[ns] = HostSpan{a, b, base + off, bytes, kind};
        chunk[ns++] = nc;
        nc += host_gather_chunks(bytes);
    };
    for (uint32_t k = 0; k < n; ++k) {
        const GridView &g = pk->boards[k]->view;
        const mrc_edges &e = inst[k].edges;
        const PackOff &o = offs[k];
        unsigned char *sm = host + small[k];
        if (e.n_x_edge_costs) std::memcpy(sm, e.x_edge_costs, (size_t)e.n_x_edge_costs * 4);
        if (e.n_y_edge_costs) std::memcpy(sm + (o.y - o.x), e.y_edge_costs, (size_t)e.n_y_edge_costs * 4);
        uint32_t *via = reinterpret_cast<uint32_t *>(sm + (o.via - o.x));
        uint32_t mask = 0;
        via[0] = 0;
        for (uint32_t i = 0; i < e.n_via_edge_costs; ++i) {
            via[i] = e.via_edge_costs[i];
            if (e.via_allowed[i]) mask |= 1u << i;
        }
        pk->boards[k]->dev.via_mask = mask;
        ctx->in_place_bytes += (size_t)g.n * 4 + (o.flags != SIZE_MAX ? g.n : 0) + (o.dir != SIZE_MAX ? (size_t)g.n * 16 : 0);
        add(src[k][0], nullptr, o.cost, (size_t)g.n * 4, 0);
        if (o.flags != SIZE_MAX) add(src[k][1], src[k][2], o.flags, g.n, g.via_forbidden ? 1 : 0);
        if (o.dir != SIZE_MAX) add(src[k][3], nullptr, o.dir, (size_t)g.n * 16, 0);
        add(host_dev + small[k], nullptr, o.x, o.via + (size_t)std::max(e.n_via_edge_costs, 1u) * 4 - o.x, 0);
    }
    // the gather list itself goes over in one copy (the kernel searches it per chunk)
    const size_t list_bytes = up16((size_t)ns * sizeof(HostSpan)) + (size_t)ns * 8;
    MRC_TRY(pk->spans.get(ctx, std::max<size_t>(list_bytes, 256), "gather list"));
    unsigned char *dl = pk->spans.as<unsigned char>();
    MRC_CUDA(cudaMemcpyAsync(dl, spans, (size_t)ns * sizeof(HostSpan), cudaMemcpyHostToDevice, ctx->stream),
             "upload gather list");
    const size_t dchunk = up16((size_t)ns * sizeof(HostSpan));
    MRC_CUDA(cudaMemcpyAsync(dl + dchunk, chunk, (size_t)ns * 8, cudaMemcpyHostToDevice, ctx->stream),
             "upload gather list");
    MRC_CUDA(host_gather_launch(reinterpret_cast<const HostSpan *>(dl), reinterpret_cast<const uint64_t *>(dl + dchunk),
                                ns, nc, (uint32_t)ctx->sms, ctx->stream),
             "gather instance boards");
    MRC_CUDA(cudaEventRecord(ctx->stage.done, ctx->stream), "stage event");
    pack_views(pk, offs);
    return MRC_OK;
}

mrc_status board_pack_build(mrc_context *ctx, const mrc_isolated_request *inst, uint32_t n, BoardPack *pk) {
    using Off = PackOff;
    std::vector<Off> offs(n);
    size_t total = 0;
    auto take = [&](size_t bytes) {
        const size_t o = total;
        total += (std::max<size_t>(bytes, 4) + 255) & ~(size_t)255;
        return o;
    };
    pk->boards.clear();
    for (uint32_t k = 0; k < n; ++k) {
        std::unique_ptr<mrc_board> b(new mrc_board());
        MRC_TRY(view_grid(inst[k].grid, &b->view));
        const GridView &g = b->view;
        const mrc_edges &e = inst[k].edges;
        const uint32_t ex = g.w ? g.w - 1 : 0, ey = g.h ? g.h - 1 : 0, ev = g.layers - 1;
        if (e.n_x_edge_costs != ex || e.n_y_edge_costs != ey || e.n_via_edge_costs != ev)
            return fail(MRC_ERR_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": edge vectors do not match its grid");
        if ((ex && !e.x_edge_costs) || (ey && !e.y_edge_costs) || (ev && (!e.via_edge_costs || !e.via_allowed)))
            return fail(MRC_ERR_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": edge price pointer is NULL");
        b->ctx = ctx;
        b->directed = e.directed_in_costs != nullptr;
        Off &o = offs[k];
        o.cost = take(g.n * 4);
        o.flags = (g.board || g.via_forbidden) ? take(g.n) : SIZE_MAX;
        o.x = take((size_t)ex * 4);
        o.y = take((size_t)ey * 4);
        o.via = take((size_t)std::max(ev, 1u) * 4);
        o.dir = b->directed ? take(g.n * 16) : SIZE_MAX;
        pk->boards.push_back(std::move(b));
    }
    // page-locked inputs (every large array of every instance mapped) are read in place
    if (n && mapped_host(pk->boards[0]->view.cost)) {
        std::vector<std::array<const void *, 4>> src(n);
        bool all = true;
        for (uint32_t k = 0; k < n && all; ++k) {
            const GridView &g = pk->boards[k]->view;
            const void *dir = inst[k].edges.directed_in_costs;
            src[k] = {mapped_host(g.cost), mapped_host(g.board), mapped_host(g.via_forbidden), mapped_host(dir)};
            all = src[k][0] && (!g.board || src[k][1]) && (!g.via_forbidden || src[k][2]) && (!dir || src[k][3]);
        }
        if (all) return board_pack_direct(ctx, inst, n, pk, offs, total, src);
    }
    MRC_TRY(pk->data.get(ctx, std::max<size_t>(total, 256), "instance boards"));
    MRC_CUDA(ctx->stage.reserve(total), "pinned staging buffer");
    ctx->staged_bytes += total;
    unsigned char *host = static_cast<unsigned char *>(ctx->stage.p);
    auto fill = [&](uint32_t k) {
        const GridView &g = pk->boards[k]->view;
        const mrc_edges &e = inst[k].edges;
        const Off &o = offs[k];
        std::memcpy(host + o.cost, g.cost, g.n * 4);
        if (o.flags != SIZE_MAX) {
            uint8_t *fl = host + o.flags;
            if (!g.via_forbidden) {
                std::memcpy(fl, g.board, g.n);
            } else {
                for (uint64_t i = 0; i < g.n; ++i)
                    fl[i] = (uint8_t)((g.board ? g.board[i] : 0) | (g.via_forbidden[i] ? kStaticVia : 0));
            }
        }
        if (e.n_x_edge_costs) std::memcpy(host + o.x, e.x_edge_costs, (size_t)e.n_x_edge_costs * 4);
        if (e.n_y_edge_costs) std::memcpy(host + o.y, e.y_edge_costs, (size_t)e.n_y_edge_costs * 4);
        uint32_t *via = reinterpret_cast<uint32_t *>(host + o.via);
        uint32_t mask = 0;
        for (uint32_t i = 0; i < e.n_via_edge_costs; ++i) {
            via[i] = e.via_edge_costs[i];
            if (e.via_allowed[i]) mask |= 1u << i;
        }
        if (o.dir != SIZE_MAX) std::memcpy(host + o.dir, e.directed_in_costs, g.n * 16);
        pk->boards[k]->dev.via_mask = mask;
    };
    // Worker threads fill instances in index order; this thread ships every
    // completed prefix of >= 32 MB to the device while the rest is still filled.
    const uint32_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const uint32_t nthreads = total > (64u << 20) ? std::min(hw, n) : 1;
    std::vector<std::atomic<uint8_t>> done(n);
    for (auto &d : done) d.store(0, std::memory_order_relaxed);
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> workers;
    auto work = [&]() {
        for (uint32_t k; (k = next.fetch_add(1, std::memory_order_relaxed)) < n;) {
            fill(k);
            done[k].store(1, std::memory_order_release);
        }
    };
    for (uint32_t t = 1; t < nthreads; ++t) workers.emplace_back(work);
    if (nthreads == 1) work();
    size_t shipped = 0;
    uint32_t ready = 0;
    cudaError_t ce = cudaSuccess;
    while (shipped < total && ce == cudaSuccess) {
        while (ready < n && done[ready].load(std::memory_order_acquire)) ++ready;
        const size_t upto = ready == n ? total : offs[ready].cost;
        if (upto > shipped && (upto - shipped >= (32u << 20) || ready == n)) {
            ce = cudaMemcpyAsync(pk->data.as<unsigned char>() + shipped, host + shipped, upto - shipped,
                                 cudaMemcpyHostToDevice, ctx->stream);
            shipped = upto;
        } else {
            std::this_thread::yield();
        }
    }
    for (auto &t : workers) t.join();
    MRC_CUDA(ce, "upload instance boards");
    MRC_CUDA(cudaEventRecord(ctx->stage.done, ctx->stream), "stage event");
    pack_views(pk, offs);
    return MRC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Results

struct mrc_result {
    uint32_t n = 0;
    uint32_t retried = 0;
    std::vector<uint64_t> offsets;
    std::vector<uint32_t> cells;
    std::vector<uint32_t> costs;
    bool has_fields = false;
    std::vector<uint64_t> field_offsets;
    std::vector<uint32_t> fields;
    std::vector<mrc_window> field_windows;
};

// ---------------------------------------------------------------------------
// Batches

struct mrc_batch {
    mrc_context *ctx = nullptr;
    std::vector<const mrc_board *> boards;  // a batch may span many boards
    uint32_t max_layers = 1;
    bool directed_any = false;
    bool has_over = false;         // some net prices its own directed overrides (not the warp schedule)
    uint32_t flags = 0;
    std::vector<NetCopy> nets;
    std::vector<mrc_window> windows;
    std::vector<DevField> fields;  // ascending lab_off (largest windows first)
    uint64_t total_cells = 0;
    uint32_t total_tiles = 0, max_tiles = 0, tile_h = 32, threads = kRelaxThreads, grid = 1;
    size_t smem = 0;
    DBuf d_tover;                  // per tile: holds price overrides of its field (has_over batches)
    DBuf d_boards, d_fields, d_pads, d_lab, d_tstamp, d_tvisit, d_lists, d_costs, d_lens, d_offsets, d_cells, d_ctl,
        d_out;
    uint32_t launches = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;  // captured launch sequence (mrc_batch_capture_graph)
    // Set before batch_build by callers that run several batches at once: a
    // fixed tile configuration, a shared-memory floor (every concurrent batch
    // has the same per-CTA footprint) and a divisor of the co-resident grid.
    uint32_t force_tile_h = 0, force_threads = 0, grid_num = 1, grid_div = 1;
    bool grid_by_work = false;  // the grid may grow past grid_num/grid_div up to what the tiles can use
    bool async_q = false;  // relax schedule: asynchronous work queue instead of rounds
    bool warp = false;     // the warp-per-tile schedule (implies the queue and a +inf-filled arena)
    bool cta_planes = true;  // the CTA queue form stages step prices from the price planes by TMA
    size_t smem_floor = 0;
    std::vector<DevBoard> devs;  // the board table (step-price plane pointers patched in by batch_layout)
    DBuf d_planes, d_pchunks;    // step-price planes of every board, chunk table of their kernel
    DBuf d_tmaps;                // one TMA tensor map per board over its planes (CTA queue form)
    uint64_t n_pchunks = 0;
    // the planes hold prices of the batch's boards, which never change: computed by
    // the first launch after a layout and kept for the launches that follow
    bool planes_valid = false;
    ~mrc_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

namespace {

// Default tile height when the context holds no autotuned choice: 8-row tiles
// (the autotuner's pick on every measured workload), else the smallest taller
// tile that fits; the caller pairs it with 256 threads and the queue schedule.
mrc_status choose_tile(mrc_context *ctx, uint32_t layers, bool directed, uint32_t *tile_h, size_t *smem) {
    const size_t hard = std::min<size_t>(ctx->smem_optin ? ctx->smem_optin : (227u << 10), 227u << 10) - 1024;
    for (size_t budget : {(size_t)(75u << 10), (size_t)(110u << 10), hard}) {
        for (uint32_t th : {8u, 16u, 32u, 64u}) {
            const size_t s = std::max(relax_smem_bytes(layers, th, directed, true), relax_smem_bytes(layers, th, directed, false));
            if (s <= budget) {
                *tile_h = th;
                *smem = s;
                return MRC_OK;
            }
        }
    }
    return fail(MRC_ERR_LIMIT, "too many layers for one shared-memory tile");
}

uint32_t tune_key(uint32_t layers, bool directed) { return layers * 2u + (directed ? 1u : 0u); }

// cuTensorMapEncodeTiled, looked up once through the runtime's driver entry
// point (the library links only the CUDA runtime).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

mrc_status encode_fn(EncodeTiledFn *out) {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (err == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    if (!fn) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "cuTensorMapEncodeTiled is not available");
    *out = fn;
    return MRC_OK;
}

// The tensor map of one board's price planes: u32 elements, dims {pitch, h,
// layers, 6}, a box of kPlaneTmaBoxW x tile_h x layers x 6 (one tile's planes).
mrc_status encode_planes_map(const DevBoard &d, uint32_t tile_h, CUtensorMap *map) {
    EncodeTiledFn enc = nullptr;
    MRC_TRY(encode_fn(&enc));
    const uint64_t wp = planes_pitch(d.w);
    const cuuint64_t dims[4] = {wp, d.h, d.layers, 6};
    const cuuint64_t strides[3] = {wp * 4, wp * d.h * 4, wp * d.h * d.layers * 4};
    const cuuint32_t box[4] = {kPlaneTmaBoxW, tile_h, d.layers, 6};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, d.planes, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "encode price-plane tensor map: error " +
                                                                   std::to_string((int)r));
    return MRC_OK;
}

// Tile-dependent layout of a staged batch: tile offsets, the CTA grid and the
// per-tile buffers.  Re-run by the autotuner for every candidate.
mrc_status batch_layout(mrc_batch *bt, uint32_t tile_h, uint32_t threads) {
    mrc_context *ctx = bt->ctx;
    if (bt->graph) {  // a captured graph bakes in the old layout
        cudaGraphExecDestroy(bt->graph);
        bt->graph = nullptr;
    }
    bt->planes_valid = false;
    if (bt->warp && bt->max_layers > kWarpMaxLayers) bt->warp = false;  // too many layers for one warp tile
    if (bt->has_over) {  // per-net price overrides: CTA tiles of one shape (the kernels compiled with them)
        if (bt->warp) {
            bt->warp = false;
            bt->cta_planes = true;
        }
        tile_h = kOverTileH;
        threads = kOverThreads;
    }
    if (bt->warp) bt->async_q = true;
    const bool cta_pl = bt->async_q && !bt->warp && bt->cta_planes;
    bt->tile_h = bt->warp ? kWarpTileH : tile_h;
    bt->threads = bt->warp ? warp_relax_threads() : threads;
    bt->smem =
        bt->warp ? 0 : std::max(relax_smem_bytes(bt->max_layers, tile_h, bt->directed_any, cta_pl), bt->smem_floor);
    uint64_t toff = 0;
    uint32_t max_tiles = 1;
    for (DevField &f : bt->fields) {
        const uint32_t tw = bt->warp ? warp_tile_w(bt->boards[f.board]->view.layers) : 32u;
        const uint64_t tiles = (uint64_t)((f.ww + tw - 1) / tw) * ((f.wh + bt->tile_h - 1) / bt->tile_h);
        f.tile_off = (uint32_t)std::min<uint64_t>(toff, 0xFFFFFFFFull);
        toff += tiles;
        max_tiles = (uint32_t)std::max<uint64_t>(max_tiles, tiles);
    }
    if (toff > 0x7FFFFFFFull) return fail(MRC_ERR_LIMIT, "batch has more than 2^31 tiles");
    bt->total_tiles = (uint32_t)std::max<uint64_t>(toff, 1);
    bt->max_tiles = max_tiles;
    int per_sm = 1;
    if (bt->warp) {
        MRC_CUDA(warp_relax_occupancy(&per_sm), "relax occupancy");
    } else {
        MRC_CUDA(relax_configure(tile_h, threads, bt->smem, bt->async_q, cta_pl, bt->has_over),
                 "configure relax kernel");
        MRC_CUDA(relax_occupancy(tile_h, threads, bt->smem, &per_sm, bt->async_q, cta_pl, bt->has_over),
                 "relax occupancy");
    }
    if (per_sm < 1) return fail(MRC_ERR_LIMIT, "relax kernel does not fit on one SM");
    // cooperative launch: every CTA must be co-resident
    const uint64_t full = (uint64_t)ctx->sms * (uint32_t)per_sm;
    uint64_t grid = full * bt->grid_num / std::max(1u, bt->grid_div);
    // a launch with work for the whole device takes it (its CTAs start as the
    // CTAs of launches already in flight exit: the queue form needs no co-residency)
    if (bt->grid_by_work && bt->async_q) grid = std::max(grid, std::min<uint64_t>(full, toff / kTilesPerCta));
    bt->grid = (uint32_t)std::max<uint64_t>(1u, grid);
    // board table, with the step-price planes of every board (warp schedule,
    // CTA queue form) and their tensor maps (CTA queue form)
    if (bt->warp || cta_pl) {
        std::vector<uint64_t> poff(bt->devs.size()), chunks(bt->devs.size() + 1, 0);
        uint64_t total = 0;
        for (size_t k = 0; k < bt->devs.size(); ++k) {
            const DevBoard &d = bt->devs[k];
            const uint64_t cells = (uint64_t)d.w * d.h * d.layers;
            poff[k] = total;
            total += ((uint64_t)planes_pitch(d.w) * d.h * d.layers * 6 * 4 + 255) & ~(uint64_t)255;
            chunks[k + 1] = chunks[k] + planes_chunks(cells);
        }
        MRC_TRY(bt->d_planes.get(ctx, std::max<uint64_t>(total, 256), "step-price planes"));
        for (size_t k = 0; k < bt->devs.size(); ++k)
            bt->devs[k].planes = reinterpret_cast<uint32_t *>(bt->d_planes.as<unsigned char>() + poff[k]);
        bt->n_pchunks = chunks.back();
        MRC_TRY(upload(ctx, bt->d_pchunks, chunks.data(), chunks.size() * 8, "plane chunk table"));
        if (cta_pl) {
            std::vector<CUtensorMap> maps(bt->devs.size());
            for (size_t k = 0; k < bt->devs.size(); ++k) MRC_TRY(encode_planes_map(bt->devs[k], tile_h, &maps[k]));
            // pool blocks are 256-byte aligned: every 128-byte map is 64-byte aligned
            MRC_TRY(upload(ctx, bt->d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), "tensor maps"));
            for (size_t k = 0; k < bt->devs.size(); ++k) bt->devs[k].tmap = bt->d_tmaps.as<CUtensorMap>() + k;
        } else {
            for (DevBoard &d : bt->devs) d.tmap = nullptr;
            bt->d_tmaps.reset();
        }
    } else {
        for (DevBoard &d : bt->devs) {
            d.planes = nullptr;
            d.tmap = nullptr;
        }
        bt->d_planes.reset();
        bt->d_tmaps.reset();
        bt->n_pchunks = 0;
    }
    MRC_TRY(upload(ctx, bt->d_boards, bt->devs.data(), bt->devs.size() * sizeof(DevBoard), "upload board table"));
    MRC_TRY(upload(ctx, bt->d_fields, bt->fields.data(), bt->fields.size() * sizeof(DevField), "upload fields"));
    MRC_TRY(bt->d_tstamp.get(ctx, (size_t)bt->total_tiles * 4, "tile stamps"));
    MRC_TRY(bt->d_tvisit.get(ctx, (size_t)bt->total_tiles * 4, "tile flags"));
    if (bt->has_over) MRC_TRY(bt->d_tover.get(ctx, (size_t)bt->total_tiles, "override tile flags"));
    else bt->d_tover.reset();
    MRC_TRY(bt->d_lists.get(ctx, (size_t)bt->total_tiles * 3 * 8, "tile lists"));
    return MRC_OK;
}

mrc_status batch_build(mrc_context *ctx, std::vector<const mrc_board *> boards, std::vector<NetCopy> nets,
                       std::vector<mrc_window> windows, uint32_t flags, mrc_batch *bt) {
    bt->ctx = ctx;
    bt->boards = std::move(boards);
    bt->flags = flags;
    bt->nets = std::move(nets);
    bt->windows = std::move(windows);
    bt->max_layers = 1;
    bt->directed_any = false;
    for (const mrc_board *b : bt->boards) {
        bt->max_layers = std::max(bt->max_layers, b->view.layers);
        bt->directed_any = bt->directed_any || b->directed;
    }
    const uint32_t n = (uint32_t)bt->nets.size();
    bt->has_over = false;
    for (const NetCopy &nc : bt->nets) bt->has_over = bt->has_over || nc.n_over;
    uint32_t tile_h = 0, threads = kRelaxThreads;
    size_t smem = 0;
    auto tuned = ctx->tuned.find(tune_key(bt->max_layers, bt->directed_any));
    if (bt->force_tile_h) {
        tile_h = bt->force_tile_h;
        threads = bt->force_threads ? bt->force_threads : kRelaxThreads;
    } else if (tuned != ctx->tuned.end()) {
        tile_h = tuned->second[0];
        threads = tuned->second[1];
        bt->async_q = tuned->second[2] != 0;
        bt->warp = tuned->second[2] == 2;
        bt->cta_planes = tuned->second[2] != 3;
    } else {
        MRC_TRY(choose_tile(ctx, bt->max_layers, bt->directed_any, &tile_h, &smem));
        bt->async_q = ctx->default_schedule != 0;
        bt->warp = ctx->default_schedule == 2;
        bt->cta_planes = ctx->default_schedule != 3;
    }
    // largest windows first: the persistent CTAs then finish together
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    auto cells_of = [&](uint32_t i) {
        const mrc_window &w = bt->windows[i];
        return (uint64_t)(w.x1 - w.x0 + 1) * (w.y1 - w.y0 + 1) * bt->boards[bt->nets[i].board]->view.layers;
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cells_of(a) > cells_of(b); });
    std::vector<uint32_t> pads;
    bt->fields.resize(n);
    uint64_t off = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t i = order[k];
        const NetCopy &nc = bt->nets[i];
        const mrc_window &w = bt->windows[i];
        DevField &f = bt->fields[k];
        f.src = nc.src;
        f.dst = nc.dst;
        f.x0 = w.x0;
        f.y0 = w.y0;
        f.ww = w.x1 - w.x0 + 1;
        f.wh = w.y1 - w.y0 + 1;
        f.lab_off = off;
        off += cells_of(i);
        f.pad_off = (uint32_t)pads.size();
        f.n_pads = (uint32_t)nc.pads.size();
        pads.insert(pads.end(), nc.pads.begin(), nc.pads.end());
        f.vpad_off = (uint32_t)pads.size();
        f.n_vpads = (uint32_t)nc.vpads.size();
        pads.insert(pads.end(), nc.vpads.begin(), nc.vpads.end());
        f.out = i;
        f.tile_off = 0;
        f.board = nc.board;
        f.n_over = nc.n_over;
        f.over_off = nc.over_off;
        f.pad_ = 0;
        if (pads.size() > 0xFFFFFFF0u) return fail(MRC_ERR_LIMIT, "pad lists exceed 2^32 entries");
    }
    bt->total_cells = off;
    bt->devs.clear();
    bt->devs.reserve(bt->boards.size());
    for (const mrc_board *b : bt->boards) bt->devs.push_back(b->dev);
    MRC_TRY(batch_layout(bt, tile_h, threads));
    MRC_TRY(upload(ctx, bt->d_pads, pads.data(), pads.size() * 4, "upload pads"));
    MRC_TRY(bt->d_lab.get(ctx, std::max<uint64_t>(off, 1) * 8, "labels"));
    MRC_TRY(bt->d_costs.get(ctx, std::max<size_t>(n, 1) * 4, "costs"));
    MRC_TRY(bt->d_lens.get(ctx, std::max<size_t>(n, 1) * 4, "lengths"));
    MRC_TRY(bt->d_offsets.get(ctx, ((size_t)n + 1) * 8, "offsets"));
    MRC_TRY(bt->d_cells.get(ctx, std::max<uint64_t>(off, 1) * 4, "path cells"));
    MRC_TRY(bt->d_ctl.get(ctx, sizeof(Ctl), "control block"));
    if (flags & MRC_FLAG_KEEP_FIELDS) MRC_TRY(bt->d_out.get(ctx, std::max<uint64_t>(off, 1) * 4, "fields"));
    if (flags & MRC_FLAG_TIME_KERNELS) {
        MRC_CUDA(cudaEventCreate(&bt->ev0), "create event");
        MRC_CUDA(cudaEventCreate(&bt->ev1), "create event");
    }
    return MRC_OK;
}

PathArgs path_args(const mrc_batch *bt) {
    PathArgs pa{};
    pa.boards = bt->d_boards.as<DevBoard>();
    pa.fields = bt->d_fields.as<DevField>();
    pa.n_fields = (uint32_t)bt->fields.size();
    pa.pads = bt->d_pads.as<uint32_t>();
    pa.lab = bt->d_lab.as<u64>();
    pa.tvisit = bt->d_tvisit.as<uint32_t>();
    pa.tover = bt->has_over ? bt->d_tover.as<uint8_t>() : nullptr;
    pa.tile_h = bt->tile_h;
    pa.arena_filled = bt->async_q ? 1u : 0u;
    const bool cta_pl = bt->async_q && !bt->warp && bt->cta_planes;
    const size_t ws = walk_smem_bytes(bt->max_layers, bt->tile_h);
    pa.walk_smem = (cta_pl && !bt->has_over && ws <= kWalkSmemLimit) ? (uint32_t)ws : 0u;
    pa.costs = bt->d_costs.as<uint32_t>();
    pa.lens = bt->d_lens.as<uint32_t>();
    pa.offsets = bt->d_offsets.as<unsigned long long>();
    pa.cells = bt->d_cells.as<uint32_t>();
    pa.status = &bt->d_ctl.as<Ctl>()->status;
    return pa;
}

// The launch sequence of one batch: reset, relax, paths (+ fields).
// Under stream capture the events become event-record nodes of the graph, so a
// replay still times the relax kernel alone.
mrc_status batch_enqueue(mrc_batch *bt, cudaStream_t st, bool capturing) {
    const uint32_t n = (uint32_t)bt->fields.size();
    uint32_t launches = 0;
    MRC_CUDA(cudaMemsetAsync(bt->d_ctl.p, 0, sizeof(Ctl), st), "reset control block");
    MRC_CUDA(cudaMemsetAsync(bt->d_tstamp.p, 0, (size_t)bt->total_tiles * 4, st), "reset tile stamps");
    MRC_CUDA(cudaMemsetAsync(bt->d_tvisit.p, 0, (size_t)bt->total_tiles * 4, st), "reset tile flags");
    RelaxArgs ra{};
    ra.boards = bt->d_boards.as<DevBoard>();
    ra.max_layers = bt->max_layers;
    ra.fields = bt->d_fields.as<DevField>();
    ra.n_fields = n;
    ra.pads = bt->d_pads.as<uint32_t>();
    ra.lab = bt->d_lab.as<u64>();
    ra.tstamp = bt->d_tstamp.as<uint32_t>();
    ra.tvisit = bt->d_tvisit.as<uint32_t>();
    ra.tover = nullptr;
    if (bt->has_over && n) {
        MRC_CUDA(cudaMemsetAsync(bt->d_tover.p, 0, (size_t)bt->total_tiles, st), "reset override tile flags");
        MRC_CUDA(mark_over_tiles_launch(bt->d_fields.as<DevField>(), n, bt->d_boards.as<DevBoard>(), bt->tile_h,
                                        bt->d_tover.as<uint8_t>(), st),
                 "mark override tiles");
        ++launches;
        ra.tover = bt->d_tover.as<uint8_t>();
    }
    ra.lists = bt->d_lists.as<u64>();
    ra.list_cap = bt->total_tiles;
    ra.ctl = bt->d_ctl.as<Ctl>();
    ra.tile_h = bt->tile_h;
    ra.round_limit = 64u * bt->max_tiles + 4096u;
    ra.activation_limit = 1024ull * bt->total_tiles + 65536ull;  // runaway guard, far above any measured need
    if (n && bt->async_q) {
        MRC_CUDA(cudaMemsetAsync(bt->d_lab.p, 0xFF, bt->total_cells * 8, st), "fill label arena");
        MRC_CUDA(cudaMemsetAsync(bt->d_lists.as<u64>() + bt->total_tiles, 0, (size_t)bt->total_tiles * 8, st),
                 "reset queue tags");
    }
    if (n) {
        const unsigned rec = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
        if (bt->ev0) MRC_CUDA(cudaEventRecordWithFlags(bt->ev0, st, rec), "record event");
        const bool cta_pl = bt->async_q && !bt->warp && bt->cta_planes;
        if ((bt->warp || cta_pl) && !bt->planes_valid) {
            MRC_CUDA(planes_launch(bt->d_boards.as<DevBoard>(), bt->d_pchunks.as<uint64_t>(),
                                   (uint32_t)bt->devs.size(), bt->n_pchunks, (uint32_t)bt->ctx->sms, st),
                     "launch step-price planes");
            launches += 1;
            // a captured graph recomputes them on every replay (it is captured with
            // valid planes, see mrc_batch_capture_graph, so this is the fallback)
            if (!capturing) bt->planes_valid = true;
        }
        if (bt->warp) {
            MRC_CUDA(warp_relax_launch(ra, bt->grid, st), "launch relax kernel");
            launches += 2;  // seeds, relax
        } else {
            MRC_CUDA(relax_launch(ra, bt->grid, bt->threads, bt->smem, st, bt->async_q, cta_pl, bt->has_over),
                     "launch relax kernel");
            launches += bt->async_q ? 2 : 1;  // (+ the seed kernel)
        }
        if (bt->ev1) MRC_CUDA(cudaEventRecordWithFlags(bt->ev1, st, rec), "record event");
    }
    const PathArgs pa = path_args(bt);
    MRC_CUDA(path_launch(pa, st), "launch path kernels");
    launches += n ? 2 : 1;
    if (bt->d_out.p && n) {
        MRC_CUDA(fields_launch(pa, bt->d_out.as<uint32_t>(), bt->total_cells, st), "launch field emit");
        launches++;
    }
    bt->launches = launches;
    return MRC_OK;
}

mrc_status batch_launch(mrc_batch *bt, cudaStream_t st) {
    bt->stream = st;
    if (bt->graph) {
        MRC_CUDA(cudaGraphLaunch(bt->graph, st), "replay graph");
        return MRC_OK;
    }
    return batch_enqueue(bt, st, false);
}

mrc_status status_error(uint32_t status) {
    if (status & (kStatusActivationLimit | kStatusRoundLimit))
        return fail(MRC_ERR_ITERATION_LIMIT, "a field hit its relaxation bound");
    if (status & kStatusBarrier) return fail(MRC_ERR_ITERATION_LIMIT, "grid barrier wait exceeded its bound");
    if (status & kStatusPathBroken) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "canonical path reconstruction failed");
    return fail(MRC_ERR_BACKEND_UNAVAILABLE, "tile queue overflow");
}

// Copy one batch's outputs (indexed like bt->nets).
mrc_status batch_collect(mrc_batch *bt, bool keep_fields, std::vector<uint32_t> *costs,
                         std::vector<std::vector<uint32_t>> *paths, std::vector<std::vector<uint32_t>> *fields) {
    cudaStream_t st = bt->stream;
    const uint32_t n = (uint32_t)bt->fields.size();
    uint32_t status = 0;
    MRC_CUDA(cudaMemcpyAsync(&status, &bt->d_ctl.as<Ctl>()->status, 4, cudaMemcpyDeviceToHost, st), "read status");
    std::vector<uint64_t> off(n + 1);
    costs->assign(n, kMax);
    if (n) MRC_CUDA(cudaMemcpyAsync(costs->data(), bt->d_costs.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "read costs");
    MRC_CUDA(cudaMemcpyAsync(off.data(), bt->d_offsets.p, ((size_t)n + 1) * 8, cudaMemcpyDeviceToHost, st), "read offsets");
    MRC_CUDA(cudaStreamSynchronize(st), "batch execution");
    if (status) return status_error(status);
    std::vector<uint32_t> cells(off[n]);
    if (off[n]) MRC_CUDA(cudaMemcpy(cells.data(), bt->d_cells.p, off[n] * 4, cudaMemcpyDeviceToHost), "read paths");
    paths->assign(n, {});
    for (uint32_t i = 0; i < n; ++i) (*paths)[i].assign(cells.begin() + off[i], cells.begin() + off[i + 1]);
    if (keep_fields) {
        fields->assign(n, {});
        std::vector<uint32_t> all(bt->total_cells);
        if (bt->total_cells && bt->d_out.p)
            MRC_CUDA(cudaMemcpy(all.data(), bt->d_out.p, bt->total_cells * 4, cudaMemcpyDeviceToHost), "read fields");
        for (const DevField &f : bt->fields) {
            const uint64_t c = (uint64_t)f.ww * f.wh * bt->boards[f.board]->view.layers;
            (*fields)[f.out].assign(all.begin() + f.lab_off, all.begin() + f.lab_off + c);
        }
    }
    return MRC_OK;
}

mrc_status finish_batch(mrc_context *ctx, mrc_batch *bt, uint32_t flags, mrc_result **out);

// Run a batch synchronously and, with MRC_FLAG_RETRY_FULL, re-solve on its full
// board every net whose window solve was unreachable (cli/src/lib.rs:574-607).
mrc_status solve(mrc_context *ctx, std::vector<const mrc_board *> boards, std::vector<NetCopy> nets,
                 std::vector<mrc_window> wins, uint32_t flags, mrc_result **out, mrc_batch *prepared) {
    std::unique_ptr<mrc_batch> own;
    mrc_batch *bt = prepared;
    if (!bt) {
        own.reset(new mrc_batch());
        bt = own.get();
        MRC_TRY(batch_build(ctx, std::move(boards), std::move(nets), std::move(wins), flags, bt));
        trace_mark("batch build");
        MRC_TRY(batch_launch(bt, ctx->stream));
        trace_mark("kernels");
    }
    MRC_TRY(finish_batch(ctx, bt, flags, out));
    trace_mark("results");
    return MRC_OK;
}

// Results of a launched batch (waits for it), with the full-board retry.
mrc_status finish_batch(mrc_context *ctx, mrc_batch *bt, uint32_t flags, mrc_result **out) {
    const bool keep = (flags & MRC_FLAG_KEEP_FIELDS) != 0;
    std::vector<uint32_t> costs;
    std::vector<std::vector<uint32_t>> paths, fields;
    MRC_TRY(batch_collect(bt, keep, &costs, &paths, &fields));
    std::unique_ptr<mrc_result> r(new mrc_result());
    const uint32_t n = (uint32_t)bt->nets.size();
    r->n = n;
    r->field_windows = bt->windows;
    if (flags & MRC_FLAG_RETRY_FULL) {
        std::vector<uint32_t> idx;
        for (uint32_t i = 0; i < n; ++i) {
            const GridView &g = bt->boards[bt->nets[i].board]->view;
            if (costs[i] == kMax && !is_full(bt->windows[i], g.w, g.h)) idx.push_back(i);
        }
        if (!idx.empty()) {
            std::vector<NetCopy> rn;
            std::vector<mrc_window> rw;
            for (uint32_t i : idx) {
                rn.push_back(bt->nets[i]);
                const GridView &g = bt->boards[bt->nets[i].board]->view;
                rw.push_back(full_window(g.w, g.h));
            }
            mrc_batch retry;
            MRC_TRY(batch_build(ctx, bt->boards, std::move(rn), std::move(rw), flags & ~MRC_FLAG_TIME_KERNELS, &retry));
            // on the engine stream, behind the retry batch's own uploads
            MRC_TRY(batch_launch(&retry, ctx->stream));
            std::vector<uint32_t> c2;
            std::vector<std::vector<uint32_t>> p2, f2;
            MRC_TRY(batch_collect(&retry, keep, &c2, &p2, &f2));
            for (size_t k = 0; k < idx.size(); ++k) {
                costs[idx[k]] = c2[k];
                paths[idx[k]] = std::move(p2[k]);
                if (keep) fields[idx[k]] = std::move(f2[k]);
                r->field_windows[idx[k]] = retry.windows[k];
            }
            r->retried = (uint32_t)idx.size();
        }
    }
    r->costs = std::move(costs);
    r->offsets.resize(n + 1);
    uint64_t o = 0;
    for (uint32_t i = 0; i < n; ++i) {
        r->offsets[i] = o;
        o += paths[i].size();
    }
    r->offsets[n] = o;
    r->cells.reserve(o);
    for (auto &p : paths) r->cells.insert(r->cells.end(), p.begin(), p.end());
    if (keep) {
        r->has_fields = true;
        r->field_offsets.resize(n + 1);
        uint64_t fo = 0;
        for (uint32_t i = 0; i < n; ++i) {
            r->field_offsets[i] = fo;
            fo += fields[i].size();
        }
        r->field_offsets[n] = fo;
        r->fields.reserve(fo);
        for (auto &f : fields) r->fields.insert(r->fields.end(), f.begin(), f.end());
    }
    *out = r.release();
    return MRC_OK;
}

mrc_status collect_windows(const GridView &g, const std::vector<NetCopy> &nets, const mrc_window *windows,
                           std::vector<mrc_window> *out) {
    out->resize(nets.size());
    for (size_t i = 0; i < nets.size(); ++i) {
        (*out)[i] = windows ? windows[i] : net_window(g.w, g.h, nets[i]);
        if (!window_valid((*out)[i], g.w, g.h))
            return fail(MRC_ERR_INVALID_ARGUMENT, "net " + std::to_string(i) + " has an invalid isolated-route window");
    }
    return MRC_OK;
}

struct Lock {
    std::unique_lock<std::mutex> lk;
    mrc_status st = MRC_OK;
    Lock(mrc_context *ctx, uint32_t flags) : lk(ctx->mu, std::defer_lock) {
        if (flags & MRC_FLAG_NO_WAIT) {
            if (!lk.try_lock()) st = fail(MRC_ERR_BUSY, "CUDA isolated batch is busy");
        } else {
            lk.lock();
        }
    }
};

mrc_status set_device(mrc_context *ctx) {
    MRC_CUDA(cudaSetDevice(ctx->device), "select device");
    return MRC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

uint32_t mrc_abi_version(void) { return MRC_ABI_VERSION; }

const char *mrc_last_error(const mrc_context *) { return g_err.c_str(); }

mrc_status mrc_context_create(int device, mrc_context **out) {
    if (!out) return fail(MRC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return fail(MRC_ERR_BACKEND_UNAVAILABLE, "no CUDA device is available");
    }
    if (device < 0 || device >= count) return fail(MRC_ERR_INVALID_ARGUMENT, "device index out of range");
    std::unique_ptr<mrc_context> ctx(new mrc_context());
    ctx->device = device;
    MRC_CUDA(cudaSetDevice(device), "select device");
    cudaDeviceProp prop;
    MRC_CUDA(cudaGetDeviceProperties(&prop, device), "device properties");
    if (prop.major < 10) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "device is not sm_100 class");
    ctx->sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    MRC_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "create stream");
    *out = ctx.release();
    return MRC_OK;
}

void mrc_context_destroy(mrc_context *ctx) {
    if (!ctx) return;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        if (ctx->stream) {
            cudaStreamSynchronize(ctx->stream);
            cudaStreamDestroy(ctx->stream);
        }
        ctx->pool.trim();
    }
    delete ctx;
}

mrc_status mrc_host_alloc(mrc_context *ctx, size_t bytes, void **out) {
    if (!ctx || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    MRC_TRY(set_device(ctx));
    void *p = nullptr;
    if (cudaHostAlloc(&p, std::max<size_t>(bytes, 16), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(MRC_ERR_OUT_OF_MEMORY, "page-locked host allocation of " + std::to_string(bytes) + " bytes failed");
    }
    *out = p;
    return MRC_OK;
}

void mrc_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

mrc_status mrc_upload_stats(mrc_context *ctx, uint64_t *staged_bytes, uint64_t *in_place_bytes) {
    if (!ctx || !staged_bytes || !in_place_bytes) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    *staged_bytes = ctx->staged_bytes;
    *in_place_bytes = ctx->in_place_bytes;
    return MRC_OK;
}

mrc_status mrc_net_windows(uint32_t w, uint32_t h, uint32_t layers, const mrc_net *nets, uint32_t n_nets,
                           mrc_window *out) {
    if ((n_nets && (!nets || !out))) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    (void)layers;
    for (uint32_t i = 0; i < n_nets; ++i) {
        NetCopy c;
        c.src = nets[i].src;
        c.dst = nets[i].dst;
        if (nets[i].n_passable_pads && !nets[i].passable_pads)
            return fail(MRC_ERR_INVALID_ARGUMENT, "pad list pointer is NULL");
        c.pads.assign(nets[i].passable_pads, nets[i].passable_pads + nets[i].n_passable_pads);
        out[i] = net_window(w, h, c);
    }
    return MRC_OK;
}

mrc_status mrc_route_isolated_batch(mrc_context *ctx, const mrc_isolated_request *req, uint32_t flags,
                                    mrc_result **out) {
    if (!ctx || !req || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, flags);
    if (lock.st != MRC_OK) return lock.st;
    MRC_TRY(set_device(ctx));
    TraceScope trace("route_isolated_batch", ctx->stream);
    GridView g;
    MRC_TRY(view_grid(req->grid, &g));
    if (req->n_nets && !req->windows) return fail(MRC_ERR_INVALID_ARGUMENT, "windows is NULL");
    std::vector<NetCopy> nets;
    MRC_TRY(validate_nets(g, req->nets, req->n_nets, &nets));
    std::vector<mrc_window> wins;
    MRC_TRY(collect_windows(g, nets, req->windows, &wins));
    trace_mark("validate");
    mrc_board board;
    MRC_TRY(board_build(ctx, req->grid, &req->edges, false, &board));
    trace_mark("board upload");
    if (nets.empty()) {
        *out = new mrc_result();
        (*out)->offsets.assign(1, 0);
        (*out)->has_fields = (flags & MRC_FLAG_KEEP_FIELDS) != 0;
        (*out)->field_offsets.assign(1, 0);
        return MRC_OK;
    }
    return solve(ctx, {&board}, std::move(nets), std::move(wins), flags, out, nullptr);
}

mrc_status mrc_route_lee(mrc_context *ctx, const mrc_grid *grid, const mrc_net *nets, uint32_t n_nets,
                         mrc_result **out) {
    if (!ctx || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    GridView g;
    MRC_TRY(view_grid(grid, &g));
    std::vector<NetCopy> nc;
    MRC_TRY(validate_nets(g, nets, n_nets, &nc));
    // LeeRouter: unit edge prices, no vias, the whole board (lee.rs:46-64)
    std::vector<uint32_t> ones(std::max<uint32_t>(std::max(g.w, g.h), 1), 1u);
    std::vector<uint32_t> via0(std::max<uint32_t>(g.layers, 1), 0u);
    std::vector<uint8_t> noallow(std::max<uint32_t>(g.layers, 1), 0);
    mrc_edges e{ones.data(), g.w ? g.w - 1 : 0, ones.data(), g.h ? g.h - 1 : 0, via0.data(), noallow.data(),
                g.layers - 1, nullptr};
    mrc_board board;
    MRC_TRY(board_build(ctx, grid, &e, false, &board));
    if (nc.empty()) {
        *out = new mrc_result();
        (*out)->offsets.assign(1, 0);
        return MRC_OK;
    }
    std::vector<mrc_window> wins(nc.size(), full_window(g.w, g.h));
    return solve(ctx, {&board}, std::move(nc), std::move(wins), 0, out, nullptr);
}

mrc_status mrc_distance_fields(mrc_context *ctx, const mrc_grid *grid, const uint32_t *sources, uint32_t n_sources,
                               uint32_t *fields) {
    if (!ctx || (n_sources && (!sources || !fields))) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    GridView g;
    MRC_TRY(view_grid(grid, &g));
    std::vector<NetCopy> nc;
    std::vector<uint32_t> slot;
    for (uint32_t i = 0; i < n_sources; ++i) {
        const uint32_t s = sources[i];
        if (g.n && s < g.n && !g.obstacle(s) && !g.board_forbidden(s)) {
            NetCopy c;
            c.src = s;
            c.dst = s;
            nc.push_back(std::move(c));
            slot.push_back(i);
        } else if (g.n) {
            std::fill(fields + (size_t)i * g.n, fields + (size_t)(i + 1) * g.n, kMax);
        }
    }
    if (nc.empty() || g.n == 0) return MRC_OK;
    std::vector<uint32_t> ones(std::max<uint32_t>(std::max(g.w, g.h), 1), 1u);
    std::vector<uint32_t> via0(std::max<uint32_t>(g.layers, 1), 0u);
    std::vector<uint8_t> noallow(std::max<uint32_t>(g.layers, 1), 0);
    mrc_edges e{ones.data(), g.w - 1, ones.data(), g.h - 1, via0.data(), noallow.data(), g.layers - 1, nullptr};
    mrc_board board;
    MRC_TRY(board_build(ctx, grid, &e, false, &board));
    std::vector<mrc_window> wins(nc.size(), full_window(g.w, g.h));
    mrc_result *r = nullptr;
    MRC_TRY(solve(ctx, {&board}, std::move(nc), std::move(wins), MRC_FLAG_KEEP_FIELDS, &r, nullptr));
    std::unique_ptr<mrc_result> hold(r);
    for (size_t k = 0; k < slot.size(); ++k)
        std::memcpy(fields + (size_t)slot[k] * g.n, r->fields.data() + r->field_offsets[k], (size_t)g.n * 4);
    return MRC_OK;
}

mrc_status mrc_route_instances(mrc_context *ctx, const mrc_isolated_request *instances, uint32_t n_instances,
                               uint32_t flags, mrc_result **out) {
    if (!ctx || !out || (n_instances && !instances)) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, flags);
    if (lock.st != MRC_OK) return lock.st;
    MRC_TRY(set_device(ctx));
    TraceScope trace("route_instances", ctx->stream);
    std::vector<NetCopy> nets;
    std::vector<mrc_window> wins;
    for (uint32_t k = 0; k < n_instances; ++k) {
        GridView g;
        MRC_TRY(view_grid(instances[k].grid, &g));
        if (instances[k].n_nets && !instances[k].windows)
            return fail(MRC_ERR_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": windows is NULL");
        std::vector<NetCopy> nk;
        MRC_TRY(validate_nets(g, instances[k].nets, instances[k].n_nets, &nk));
        std::vector<mrc_window> wk;
        MRC_TRY(collect_windows(g, nk, instances[k].windows, &wk));
        for (NetCopy &c : nk) c.board = k;
        nets.insert(nets.end(), std::make_move_iterator(nk.begin()), std::make_move_iterator(nk.end()));
        wins.insert(wins.end(), wk.begin(), wk.end());
    }
    if (nets.empty()) {
        *out = new mrc_result();
        (*out)->offsets.assign(1, 0);
        (*out)->has_fields = (flags & MRC_FLAG_KEEP_FIELDS) != 0;
        (*out)->field_offsets.assign(1, 0);
        return MRC_OK;
    }
    trace_mark("validate");
    BoardPack pk;
    MRC_TRY(board_pack_build(ctx, instances, n_instances, &pk));
    trace_mark("board upload");
    std::vector<const mrc_board *> boards;
    for (auto &b : pk.boards) boards.push_back(b.get());
    return solve(ctx, std::move(boards), std::move(nets), std::move(wins), flags, out, nullptr);
}

uint32_t mrc_result_count(const mrc_result *r) { return r ? r->n : 0; }
const uint64_t *mrc_result_path_offsets(const mrc_result *r) { return r ? r->offsets.data() : nullptr; }
const uint32_t *mrc_result_path_cells(const mrc_result *r) { return r ? r->cells.data() : nullptr; }
const uint32_t *mrc_result_search_costs(const mrc_result *r) { return r ? r->costs.data() : nullptr; }
const uint64_t *mrc_result_field_offsets(const mrc_result *r) {
    return r && r->has_fields ? r->field_offsets.data() : nullptr;
}
const uint32_t *mrc_result_fields(const mrc_result *r) { return r && r->has_fields ? r->fields.data() : nullptr; }
const mrc_window *mrc_result_field_windows(const mrc_result *r) { return r ? r->field_windows.data() : nullptr; }
uint32_t mrc_result_retried(const mrc_result *r) { return r ? r->retried : 0; }
void mrc_result_free(mrc_result *r) { delete r; }

mrc_status mrc_board_create(mrc_context *ctx, const mrc_grid *grid, const mrc_edges *edges, mrc_board **out) {
    if (!ctx || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    std::unique_ptr<mrc_board> b(new mrc_board());
    MRC_TRY(board_build(ctx, grid, edges, true, b.get()));
    MRC_CUDA(cudaStreamSynchronize(ctx->stream), "upload board");
    *out = b.release();
    return MRC_OK;
}

void mrc_board_destroy(mrc_board *board) {
    if (!board) return;
    mrc_context *ctx = board->ctx;
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        delete board;
    } else {
        delete board;
    }
}

mrc_status mrc_batch_create(mrc_context *ctx, const mrc_board *board, const mrc_net *nets, uint32_t n_nets,
                            const mrc_window *windows, uint32_t flags, mrc_batch **out) {
    if (!ctx || !board || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, flags);
    if (lock.st != MRC_OK) return lock.st;
    MRC_TRY(set_device(ctx));
    std::vector<NetCopy> nc;
    MRC_TRY(validate_nets(board->view, nets, n_nets, &nc));
    std::vector<mrc_window> wins;
    MRC_TRY(collect_windows(board->view, nc, windows, &wins));
    std::unique_ptr<mrc_batch> bt(new mrc_batch());
    MRC_TRY(batch_build(ctx, {board}, std::move(nc), std::move(wins), flags, bt.get()));
    MRC_CUDA(cudaStreamSynchronize(ctx->stream), "stage batch");
    *out = bt.release();
    return MRC_OK;
}

mrc_status mrc_batch_create_multi(mrc_context *ctx, const mrc_board *const *boards, uint32_t n_boards,
                                  const mrc_net *nets, const uint32_t *net_board, uint32_t n_nets,
                                  const mrc_window *windows, uint32_t flags, mrc_batch **out) {
    if (!ctx || !out || !boards || !n_boards || (n_nets && !net_board))
        return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, flags);
    if (lock.st != MRC_OK) return lock.st;
    MRC_TRY(set_device(ctx));
    std::vector<NetCopy> nc(n_nets);
    std::vector<mrc_window> wins(n_nets);
    for (uint32_t i = 0; i < n_nets; ++i) {
        const uint32_t k = net_board[i];
        if (k >= n_boards || !boards[k]) return fail(MRC_ERR_INVALID_ARGUMENT, "net board index out of range");
        std::vector<NetCopy> one;
        MRC_TRY(validate_nets(boards[k]->view, nets + i, 1, &one));
        std::vector<mrc_window> w;
        MRC_TRY(collect_windows(boards[k]->view, one, windows ? windows + i : nullptr, &w));
        nc[i] = std::move(one[0]);
        nc[i].board = k;
        wins[i] = w[0];
    }
    std::unique_ptr<mrc_batch> bt(new mrc_batch());
    MRC_TRY(batch_build(ctx, std::vector<const mrc_board *>(boards, boards + n_boards), std::move(nc), std::move(wins),
                        flags, bt.get()));
    MRC_CUDA(cudaStreamSynchronize(ctx->stream), "stage batch");
    *out = bt.release();
    return MRC_OK;
}

mrc_status mrc_batch_capture_graph(mrc_context *ctx, mrc_batch *batch) {
    if (!ctx || !batch) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    if (batch->graph) {
        cudaGraphExecDestroy(batch->graph);
        batch->graph = nullptr;
    }
    // the boards' price planes first, outside the graph: they stay valid for
    // every replay of this layout
    const bool cta_pl = batch->async_q && !batch->warp && batch->cta_planes;
    if ((batch->warp || cta_pl) && !batch->planes_valid && !batch->fields.empty()) {
        MRC_CUDA(planes_launch(batch->d_boards.as<DevBoard>(), batch->d_pchunks.as<uint64_t>(),
                               (uint32_t)batch->devs.size(), batch->n_pchunks, (uint32_t)ctx->sms, ctx->stream),
                 "launch step-price planes");
        MRC_CUDA(cudaStreamSynchronize(ctx->stream), "step-price planes");
        batch->planes_valid = true;
    }
    cudaStream_t cs = nullptr;
    MRC_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    mrc_status rc = MRC_OK;
    if (e == cudaSuccess) {
        rc = batch_enqueue(batch, cs, true);
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (rc == MRC_OK && e2 != cudaSuccess) rc = fail(MRC_ERR_BACKEND_UNAVAILABLE, std::string("end capture: ") + cudaGetErrorString(e2));
    } else {
        rc = fail(MRC_ERR_BACKEND_UNAVAILABLE, std::string("begin capture: ") + cudaGetErrorString(e));
    }
    if (rc == MRC_OK) {
        e = cudaGraphInstantiate(&batch->graph, g, 0);
        if (e != cudaSuccess) rc = fail(MRC_ERR_BACKEND_UNAVAILABLE, std::string("instantiate graph: ") + cudaGetErrorString(e));
    }
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    (void)cudaGetLastError();
    return rc;
}

mrc_status mrc_batch_launch(mrc_context *ctx, mrc_batch *batch, void *stream) {
    if (!ctx || !batch) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    return batch_launch(batch, stream ? (cudaStream_t)stream : ctx->stream);
}

mrc_status mrc_batch_finish(mrc_context *ctx, mrc_batch *batch, mrc_result **out) {
    if (!ctx || !batch || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    if (!batch->stream) return fail(MRC_ERR_INVALID_ARGUMENT, "batch was never launched");
    return solve(ctx, batch->boards, {}, {}, batch->flags, out, batch);
}

mrc_status mrc_batch_autotune(mrc_context *ctx, mrc_batch *batch, uint32_t *tile_h, uint32_t *threads,
                              float *best_ms) {
    if (!ctx || !batch) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    const uint32_t layers = batch->max_layers;
    const size_t hard = std::min<size_t>(ctx->smem_optin ? ctx->smem_optin : (227u << 10), 227u << 10) - 1024;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MRC_CUDA(cudaEventCreate(&e0), "create event");
    MRC_CUDA(cudaEventCreate(&e1), "create event");
    float best = -1.0f;
    uint32_t best_th = batch->tile_h, best_nt = batch->threads;
    uint32_t best_sched = batch->warp ? 2u : !batch->async_q ? 0u : batch->cta_planes ? 1u : 3u;
    mrc_status rc = MRC_OK;
    // candidates: (tile height, CTA width, schedule); the warp schedule has one shape
    std::vector<std::array<uint32_t, 3>> cands;
    if (layers <= kWarpMaxLayers) cands.push_back({kWarpTileH, warp_relax_threads(), 2u});
    for (uint32_t th : {8u, 16u, 32u, 64u}) {
        if (relax_smem_bytes(layers, th, batch->directed_any, true) > hard ||
            relax_smem_bytes(layers, th, batch->directed_any, false) > hard)
            continue;
        for (uint32_t nt : {128u, 256u}) {
            if (4u * layers * th < nt / 2) continue;  // most lanes would idle in the line passes
            for (uint32_t sched : {0u, 1u, 3u}) cands.push_back({th, nt, sched});
        }
    }
    for (const auto &cand : cands) {
        {
            const uint32_t th = cand[0], nt = cand[1], sched = cand[2];
            batch->async_q = sched != 0;
            batch->warp = sched == 2;
            batch->cta_planes = sched != 3;
            rc = batch_layout(batch, th, nt);
            if (rc != MRC_OK) break;
            float ms = 0.0f, sum = 0.0f;
            sum = -1.0f;  // the fastest of three timed launches after one that warms the configuration
            for (int rep = 0; rep < 4 && rc == MRC_OK; ++rep) {
                cudaEventRecord(e0, ctx->stream);
                rc = batch_launch(batch, ctx->stream);
                cudaEventRecord(e1, ctx->stream);
                if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = fail(MRC_ERR_BACKEND_UNAVAILABLE, "autotune");
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep && (sum < 0.0f || ms < sum)) sum = ms;
            }
            if (rc != MRC_OK) break;
            if (best < 0.0f || sum < best) {
                best = sum;
                best_th = th;
                best_nt = nt;
                best_sched = sched;
            }
        }
        if (rc != MRC_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != MRC_OK) return rc;
    batch->async_q = best_sched != 0;
    batch->warp = best_sched == 2;
    batch->cta_planes = best_sched != 3;
    MRC_TRY(batch_layout(batch, best_th, best_nt));
    ctx->tuned[tune_key(layers, batch->directed_any)] = {best_th, best_nt, best_sched};
    if (tile_h) *tile_h = best_th;
    if (threads) *threads = best_nt;
    if (best_ms) *best_ms = best;
    return MRC_OK;
}

mrc_status mrc_batch_set_config(mrc_context *ctx, mrc_batch *batch, uint32_t tile_h, uint32_t threads) {
    if (!ctx || !batch) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((tile_h != 8 && tile_h != 16 && tile_h != 32 && tile_h != 64) || (threads != 128 && threads != 256))
        return fail(MRC_ERR_INVALID_ARGUMENT, "tile height must be 8/16/32/64 and threads 128/256");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    const size_t hard = std::min<size_t>(ctx->smem_optin ? ctx->smem_optin : (227u << 10), 227u << 10) - 1024;
    if (relax_smem_bytes(batch->max_layers, tile_h, batch->directed_any, true) > hard ||
        relax_smem_bytes(batch->max_layers, tile_h, batch->directed_any, false) > hard)
        return fail(MRC_ERR_LIMIT, "tile does not fit in shared memory");
    return batch_layout(batch, tile_h, threads);
}

mrc_status mrc_batch_set_schedule(mrc_context *ctx, mrc_batch *batch, uint32_t schedule) {
    if (!ctx || !batch) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (schedule > 3)
        return fail(MRC_ERR_INVALID_ARGUMENT,
                    "schedule must be 0 (rounds), 1 (queue), 2 (warp tiles) or 3 (queue, prices computed per tile)");
    if (schedule == 2 && batch->max_layers > kWarpMaxLayers)
        return fail(MRC_ERR_LIMIT, "the warp schedule takes boards of at most 16 layers");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    const bool was_warp = batch->warp;
    batch->async_q = schedule >= 1;
    batch->warp = schedule == 2;
    batch->cta_planes = schedule != 3;
    // leaving the warp schedule: the default CTA tile (8 rows, 256 threads)
    return batch_layout(batch, was_warp ? 8u : batch->tile_h, was_warp ? 256u : batch->threads);
}

mrc_status mrc_context_set_schedule(mrc_context *ctx, uint32_t schedule) {
    if (!ctx) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (schedule > 3) return fail(MRC_ERR_INVALID_ARGUMENT, "default schedule must be 0, 1, 2 or 3");
    Lock lock(ctx, 0);
    ctx->default_schedule = schedule;
    return MRC_OK;
}

mrc_status mrc_batch_config(const mrc_batch *batch, uint32_t *tile_h, uint32_t *threads, uint32_t *schedule) {
    if (!batch) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (tile_h) *tile_h = batch->tile_h;
    if (threads) *threads = batch->threads;
    if (schedule) *schedule = batch->warp ? 2u : !batch->async_q ? 0u : batch->cta_planes ? 1u : 3u;
    return MRC_OK;
}

uint32_t mrc_batch_kernel_launches(const mrc_batch *batch) { return batch ? batch->launches : 0; }
uint64_t mrc_batch_window_cells(const mrc_batch *batch) { return batch ? batch->total_cells : 0; }

mrc_status mrc_batch_stats(const mrc_batch *batch, uint64_t out[4]) {
    if (!batch || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    if (batch->d_ctl.p) MRC_CUDA(cudaMemcpy(&c, batch->d_ctl.p, sizeof(Ctl), cudaMemcpyDeviceToHost), "read counters");
    out[0] = c.activations;
    out[1] = c.sweeps;
    out[2] = batch->warp ? c.rows : c.rounds;
    out[3] = batch->total_tiles;
    return MRC_OK;
}

float mrc_batch_relax_ms(const mrc_batch *batch) {
    if (!batch || !batch->ev0 || !batch->ev1) return -1.0f;
    float ms = -1.0f;
    if (cudaEventElapsedTime(&ms, batch->ev0, batch->ev1) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1.0f;
    }
    return ms;
}

void mrc_batch_destroy(mrc_batch *batch) {
    if (!batch) return;
    mrc_context *ctx = batch->ctx;
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        delete batch;
    } else {
        delete batch;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Snapshot negotiation rounds (negotiated.rs:1610-1991 on directed planar edge
// slots; the device kernels are in negotiate.cu).

struct mrc_negotiation {
    mrc_context *ctx = nullptr;
    std::unique_ptr<mrc_board> base;   // base board; dev.directed = base prices
    std::unique_ptr<mrc_board> snap;   // the same board priced by the snapshot
    mrc_negotiation_params params{16, 1};
    std::vector<NetCopy> nets;
    std::vector<mrc_window> windows;
    std::vector<std::vector<uint32_t>> paths;
    std::vector<uint64_t> offsets;     // CSR of `paths` (host copy of d_off/d_cells)
    std::vector<uint32_t> cells;
    std::vector<uint32_t> dirty;       // nets of the next round
    std::vector<uint8_t> owned;        // nets this object routes (a shard routes a subset)
    bool sharded = false;              // occupancy of all shards arrives in d_global between phases
    uint32_t round = 0;
    uint32_t phase = 0;                // 0 ready, 1 ripped up, 2 routed and merged
    mrc_round_stats pending{};         // statistics of the round in progress
    DBuf d_present, d_history, d_snap, d_off, d_cells, d_list, d_flags, d_count;
    DBuf d_global;                     // sharded: sum of every shard's d_present
    bool grouped = false;              // overuse counts connection groups, not nets
    DBuf d_group, d_first, d_over;     // group of every net; per slot: first group seen, overused flag
    // clearance-active rounds (mrc_negotiation_set_clearance): footprint counts
    // per cell and the per-net price overrides of the round being routed
    bool clear = false;
    uint32_t clearance = 0, via_keepout = 0, halo_weight = 16;
    DBuf d_halo, d_emit_off, d_via_off, d_via_k, d_keys, d_vals, d_keys2, d_vals2, d_run_keys, d_run_vals, d_nruns;
    DBuf d_cub, d_over_cells, d_over_price, d_range;
    size_t cub_bytes = 0;
    const uint4 *global() const { return sharded ? d_global.as<uint4>() : d_present.as<uint4>(); }
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~mrc_negotiation() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

namespace {

mrc_status negotiation_upload_paths(mrc_negotiation *ng) {
    mrc_context *ctx = ng->ctx;
    const uint32_t n = (uint32_t)ng->nets.size();
    ng->offsets.assign(n + 1, 0);
    uint64_t o = 0;
    for (uint32_t i = 0; i < n; ++i) {
        ng->offsets[i] = o;
        o += ng->paths[i].size();
    }
    ng->offsets[n] = o;
    ng->cells.clear();
    ng->cells.reserve(o);
    for (auto &p : ng->paths) ng->cells.insert(ng->cells.end(), p.begin(), p.end());
    MRC_TRY(upload(ctx, ng->d_off, ng->offsets.data(), ng->offsets.size() * 8, "upload path offsets"));
    MRC_TRY(upload(ctx, ng->d_cells, ng->cells.data(), ng->cells.size() * 4, "upload path cells"));
    return MRC_OK;
}

HaloArgs negotiation_halo(mrc_negotiation *ng, uint32_t n_list, bool add) {
    HaloArgs a;
    a.offsets = ng->d_off.as<unsigned long long>();
    a.cells = ng->d_cells.as<uint32_t>();
    a.list = ng->d_list.as<uint32_t>();
    a.n_list = n_list;
    a.w = ng->base->view.w;
    a.h = ng->base->view.h;
    a.layers = ng->base->view.layers;
    a.cost = ng->base->dev.cost;
    a.r = ng->clearance;
    a.vr = std::max(ng->clearance, ng->via_keepout);
    a.halo = ng->d_halo.as<uint32_t>();
    a.add = add;
    return a;
}

// Each dirty net's own path slots and clearance footprint, as directed-price
// overrides of the snapshot (the net's prices with its own contribution
// subtracted); `range` gets (first, end) of every dirty net's run of
// overrides, in dirty-list order.  The dirty list is on the device (d_list)
// and d_off/d_cells still hold the paths of the previous round.
mrc_status negotiation_overrides(mrc_negotiation *ng, uint32_t pfac, std::vector<uint32_t> *range) {
    mrc_context *ctx = ng->ctx;
    cudaStream_t s = ctx->stream;
    const GridView &g = ng->base->view;
    const uint32_t plane = g.w * g.h;
    const uint32_t n_dirty = (uint32_t)ng->dirty.size();
    const uint64_t r = ng->clearance, vr = std::max(ng->clearance, ng->via_keepout);
    const uint64_t B = r ? (2 * r + 1) * (2 * r + 1) : 0, BV = vr ? (2 * vr + 1) * (2 * vr + 1) : 0;
    std::vector<uint64_t> emit_off(n_dirty + 1, 0), via_off(n_dirty + 1, 0);
    std::vector<uint32_t> via_k;
    uint64_t total = 0;
    for (uint32_t j = 0; j < n_dirty; ++j) {
        const std::vector<uint32_t> &p = ng->paths[ng->dirty[j]];
        emit_off[j] = total;
        via_off[j] = via_k.size();
        for (size_t k = 0; k + 1 < p.size(); ++k)
            if (p[k] % plane == p[k + 1] % plane) via_k.push_back((uint32_t)k);
        total += p.size() * B + p.size() + (via_k.size() - via_off[j]) * 2 * BV;
    }
    emit_off[n_dirty] = total;
    via_off[n_dirty] = via_k.size();
    range->assign((size_t)2 * n_dirty, 0);
    if (total == 0) return MRC_OK;
    if (total > 0xFFFFFFF0ull) return fail(MRC_ERR_LIMIT, "clearance footprints exceed 2^32 entries");
    MRC_TRY(upload(ctx, ng->d_emit_off, emit_off.data(), emit_off.size() * 8, "upload footprint offsets"));
    MRC_TRY(upload(ctx, ng->d_via_off, via_off.data(), via_off.size() * 8, "upload via offsets"));
    MRC_TRY(upload(ctx, ng->d_via_k, via_k.data(), via_k.size() * 4, "upload via steps"));
    MRC_TRY(ng->d_keys.get(ctx, total * 8, "footprint keys"));
    MRC_TRY(ng->d_vals.get(ctx, total * 4, "footprint values"));
    MRC_TRY(ng->d_keys2.get(ctx, total * 8, "sorted footprint keys"));
    MRC_TRY(ng->d_vals2.get(ctx, total * 4, "sorted footprint values"));
    MRC_TRY(ng->d_run_keys.get(ctx, total * 8, "footprint runs"));
    MRC_TRY(ng->d_run_vals.get(ctx, total * 4, "footprint run values"));
    MRC_TRY(ng->d_nruns.get(ctx, 8, "run count"));
    MRC_TRY(ng->d_over_cells.get(ctx, total * 4, "override cells"));
    MRC_TRY(ng->d_over_price.get(ctx, total * 16, "override prices"));
    MRC_TRY(ng->d_range.get(ctx, (size_t)2 * n_dirty * 4, "override ranges"));
    MRC_CUDA(cudaMemsetAsync(ng->d_range.p, 0, (size_t)2 * n_dirty * 4, s), "clear override ranges");
    EmitArgs ea;
    ea.offsets = ng->d_off.as<unsigned long long>();
    ea.cells = ng->d_cells.as<uint32_t>();
    ea.list = ng->d_list.as<uint32_t>();
    ea.n_list = n_dirty;
    ea.emit_off = ng->d_emit_off.as<unsigned long long>();
    ea.via_off = ng->d_via_off.as<unsigned long long>();
    ea.via_k = ng->d_via_k.as<uint32_t>();
    ea.w = g.w;
    ea.h = g.h;
    ea.layers = g.layers;
    ea.cost = ng->base->dev.cost;
    ea.r = (uint32_t)r;
    ea.vr = (uint32_t)vr;
    ea.keys = ng->d_keys.as<unsigned long long>();
    ea.vals = ng->d_vals.as<uint32_t>();
    MRC_CUDA(emit_launch(ea, s), "emit footprints");
    size_t need = 0;
    auto reduce = [&](void *temp, size_t *bytes) {
        return footprint_reduce(ng->d_keys.as<unsigned long long>(), ng->d_vals.as<uint32_t>(),
                                ng->d_keys2.as<unsigned long long>(), ng->d_vals2.as<uint32_t>(),
                                ng->d_run_keys.as<unsigned long long>(), ng->d_run_vals.as<uint32_t>(),
                                ng->d_nruns.as<uint32_t>(), total, 64, temp, bytes, s);
    };
    MRC_CUDA(reduce(nullptr, &need), "size the footprint sort");
    if (ng->cub_bytes < need || !ng->d_cub.p) {
        MRC_TRY(ng->d_cub.get(ctx, std::max<size_t>(need, 16), "footprint sort scratch"));
        ng->cub_bytes = std::max<size_t>(need, 16);
    }
    size_t have = ng->cub_bytes;
    MRC_CUDA(reduce(ng->d_cub.p, &have), "sort and sum footprints");
    OverrideArgs oa;
    oa.keys = ng->d_run_keys.as<unsigned long long>();
    oa.vals = ng->d_run_vals.as<uint32_t>();
    oa.n_runs = ng->d_nruns.as<uint32_t>();
    oa.cap = total;
    oa.base = ng->base->dev.directed;
    oa.present = ng->global();
    oa.history = ng->d_history.as<uint4>();
    oa.halo = ng->d_halo.as<uint32_t>();
    oa.pf = (uint64_t)pfac * ng->params.present_weight;
    oa.hf = (uint64_t)pfac * ng->halo_weight;
    oa.out_cells = ng->d_over_cells.as<uint32_t>();
    oa.out_price = ng->d_over_price.as<uint4>();
    oa.range = ng->d_range.as<uint32_t>();
    MRC_CUDA(override_launch(oa, s), "price overrides");
    MRC_CUDA(cudaMemcpyAsync(range->data(), ng->d_range.p, (size_t)2 * n_dirty * 4, cudaMemcpyDeviceToHost, s),
             "read override ranges");
    MRC_CUDA(cudaStreamSynchronize(s), "price overrides");
    return MRC_OK;
}

OccupancyArgs negotiation_occupancy(mrc_negotiation *ng, uint32_t n_list, bool add) {
    OccupancyArgs a;
    a.offsets = ng->d_off.as<unsigned long long>();
    a.cells = ng->d_cells.as<uint32_t>();
    a.list = ng->d_list.as<uint32_t>();
    a.n_list = n_list;
    a.w = ng->base->view.w;
    a.plane = ng->base->view.w * ng->base->view.h;
    a.present = ng->d_present.as<uint32_t>();
    a.add = add;
    return a;
}

}  // namespace

extern "C" {

mrc_status negotiation_create(mrc_context *ctx, const mrc_isolated_request *req, const mrc_negotiation_params *params,
                              const uint8_t *owned, mrc_negotiation **out);

mrc_status mrc_negotiation_create(mrc_context *ctx, const mrc_isolated_request *req,
                                  const mrc_negotiation_params *params, mrc_negotiation **out) {
    return negotiation_create(ctx, req, params, nullptr, out);
}

mrc_status mrc_negotiation_create_shard(mrc_context *ctx, const mrc_isolated_request *req,
                                        const mrc_negotiation_params *params, const uint8_t *owned,
                                        mrc_negotiation **out) {
    if (!owned) return fail(MRC_ERR_INVALID_ARGUMENT, "owned mask is NULL");
    return negotiation_create(ctx, req, params, owned, out);
}

}  // extern "C"

mrc_status negotiation_create(mrc_context *ctx, const mrc_isolated_request *req, const mrc_negotiation_params *params,
                              const uint8_t *owned, mrc_negotiation **out) {
    if (!ctx || !req || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    std::unique_ptr<mrc_negotiation> ng(new mrc_negotiation());
    ng->ctx = ctx;
    if (params) ng->params = *params;
    GridView g;
    MRC_TRY(view_grid(req->grid, &g));
    const mrc_edges &e = req->edges;
    std::vector<uint32_t> dir;
    mrc_edges eb = e;
    if (!e.directed_in_costs) {
        // per-axis prices as in-prices; slots without a neighbour are never read
        const uint32_t ex = g.w ? g.w - 1 : 0, ey = g.h ? g.h - 1 : 0;
        if (e.n_x_edge_costs != ex || e.n_y_edge_costs != ey || (ex && !e.x_edge_costs) || (ey && !e.y_edge_costs))
            return fail(MRC_ERR_INVALID_ARGUMENT, "edge price vectors do not match the grid");
        dir.resize(g.n * 4);
        for (uint64_t c = 0; c < g.n; ++c) {
            const uint32_t r = (uint32_t)(c % ((uint64_t)g.w * g.h)), x = r % g.w, y = r / g.w;
            dir[4 * c + 0] = y > 0 ? e.y_edge_costs[y - 1] : kMax;
            dir[4 * c + 1] = x > 0 ? e.x_edge_costs[x - 1] : kMax;
            dir[4 * c + 2] = x + 1 < g.w ? e.x_edge_costs[x] : kMax;
            dir[4 * c + 3] = y + 1 < g.h ? e.y_edge_costs[y] : kMax;
        }
        eb.directed_in_costs = dir.data();
    }
    ng->base.reset(new mrc_board());
    MRC_TRY(board_build(ctx, req->grid, &eb, true, ng->base.get()));
    MRC_TRY(validate_nets(ng->base->view, req->nets, req->n_nets, &ng->nets));
    MRC_TRY(collect_windows(ng->base->view, ng->nets, req->windows, &ng->windows));
    const uint32_t n = req->n_nets;
    const size_t slots = (size_t)g.n * 16;
    MRC_TRY(ng->d_present.get(ctx, std::max<size_t>(slots, 16), "occupancy"));
    MRC_TRY(ng->d_history.get(ctx, std::max<size_t>(slots, 16), "history"));
    MRC_TRY(ng->d_snap.get(ctx, std::max<size_t>(slots, 16), "snapshot prices"));
    MRC_CUDA(cudaMemsetAsync(ng->d_present.p, 0, slots, ctx->stream), "clear occupancy");
    MRC_CUDA(cudaMemsetAsync(ng->d_history.p, 0, slots, ctx->stream), "clear history");
    MRC_TRY(ng->d_flags.get(ctx, std::max<size_t>(n, 4), "dirty flags"));
    MRC_TRY(ng->d_count.get(ctx, 8, "overuse count"));
    ng->snap.reset(new mrc_board());
    ng->snap->ctx = ctx;
    ng->snap->view = ng->base->view;
    ng->snap->directed = true;
    ng->snap->dev = ng->base->dev;
    ng->snap->dev.directed = ng->d_snap.as<uint4>();
    ng->paths.assign(n, {});
    ng->sharded = owned != nullptr;
    ng->owned.assign(n, 1);
    if (owned)
        for (uint32_t i = 0; i < n; ++i) ng->owned[i] = owned[i] ? 1 : 0;
    if (ng->sharded) {
        MRC_TRY(ng->d_global.get(ctx, std::max<size_t>(slots, 16), "global occupancy"));
        MRC_CUDA(cudaMemsetAsync(ng->d_global.p, 0, slots, ctx->stream), "clear global occupancy");
    }
    ng->dirty.clear();
    for (uint32_t i = 0; i < n; ++i)
        if (ng->owned[i]) ng->dirty.push_back(i);
    MRC_TRY(negotiation_upload_paths(ng.get()));
    MRC_CUDA(cudaEventCreate(&ng->ev0), "create event");
    MRC_CUDA(cudaEventCreate(&ng->ev1), "create event");
    MRC_CUDA(cudaStreamSynchronize(ctx->stream), "negotiation setup");
    *out = ng.release();
    return MRC_OK;
}

extern "C" {

// Phase 1: the dirty nets this object owns leave its occupancy.
mrc_status mrc_negotiation_ripup(mrc_context *ctx, mrc_negotiation *ng) {
    if (!ctx || !ng) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ng->phase != 0) return fail(MRC_ERR_INVALID_ARGUMENT, "negotiation phase out of order (rip-up)");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    std::memset(&ng->pending, 0, sizeof(ng->pending));
    ng->pending.round = ng->round;
    ng->pending.pfac = 1 + ng->round;
    const uint32_t n_dirty = (uint32_t)ng->dirty.size();
    ng->pending.dirty = n_dirty;
    cudaStream_t s = ctx->stream;
    MRC_CUDA(cudaEventRecord(ng->ev0, s), "record event");
    if (n_dirty && !ng->clear) {  // with a clearance every path stays in the snapshot until the merge
        MRC_TRY(upload(ctx, ng->d_list, ng->dirty.data(), (size_t)n_dirty * 4, "upload dirty nets"));
        MRC_CUDA(occupancy_launch(negotiation_occupancy(ng, n_dirty, false), s), "rip-up");
    }
    MRC_CUDA(cudaStreamSynchronize(s), "rip-up");
    ng->phase = 1;
    return MRC_OK;
}

// Phase 2: the frozen snapshot from the global occupancy (after every shard's
// rip-up) and history, the owned dirty nets routed alone on it, and merged
// into this object's occupancy.
mrc_status mrc_negotiation_route(mrc_context *ctx, mrc_negotiation *ng, mrc_round_stats *out) {
    if (!ctx || !ng) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ng->phase != 1) return fail(MRC_ERR_INVALID_ARGUMENT, "negotiation phase out of order (route)");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    mrc_round_stats *st = &ng->pending;
    const GridView &g = ng->base->view;
    cudaStream_t s = ctx->stream;
    const uint32_t n_dirty = (uint32_t)ng->dirty.size();
    SnapshotArgs sa;
    sa.base = ng->base->dev.directed;
    sa.present = ng->global();
    sa.history = ng->d_history.as<uint4>();
    sa.halo = ng->clear ? ng->d_halo.as<uint32_t>() : nullptr;
    sa.out = ng->d_snap.as<uint4>();
    sa.n = g.n;
    sa.pfac = st->pfac;
    sa.weight = ng->params.present_weight;
    sa.halo_weight = ng->halo_weight;
    MRC_CUDA(snapshot_launch(sa, s), "price snapshot");
    if (n_dirty) {
        std::vector<NetCopy> nets;
        std::vector<mrc_window> wins;
        nets.reserve(n_dirty);
        for (uint32_t i : ng->dirty) {
            nets.push_back(ng->nets[i]);
            wins.push_back(ng->windows[i]);
        }
        if (ng->clear) {
            MRC_TRY(upload(ctx, ng->d_list, ng->dirty.data(), (size_t)n_dirty * 4, "upload dirty nets"));
            std::vector<uint32_t> range;
            MRC_TRY(negotiation_overrides(ng, st->pfac, &range));
            for (uint32_t k = 0; k < n_dirty; ++k) {
                nets[k].over_off = range[2 * k];
                nets[k].n_over = range[2 * k + 1] - range[2 * k];
            }
            ng->snap->dev.over_cells = ng->d_over_cells.as<uint32_t>();
            ng->snap->dev.over_price = ng->d_over_price.as<uint4>();
        }
        mrc_result *raw = nullptr;
        const mrc_status rs =
            solve(ctx, {ng->snap.get()}, std::move(nets), std::move(wins), MRC_FLAG_RETRY_FULL, &raw, nullptr);
        ng->snap->dev.over_cells = nullptr;
        ng->snap->dev.over_price = nullptr;
        MRC_TRY(rs);
        std::unique_ptr<mrc_result> res(raw);
        if (ng->clear) {  // the routed nets' old copper and footprints leave before the new ones enter
            MRC_CUDA(occupancy_launch(negotiation_occupancy(ng, n_dirty, false), s), "rip-up old paths");
            MRC_CUDA(halo_launch(negotiation_halo(ng, n_dirty, false), s), "remove old footprints");
        }
        for (uint32_t k = 0; k < n_dirty; ++k) {
            const uint32_t i = ng->dirty[k];
            ng->paths[i].assign(res->cells.begin() + res->offsets[k], res->cells.begin() + res->offsets[k + 1]);
            if (!ng->paths[i].empty()) st->routed++;
            const mrc_window &w0 = ng->windows[i], &w1 = res->field_windows[k];
            const uint64_t c0 = (uint64_t)(w0.x1 - w0.x0 + 1) * (w0.y1 - w0.y0 + 1) * g.layers;
            const bool retried = w1.x0 != w0.x0 || w1.y0 != w0.y0 || w1.x1 != w0.x1 || w1.y1 != w0.y1;
            st->window_cells += c0 + (retried ? g.n : 0);
            st->retried += retried;
        }
        MRC_TRY(negotiation_upload_paths(ng));
        MRC_TRY(upload(ctx, ng->d_list, ng->dirty.data(), (size_t)n_dirty * 4, "upload dirty nets"));
        MRC_CUDA(occupancy_launch(negotiation_occupancy(ng, n_dirty, true), s), "merge paths");
        if (ng->clear) MRC_CUDA(halo_launch(negotiation_halo(ng, n_dirty, true), s), "add footprints");
    }
    MRC_CUDA(cudaStreamSynchronize(s), "route");
    ng->phase = 2;
    if (out) *out = *st;
    return MRC_OK;
}

// Phase 3: history on the edges the global occupancy overuses, then the owned
// nets the next round routes.
mrc_status mrc_negotiation_settle(mrc_context *ctx, mrc_negotiation *ng, mrc_round_stats *out) {
    if (!ctx || !ng) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ng->phase != 2) return fail(MRC_ERR_INVALID_ARGUMENT, "negotiation phase out of order (settle)");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    mrc_round_stats *st = &ng->pending;
    const GridView &g = ng->base->view;
    cudaStream_t s = ctx->stream;
    MRC_CUDA(cudaMemsetAsync(ng->d_count.p, 0, 8, s), "clear count");
    const uint32_t n = (uint32_t)ng->nets.size();
    if (ng->grouped) {
        // group-aware overuse of the current paths of every net
        MRC_CUDA(cudaMemsetAsync(ng->d_first.p, 0xFF, (size_t)g.n * 16, s), "clear group claims");
        MRC_CUDA(cudaMemsetAsync(ng->d_over.p, 0, (size_t)g.n * 4, s), "clear overuse flags");
        GroupArgs ga;
        ga.offsets = ng->d_off.as<unsigned long long>();
        ga.cells = ng->d_cells.as<uint32_t>();
        ga.group = ng->d_group.as<uint32_t>();
        ga.n_nets = n;
        ga.w = g.w;
        ga.plane = g.w * g.h;
        ga.first = ng->d_first.as<uint32_t>();
        ga.over = ng->d_over.as<uint8_t>();
        MRC_CUDA(group_overuse_launch(ga, s), "group overuse scan");
    }
    const uint8_t *over = ng->grouped ? ng->d_over.as<uint8_t>() : nullptr;
    OveruseArgs oa;
    oa.present = ng->global();
    oa.over = over;
    oa.history = ng->d_history.as<uint4>();
    oa.n = g.n;
    oa.step = ng->params.history_step;
    oa.count = ng->d_count.as<unsigned long long>();
    MRC_CUDA(overuse_launch(oa, s), "overuse scan");
    DirtyArgs da;
    da.offsets = ng->d_off.as<unsigned long long>();
    da.cells = ng->d_cells.as<uint32_t>();
    da.n_nets = n;
    da.w = g.w;
    da.plane = g.w * g.h;
    da.present = reinterpret_cast<const uint32_t *>(ng->global());
    da.over = over;
    da.flags = ng->d_flags.as<uint8_t>();
    MRC_CUDA(dirty_launch(da, s), "dirty scan");
    MRC_CUDA(cudaEventRecord(ng->ev1, s), "record event");
    std::vector<uint8_t> flags(n);
    unsigned long long slots = 0;
    if (n) MRC_CUDA(cudaMemcpyAsync(flags.data(), ng->d_flags.p, n, cudaMemcpyDeviceToHost, s), "read dirty flags");
    MRC_CUDA(cudaMemcpyAsync(&slots, ng->d_count.p, 8, cudaMemcpyDeviceToHost, s), "read overuse count");
    MRC_CUDA(cudaStreamSynchronize(s), "negotiation round");
    MRC_CUDA(cudaEventElapsedTime(&st->round_ms, ng->ev0, ng->ev1), "round time");
    ng->dirty.clear();
    if (ng->clear) {  // every net again until a round ends without overuse (negotiated.rs:1631-1634, :1986)
        if (slots)
            for (uint32_t i = 0; i < n; ++i) ng->dirty.push_back(i);
    } else {
        for (uint32_t i = 0; i < n; ++i)
            if (flags[i] && ng->owned[i]) ng->dirty.push_back(i);  // the dirty scan marks unrouted nets too
    }
    st->overused_edges = slots / 2;
    st->next_dirty = (uint32_t)ng->dirty.size();
    st->path_cells = ng->cells.size();
    ng->round++;
    ng->phase = 0;
    if (out) *out = *st;
    return MRC_OK;
}

mrc_status mrc_negotiation_set_groups(mrc_context *ctx, mrc_negotiation *ng, const uint32_t *groups) {
    if (!ctx || !ng || !groups) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ng->sharded) return fail(MRC_ERR_INVALID_ARGUMENT, "connection groups need every path: not on a shard");
    if (ng->round != 0 || ng->phase != 0)
        return fail(MRC_ERR_INVALID_ARGUMENT, "connection groups are set before the first round");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    const uint32_t n = (uint32_t)ng->nets.size();
    for (uint32_t i = 0; i < n; ++i)
        if (groups[i] == kNoGroup) return fail(MRC_ERR_INVALID_ARGUMENT, "group id 0xFFFFFFFF is reserved");
    const size_t cells = (size_t)ng->base->view.n;
    MRC_TRY(upload(ctx, ng->d_group, groups, (size_t)n * 4, "upload connection groups"));
    MRC_TRY(ng->d_first.get(ctx, std::max<size_t>(cells * 16, 16), "group claims"));
    MRC_TRY(ng->d_over.get(ctx, std::max<size_t>(cells * 4, 16), "overuse flags"));
    MRC_CUDA(cudaStreamSynchronize(ctx->stream), "upload connection groups");
    ng->grouped = true;
    return MRC_OK;
}

mrc_status mrc_negotiation_set_clearance(mrc_context *ctx, mrc_negotiation *ng, uint32_t clearance_cells,
                                         uint32_t via_keepout_cells, uint32_t halo_weight) {
    if (!ctx || !ng) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ng->sharded) return fail(MRC_ERR_INVALID_ARGUMENT, "clearance pricing needs every path: not on a shard");
    if (ng->round != 0 || ng->phase != 0)
        return fail(MRC_ERR_INVALID_ARGUMENT, "the clearance is set before the first round");
    if (clearance_cells > kMaxClearanceCells || via_keepout_cells > kMaxClearanceCells)
        return fail(MRC_ERR_INVALID_ARGUMENT, "clearance radius above 255 cells");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    ng->clearance = clearance_cells;
    ng->via_keepout = via_keepout_cells;
    ng->halo_weight = halo_weight;
    ng->clear = clearance_cells > 0 || via_keepout_cells > 0;
    if (ng->clear) {
        const size_t bytes = std::max<size_t>((size_t)ng->base->view.n * 4, 16);
        MRC_TRY(ng->d_halo.get(ctx, bytes, "clearance footprints"));
        MRC_CUDA(cudaMemsetAsync(ng->d_halo.p, 0, bytes, ctx->stream), "clear footprints");
        MRC_CUDA(cudaStreamSynchronize(ctx->stream), "clear footprints");
    }
    return MRC_OK;
}

mrc_status mrc_negotiation_read_halo(mrc_context *ctx, mrc_negotiation *ng, uint32_t *halo) {
    if (!ctx || !ng || !halo) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!ng->clear) return fail(MRC_ERR_INVALID_ARGUMENT, "no clearance set");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    MRC_CUDA(cudaMemcpy(halo, ng->d_halo.p, (size_t)ng->base->view.n * 4, cudaMemcpyDeviceToHost), "read footprints");
    return MRC_OK;
}

mrc_status mrc_negotiation_buffers(mrc_negotiation *ng, void **local_present, void **global_present,
                                   uint64_t *bytes) {
    if (!ng || !local_present || !global_present || !bytes) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *local_present = ng->d_present.p;
    *global_present = const_cast<uint4 *>(ng->global());
    *bytes = (uint64_t)ng->base->view.n * 16;
    return MRC_OK;
}

// One whole round of an unsharded negotiation (its occupancy is the global one).
mrc_status mrc_negotiation_round(mrc_context *ctx, mrc_negotiation *ng, mrc_round_stats *st) {
    if (!ctx || !ng || !st) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ng->sharded) return fail(MRC_ERR_INVALID_ARGUMENT, "a shard runs its rounds phase by phase");
    if (ng->dirty.empty()) {  // converged: nothing to do
        std::memset(st, 0, sizeof(*st));
        st->round = ng->round;
        st->pfac = 1 + ng->round;
        st->path_cells = ng->cells.size();
        return MRC_OK;
    }
    MRC_TRY(mrc_negotiation_ripup(ctx, ng));
    MRC_TRY(mrc_negotiation_route(ctx, ng, nullptr));
    return mrc_negotiation_settle(ctx, ng, st);
}

mrc_status mrc_negotiation_paths(const mrc_negotiation *ng, uint32_t *n_nets, const uint64_t **offsets,
                                 const uint32_t **cells) {
    if (!ng || !n_nets || !offsets || !cells) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *n_nets = (uint32_t)ng->nets.size();
    *offsets = ng->offsets.data();
    *cells = ng->cells.data();
    return MRC_OK;
}

mrc_status mrc_negotiation_read(mrc_context *ctx, mrc_negotiation *ng, uint32_t *present, uint32_t *history,
                                uint32_t *snapshot) {
    if (!ctx || !ng) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    const size_t bytes = (size_t)ng->base->view.n * 16;
    if (present) MRC_CUDA(cudaMemcpy(present, ng->d_present.p, bytes, cudaMemcpyDeviceToHost), "read occupancy");
    if (history) MRC_CUDA(cudaMemcpy(history, ng->d_history.p, bytes, cudaMemcpyDeviceToHost), "read history");
    if (snapshot) MRC_CUDA(cudaMemcpy(snapshot, ng->d_snap.p, bytes, cudaMemcpyDeviceToHost), "read snapshot");
    return MRC_OK;
}

mrc_status mrc_negotiation_dirty(const mrc_negotiation *ng, uint32_t *n, const uint32_t **nets) {
    if (!ng || !n || !nets) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *n = (uint32_t)ng->dirty.size();
    *nets = ng->dirty.data();
    return MRC_OK;
}

void mrc_negotiation_destroy(mrc_negotiation *ng) {
    if (!ng) return;
    mrc_context *ctx = ng->ctx;
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        delete ng;
    } else {
        delete ng;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving: a dispatcher thread that admits requests by device-memory footprint,
// merges them into multi-board launches and keeps several launches in flight.

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct ServerRequest {
    uint64_t ticket = 0;
    uint32_t flags = 0;
    mrc_isolated_request req{};   // borrowed arrays
    mrc_grid grid{};
    const mrc_board *resident = nullptr;  // a board already in HBM (no upload)
    std::vector<NetCopy> nets;
    std::vector<mrc_window> windows;
    uint64_t cells = 0;           // window cells of all nets
    size_t footprint = 0;         // device bytes while in flight
    Clock::time_point t_submit, t_stage, t_done;
    bool done = false;
    mrc_status status = MRC_OK;
    std::string error;
    std::unique_ptr<mrc_result> result;
    uint32_t batch_requests = 0;
    uint64_t batch_id = 0;
};

struct ServerBatch {
    uint64_t id = 0;
    mrc_server *srv = nullptr;
    std::vector<std::shared_ptr<ServerRequest>> reqs;
    BoardPack pack;
    std::unique_ptr<mrc_batch> bt;
    std::vector<uint32_t> slots;  // claimed slots; the launch runs on the first one's stream
    uint32_t flags = 0;
    size_t footprint = 0;
    bool finished = false;        // set by the stream callback (under the server mutex)
};

}  // namespace

struct mrc_server {
    mrc_context *ctx = nullptr;
    mrc_server_params p{};
    std::mutex mu;
    std::condition_variable cv;       // dispatcher wake-ups
    std::condition_variable cv_done;  // waiters
    std::deque<std::shared_ptr<ServerRequest>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<ServerRequest>> tickets;
    std::vector<std::unique_ptr<ServerBatch>> inflight;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> staged;
    std::vector<bool> slot_busy;
    size_t budget = 0, inflight_bytes = 0, peak_bytes = 0, smem_floor = 0;
    uint32_t tile_h = 8, threads = kRelaxThreads;
    uint64_t next_ticket = 1, next_batch = 1;
    uint64_t submitted = 0, completed = 0, failed = 0, launches = 0, largest = 0;
    bool stop = false, wake = false;
    std::thread th;
};

namespace {

// Device bytes a request holds while in flight (board + per-net state).
size_t request_footprint(const ServerRequest &r, uint32_t tile_h) {
    auto al = [](size_t b) { return (std::max<size_t>(b, 4) + 255) & ~(size_t)255; };
    const GridView g{r.grid.w, r.grid.h, r.grid.layers ? r.grid.layers : 1u,
                     (uint64_t)r.grid.w * r.grid.h * (r.grid.layers ? r.grid.layers : 1u)};
    size_t b = 0;
    if (!r.resident) {
        b += al(g.n * 4) + al((size_t)g.w * 4) + al((size_t)g.h * 4) + al(128);
        if (r.grid.board_constraint || r.grid.via_forbidden) b += al(g.n);
        if (r.req.edges.directed_in_costs) b += al(g.n * 16);
    }
    const bool keep = (r.flags & MRC_FLAG_KEEP_FIELDS) != 0;
    for (size_t i = 0; i < r.nets.size(); ++i) {
        const mrc_window &w = r.windows[i];
        const uint64_t ww = w.x1 - w.x0 + 1, wh = w.y1 - w.y0 + 1;
        const uint64_t cells = ww * wh * g.layers;
        const uint64_t tiles = ((ww + 31) / 32) * ((wh + tile_h - 1) / tile_h);
        b += cells * (8 + 4 + (keep ? 4 : 0)) + tiles * (4 + 4 + 24) + sizeof(DevField) + 32 +
             4 * (r.nets[i].pads.size() + r.nets[i].vpads.size());
    }
    return b + (1u << 20);
}

mrc_status server_validate(mrc_server *s, const mrc_isolated_request *req, ServerRequest *r) {
    if (!req) return fail(MRC_ERR_INVALID_ARGUMENT, "request is NULL");
    GridView g;
    MRC_TRY(view_grid(req->grid, &g));
    if (g.layers > s->p.max_layers) return fail(MRC_ERR_LIMIT, "request has more layers than the server accepts");
    const mrc_edges &e = req->edges;
    const uint32_t ex = g.w ? g.w - 1 : 0, ey = g.h ? g.h - 1 : 0, ev = g.layers - 1;
    if (e.n_x_edge_costs != ex || e.n_y_edge_costs != ey || e.n_via_edge_costs != ev)
        return fail(MRC_ERR_INVALID_ARGUMENT, "isolated batch shape does not match grid/nets");
    if ((ex && !e.x_edge_costs) || (ey && !e.y_edge_costs) || (ev && (!e.via_edge_costs || !e.via_allowed)))
        return fail(MRC_ERR_INVALID_ARGUMENT, "edge price pointer is NULL");
    MRC_TRY(validate_nets(g, req->nets, req->n_nets, &r->nets));
    MRC_TRY(collect_windows(g, r->nets, req->windows, &r->windows));
    r->req = *req;
    r->grid = *req->grid;
    r->req.grid = &r->grid;
    for (const mrc_window &w : r->windows) r->cells += (uint64_t)(w.x1 - w.x0 + 1) * (w.y1 - w.y0 + 1) * g.layers;
    r->footprint = request_footprint(*r, s->tile_h);
    return MRC_OK;
}

void CUDART_CB server_on_done(void *p) {
    ServerBatch *b = static_cast<ServerBatch *>(p);
    mrc_server *s = b->srv;
    {
        std::lock_guard<std::mutex> g(s->mu);
        b->finished = true;
        s->wake = true;
    }
    s->cv.notify_all();
}

// Stage every request of the batch (one packed board upload, one batch) and
// enqueue it on the slot's stream behind the staging copies.
mrc_status server_launch(mrc_server *s, ServerBatch *b) {
    mrc_context *ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    MRC_TRY(set_device(ctx));
    std::vector<mrc_isolated_request> inst;
    inst.reserve(b->reqs.size());
    for (auto &r : b->reqs)
        if (!r->resident) inst.push_back(r->req);
    if (!inst.empty()) MRC_TRY(board_pack_build(ctx, inst.data(), (uint32_t)inst.size(), &b->pack));
    std::vector<const mrc_board *> boards;
    std::vector<NetCopy> nets;
    std::vector<mrc_window> wins;
    uint32_t packed = 0;
    for (uint32_t k = 0; k < b->reqs.size(); ++k) {
        boards.push_back(b->reqs[k]->resident ? b->reqs[k]->resident : b->pack.boards[packed++].get());
        for (const NetCopy &nc : b->reqs[k]->nets) {
            nets.push_back(nc);
            nets.back().board = k;
        }
        wins.insert(wins.end(), b->reqs[k]->windows.begin(), b->reqs[k]->windows.end());
    }
    b->bt.reset(new mrc_batch());
    b->bt->force_tile_h = s->tile_h;
    b->bt->force_threads = s->threads;
    b->bt->async_q = true;  // the queue schedule: no grid barrier, no co-residency needed
    b->bt->grid_num = (uint32_t)b->slots.size();
    b->bt->grid_div = s->p.slots;
    b->bt->grid_by_work = true;
    b->bt->smem_floor = s->smem_floor;
    MRC_TRY(batch_build(ctx, std::move(boards), std::move(nets), std::move(wins), b->flags, b->bt.get()));
    cudaStream_t st = s->streams[b->slots[0]];
    MRC_CUDA(cudaEventRecord(s->staged[b->slots[0]], ctx->stream), "record staging");
    MRC_CUDA(cudaStreamWaitEvent(st, s->staged[b->slots[0]], 0), "wait for staging");
    MRC_TRY(batch_launch(b->bt.get(), st));
    MRC_CUDA(cudaLaunchHostFunc(st, server_on_done, b), "completion callback");
    return MRC_OK;
}

// Results of one finished launch, split per request.
void server_reap(mrc_server *s, ServerBatch *b) {
    mrc_context *ctx = s->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    mrc_result *raw = nullptr;
    mrc_status st = set_device(ctx);
    if (st == MRC_OK) st = finish_batch(ctx, b->bt.get(), b->flags, &raw);
    std::unique_ptr<mrc_result> res(raw);
    const std::string err = st == MRC_OK ? std::string() : g_err;
    uint32_t first = 0;
    for (auto &r : b->reqs) {
        const uint32_t n = (uint32_t)r->nets.size();
        r->batch_requests = (uint32_t)b->reqs.size();
        r->batch_id = b->id;
        if (st != MRC_OK) {
            r->status = st;
            r->error = err;
        } else {
            std::unique_ptr<mrc_result> o(new mrc_result());
            o->n = n;
            const uint64_t c0 = res->offsets[first], c1 = res->offsets[first + n];
            o->costs.assign(res->costs.begin() + first, res->costs.begin() + first + n);
            o->offsets.resize(n + 1);
            for (uint32_t i = 0; i <= n; ++i) o->offsets[i] = res->offsets[first + i] - c0;
            o->cells.assign(res->cells.begin() + c0, res->cells.begin() + c1);
            o->field_windows.assign(res->field_windows.begin() + first, res->field_windows.begin() + first + n);
            for (uint32_t i = 0; i < n; ++i) {
                const mrc_window &a = r->windows[i], &w = o->field_windows[i];
                o->retried += (a.x0 != w.x0 || a.y0 != w.y0 || a.x1 != w.x1 || a.y1 != w.y1) ? 1 : 0;
            }
            if (res->has_fields) {
                o->has_fields = true;
                const uint64_t f0 = res->field_offsets[first], f1 = res->field_offsets[first + n];
                o->field_offsets.resize(n + 1);
                for (uint32_t i = 0; i <= n; ++i) o->field_offsets[i] = res->field_offsets[first + i] - f0;
                o->fields.assign(res->fields.begin() + f0, res->fields.begin() + f1);
            }
            r->result = std::move(o);
        }
        first += n;
    }
    // free the launch's device memory while the engine lock is held
    b->bt.reset();
    b->pack.boards.clear();
    b->pack.data.reset();
}

constexpr uint32_t kMergeScan = 256;  // queued requests a forming launch looks at

void server_loop(mrc_server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto free_slot = [&]() -> int {
        for (uint32_t i = 0; i < s->slot_busy.size(); ++i)
            if (!s->slot_busy[i]) return (int)i;
        return -1;
    };
    for (;;) {
        s->cv.wait(lk, [&] {
            if (s->stop || s->wake) return true;
            if (s->queue.empty() || free_slot() < 0) return false;
            return s->inflight.empty() || s->inflight_bytes + s->queue.front()->footprint <= s->budget;
        });
        s->wake = false;
        // ---- reap finished launches ----------------------------------------
        std::vector<std::unique_ptr<ServerBatch>> done;
        for (auto it = s->inflight.begin(); it != s->inflight.end();) {
            if ((*it)->finished) {
                done.push_back(std::move(*it));
                it = s->inflight.erase(it);
            } else {
                ++it;
            }
        }
        if (!done.empty()) {
            lk.unlock();
            for (auto &b : done) server_reap(s, b.get());
            lk.lock();
            const auto now = Clock::now();
            for (auto &b : done) {
                s->inflight_bytes -= b->footprint;
                for (uint32_t sl : b->slots) s->slot_busy[sl] = false;
                for (auto &r : b->reqs) {
                    r->t_done = now;
                    r->done = true;
                    if (r->status == MRC_OK) s->completed++;
                    else s->failed++;
                }
            }
            s->cv_done.notify_all();
            done.clear();
        }
        // ---- admit queued requests into new launches -------------------------
        while (!s->queue.empty()) {
            const int slot = free_slot();
            if (slot < 0) break;
            std::shared_ptr<ServerRequest> head = s->queue.front();
            if (head->footprint > s->budget) {  // can never fit
                s->queue.pop_front();
                head->status = MRC_ERR_LIMIT;
                head->error = "request needs more device memory than the admission budget";
                head->t_stage = head->t_done = Clock::now();
                head->done = true;
                s->failed++;
                s->cv_done.notify_all();
                continue;
            }
            if (s->inflight_bytes + head->footprint > s->budget) break;  // wait for a launch to finish
            std::unique_ptr<ServerBatch> b(new ServerBatch());
            b->id = s->next_batch++;
            b->srv = s;
            b->flags = head->flags;
            uint64_t cells = 0;
            const auto now = Clock::now();
            // The queue head always goes; later requests join in queue order when
            // they have the same flags, fit the budget and the cell limit and, with
            // a merge ratio, are of a similar size (window cells within the ratio of
            // the head's, either way).  A request that does not join keeps its place
            // for the next launch, which may start on another free slot at once.
            const uint64_t head_cells = std::max<uint64_t>(head->cells, 1);
            const uint64_t ratio = s->p.merge_ratio;
            uint32_t scanned = 0;
            for (auto it = s->queue.begin(); it != s->queue.end() && b->reqs.size() < s->p.max_batch_requests &&
                                             scanned < kMergeScan;
                 ++scanned) {
                std::shared_ptr<ServerRequest> r = *it;
                const uint64_t rc = std::max<uint64_t>(r->cells, 1);
                bool join = b->reqs.empty();
                if (!join) {
                    join = r->flags == b->flags &&
                           !(s->p.max_batch_cells && cells + r->cells > s->p.max_batch_cells) &&
                           s->inflight_bytes + b->footprint + r->footprint <= s->budget &&
                           (!ratio || (rc <= head_cells * ratio && head_cells <= rc * ratio));
                }
                if (!join) {
                    ++it;
                    continue;
                }
                it = s->queue.erase(it);
                r->t_stage = now;
                cells += r->cells;
                b->footprint += r->footprint;
                b->reqs.push_back(std::move(r));
            }
            // Co-resident grids: a launch takes 1/slots of the grid per slot it
            // claims, so all launches in flight always fit on the device at once.
            // With nothing left in the queue it claims every free slot (the whole
            // idle device); otherwise one, leaving room for the next launch.
            b->slots.push_back((uint32_t)slot);
            s->slot_busy[slot] = true;
            if (s->queue.empty()) {
                for (uint32_t i = 0; i < s->slot_busy.size(); ++i) {
                    if (s->slot_busy[i]) continue;
                    s->slot_busy[i] = true;
                    b->slots.push_back(i);
                }
            }
            s->inflight_bytes += b->footprint;
            s->peak_bytes = std::max(s->peak_bytes, s->inflight_bytes);
            s->launches++;
            s->largest = std::max<uint64_t>(s->largest, b->reqs.size());
            ServerBatch *raw = b.get();
            s->inflight.push_back(std::move(b));
            lk.unlock();
            const mrc_status st = server_launch(s, raw);
            const std::string err = st == MRC_OK ? std::string() : g_err;
            if (st != MRC_OK) {
                std::lock_guard<std::mutex> g(s->ctx->mu);
                raw->bt.reset();
                raw->pack.boards.clear();
                raw->pack.data.reset();
            }
            lk.lock();
            if (st != MRC_OK) {
                for (auto it = s->inflight.begin(); it != s->inflight.end(); ++it) {
                    if (it->get() != raw) continue;
                    s->inflight_bytes -= raw->footprint;
                    for (uint32_t sl : raw->slots) s->slot_busy[sl] = false;
                    for (auto &r : raw->reqs) {
                        r->status = st;
                        r->error = err;
                        r->t_done = Clock::now();
                        r->done = true;
                        s->failed++;
                    }
                    s->inflight.erase(it);
                    break;
                }
                s->cv_done.notify_all();
            }
        }
        if (s->stop && s->queue.empty() && s->inflight.empty()) break;
    }
}

}  // namespace

extern "C" {

mrc_status mrc_server_create(mrc_context *ctx, const mrc_server_params *params, mrc_server **out) {
    if (!ctx || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    std::unique_ptr<mrc_server> s(new mrc_server());
    s->ctx = ctx;
    s->p = params ? *params : mrc_server_params{0.8f, 2, 64, 0, 8, 8};
    if (s->p.hbm_fraction <= 0.f || s->p.hbm_fraction > 1.f) s->p.hbm_fraction = 0.8f;
    s->p.slots = std::max(1u, std::min(s->p.slots, 8u));
    s->p.max_batch_requests = std::max(1u, s->p.max_batch_requests);
    if (!s->p.max_layers) s->p.max_layers = 8;
    if (s->p.max_layers > 16) return fail(MRC_ERR_LIMIT, "a server tile holds at most 16 layers");
    {
        Lock lock(ctx, 0);
        MRC_TRY(set_device(ctx));
        // the pool's free blocks count as available: they are kept (not
        // released, which would synchronise the device) so that large requests
        // find a block instead of waiting on a fresh cudaMalloc
        size_t free_b = 0, total_b = 0;
        MRC_CUDA(cudaMemGetInfo(&free_b, &total_b), "device memory");
        const double used = (double)(total_b - free_b) - (double)ctx->pool.cached();
        const double allowed = (double)s->p.hbm_fraction * (double)total_b - std::max(used, 0.0);
        s->budget = allowed > 0 ? (size_t)allowed : 0;
        s->tile_h = 8;
        s->threads = kRelaxThreads;
        s->smem_floor = relax_smem_bytes(s->p.max_layers, s->tile_h, true, true);
        int per_sm = 0;
        MRC_CUDA(relax_configure(s->tile_h, s->threads, s->smem_floor, true, true), "configure relax kernel");
        MRC_CUDA(relax_occupancy(s->tile_h, s->threads, s->smem_floor, &per_sm, true, true), "relax occupancy");
        if ((uint32_t)per_sm * (uint32_t)ctx->sms < s->p.slots) return fail(MRC_ERR_LIMIT, "too many slots");
        s->streams.resize(s->p.slots);
        s->staged.resize(s->p.slots);
        s->slot_busy.assign(s->p.slots, false);
        for (uint32_t i = 0; i < s->p.slots; ++i) {
            MRC_CUDA(cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking), "server stream");
            MRC_CUDA(cudaEventCreateWithFlags(&s->staged[i], cudaEventDisableTiming), "server event");
        }
    }
    mrc_server *raw = s.get();
    s->th = std::thread(server_loop, raw);
    *out = s.release();
    return MRC_OK;
}

mrc_status mrc_server_submit(mrc_server *s, const mrc_isolated_request *req, uint32_t flags, uint64_t *ticket) {
    if (!s || !ticket) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    auto r = std::make_shared<ServerRequest>();
    r->flags = flags & (MRC_FLAG_RETRY_FULL | MRC_FLAG_KEEP_FIELDS);
    MRC_TRY(server_validate(s, req, r.get()));
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "server is stopping");
        r->ticket = s->next_ticket++;
        *ticket = r->ticket;
        s->tickets[r->ticket] = r;
        s->queue.push_back(r);
        s->submitted++;
    }
    s->cv.notify_all();
    return MRC_OK;
}

mrc_status mrc_server_submit_resident(mrc_server *s, const mrc_board *board, const mrc_net *nets, uint32_t n_nets,
                                      const mrc_window *windows, uint32_t flags, uint64_t *ticket) {
    if (!s || !board || !ticket) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (board->ctx != s->ctx) return fail(MRC_ERR_INVALID_ARGUMENT, "board belongs to another context");
    auto r = std::make_shared<ServerRequest>();
    r->flags = flags & (MRC_FLAG_RETRY_FULL | MRC_FLAG_KEEP_FIELDS);
    const GridView &g = board->view;
    if (g.layers > s->p.max_layers) return fail(MRC_ERR_LIMIT, "request has more layers than the server accepts");
    MRC_TRY(validate_nets(g, nets, n_nets, &r->nets));
    MRC_TRY(collect_windows(g, r->nets, windows, &r->windows));
    r->resident = board;
    r->grid = mrc_grid{g.w, g.h, g.layers, g.cost, g.board, g.via_forbidden};
    r->req.grid = &r->grid;
    for (const mrc_window &w : r->windows) r->cells += (uint64_t)(w.x1 - w.x0 + 1) * (w.y1 - w.y0 + 1) * g.layers;
    r->footprint = request_footprint(*r, s->tile_h);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "server is stopping");
        r->ticket = s->next_ticket++;
        *ticket = r->ticket;
        s->tickets[r->ticket] = r;
        s->queue.push_back(r);
        s->submitted++;
    }
    s->cv.notify_all();
    return MRC_OK;
}

mrc_status mrc_server_wait(mrc_server *s, uint64_t ticket, uint32_t timeout_ms, mrc_result **out,
                           mrc_request_info *info) {
    if (!s || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(MRC_ERR_INVALID_ARGUMENT, "unknown ticket");
    std::shared_ptr<ServerRequest> r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms) {
        if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return fail(MRC_ERR_BUSY, "request is still queued or running");
    } else {
        s->cv_done.wait(lk, ready);
    }
    s->tickets.erase(ticket);
    if (info) {
        info->queue_ms = ms_between(r->t_submit, r->t_stage);
        info->run_ms = ms_between(r->t_stage, r->t_done);
        info->total_ms = ms_between(r->t_submit, r->t_done);
        info->batch_requests = r->batch_requests;
        info->status = (uint32_t)r->status;
        info->batch_id = r->batch_id;
    }
    if (r->status != MRC_OK) return fail(r->status, r->error);
    *out = r->result.release();
    return MRC_OK;
}

mrc_status mrc_server_stats(mrc_server *s, uint64_t out[8]) {
    if (!s || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> g(s->mu);
    out[0] = s->submitted;
    out[1] = s->completed;
    out[2] = s->failed;
    out[3] = s->launches;
    out[4] = s->largest;
    out[5] = s->peak_bytes;
    out[6] = s->budget;
    out[7] = s->queue.size();
    return MRC_OK;
}

void mrc_server_destroy(mrc_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->th.joinable()) s->th.join();
    {
        std::lock_guard<std::mutex> g(s->ctx->mu);
        cudaSetDevice(s->ctx->device);
        for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
        for (cudaEvent_t e : s->staged) cudaEventDestroy(e);
    }
    delete s;
}

}  // extern "C"

extern "C" mrc_status mrc_selftest_wait_timeout(mrc_context *ctx, uint32_t spin_limit, uint32_t *status,
                                                float *elapsed_ms) {
    if (!ctx || !status) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    Lock lock(ctx, 0);
    MRC_TRY(set_device(ctx));
    DBuf ctl;
    MRC_TRY(ctl.get(ctx, sizeof(Ctl), "control block"));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MRC_CUDA(cudaEventCreate(&e0), "create event");
    MRC_CUDA(cudaEventCreate(&e1), "create event");
    cudaError_t ce = cudaMemsetAsync(ctl.p, 0, sizeof(Ctl), ctx->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(e0, ctx->stream);
    if (ce == cudaSuccess) ce = wait_selftest_launch(ctl.as<Ctl>(), spin_limit, ctx->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, ctx->stream);
    uint32_t st = 0;
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(&st, &ctl.as<Ctl>()->status, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
    float ms = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MRC_CUDA(ce, "wait self-test");
    *status = st;
    if (elapsed_ms) *elapsed_ms = ms;
    return MRC_OK;
}

// ---------------------------------------------------------------------------
// The plain form: one net per launch sequence, a host read of the changed
// flag after every Jacobi round (the reference's M3 loop, gpu.rs:1242-1303).

namespace {

mrc_status plain_one(mrc_context *ctx, const mrc_board *board, const NetCopy &net, const mrc_window &win,
                     uint32_t *cost, std::vector<uint32_t> *path, std::vector<uint32_t> *field) {
    const GridView &g = board->view;
    cudaStream_t st = ctx->stream;
    constexpr uint32_t kPlainTileH = 32;
    DevField f{};
    f.src = net.src;
    f.dst = net.dst;
    f.x0 = win.x0;
    f.y0 = win.y0;
    f.ww = win.x1 - win.x0 + 1;
    f.wh = win.y1 - win.y0 + 1;
    f.lab_off = 0;
    f.pad_off = 0;
    f.n_pads = (uint32_t)net.pads.size();
    f.vpad_off = f.n_pads;
    f.n_vpads = (uint32_t)net.vpads.size();
    f.out = 0;
    f.tile_off = 0;
    const uint64_t wc = (uint64_t)f.ww * f.wh * g.layers;
    const uint64_t tiles = (uint64_t)((f.ww + 31) / 32) * ((f.wh + kPlainTileH - 1) / kPlainTileH);
    std::vector<uint32_t> pads(net.pads);
    pads.insert(pads.end(), net.vpads.begin(), net.vpads.end());
    DBuf d_pads, d_a, d_b, d_ctl, d_field, d_costs, d_lens, d_off, d_cells, d_vis, d_out, d_board;
    MRC_TRY(upload(ctx, d_board, &board->dev, sizeof(DevBoard), "plain board"));
    MRC_TRY(upload(ctx, d_pads, pads.data(), pads.size() * 4, "plain pads"));
    MRC_TRY(upload(ctx, d_field, &f, sizeof(f), "plain field"));
    MRC_TRY(d_a.get(ctx, wc * 8, "plain labels"));
    MRC_TRY(d_b.get(ctx, wc * 8, "plain labels"));
    MRC_TRY(d_ctl.get(ctx, 64, "plain flags"));
    MRC_TRY(d_vis.get(ctx, tiles * 4, "plain tile flags"));
    MRC_CUDA(cudaMemsetAsync(d_a.p, 0xFF, wc * 8, st), "plain init");
    MRC_CUDA(cudaMemsetAsync(d_ctl.p, 0, 64, st), "plain init");
    MRC_CUDA(cudaMemsetAsync(d_vis.p, 0x01, tiles * 4, st), "plain init");  // every tile holds labels
    const uint32_t plane = g.w * g.h;
    const uint32_t sx = (net.src % plane) % g.w, sy = (net.src % plane) / g.w, sl = net.src / plane;
    const bool src_ok = sx >= win.x0 && sx <= win.x1 && sy >= win.y0 && sy <= win.y1 &&
                        !g.board_forbidden(net.src) && (!g.obstacle(net.src) || sorted_contains(net.pads, net.src));
    static const u64 zero = 0;
    if (src_ok) {
        const uint64_t lc = ((uint64_t)sl * f.wh + (sy - f.y0)) * f.ww + (sx - f.x0);
        MRC_CUDA(cudaMemcpyAsync(d_a.as<u64>() + lc, &zero, 8, cudaMemcpyHostToDevice, st), "plain seed");
    }
    PlainArgs pa;
    pa.board = board->dev;
    pa.field = f;
    pa.pads = d_pads.as<uint32_t>();
    pa.changed = d_ctl.as<uint32_t>();
    u64 *in = d_a.as<u64>(), *out = d_b.as<u64>();
    const uint64_t round_limit = wc + 2;
    for (uint64_t round = 0; src_ok; ++round) {
        if (round > round_limit) return fail(MRC_ERR_ITERATION_LIMIT, "plain relaxation did not converge");
        uint32_t changed = 0;
        MRC_CUDA(cudaMemsetAsync(pa.changed, 0, 4, st), "plain round");
        pa.in = in;
        pa.out = out;
        MRC_CUDA(plain_round_launch(pa, wc, st), "plain round");
        MRC_CUDA(cudaMemcpyAsync(&changed, pa.changed, 4, cudaMemcpyDeviceToHost, st), "plain flag");
        MRC_CUDA(cudaStreamSynchronize(st), "plain round");
        std::swap(in, out);
        if (!changed) break;
    }
    MRC_TRY(d_costs.get(ctx, 4, "plain cost"));
    MRC_TRY(d_lens.get(ctx, 4, "plain len"));
    MRC_TRY(d_off.get(ctx, 16, "plain offsets"));
    MRC_TRY(d_cells.get(ctx, wc * 4, "plain path"));
    PathArgs pt{};
    pt.boards = d_board.as<DevBoard>();
    pt.fields = d_field.as<DevField>();
    pt.n_fields = 1;
    pt.pads = d_pads.as<uint32_t>();
    pt.lab = in;
    pt.tvisit = d_vis.as<uint32_t>();
    pt.tile_h = kPlainTileH;
    pt.arena_filled = 0;
    pt.costs = d_costs.as<uint32_t>();
    pt.lens = d_lens.as<uint32_t>();
    pt.offsets = d_off.as<unsigned long long>();
    pt.cells = d_cells.as<uint32_t>();
    pt.status = d_ctl.as<uint32_t>() + 1;
    MRC_CUDA(path_launch(pt, st), "plain path");
    if (field) {
        MRC_TRY(d_out.get(ctx, wc * 4, "plain field"));
        MRC_CUDA(fields_launch(pt, d_out.as<uint32_t>(), wc, st), "plain field");
    }
    uint32_t status = 0;
    uint64_t off[2];
    MRC_CUDA(cudaMemcpyAsync(&status, pt.status, 4, cudaMemcpyDeviceToHost, st), "plain status");
    MRC_CUDA(cudaMemcpyAsync(cost, pt.costs, 4, cudaMemcpyDeviceToHost, st), "plain cost");
    MRC_CUDA(cudaMemcpyAsync(off, pt.offsets, 16, cudaMemcpyDeviceToHost, st), "plain offsets");
    MRC_CUDA(cudaStreamSynchronize(st), "plain path");
    if (status) return status_error(status);
    path->resize(off[1]);
    if (off[1]) MRC_CUDA(cudaMemcpy(path->data(), pt.cells, off[1] * 4, cudaMemcpyDeviceToHost), "plain path");
    if (field) {
        field->resize(wc);
        MRC_CUDA(cudaMemcpy(field->data(), d_out.p, wc * 4, cudaMemcpyDeviceToHost), "plain field");
    }
    return MRC_OK;
}

}  // namespace

extern "C" mrc_status mrc_route_isolated_plain(mrc_context *ctx, const mrc_isolated_request *req, uint32_t flags,
                                               mrc_result **out) {
    if (!ctx || !req || !out) return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    Lock lock(ctx, flags);
    if (lock.st != MRC_OK) return lock.st;
    MRC_TRY(set_device(ctx));
    GridView g;
    MRC_TRY(view_grid(req->grid, &g));
    if (req->n_nets && !req->windows) return fail(MRC_ERR_INVALID_ARGUMENT, "windows is NULL");
    std::vector<NetCopy> nets;
    MRC_TRY(validate_nets(g, req->nets, req->n_nets, &nets));
    std::vector<mrc_window> wins;
    MRC_TRY(collect_windows(g, nets, req->windows, &wins));
    mrc_board board;
    MRC_TRY(board_build(ctx, req->grid, &req->edges, false, &board));
    const bool keep = (flags & MRC_FLAG_KEEP_FIELDS) != 0;
    std::unique_ptr<mrc_result> r(new mrc_result());
    const uint32_t n = (uint32_t)nets.size();
    r->n = n;
    r->costs.assign(n, kMax);
    r->offsets.assign(n + 1, 0);
    r->field_windows = wins;
    r->has_fields = keep;
    r->field_offsets.assign(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) {
        std::vector<uint32_t> path, field;
        uint32_t cost = kMax;
        MRC_TRY(plain_one(ctx, &board, nets[i], wins[i], &cost, &path, keep ? &field : nullptr));
        if (cost == kMax && (flags & MRC_FLAG_RETRY_FULL) && !is_full(wins[i], g.w, g.h)) {
            r->field_windows[i] = full_window(g.w, g.h);
            r->retried++;
            MRC_TRY(plain_one(ctx, &board, nets[i], r->field_windows[i], &cost, &path, keep ? &field : nullptr));
        }
        r->costs[i] = cost;
        r->offsets[i + 1] = r->offsets[i] + path.size();
        r->cells.insert(r->cells.end(), path.begin(), path.end());
        if (keep) {
            r->field_offsets[i + 1] = r->field_offsets[i] + field.size();
            r->fields.insert(r->fields.end(), field.begin(), field.end());
        }
    }
    *out = r.release();
    return MRC_OK;
}

// ---------------------------------------------------------------------------
// No device allocation: every scratch buffer of one window solve is carved
// from a file-scope device array.  Callers that cannot call cudaMalloc (their
// allocator owns the HBM, or the call sits on a path where cudaMalloc/cudaFree
// may not synchronise the device) use mrc_route_isolated_batch_noalloc.

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[MRC_NOALLOC_SCRATCH_BYTES];

struct NoallocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
    int sms = 0;
    size_t smem_optin = 0;
};

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc_dev[kNoallocMaxDevices];

// Once per device, with that device current: look up the array's device address.
mrc_status noalloc_setup(int device, NoallocDevice **out) {
    if (device < 0 || device >= kNoallocMaxDevices) return fail(MRC_ERR_LIMIT, "device ordinal beyond 63");
    NoallocDevice &d = g_noalloc_dev[device];
    if (!d.ready) {
        void *p = nullptr;
        MRC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "look up the no-allocation scratch array");
        cudaDeviceProp prop;
        MRC_CUDA(cudaGetDeviceProperties(&prop, device), "device properties");
        if (prop.major < 10) return fail(MRC_ERR_BACKEND_UNAVAILABLE, "device is not sm_100 class");
        d.scratch = static_cast<unsigned char *>(p);
        d.sms = prop.multiProcessorCount;
        d.smem_optin = prop.sharedMemPerBlockOptin;
        d.ready = true;
    }
    *out = &d;
    return MRC_OK;
}

// Bump allocator over the scratch array (offsets only, 256-byte aligned).
struct Carve {
    size_t off = 0;
    size_t take(size_t bytes) {
        const size_t o = off;
        off = (off + std::max<size_t>(bytes, 4) + 255) & ~(size_t)255;
        return o;
    }
};

}  // namespace

extern "C" mrc_status mrc_route_isolated_batch_noalloc(const mrc_isolated_request *req, void *stream,
                                                       uint32_t *search_costs, uint64_t *path_offsets,
                                                       uint32_t *path_cells, uint64_t path_cells_capacity) {
    if (!req || !path_offsets || (req->n_nets && !search_costs) || (path_cells_capacity && !path_cells))
        return fail(MRC_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    int device = 0;
    MRC_CUDA(cudaGetDevice(&device), "current device");
    NoallocDevice *dev = nullptr;
    MRC_TRY(noalloc_setup(device, &dev));
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    GridView g;
    MRC_TRY(view_grid(req->grid, &g));
    const mrc_edges &e = req->edges;
    const uint32_t ex = g.w ? g.w - 1 : 0, ey = g.h ? g.h - 1 : 0, ev = g.layers - 1;
    if (e.n_x_edge_costs != ex || e.n_y_edge_costs != ey || e.n_via_edge_costs != ev)
        return fail(MRC_ERR_INVALID_ARGUMENT, "isolated batch shape does not match grid/nets");
    if ((ex && !e.x_edge_costs) || (ey && !e.y_edge_costs) || (ev && (!e.via_edge_costs || !e.via_allowed)))
        return fail(MRC_ERR_INVALID_ARGUMENT, "edge price pointer is NULL");
    if (req->n_nets && !req->windows) return fail(MRC_ERR_INVALID_ARGUMENT, "windows is NULL");
    std::vector<NetCopy> nets;
    MRC_TRY(validate_nets(g, req->nets, req->n_nets, &nets));
    std::vector<mrc_window> wins;
    MRC_TRY(collect_windows(g, nets, req->windows, &wins));
    const uint32_t n = (uint32_t)nets.size();
    path_offsets[0] = 0;
    if (n == 0) return MRC_OK;

    // tile height: the largest whose shared tile fits the per-CTA budget
    const bool directed = e.directed_in_costs != nullptr;
    uint32_t tile_h = 0;
    size_t smem = 0;
    const size_t budget = std::min<size_t>(dev->smem_optin ? dev->smem_optin : (227u << 10), 227u << 10) - 1024;
    for (size_t b : {(size_t)(110u << 10), budget}) {
        for (uint32_t th : {32u, 16u, 8u}) {
            if (!tile_h && relax_smem_bytes(g.layers, th, directed) <= b) {
                tile_h = th;
                smem = relax_smem_bytes(g.layers, th, directed);
            }
        }
    }
    if (!tile_h) return fail(MRC_ERR_LIMIT, "too many layers for one shared-memory tile");

    // field descriptors, largest windows first, and the pad arena
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    auto cells_of = [&](uint32_t i) {
        return (uint64_t)(wins[i].x1 - wins[i].x0 + 1) * (wins[i].y1 - wins[i].y0 + 1) * g.layers;
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cells_of(a) > cells_of(b); });
    std::vector<DevField> fields(n);
    std::vector<uint32_t> pads;
    uint64_t cells = 0, tiles = 0;
    uint32_t max_tiles = 1;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t i = order[k];
        DevField &f = fields[k];
        f.src = nets[i].src;
        f.dst = nets[i].dst;
        f.x0 = wins[i].x0;
        f.y0 = wins[i].y0;
        f.ww = wins[i].x1 - wins[i].x0 + 1;
        f.wh = wins[i].y1 - wins[i].y0 + 1;
        f.lab_off = cells;
        cells += cells_of(i);
        f.pad_off = (uint32_t)pads.size();
        f.n_pads = (uint32_t)nets[i].pads.size();
        pads.insert(pads.end(), nets[i].pads.begin(), nets[i].pads.end());
        f.vpad_off = (uint32_t)pads.size();
        f.n_vpads = (uint32_t)nets[i].vpads.size();
        pads.insert(pads.end(), nets[i].vpads.begin(), nets[i].vpads.end());
        f.out = i;
        const uint64_t t = (uint64_t)((f.ww + 31) / 32) * ((f.wh + tile_h - 1) / tile_h);
        f.tile_off = (uint32_t)std::min<uint64_t>(tiles, 0xFFFFFFFFull);
        f.board = 0;
        f.pad_ = 0;
        tiles += t;
        max_tiles = (uint32_t)std::max<uint64_t>(max_tiles, t);
    }

    // carve the scratch array; reject before any device work when it does not fit
    const bool has_flags = g.board || g.via_forbidden;
    Carve c;
    const size_t o_ctl = c.take(sizeof(Ctl)), o_fields = c.take(n * sizeof(DevField)), o_pads = c.take(pads.size() * 4);
    const size_t o_btab = c.take(sizeof(DevBoard));
    const size_t o_cost = c.take(g.n * 4), o_flags = has_flags ? c.take(g.n) : 0;
    const size_t o_vf = g.via_forbidden ? c.take(g.n) : 0, o_dir = directed ? c.take(g.n * 16) : 0;
    const size_t o_x = c.take((size_t)ex * 4), o_y = c.take((size_t)ey * 4), o_via = c.take((size_t)std::max(ev, 1u) * 4);
    const size_t o_tstamp = c.take(tiles * 4), o_tvisit = c.take(tiles * 4), o_lists = c.take(tiles * 24);
    const size_t o_lab = c.take(cells * 8), o_costs = c.take((size_t)n * 4), o_lens = c.take((size_t)n * 4);
    const size_t o_offsets = c.take(((size_t)n + 1) * 8), o_cells = c.take(cells * 4);
    if (c.off > (size_t)MRC_NOALLOC_SCRATCH_BYTES || tiles > 0x7FFFFFFFull)
        return fail(MRC_ERR_LIMIT, "request needs " + std::to_string(c.off) + " bytes of scratch; the no-allocation "
                                   "entry point has MRC_NOALLOC_SCRATCH_BYTES = " +
                                       std::to_string((size_t)MRC_NOALLOC_SCRATCH_BYTES) + " bytes");
    unsigned char *s = dev->scratch;
    // From the first enqueued copy on, every return (an error included) waits
    // for the stream before the lock is released, so no device work of this
    // call can still read or write the array when the next call starts.
    // Declared after the lock, so it runs first.
    struct DrainOnExit {
        cudaStream_t st;
        ~DrainOnExit() { cudaStreamSynchronize(st); }
    } drain{st};

    // inputs into the scratch array
    MRC_CUDA(cudaMemcpyAsync(s + o_fields, fields.data(), n * sizeof(DevField), cudaMemcpyHostToDevice, st), "upload fields");
    if (!pads.empty())
        MRC_CUDA(cudaMemcpyAsync(s + o_pads, pads.data(), pads.size() * 4, cudaMemcpyHostToDevice, st), "upload pads");
    MRC_CUDA(cudaMemcpyAsync(s + o_cost, g.cost, g.n * 4, cudaMemcpyHostToDevice, st), "upload cost");
    if (has_flags) {
        if (g.board) MRC_CUDA(cudaMemcpyAsync(s + o_flags, g.board, g.n, cudaMemcpyHostToDevice, st), "upload board mask");
        else MRC_CUDA(cudaMemsetAsync(s + o_flags, 0, g.n, st), "clear flags");
        if (g.via_forbidden) {
            MRC_CUDA(cudaMemcpyAsync(s + o_vf, g.via_forbidden, g.n, cudaMemcpyHostToDevice, st), "upload via mask");
            MRC_CUDA(combine_flags_launch(s + o_flags, s + o_vf, g.n, st), "combine masks");
        }
    }
    if (directed)
        MRC_CUDA(cudaMemcpyAsync(s + o_dir, e.directed_in_costs, g.n * 16, cudaMemcpyHostToDevice, st), "upload prices");
    uint32_t via_mask = 0;
    std::vector<uint32_t> vias(std::max(ev, 1u), 0);
    for (uint32_t k = 0; k < ev; ++k) {
        vias[k] = e.via_edge_costs[k];
        if (e.via_allowed[k]) via_mask |= 1u << k;
    }
    if (ex) MRC_CUDA(cudaMemcpyAsync(s + o_x, e.x_edge_costs, (size_t)ex * 4, cudaMemcpyHostToDevice, st), "upload x");
    if (ey) MRC_CUDA(cudaMemcpyAsync(s + o_y, e.y_edge_costs, (size_t)ey * 4, cudaMemcpyHostToDevice, st), "upload y");
    MRC_CUDA(cudaMemcpyAsync(s + o_via, vias.data(), vias.size() * 4, cudaMemcpyHostToDevice, st), "upload vias");
    // state that must start at zero (the array keeps the previous call's contents)
    MRC_CUDA(cudaMemsetAsync(s + o_ctl, 0, sizeof(Ctl), st), "clear control block");
    MRC_CUDA(cudaMemsetAsync(s + o_tstamp, 0, tiles * 4, st), "clear tile stamps");
    MRC_CUDA(cudaMemsetAsync(s + o_tvisit, 0, tiles * 4, st), "clear tile flags");

    DevBoard b{};
    b.w = g.w;
    b.h = g.h;
    b.layers = g.layers;
    b.via_mask = via_mask;
    b.cost = reinterpret_cast<const uint32_t *>(s + o_cost);
    b.flags = has_flags ? s + o_flags : nullptr;
    b.x_edge = reinterpret_cast<const uint32_t *>(s + o_x);
    b.y_edge = reinterpret_cast<const uint32_t *>(s + o_y);
    b.via_edge = reinterpret_cast<const uint32_t *>(s + o_via);
    b.directed = directed ? reinterpret_cast<const uint4 *>(s + o_dir) : nullptr;

    MRC_CUDA(cudaMemcpyAsync(s + o_btab, &b, sizeof(DevBoard), cudaMemcpyHostToDevice, st), "upload board table");
    int per_sm = 0;
    MRC_CUDA(relax_configure(tile_h, kRelaxThreads, smem), "configure relax kernel");
    MRC_CUDA(relax_occupancy(tile_h, kRelaxThreads, smem, &per_sm), "relax occupancy");
    if (per_sm < 1) return fail(MRC_ERR_LIMIT, "relax kernel does not fit on one SM");
    RelaxArgs ra{};
    ra.boards = reinterpret_cast<const DevBoard *>(s + o_btab);
    ra.max_layers = g.layers;
    ra.fields = reinterpret_cast<const DevField *>(s + o_fields);
    ra.n_fields = n;
    ra.pads = reinterpret_cast<const uint32_t *>(s + o_pads);
    ra.lab = reinterpret_cast<u64 *>(s + o_lab);
    ra.tstamp = reinterpret_cast<uint32_t *>(s + o_tstamp);
    ra.tvisit = reinterpret_cast<uint32_t *>(s + o_tvisit);
    ra.lists = reinterpret_cast<u64 *>(s + o_lists);
    ra.list_cap = (uint32_t)tiles;
    ra.ctl = reinterpret_cast<Ctl *>(s + o_ctl);
    ra.tile_h = tile_h;
    ra.round_limit = 64u * max_tiles + 4096u;
    ra.activation_limit = ~0ull;
    MRC_CUDA(relax_launch(ra, (uint32_t)dev->sms * (uint32_t)per_sm, kRelaxThreads, smem, st), "launch relax kernel");
    PathArgs pa{};
    pa.boards = ra.boards;
    pa.fields = ra.fields;
    pa.n_fields = n;
    pa.pads = ra.pads;
    pa.lab = ra.lab;
    pa.tvisit = ra.tvisit;
    pa.tile_h = tile_h;
    pa.arena_filled = 0;
    pa.costs = reinterpret_cast<uint32_t *>(s + o_costs);
    pa.lens = reinterpret_cast<uint32_t *>(s + o_lens);
    pa.offsets = reinterpret_cast<unsigned long long *>(s + o_offsets);
    pa.cells = reinterpret_cast<uint32_t *>(s + o_cells);
    pa.status = &ra.ctl->status;
    MRC_CUDA(path_launch(pa, st), "launch path kernels");

    uint32_t status = 0;
    MRC_CUDA(cudaMemcpyAsync(&status, pa.status, 4, cudaMemcpyDeviceToHost, st), "read status");
    MRC_CUDA(cudaMemcpyAsync(search_costs, pa.costs, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "read costs");
    MRC_CUDA(cudaMemcpyAsync(path_offsets, pa.offsets, ((size_t)n + 1) * 8, cudaMemcpyDeviceToHost, st),
             "read offsets");
    MRC_CUDA(cudaStreamSynchronize(st), "no-allocation batch");
    if (status) return status_error(status);
    const uint64_t total = path_offsets[n];
    if (total > path_cells_capacity)
        return fail(MRC_ERR_LIMIT, "paths need " + std::to_string(total) + " cells; path_cells_capacity is " +
                                       std::to_string(path_cells_capacity));
    if (total) {
        MRC_CUDA(cudaMemcpyAsync(path_cells, pa.cells, total * 4, cudaMemcpyDeviceToHost, st), "read paths");
        MRC_CUDA(cudaStreamSynchronize(st), "read paths");
    }
    return MRC_OK;
}
