// capi.cpp -- C ABI of libplp_b200.so: instances, results, the batched
// persistent solver, the serving loop and the kernel test hooks.
//
// Device memory of a batch comes from the stream-ordered allocator
// (cudaMallocAsync/cudaFreeAsync) so waves on different streams never force a
// device-wide synchronisation; the handle's budget bounds the bytes of all
// batches in flight.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>

#include <unistd.h>

#include "capi_internal.hpp"
#include "engine.hpp"

using namespace plpb;

// ===========================================================================
// errors
// ===========================================================================
namespace {
thread_local std::string g_err;
}

namespace plpb {

int set_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

std::string plpb_last() { return g_err; }

int set_cuda_error(const char* what, cudaError_t e) {
    g_err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return PLP_E_CUDA;
}

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void mt_init_table(uint32_t out[624]) {
    out[0] = 19650218u;
    for (uint32_t i = 1; i < 624; i++) out[i] = 1812433253u * (out[i - 1] ^ (out[i - 1] >> 30)) + i;
}

const uint32_t* device_mt_init(int* status) {
    static std::mutex mu;
    static std::map<int, uint32_t*> per_dev;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { *status = set_cuda_error("cudaGetDevice", e); return nullptr; }
    std::lock_guard<std::mutex> g(mu);
    auto it = per_dev.find(dev);
    if (it != per_dev.end()) { *status = PLP_OK; return it->second; }
    uint32_t tab[624];
    mt_init_table(tab);
    uint32_t* d = nullptr;
    e = cudaMalloc(&d, sizeof tab);
    if (e != cudaSuccess) { *status = set_cuda_error("MT init table allocation", e); return nullptr; }
    e = cudaMemcpy(d, tab, sizeof tab, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { *status = set_cuda_error("MT init table copy", e); return nullptr; }
    per_dev[dev] = d;
    *status = PLP_OK;
    return d;
}

}  // namespace plpb

struct plp_handle;

namespace {

std::mutex g_handle_err_mu;

void record(plp_handle* h, int status);

// ===========================================================================
// batch: device tables + one persistent decoder launch (+ retries)
// ===========================================================================
struct TileConfig {
    // default: the tile the autotuner picks on every bench workload (one
    // decoder per CTA spreads a launch over all SMs; these depths hold the
    // 400-item instances without capacity retries)
    int P = 256;       // placed-box tile depth per decoder
    int C = 512;       // live-point tile depth per decoder
    int G = 1;         // warps per decoder
    int D = 1;         // decoders per CTA
    int M = 1;         // minimum resident CTAs per SM (register cap)
    // test hook of the bounded barrier wait (plp_debug_sync_bound), multi-warp
    // decoders only: tries per wait (0 = the kernel's bound) and 1 + the warp
    // of every decoder that skips its first arrive (0 = none)
    int sync_limit = 0;
    int sync_skip = 0;
};

// Tiles only deepen: a retry that needed a deeper tile is remembered so the
// next batch of this handle starts there.
void remember_tile(TileConfig& keep, const TileConfig& used) {
    keep.P = std::max(keep.P, used.P);
    keep.C = std::max(keep.C, used.C);
    while (keep.D > 1 && decoder_smem_bytes(keep.P, keep.C, 0, keep.G) * keep.D > 200 * 1024) keep.D >>= 1;
    if (!decoder_config_supported(keep.G, keep.D, keep.M)) keep.M = 1;
}



constexpr int P_MAX = 2048;
constexpr long long SEED_TABLE_MAX = 8192;   // seeded states kept per batch (2.5 KB each)
constexpr int C_MAX = 8192;

struct Batch;
// shared-memory bytes, supported launch shape and occupancy of a tile for a
// batch's engine (extreme-point decoder or block engine)
int tile_smem(const Batch& b, const TileConfig& t);
bool tile_supported(const Batch& b, const TileConfig& t);
cudaError_t tile_occupancy(const Batch& b, const TileConfig& t, int* occ);

// Host tables of the block-building engine for one instance
// (blockproof/plp_block.cpp:237-262): the shape catalogue; each type's shapes
// in precedence order (most copies, tallest stack, widest base, orientation);
// for each type the first shape fitting r remaining copies, for every r below
// the type's largest count; the placement rank of every shape (block volume
// desc, type, orientation, k desc, a desc, b desc) and the shapes by rank; the
// type order (volume desc, index) and the copies per type.
struct BlockTables {
    std::vector<BlkShape> cat;
    std::vector<int> tab;
    // offsets into tab
    int bo_order = 0, bo_qty = 0, bo_list_off = 0, bo_list = 0, bo_start_off = 0, bo_start = 0,
        bo_shape_of_rank = 0;
    size_t bytes() const { return cat.size() * sizeof(BlkShape) + tab.size() * sizeof(int); }
};

int make_block_tables(const Instance& I, const std::vector<TypeOrs>& ors, int amax, int bmax, int kmax,
                      BlockTables& out) {
    std::vector<int>& tab = out.tab;
    BlockTables& d = out;
    const int nt = (int)I.types.size();
    std::vector<BlkShape> cat;
    for (int ti = 0; ti < nt; ti++) {
        for (int oi = 0; oi < ors[ti].n; oi++) {
            const int w = ors[ti].w[oi], dd = ors[ti].d[oi], h = ors[ti].h[oi];
            for (int a = 1; a <= amax; a++) {
                if ((long long)a * w > I.L) break;
                for (int b = 1; b <= bmax; b++) {
                    if ((long long)b * dd > I.W) break;
                    for (int k = 1; k <= kmax; k++) {
                        if ((long long)k * h > I.H) break;
                        const long long cnt = 1LL * a * b * k;
                        if (cnt > I.types[ti].qty) break;
                        if (cat.size() >= (size_t)(1 << 22))
                            return set_error(PLP_E_CAPACITY, "block catalogue larger than 4M shapes");
                        cat.push_back(BlkShape{ti, oi, a, b, k, (int)cnt, a * w, b * dd, k * h, 0});
                    }
                }
            }
        }
    }
    const int nc = (int)cat.size();
    std::vector<std::vector<int>> by(nt);
    for (int i = 0; i < nc; i++) by[cat[i].ti].push_back(i);
    for (auto& v : by)
        std::sort(v.begin(), v.end(), [&](int x, int y) {
            const BlkShape &p = cat[x], &q = cat[y];
            if (p.cnt != q.cnt) return p.cnt > q.cnt;
            if (p.bh != q.bh) return p.bh > q.bh;
            if (p.a != q.a) return p.a > q.a;
            if (p.b != q.b) return p.b > q.b;
            return p.oi < q.oi;
        });
    std::vector<int> by_rank(nc);
    for (int i = 0; i < nc; i++) by_rank[i] = i;
    std::sort(by_rank.begin(), by_rank.end(), [&](int x, int y) {
        const BlkShape &p = cat[x], &q = cat[y];
        const long long vp = 1LL * p.bw * p.bd * p.bh, vq = 1LL * q.bw * q.bd * q.bh;
        if (vp != vq) return vp > vq;
        if (p.ti != q.ti) return p.ti < q.ti;
        if (p.oi != q.oi) return p.oi < q.oi;
        if (p.k != q.k) return p.k > q.k;
        if (p.a != q.a) return p.a > q.a;
        return p.b > q.b;
    });
    for (int r = 0; r < nc; r++) cat[by_rank[r]].rank = r;
    std::vector<int> tord(nt);
    for (int t = 0; t < nt; t++) tord[t] = t;
    std::sort(tord.begin(), tord.end(), [&](int x, int y) {
        const long long vx = I.types[x].volume(), vy = I.types[y].volume();
        if (vx != vy) return vx > vy;
        return x < y;
    });
    d.bo_order = (int)tab.size();
    tab.insert(tab.end(), tord.begin(), tord.end());
    d.bo_qty = (int)tab.size();
    for (int t = 0; t < nt; t++) tab.push_back(I.types[t].qty);
    d.bo_list_off = (int)tab.size();
    {
        int off = 0;
        for (int t = 0; t < nt; t++) { tab.push_back(off); off += (int)by[t].size(); }
        tab.push_back(off);
    }
    d.bo_list = (int)tab.size();
    for (int t = 0; t < nt; t++) tab.insert(tab.end(), by[t].begin(), by[t].end());
    d.bo_start_off = (int)tab.size();
    {
        int off = 0;
        for (int t = 0; t < nt; t++) {
            tab.push_back(off);
            off += by[t].empty() ? 0 : cat[by[t][0]].cnt - 1;
        }
        tab.push_back(off);
    }
    d.bo_start = (int)tab.size();
    for (int t = 0; t < nt; t++) {
        if (by[t].empty()) continue;
        const int maxc = cat[by[t][0]].cnt, ns = (int)by[t].size();
        for (int r = 1; r < maxc; r++) {   // shapes are cnt-desc: the fitting ones form a suffix
            int start = ns;
            while (start > 0 && cat[by[t][start - 1]].cnt <= r) start--;
            tab.push_back(start);
        }
    }
    d.bo_shape_of_rank = (int)tab.size();
    tab.insert(tab.end(), by_rank.begin(), by_rank.end());
    out.cat = std::move(cat);
    return PLP_OK;
}

// The tables depend only on the container, the types and (amax, bmax, kmax),
// so they are kept per process (up to PLP_BLOCK_CACHE_MB, default 1024 MiB,
// oldest first out): a batch that solves the same instances again appends
// them instead of rebuilding the catalogue and its sorts.
std::shared_ptr<const BlockTables> block_tables(const Instance& I, const std::vector<TypeOrs>& ors,
                                                 int amax, int bmax, int kmax, int* status) {
    static std::mutex mu;
    static std::unordered_map<std::string, std::shared_ptr<const BlockTables>> cache;
    static std::deque<std::string> order;
    static size_t held = 0;
    static const size_t limit = [] {
        size_t mb = 1024;
        if (const char* v = std::getenv("PLP_BLOCK_CACHE_MB")) {
            char* end = nullptr;
            const unsigned long long x = std::strtoull(v, &end, 10);
            if (end != v) mb = (size_t)x;
        }
        return mb << 20;
    }();
    std::string key;
    key.reserve(32 + I.types.size() * 28);
    auto put = [&](int v) { key.append(reinterpret_cast<const char*>(&v), sizeof v); };
    for (int v : {I.L, I.W, I.H, amax, bmax, kmax, (int)I.types.size()}) put(v);
    for (const auto& t : I.types)
        for (int v : {t.l, (int)t.lf, t.w, (int)t.wf, t.h, (int)t.hf, t.qty}) put(v);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            *status = PLP_OK;
            return it->second;
        }
    }
    auto bt = std::make_shared<BlockTables>();
    *status = make_block_tables(I, ors, amax, bmax, kmax, *bt);
    if (*status != PLP_OK) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (bt->bytes() <= limit && !cache.count(key)) {
        while (held + bt->bytes() > limit && !order.empty()) {
            auto old = cache.find(order.front());
            held -= old->second->bytes();
            cache.erase(old);
            order.pop_front();
        }
        cache.emplace(key, bt);
        order.push_back(key);
        held += bt->bytes();
    }
    return bt;
}

// Appends one instance's block tables to the batch's catalogue and table,
// with its descriptor's offsets.
int build_block_tables(const Instance& I, const std::vector<TypeOrs>& ors, const plp_run_opts& o,
                       std::vector<BlkShape>& cat_all, std::vector<int>& tab, InstDesc& d) {
    int status = PLP_OK;
    const auto bt = block_tables(I, ors, std::max(1, o.blk_amax), std::max(1, o.blk_bmax),
                                 std::max(1, o.blk_kmax), &status);
    if (!bt) return status;
    const int base = (int)tab.size();
    d.n_types = (int)I.types.size();
    d.bo_order = base + bt->bo_order;
    d.bo_qty = base + bt->bo_qty;
    d.bo_list_off = base + bt->bo_list_off;
    d.bo_list = base + bt->bo_list;
    d.bo_start_off = base + bt->bo_start_off;
    d.bo_start = base + bt->bo_start;
    d.bo_shape_of_rank = base + bt->bo_shape_of_rank;
    d.cat_off = (int)cat_all.size();
    d.n_cat = (int)bt->cat.size();
    tab.insert(tab.end(), bt->tab.begin(), bt->tab.end());
    cat_all.insert(cat_all.end(), bt->cat.begin(), bt->cat.end());
    d.blk_topk = std::max(1, o.blk_topk);
    d.blk_pick = o.blk_pick;
    if (tab.size() > (size_t)INT_MAX / 2 || cat_all.size() > (size_t)INT_MAX / 2)
        return set_error(PLP_E_CAPACITY, "block tables too large for one batch");
    return PLP_OK;
}

// Orientation table of every box type of an instance; clears *small when an
// orientation's footprint area reaches 65536 (its contact areas need 32 bits).
std::vector<TypeOrs> type_orientations(const Instance& I, int* small) {
    std::vector<TypeOrs> ot;
    ot.reserve(I.types.size());
    for (const auto& t : I.types) {
        TypeOrs to{};
        const auto v = orientations(t);
        to.n = (int)v.size();
        for (int k = 0; k < to.n; k++) { to.w[k] = v[k][0]; to.d[k] = v[k][1]; to.h[k] = v[k][2]; }
        for (int k = 0; k < to.n; k++)
            if (1LL * to.w[k] * to.d[k] >= 65536) *small = 0;
        ot.push_back(to);
    }
    return ot;
}

struct Batch {
    std::vector<const Instance*> insts;
    std::vector<plp_run_opts> opts;
    // host tables
    std::vector<InstDesc> desc;
    std::vector<int> steps;
    std::vector<TypeOrs> types;
    std::vector<std::vector<TypeOrs>> inst_ors;
    std::vector<int2> work;
    long long n_slots = 0, n_places = 0;
    int max_stride = 1, max_steps = 0, Hz = 0;
    bool multi_pass = false;
    // block-building engine: shape catalogue and per-instance orderings
    int engine = 0, max_types = 0;
    // contact areas of the decoder in 16 bits: allowed when every
    // orientation's footprint area is below 65536, chosen (plan) when the
    // batch's restarts exceed one wave at 32-bit residency
    int sup16_ok = 1, sup16 = 0;
    // seeded MT states computed once per distinct restart seed when the
    // batch's restarts share seeds (every instance seeding 0 .. R - 1, say):
    // seeds seed_lo .. seed_lo + seed_n - 1, or seed_n = 0 to seed in place
    long long seed_lo = 0;
    int seed_n = 0;
    std::vector<BlkShape> bcat;
    std::vector<int> btab;
    // device
    char* d_mem = nullptr;
    size_t bytes = 0;
    size_t o_desc, o_steps, o_types, o_bcat, o_btab, o_work, o_next, o_heads, o_places, o_best, o_scratch, o_gather, o_redo,
        o_seedtab;
    const uint32_t* mt_init = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    char* h_flag = nullptr;                // pinned error-flag word
    bool own_ctx = true;                   // h_flag and ev allocated by this batch
    std::vector<int2> redo_host;
    int2* h_redo_stage(size_t n) { redo_host.resize(n); return redo_host.data(); }
    size_t scratch_bytes = 0;
    int ctas = 0;
    TileConfig tile;
    // one-graph replay of a clean execution (flag reset, decoder, flag copy,
    // select, gather), kept for later executions with the same tile
    cudaGraphExec_t gexec = nullptr;
    cudaGraphExec_t gexec2 = nullptr;      // the part after the first decoder (retry stage, flags, select)
    TileConfig gtile;
    int glaunches = 0;
    bool gstaged = false;                  // the graph holds the device retry stage
    size_t stage_slots = 0;                // work size that decides the retry stage (0: this batch's)
    // host results: one block of [slot heads | best per instance | packed
    // placements (all slots, or the gathered best per instance)], shared
    // with the result objects that read it in place
    std::vector<SlotHead> heads;              // scratch of the capacity-retry loop
    std::shared_ptr<char> host;
    const SlotHead* heads_ptr = nullptr;
    const int2* best_ptr = nullptr;
    const unsigned long long* places_ptr = nullptr;
    bool best_only = false;
    double t_start = 0, t_end = 0;

    // validate and build the host tables; returns a status
    int build(const std::vector<const Instance*>& in, const std::vector<plp_run_opts>& op) {
        insts = in;
        opts = op;
        desc.clear(); steps.clear(); types.clear(); work.clear(); inst_ors.clear();
        bcat.clear(); btab.clear();
        engine = op.empty() ? 0 : op[0].engine;
        max_types = 0;
        sup16_ok = 1;
        sup16 = 0;
        n_slots = 0; n_places = 0; max_stride = 1; max_steps = 0; multi_pass = false;
        int maxH = 0;
        best_only = true;
        // item sequences and orientation tables of a large batch are built on
        // several threads; the rest of the build is appends in instance order
        std::vector<std::vector<int>> seqs;
        std::vector<std::vector<TypeOrs>> ors;
        std::vector<int> ors_small;
        if (in.size() >= 256) {
            seqs.resize(in.size());
            ors.resize(in.size());
            ors_small.assign(in.size(), 1);
            const unsigned hw = std::thread::hardware_concurrency();
            const int nt = (int)std::max(1u, std::min(16u, hw ? hw : 1u));
            std::atomic<size_t> next{0};
            auto job = [&] {
                for (size_t i0; (i0 = next.fetch_add(64)) < in.size();)
                    for (size_t k = i0; k < std::min(in.size(), i0 + 64); k++) {
                        if (op[k].order == 0 || op[k].order == 1) seqs[k] = item_sequence(*in[k], op[k].order);
                        ors[k] = type_orientations(*in[k], &ors_small[k]);
                    }
            };
            std::vector<std::thread> pool;
            for (int t = 1; t < nt; t++) pool.emplace_back(job);
            job();
            for (auto& th : pool) th.join();
        }
        {
            size_t n_types = 0, n_steps = 0;
            for (size_t i = 0; i < in.size(); i++) {
                n_types += in[i]->types.size();
                if (!seqs.empty()) n_steps += seqs[i].size();
            }
            desc.reserve(in.size());
            inst_ors.reserve(in.size());
            types.reserve(n_types);
            steps.reserve(n_steps);
        }
        for (size_t i = 0; i < in.size(); i++) {
            const Instance& I = *in[i];
            const plp_run_opts& o = op[i];
            const bool budget = o.time_limit_s >= 0;   // wall-clock budget, passes = cap (0: none)
            if (o.restarts < 1 || o.passes < 0 || (!budget && o.passes < 1))
                return set_error(PLP_E_INVALID, "restarts must be >= 1 and passes >= 1 (>= 0 with a time limit)");
            if (o.order != 0 && o.order != 1) return set_error(PLP_E_INVALID, "order must be 0 or 1");
            if (o.engine != 0 && o.engine != 1) return set_error(PLP_E_INVALID, "engine must be 0 or 1");
            if (o.engine != engine)
                return set_error(PLP_E_INVALID, "all instances of one batch must use the same engine");
            if (o.engine == 1 && (o.blk_pick < 0 || o.blk_pick > 2))
                return set_error(PLP_E_INVALID, "blk_pick must be 0 (first), 1 (support) or 2 (contact)");
            if (o.engine == 1 && I.types.size() > 2048)
                return set_error(PLP_E_CAPACITY, "the block engine takes at most 2048 box types");
            int xb = 0, yb = 0, zb = 0;
            for (int v = I.L; v; v >>= 1) xb++;
            for (int v = I.W; v; v >>= 1) yb++;
            for (int v = I.H; v; v >>= 1) zb++;
            if (xb + yb + zb > 32 || I.L >= 65536 || I.W >= 65536 || I.H >= 65536)
                return set_error(PLP_E_CAPACITY,
                                 "container too large for 32-bit point keys (bit lengths of L, W, H "
                                 "must sum to <= 32)");
            if ((int)I.types.size() >= 8192)
                return set_error(PLP_E_CAPACITY, "more than 8191 box types");
            const std::vector<int> seq = seqs.empty() ? item_sequence(I, o.order) : std::move(seqs[i]);
            InstDesc d{};
            d.L = I.L; d.W = I.W; d.H = I.H;
            d.n_steps = (int)seq.size();
            d.step_off = (int)steps.size();
            d.type_off = (int)types.size();
            d.xb = xb; d.yb = yb;
            d.restarts = o.restarts;
            d.slot_base = (int)n_slots;
            d.place_stride = std::max(1, d.n_steps);
            d.passes = budget && o.passes == 0 ? INT_MAX : o.passes;
            d.budget_ns = budget ? (long long)std::min(o.time_limit_s * 1e9, 9.0e18) : -1;
            d.place_off = n_places;
            d.seed = o.seed;
            d.eps = o.eps;
            d.has_theta = std::isnan(o.theta) ? 0 : 1;
            d.theta = d.has_theta ? o.theta : 0.0;
            d.mu = o.mu;
            d.first_fit = o.first_fit ? 1 : 0;
            desc.push_back(d);
            steps.insert(steps.end(), seq.begin(), seq.end());
            int small = 1;
            std::vector<TypeOrs> ot;
            if (ors.empty()) {
                ot = type_orientations(I, &small);
            } else {
                ot = std::move(ors[i]);
                small = ors_small[i];
            }
            if (!small) sup16_ok = 0;
            types.insert(types.end(), ot.begin(), ot.end());
            desc.back().engine = o.engine;
            desc.back().n_types = (int)I.types.size();
            max_types = std::max(max_types, (int)I.types.size());
            if (o.engine == 1) {
                const int sb = build_block_tables(I, ot, o, bcat, btab, desc.back());
                if (sb != PLP_OK) return sb;
            }
            inst_ors.push_back(std::move(ot));
            n_slots += o.restarts;
            n_places += (long long)o.restarts * d.place_stride;
            max_stride = std::max(max_stride, d.place_stride);
            max_steps = std::max(max_steps, d.n_steps);
            multi_pass = multi_pass || d.passes > 1;
            best_only = best_only && o.best_only;
            maxH = std::max(maxH, I.H);
        }
        // top-z index: one u16 per height level 0 .. H + 1 (binary search above 4094)
        Hz = maxH + 2 <= 4096 ? ((maxH + 2 + 7) & ~7) : 0;
        // a table of seeded states pays when at least two restarts share each seed
        seed_lo = 0;
        seed_n = 0;
        if (engine == 0 && !desc.empty()) {
            long long lo = LLONG_MAX, hi = LLONG_MIN;
            for (const auto& d : desc) {
                lo = std::min(lo, d.seed);
                hi = std::max(hi, d.seed + d.restarts - 1);
            }
            const long long span = hi - lo + 1;
            if (span >= 1 && span <= SEED_TABLE_MAX && n_slots >= 2 * span) {
                seed_lo = lo;
                seed_n = (int)span;
            }
        }
        if (n_slots > INT_MAX / 2) return set_error(PLP_E_CAPACITY, "too many restarts in one batch");
        // longest instances first (dynamic scheduling then balances the tail)
        std::vector<int> order(in.size());
        for (size_t i = 0; i < in.size(); i++) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return (long long)desc[a].n_steps * std::min(desc[a].passes, 1 << 16) >
                   (long long)desc[b].n_steps * std::min(desc[b].passes, 1 << 16);
        });
        work.reserve(n_slots);
        for (int i : order)
            for (int r = 0; r < desc[i].restarts; r++) work.push_back(make_int2(i, r));
        return PLP_OK;
    }

    static size_t al(size_t v) { return (v + 255) & ~size_t(255); }

    void plan(int sms, const TileConfig& t) {
        tile = t;
        // a latency-bound launch (one wave) gains nothing from the smaller
        // footprint and the 32-bit areas are a little faster to update
        sup16 = 0;
        if (engine == 0 && sup16_ok && t.G == 1) {
            int occ32 = 1;
            if (tile_occupancy(*this, t, &occ32) != cudaSuccess || occ32 < 1) occ32 = 1;
            sup16 = n_slots > (long long)sms * occ32 * t.D ? 1 : 0;
        }
        int occ = 1;
        if (tile_occupancy(*this, t, &occ) != cudaSuccess || occ < 1) occ = 1;
        const long long need = (n_slots + t.D - 1) / t.D;
        ctas = (int)std::max(1LL, std::min<long long>(need, (long long)sms * occ));
        scratch_bytes = multi_pass ? (size_t)ctas * t.D * max_stride * 8 : 0;
        size_t o = 0;
        o_desc = o;    o = al(o + desc.size() * sizeof(InstDesc));
        o_steps = o;   o = al(o + std::max<size_t>(1, steps.size()) * sizeof(int));
        o_types = o;   o = al(o + std::max<size_t>(1, types.size()) * sizeof(TypeOrs));
        o_bcat = o;    o = al(o + std::max<size_t>(1, bcat.size()) * sizeof(BlkShape));
        o_btab = o;    o = al(o + std::max<size_t>(1, btab.size()) * sizeof(int));
        o_work = o;    o = al(o + work.size() * sizeof(int2));
        // counters and flags: [0] work counter, [4] retry-stage work counter,
        // [8] error flag, [12] abort, [16] retry-stage error flag, [20] retry count
        o_next = o;    o = al(o + 32);
        o_heads = o;   o = al(o + n_slots * sizeof(SlotHead));
        o_places = o;  o = al(o + std::max<long long>(1, n_places) * 8);
        o_best = o;    o = al(o + desc.size() * sizeof(int2));
        o_gather = o;  o = al(o + desc.size() * (size_t)max_stride * 8);
        o_scratch = o; o = al(o + std::max<size_t>(8, scratch_bytes));
        o_redo = o;    o = al(o + work.size() * sizeof(int2));
        o_seedtab = o; o = al(o + (size_t)seed_n * 624 * sizeof(uint32_t));
        bytes = o;
    }

    size_t upload_bytes() const { return o_next; }   // desc .. work are contiguous at the front
};

int tile_smem(const Batch& b, const TileConfig& t) {
    return b.engine == 1 ? block_smem_bytes(t.P, t.C, std::max(1, b.max_steps), std::max(1, b.max_types), b.Hz)
                         : decoder_smem_bytes(t.P, t.C, b.Hz, t.G, b.sup16);
}

bool tile_supported(const Batch& b, const TileConfig& t) {
    return b.engine == 1 ? t.G == 1 && block_config_supported(t.D, t.M) : decoder_config_supported(t.G, t.D, t.M);
}

cudaError_t tile_occupancy(const Batch& b, const TileConfig& t, int* occ) {
    if (b.engine == 1)
        return block_occupancy(t.P, t.C, std::max(1, b.max_steps), std::max(1, b.max_types), b.Hz, t.D, t.M, occ);
    return decoder_occupancy(t.P, t.C, b.Hz, t.G, t.D, t.M, occ, b.sup16);
}

// Fewer decoders per CTA when the tile plus this batch's top-z index (and,
// for the block engine, its item and type tables) would not fit one CTA's
// shared memory. The block engine runs one warp per restart.
void fit_tile(TileConfig& t, const Batch& b) {
    if (b.engine == 1) t.G = 1;
    while (t.D > 1 && tile_smem(b, t) * t.D > 227 * 1024) t.D >>= 1;
    while (!tile_supported(b, t) && t.D > 1) t.D >>= 1;
    if (!tile_supported(b, t)) t.M = 1;
}

// pinned staging buffer per thread (grows)
struct Pinned {
    char* p = nullptr;
    size_t cap = 0;
    // error-flag word and timing events lent to this thread's one-shot
    // batches (pinned allocation and event creation cost more than a solve's
    // whole host side)
    char* flag = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // outgrown buffers, freed with the context: freeing pinned memory
    // synchronises the device, which would stall other streams mid-run
    std::vector<char*> retired;
    ~Pinned() {
        if (p) cudaFreeHost(p);
        for (char* q : retired) cudaFreeHost(q);
        if (flag) cudaFreeHost(flag);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    cudaError_t ensure_ctx() {
        cudaError_t e = cudaSuccess;
        if (!flag) e = cudaMallocHost(&flag, 64);
        for (auto& v : ev)
            if (e == cudaSuccess && !v) e = cudaEventCreate(&v);
        return e;
    }
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) retired.push_back(p);
        p = nullptr;
        cap = 0;
        size_t c = 1 << 20;
        while (c < n) c <<= 1;
        cudaError_t e = cudaMallocHost(&p, c);
        if (e == cudaSuccess) cap = c;
        return e;
    }
};

// Pinned host blocks that the results of synchronous solves are read from in
// place: the device writes each result byte once, into memory the result
// objects keep. A block returns to the free list when the last result
// viewing it is freed, and the pool pins at most a quarter of host memory, or
// PLP_PINNED_POOL_MB (a solve that finds no room copies into pageable memory
// instead). Pinned memory is freed
// only when the pool is destroyed with its handle: freeing it synchronises
// the device.
struct HostPool {
    std::mutex mu;
    std::vector<std::pair<char*, size_t>> free_list;   // (block, capacity)
    size_t held = 0;
    size_t limit = 0;
    HostPool() {
        const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
        const size_t phys = pages > 0 && page > 0 ? (size_t)pages * (size_t)page : ((size_t)16 << 30);
        limit = phys / 4;
        if (const char* v = std::getenv("PLP_PINNED_POOL_MB")) {   // operator override, 0 = off
            char* end = nullptr;
            const unsigned long long mb = std::strtoull(v, &end, 10);
            if (end != v) limit = (size_t)mb << 20;
        }
    }
    ~HostPool() {
        for (auto& f : free_list) cudaFreeHost(f.first);
    }
};

// a block of at least n bytes from the pool, or null when the pool is full
std::shared_ptr<char> pool_take(const std::shared_ptr<HostPool>& pool, size_t n) {
    n = std::max<size_t>(n, 1);
    size_t cap = (size_t)1 << 20;             // 1 MiB, then 1/8-power-of-two steps
    while (cap < n) cap <<= 1;
    if (cap > ((size_t)8 << 20)) {
        const size_t step = cap >> 3;
        cap = (n + step - 1) / step * step;
    }
    char* p = nullptr;
    {
        std::lock_guard<std::mutex> lk(pool->mu);
        int pick = -1;
        for (size_t i = 0; i < pool->free_list.size(); i++)
            if (pool->free_list[i].second >= n &&
                (pick < 0 || pool->free_list[i].second < pool->free_list[pick].second))
                pick = (int)i;
        if (pick >= 0) {
            p = pool->free_list[pick].first;
            cap = pool->free_list[pick].second;
            pool->free_list.erase(pool->free_list.begin() + pick);
        } else {
            if (pool->held + cap > pool->limit) return nullptr;
            pool->held += cap;                // reserved; allocated outside the lock
        }
    }
    if (!p && cudaMallocHost(&p, cap) != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(pool->mu);
        pool->held -= cap;
        return nullptr;
    }
    std::weak_ptr<HostPool> wp = pool;
    return std::shared_ptr<char>(p, [wp, cap](char* q) {
        if (auto sp = wp.lock()) {
            std::lock_guard<std::mutex> lk(sp->mu);
            sp->free_list.push_back({q, cap});
        } else {
            cudaFreeHost(q);
        }
    });
}

}  // namespace

// gather of the best restart's placements (decoder.cu); fixed scratch (noalloc.cu)
namespace plpb {
cudaError_t noalloc_scratch(void** ptr, size_t* bytes);
cudaError_t launch_gather_best(const InstDesc* inst, int n_inst, const int2* best,
                               const unsigned long long* places, unsigned long long* out,
                               int out_stride, cudaStream_t st);
}

namespace {

// ---------------------------------------------------------------------------
// batch stages: prepare (tables to the device), execute (decode + select,
// CUDA-event timed, capacity retries), fetch (results to the host), release.
// Device memory comes from the stream-ordered pool.
// ---------------------------------------------------------------------------
struct ExecStats {
    double device_ms = 0, decoder_ms = 0;
    int launches = 0;
    int redo = 0;                 // restarts the device retry stage ran again
    long long redo_wave = 0;      // resident decoders of the retry stage's tile
};

int batch_release(Batch& b, cudaStream_t st) {
    if (b.gexec) {
        cudaGraphExecDestroy(b.gexec);
        b.gexec = nullptr;
    }
    if (b.gexec2) {
        cudaGraphExecDestroy(b.gexec2);
        b.gexec2 = nullptr;
    }
    cudaError_t e = cudaSuccess;
    if (b.d_mem) e = cudaFreeAsync(b.d_mem, st);
    b.d_mem = nullptr;
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (b.own_ctx) {
        for (auto& ev : b.ev)
            if (ev) cudaEventDestroy(ev);
        if (b.h_flag) cudaFreeHost(b.h_flag);
    }
    for (auto& ev : b.ev) ev = nullptr;
    b.h_flag = nullptr;
    if (e != cudaSuccess) return set_cuda_error("batch free", e);
    if (e2 != cudaSuccess) return set_cuda_error("batch completion", e2);
    return PLP_OK;
}

// one_shot: the batch runs once and is released before this thread prepares
// another, so it borrows the thread's flag word and events and its upload
// needs no synchronisation of its own (the execution synchronises).
int batch_prepare(Batch& b, cudaStream_t st, Pinned& pin, int sms, const TileConfig& tc,
                  bool one_shot) {
    int status = PLP_OK;
    b.mt_init = device_mt_init(&status);
    if (!b.mt_init) return status;
    b.plan(sms, tc);
    auto fail = [&](const char* what, cudaError_t err) {
        const int s = set_cuda_error(what, err);
        std::string keep = plpb_last();
        batch_release(b, st);
        set_error(s, keep);
        return s;
    };
    cudaError_t e;
    if (one_shot) {
        e = pin.ensure_ctx();
        if (e != cudaSuccess) return fail("pinned flag", e);
        b.own_ctx = false;
        b.h_flag = pin.flag;
        for (int k = 0; k < 4; k++) b.ev[k] = pin.ev[k];
    } else {
        for (auto& ev : b.ev) {
            e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return fail("event creation", e);
        }
        e = cudaMallocHost(&b.h_flag, 64);
        if (e != cudaSuccess) return fail("pinned flag", e);
    }
    e = cudaMallocAsync(&b.d_mem, b.bytes, st);
    if (e != cudaSuccess) return fail("batch allocation", e);
    const size_t up = b.upload_bytes();
    e = pin.ensure(std::max(up, (size_t)1));
    if (e != cudaSuccess) return fail("pinned staging", e);
    std::memcpy(pin.p + b.o_desc, b.desc.data(), b.desc.size() * sizeof(InstDesc));
    std::memcpy(pin.p + b.o_steps, b.steps.data(), b.steps.size() * sizeof(int));
    std::memcpy(pin.p + b.o_types, b.types.data(), b.types.size() * sizeof(TypeOrs));
    if (!b.bcat.empty()) std::memcpy(pin.p + b.o_bcat, b.bcat.data(), b.bcat.size() * sizeof(BlkShape));
    if (!b.btab.empty()) std::memcpy(pin.p + b.o_btab, b.btab.data(), b.btab.size() * sizeof(int));
    std::memcpy(pin.p + b.o_work, b.work.data(), b.work.size() * sizeof(int2));
    e = cudaMemcpyAsync(b.d_mem, pin.p, up, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail("batch upload", e);
    e = launch_seed_table(b.seed_lo, b.seed_n, b.mt_init, reinterpret_cast<uint32_t*>(b.d_mem + b.o_seedtab), st);
    if (e != cudaSuccess) return fail("seed table", e);
    // the staging buffer is reused by the next batch of this thread
    if (!one_shot) {
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail("batch upload", e);
    }
    return PLP_OK;
}

static DecodeLaunch make_launch(const Batch& b, const TileConfig& t, const int2* work, int n_work, int sms) {
    DecodeLaunch L{};
    L.inst = reinterpret_cast<const InstDesc*>(b.d_mem + b.o_desc);
    L.step_type = reinterpret_cast<const int*>(b.d_mem + b.o_steps);
    L.types = reinterpret_cast<const TypeOrs*>(b.d_mem + b.o_types);
    L.work = work;
    L.n_work = n_work;
    L.work_next = reinterpret_cast<int*>(b.d_mem + b.o_next);
    L.err_flag = reinterpret_cast<int*>(b.d_mem + b.o_next + 8);
    L.abort = reinterpret_cast<int*>(b.d_mem + b.o_next + 12);
    L.heads = reinterpret_cast<SlotHead*>(b.d_mem + b.o_heads);
    L.places = reinterpret_cast<unsigned long long*>(b.d_mem + b.o_places);
    L.scratch = reinterpret_cast<unsigned long long*>(b.d_mem + b.o_scratch);
    L.mt_init = b.mt_init;
    L.seed_tab = b.seed_n ? reinterpret_cast<const uint32_t*>(b.d_mem + b.o_seedtab) : nullptr;
    L.seed_lo = b.seed_lo;
    L.seed_n = b.seed_n;
    L.P = t.P;
    L.C = t.C;
    L.Hz = b.Hz;
    L.engine = b.engine;
    L.sup16 = b.sup16;
    L.bcat = reinterpret_cast<const BlkShape*>(b.d_mem + b.o_bcat);
    L.btab = reinterpret_cast<const int*>(b.d_mem + b.o_btab);
    L.N = std::max(1, b.max_steps);
    L.T = std::max(1, b.max_types);
    L.warps_per_decoder = t.G;
    L.decoders_per_cta = t.D;
    L.min_blocks = t.M;
    L.sync_limit = t.sync_limit;
    L.sync_skip = t.sync_skip;
    int occ = 1;
    if (tile_occupancy(b, t, &occ) != cudaSuccess || occ < 1) occ = 1;
    L.ctas = (int)std::max<long long>(1, std::min<long long>((n_work + t.D - 1) / t.D, (long long)sms * occ));
    // multi-pass scratch holds one placement row per resident decoder
    if (b.multi_pass) {
        const size_t per_cta = (size_t)t.D * b.max_stride * 8;
        L.ctas = (int)std::max<size_t>(1, std::min<size_t>((size_t)L.ctas, b.scratch_bytes / per_cta));
    }
    return L;
}

bool same_tile(const TileConfig& a, const TileConfig& b) {
    return a.P == b.P && a.C == b.C && a.G == b.G && a.D == b.D && a.M == b.M &&
           a.sync_limit == b.sync_limit && a.sync_skip == b.sync_skip;
}

// After-decoder part of an execution: best restart per instance and, for
// best-only batches, the gather of its placements.
cudaError_t enqueue_select(Batch& b, cudaStream_t st, int* launches) {
    int2* d_best = reinterpret_cast<int2*>(b.d_mem + b.o_best);
    const InstDesc* d_inst = reinterpret_cast<const InstDesc*>(b.d_mem + b.o_desc);
    const SlotHead* d_heads = reinterpret_cast<const SlotHead*>(b.d_mem + b.o_heads);
    cudaError_t e = launch_select_best(d_inst, (int)b.desc.size(), d_heads, d_best, st);
    if (e != cudaSuccess) return e;
    (*launches)++;
    if (b.best_only) {
        unsigned long long* d_g = reinterpret_cast<unsigned long long*>(b.d_mem + b.o_gather);
        e = launch_gather_best(d_inst, (int)b.desc.size(), d_best,
                               reinterpret_cast<const unsigned long long*>(b.d_mem + b.o_places), d_g,
                               b.max_stride, st);
        if (e != cudaSuccess) return e;
        (*launches)++;
    }
    return cudaSuccess;
}

constexpr int FATAL_BITS = (1 << ERR_RNG) | (1 << ERR_SYNC);

// The device retry stage. In a batch whose restarts take more than one wave of
// resident decoders, a tile deep enough for the largest restart costs every
// restart occupancy. Such a batch instead runs at its tile and, in the same
// stream pass, runs the restarts that overflowed it again at a deeper tile
// (P and C doubled) over a list the device builds. Returns whether the stage
// applies and its tile.
bool redo_stage(const Batch& b, const TileConfig& t, int sms, TileConfig* deep, long long* deep_wave = nullptr) {
    int occ = 1;
    if (tile_occupancy(b, t, &occ) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        return false;
    }
    const size_t slots = b.stage_slots ? b.stage_slots : b.work.size();
    if ((long long)slots <= (long long)sms * occ * t.D) return false;   // one wave
    TileConfig d = t;
    d.P = std::min(P_MAX, t.P * 2);
    d.C = std::min(C_MAX, t.C * 2);
    if (d.P == t.P && d.C == t.C) return false;
    while (d.D > 1 && tile_smem(b, d) * d.D > 200 * 1024) d.D >>= 1;
    fit_tile(d, b);
    if (tile_smem(b, d) > 227 * 1024 || !tile_supported(b, d)) return false;
    if (deep_wave) {
        int occ2 = 1;
        if (tile_occupancy(b, d, &occ2) != cudaSuccess || occ2 < 1) {
            cudaGetLastError();
            occ2 = 1;
        }
        *deep_wave = (long long)sms * occ2 * d.D;
    }
    *deep = d;
    return true;
}

// the retry stage's decoder launch: the device-built list, its own work
// counter and error flag, the count read at kernel start
DecodeLaunch redo_launch(const Batch& b, const TileConfig& deep, int sms) {
    DecodeLaunch L = make_launch(b, deep, reinterpret_cast<const int2*>(b.d_mem + b.o_redo), (int)b.work.size(), sms);
    L.n_work_dev = reinterpret_cast<const int*>(b.d_mem + b.o_next + 20);
    L.work_next = reinterpret_cast<int*>(b.d_mem + b.o_next + 4);
    L.err_flag = reinterpret_cast<int*>(b.d_mem + b.o_next + 16);
    return L;
}

// stream operations of the retry stage (capturable): list, then decoder
cudaError_t enqueue_redo(Batch& b, const DecodeLaunch& L, int sms, cudaStream_t st, int* launches) {
    cudaError_t e = launch_redo_collect(reinterpret_cast<const int2*>(b.d_mem + b.o_work), (int)b.work.size(),
                                        reinterpret_cast<const InstDesc*>(b.d_mem + b.o_desc),
                                        reinterpret_cast<const SlotHead*>(b.d_mem + b.o_heads),
                                        reinterpret_cast<int2*>(b.d_mem + b.o_redo),
                                        reinterpret_cast<int*>(b.d_mem + b.o_next + 20), sms, st);
    if (e != cudaSuccess) return e;
    (*launches)++;
    e = enqueue_decoder(L, st);
    if (e != cudaSuccess) return e;
    (*launches)++;
    return cudaSuccess;
}

// Flags of an execution, as copied to the pinned words [flag, abort, retry
// flag, retry count]: the bits still to handle on the host -- fatal bits of
// either launch, and capacity bits of the last launch that ran each restart.
int pending_bits(const Batch& b, bool staged) {
    const volatile int* fl = reinterpret_cast<const volatile int*>(b.h_flag);
    return staged ? (fl[2] | (fl[0] & FATAL_BITS)) : fl[0];
}

// Records a clean execution of the batch with tile t as one CUDA graph:
// error-flag reset, the persistent decoder, the retry stage where it applies,
// the flag copy to the pinned words, selection and gather, as two graphs
// (the first ends after the first decoder, so an event between their
// launches gives the decoder's own time under replay). A capture that fails leaves the batch on direct
// launches.
void batch_capture(Batch& b, cudaStream_t st, int sms, const TileConfig& t) {
    if (b.gexec) {
        cudaGraphExecDestroy(b.gexec);
        b.gexec = nullptr;
    }
    if (b.gexec2) {
        cudaGraphExecDestroy(b.gexec2);
        b.gexec2 = nullptr;
    }
    // launch shapes and function attributes: before capture
    const DecodeLaunch L = make_launch(b, t, reinterpret_cast<const int2*>(b.d_mem + b.o_work),
                                       (int)b.work.size(), sms);
    if (configure_decoder(L) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    TileConfig deep;
    const bool staged = redo_stage(b, t, sms, &deep);
    DecodeLaunch L2{};
    if (staged) {
        L2 = redo_launch(b, deep, sms);
        if (configure_decoder(L2) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
    }
    char* d_flag = b.d_mem + b.o_next + 8;
    // two graphs, so that events recorded between their launches time the
    // decoder alone: [flag reset, decoder] and [retry stage, flag copy, select]
    cudaGraph_t g = nullptr, g2 = nullptr;
    int n = 0;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    e = cudaMemsetAsync(d_flag, 0, 16, st);
    if (e == cudaSuccess) e = enqueue_decoder(L, st);
    if (e == cudaSuccess) n++;
    cudaError_t e2 = cudaStreamEndCapture(st, &g);
    if (e == cudaSuccess && e2 == cudaSuccess) {
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            if (staged) e = enqueue_redo(b, L2, sms, st, &n);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b.h_flag, d_flag, 16, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = enqueue_select(b, st, &n);
            e2 = cudaStreamEndCapture(st, &g2);
        }
    }
    if (e == cudaSuccess && e2 == cudaSuccess && g && g2) {
        cudaGraphExec_t x = nullptr, x2 = nullptr;
        if (cudaGraphInstantiate(&x, g, 0) == cudaSuccess && cudaGraphInstantiate(&x2, g2, 0) == cudaSuccess) {
            b.gexec = x;
            b.gexec2 = x2;
            b.gtile = t;
            b.glaunches = n;
            b.gstaged = staged;
        } else {
            if (x) cudaGraphExecDestroy(x);
            if (x2) cudaGraphExecDestroy(x2);
        }
    }
    if (g2) cudaGraphDestroy(g2);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
}

// Host destination of a batch's results: [slot heads | best per instance |
// packed placements (all slots, or the gathered best per instance)]. With a
// pool, a pooled pinned block that the results keep; else a pageable block,
// staged through the thread's pinned buffer when it is large enough (that
// buffer is reused by the thread's next batch, so it is copied out).
struct ResultCopy {
    std::shared_ptr<char> blk;
    char* dst = nullptr;
    char* stage = nullptr;
    size_t hb = 0, bb = 0, pb = 0;
};

int result_dst(const Batch& b, Pinned* pin, const std::shared_ptr<HostPool>* pool, ResultCopy& rc) {
    rc.hb = b.n_slots * sizeof(SlotHead);
    rc.bb = b.desc.size() * sizeof(int2);
    rc.pb = b.best_only ? b.desc.size() * (size_t)b.max_stride * 8 : (size_t)b.n_places * 8;
    const size_t total = rc.hb + rc.bb + rc.pb;
    if (pool && *pool) rc.blk = pool_take(*pool, total);
    if (!rc.blk) {
        if (pin && pin->p && total <= pin->cap) rc.stage = pin->p;
        rc.blk = std::shared_ptr<char>(new (std::nothrow) char[std::max<size_t>(total, 1)], std::default_delete<char[]>());
        if (!rc.blk) return set_error(PLP_E_CAPACITY, "host memory for the results could not be allocated");
    }
    rc.dst = rc.stage ? rc.stage : rc.blk.get();
    return PLP_OK;
}

cudaError_t result_enqueue(const Batch& b, const ResultCopy& rc, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(rc.dst, b.d_mem + b.o_heads, rc.hb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rc.dst + rc.hb, b.d_mem + b.o_best, rc.bb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && rc.pb)
        e = cudaMemcpyAsync(rc.dst + rc.hb + rc.bb, b.d_mem + (b.best_only ? b.o_gather : b.o_places), rc.pb,
                            cudaMemcpyDeviceToHost, st);
    return e;
}

// after the copies completed: the batch's results view the block
void result_take(Batch& b, ResultCopy& rc) {
    if (rc.stage) std::memcpy(rc.blk.get(), rc.stage, rc.hb + rc.bb + rc.pb);
    b.host = std::move(rc.blk);
    b.heads_ptr = reinterpret_cast<const SlotHead*>(b.host.get());
    b.best_ptr = reinterpret_cast<const int2*>(b.host.get() + rc.hb);
    b.places_ptr = reinterpret_cast<const unsigned long long*>(b.host.get() + rc.hb + rc.bb);
}

// tile: in = tile to use, out = tile to start the next execution with (deeper
// after host retries of a one-wave batch, or when the retry stage ran more
// than a quarter of the restarts). graph: capture a clean execution and
// replay it on later calls (batches that run more than once). rc: copy the
// results there in the same stream pass, after the final selection, so one
// synchronisation covers execution and result copy.
int batch_execute(Batch& b, cudaStream_t st, int sms, TileConfig& tile, ExecStats* xs, bool graph,
                  const ResultCopy* rc = nullptr) {
    auto fail = [&](const char* what, cudaError_t err) {
        const int s = set_cuda_error(what, err);
        std::string keep = plpb_last();
        batch_release(b, st);
        set_error(s, keep);
        return s;
    };
    const volatile int* fl = reinterpret_cast<const volatile int*>(b.h_flag);
    ExecStats x;
    TileConfig t = tile;
    fit_tile(t, b);
    if (b.gexec && same_tile(t, b.gtile)) {
        // replay: one graph launch, one synchronisation
        cudaError_t e = cudaEventRecord(b.ev[0], st);
        if (e == cudaSuccess) e = cudaGraphLaunch(b.gexec, st);
        if (e == cudaSuccess) e = cudaEventRecord(b.ev[1], st);
        if (e == cudaSuccess) e = cudaGraphLaunch(b.gexec2, st);
        if (e == cudaSuccess) e = cudaEventRecord(b.ev[2], st);
        if (e == cudaSuccess && rc) e = result_enqueue(b, *rc, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail("graph execution", e);
        if (pending_bits(b, b.gstaged) == 0) {
            float ms = 0, dms = 0;
            cudaEventElapsedTime(&ms, b.ev[0], b.ev[2]);
            if (cudaEventElapsedTime(&dms, b.ev[0], b.ev[1]) != cudaSuccess) {
                cudaGetLastError();
                dms = ms;
            }
            x.device_ms = ms;
            x.decoder_ms = dms;
            x.launches = b.glaunches;
            tile = t;
            if (xs) *xs = x;
            return PLP_OK;
        }
        // flags left to handle: run again on direct launches, which handle them
    }
    const int2* d_work = reinterpret_cast<const int2*>(b.d_mem + b.o_work);
    char* d_flag = b.d_mem + b.o_next + 8;
    // decoder, retry stage, flag copy and selection in one stream pass with a
    // single synchronisation; flags left over (rare) re-run the affected
    // restarts below and select again
    TileConfig deep;
    const bool staged = redo_stage(b, t, sms, &deep, &x.redo_wave);
    cudaError_t e = cudaMemsetAsync(d_flag, 0, 16, st);
    if (e != cudaSuccess) return fail("flag reset", e);
    e = cudaEventRecord(b.ev[0], st);
    if (e == cudaSuccess) e = launch_decoder(make_launch(b, t, d_work, (int)b.work.size(), sms), st);
    if (e == cudaSuccess) e = cudaEventRecord(b.ev[1], st);
    if (e != cudaSuccess) return fail("decoder launch", e);
    x.launches++;
    if (staged) {
        const DecodeLaunch L2 = redo_launch(b, deep, sms);
        e = configure_decoder(L2);
        if (e == cudaSuccess) e = enqueue_redo(b, L2, sms, st, &x.launches);
        if (e != cudaSuccess) return fail("retry stage launch", e);
    }
    e = cudaMemcpyAsync(b.h_flag, d_flag, 16, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return fail("flag copy", e);
    {
        int n = 0;
        e = enqueue_select(b, st, &n);
        x.launches += n;
        if (e != cudaSuccess) return fail("select launch", e);
    }
    e = cudaEventRecord(b.ev[2], st);
    if (e == cudaSuccess && rc) e = result_enqueue(b, *rc, st);   // valid unless host retries follow
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail("decoder", e);
    float ms = 0;
    cudaEventElapsedTime(&ms, b.ev[0], b.ev[1]);
    x.decoder_ms = ms;
    const int staged_count = staged ? fl[3] : 0;
    x.redo = staged_count;
    // host retries: restarts whose live points or boxes outgrew the last
    // tile they ran with run again with a deeper one (same slots, so results
    // land in place)
    TileConfig tr = staged ? deep : t;
    bool retried = false;
    for (int attempt = 0, bits = pending_bits(b, staged); bits != 0; attempt++, bits = fl[0]) {
        retried = true;
        if (bits & (1 << ERR_RNG)) {
            batch_release(b, st);
            return set_error(PLP_E_DEVICE, "decoder reported an RNG rejection-bound error");
        }
        if (bits & (1 << ERR_SYNC)) {
            batch_release(b, st);
            return set_error(PLP_E_DEVICE, "decoder warps stopped meeting at a barrier (bounded wait gave up)");
        }
        b.heads.resize(b.n_slots);
        e = cudaMemcpyAsync(b.heads.data(), b.d_mem + b.o_heads, b.n_slots * sizeof(SlotHead),
                            cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail("head copy", e);
        std::vector<int2> redo;
        bool grow_p = false, grow_c = false;
        for (const int2& w : b.work) {
            const SlotHead& h = b.heads[b.desc[w.x].slot_base + w.y];
            if (h.err == ERR_BOX_CAP) { grow_p = true; redo.push_back(w); }
            else if (h.err == ERR_CAND_CAP) { grow_c = true; redo.push_back(w); }
        }
        if (redo.empty() || attempt == 6) {
            batch_release(b, st);
            return set_error(PLP_E_CAPACITY, "decoder tile capacity exceeded after retries");
        }
        if (grow_p) tr.P = std::min(P_MAX, std::max(tr.P * 2, 32));
        if (grow_c) tr.C = std::min(C_MAX, tr.C * 2);
        // deeper tiles: fewer decoders per CTA keeps one CTA within 227 KB
        while (tr.D > 1 && tile_smem(b, tr) * tr.D > 200 * 1024) tr.D >>= 1;
        fit_tile(tr, b);
        if (tile_smem(b, tr) > 227 * 1024 || !tile_supported(b, tr)) {
            batch_release(b, st);
            return set_error(PLP_E_CAPACITY, "instance needs a larger tile than shared memory holds");
        }
        std::memcpy(b.h_redo_stage(redo.size()), redo.data(), redo.size() * sizeof(int2));
        int2* d_redo = reinterpret_cast<int2*>(b.d_mem + b.o_redo);
        e = cudaMemcpyAsync(d_redo, b.redo_host.data(), redo.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_flag, 0, 8, st);
        if (e == cudaSuccess) e = launch_decoder(make_launch(b, tr, d_redo, (int)redo.size(), sms), st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b.h_flag, d_flag, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail("decoder relaunch", e);
        x.launches++;
    }
    if (retried) {   // the first selection read unfinished restarts
        int n = 0;
        e = enqueue_select(b, st, &n);
        x.launches += n;
        if (e != cudaSuccess) return fail("select launch", e);
        e = cudaEventRecord(b.ev[2], st);
        if (e == cudaSuccess && rc) e = result_enqueue(b, *rc, st);   // again, after the retries
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail("select", e);
    }
    cudaEventElapsedTime(&ms, b.ev[0], b.ev[2]);
    x.device_ms = ms;
    if (graph && !retried) batch_capture(b, st, sms, t);
    if (staged) {
        if ((long long)staged_count * 4 > (long long)b.work.size()) tile = deep;
        else tile = t;
    } else {
        tile = tr;
    }
    if (xs) *xs = x;
    return PLP_OK;
}

// Copies a finished batch's results to the host (destination as result_dst).
int batch_fetch(Batch& b, cudaStream_t st, Pinned* pin = nullptr, const std::shared_ptr<HostPool>* pool = nullptr) {
    ResultCopy rc;
    int s = result_dst(b, pin, pool, rc);
    if (s != PLP_OK) {
        std::string keep = plpb_last();
        batch_release(b, st);
        set_error(s, keep);
        return s;
    }
    cudaError_t e = result_enqueue(b, rc, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        s = set_cuda_error("result copy", e);
        std::string keep = plpb_last();
        batch_release(b, st);
        set_error(s, keep);
        return s;
    }
    result_take(b, rc);
    return PLP_OK;
}

// bytes copied host->device per execution and device->host per fetch
size_t batch_h2d_bytes(const Batch& b) { return b.upload_bytes(); }
size_t batch_d2h_bytes(const Batch& b) {
    return b.n_slots * sizeof(SlotHead) + b.desc.size() * sizeof(int2) +
           (b.best_only ? b.desc.size() * (size_t)b.max_stride * 8 : (size_t)b.n_places * 8);
}

// full synchronous run used by plp_solve and the serving workers
int run_batch(Batch& b, cudaStream_t st, Pinned& pin, int sms, TileConfig& tile,
              const std::shared_ptr<HostPool>* pool = nullptr) {
    int s = batch_prepare(b, st, pin, sms, tile, true);
    if (s != PLP_OK) return s;
    ResultCopy rc;
    s = result_dst(b, &pin, pool, rc);
    if (s != PLP_OK) {
        std::string keep = plpb_last();
        batch_release(b, st);
        set_error(s, keep);
        return s;
    }
    s = batch_execute(b, st, sms, tile, nullptr, false, &rc);   // results copied in the same pass
    if (s != PLP_OK) return s;
    result_take(b, rc);
    return batch_release(b, st);
}

// Builds the per-instance result objects of a finished batch; they view the
// batch's host block in place.
std::vector<plp_result*> collect(const Batch& b, double time_s) {
    std::vector<plp_result*> out;
    out.reserve(b.desc.size());
    for (size_t i = 0; i < b.desc.size(); i++) {
        const InstDesc& d = b.desc[i];
        auto* r = new plp_result;
        r->restarts = d.restarts;
        r->stride = d.place_stride;
        r->ors = b.inst_ors[i];
        r->L = d.L; r->W = d.W; r->H = d.H;
        r->steps.assign(b.steps.begin() + d.step_off, b.steps.begin() + d.step_off + d.n_steps);
        r->block = b.host;
        r->heads = b.heads_ptr + d.slot_base;
        r->seed0 = d.seed;
        r->time_s = time_s;
        r->best = b.best_ptr[i].x;
        r->best_fallback = b.best_ptr[i].y;
        r->kept_all = !b.best_only;
        r->packed = b.places_ptr + (b.best_only ? (long long)i * b.max_stride : d.place_off);
        out.push_back(r);
    }
    return out;
}

}  // namespace

// ===========================================================================
// handle: budget, streams, serving loop
// ===========================================================================
struct Request {
    int64_t id;
    Instance inst;
    plp_run_opts opts;
    size_t bytes = 0;
    int status = PLP_E_PENDING;   // PLP_E_PENDING until finished
    bool running = false, cancelled = false;
    std::string err;
    plp_result* result = nullptr;
    double t_submit = 0, t_start = 0, t_done = 0;
};

namespace {
struct ServeEngine;
}

struct plp_handle {
    int device = 0;
    int sms = 148;
    size_t budget = 0;
    size_t in_use = 0;
    TileConfig tile;
    std::string err;
    std::mutex mu;
    std::condition_variable cv;       // request state changes
    std::condition_variable cv_sched; // work for the scheduler
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_id = 1;
    bool stop = false;
    int n_workers = 4;
    int busy_workers = 0;
    int workers_ready = 0;
    std::vector<std::thread> workers;
    std::vector<cudaStream_t> streams;
    // synchronous solves
    cudaStream_t sync_stream = nullptr;
    std::mutex sync_mu;
    Pinned sync_pin;
    std::shared_ptr<HostPool> pool = std::make_shared<HostPool>();   // result blocks of synchronous solves
    // serving engine (one persistent launch that requests join), made on the
    // first eligible request; off with PLP_SERVE=0 or when it cannot be set up
    ServeEngine* serve = nullptr;
    bool serve_off = false;
    std::mutex serve_mu;
};

namespace {

void record(plp_handle* h, int status) {
    if (h && status != PLP_OK && status != PLP_E_PENDING) {
        std::lock_guard<std::mutex> g(g_handle_err_mu);
        h->err = g_err;
    }
}

// rough device bytes of one request (tables + results + scratch share)
size_t request_bytes(const Instance& I, const plp_run_opts& o) {
    const size_t steps = (size_t)std::max(1, I.n_items());
    return 4096 + I.types.size() * sizeof(TypeOrs) + steps * 4 +
           (size_t)o.restarts * (sizeof(int2) + sizeof(SlotHead) + steps * 8) +
           (o.passes > 1 || (o.time_limit_s >= 0 && o.passes == 0) ? (size_t)148 * 64 * steps * 8 : 0);
}

void worker_main(plp_handle* h, int wi) {
    cudaSetDevice(h->device);
    Pinned pin;
    cudaStream_t st = h->streams[wi];
    // pinned flag word, events and a staging buffer for a typical request,
    // made before the first request rather than inside its latency
    if (pin.ensure_ctx() != cudaSuccess || pin.ensure((size_t)4 << 20) != cudaSuccess) cudaGetLastError();
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->workers_ready++;
    }
    h->cv.notify_all();
    for (;;) {
        std::vector<Request*> wave;
        size_t wave_bytes = 0;
        {
            std::unique_lock<std::mutex> lk(h->mu);
            h->cv_sched.wait(lk, [&] {
                if (h->stop) return true;
                if (h->queue.empty()) return false;
                auto it = h->reqs.find(h->queue.front());
                if (it == h->reqs.end()) return true;
                Request* r = it->second.get();
                return r->cancelled || h->in_use + r->bytes <= h->budget;
            });
            if (h->stop) return;
            // admit queued requests in arrival order while the budget allows
            while (!h->queue.empty()) {
                auto it = h->reqs.find(h->queue.front());
                if (it == h->reqs.end() || it->second->cancelled) {
                    h->queue.pop_front();
                    continue;
                }
                Request* r = it->second.get();
                if (h->in_use + wave_bytes + r->bytes > h->budget) break;
                wave_bytes += r->bytes;
                r->running = true;
                r->t_start = now_seconds();
                wave.push_back(r);
                h->queue.pop_front();
                if (wave.size() >= 4096) break;
            }
            h->in_use += wave_bytes;
            h->busy_workers++;
        }
        if (wave.empty()) {
            std::lock_guard<std::mutex> lk(h->mu);
            h->busy_workers--;
            continue;
        }
        Batch b;
        std::vector<const Instance*> in;
        std::vector<plp_run_opts> op;
        for (Request* r : wave) {
            in.push_back(&r->inst);
            op.push_back(r->opts);
        }
        const double t0 = now_seconds();
        int s = b.build(in, op);
        TileConfig tile;
        {
            std::lock_guard<std::mutex> lk(h->mu);
            tile = h->tile;
        }
        if (s == PLP_OK) s = run_batch(b, st, pin, h->sms, tile);
        if (s == PLP_OK) {
            std::lock_guard<std::mutex> lk(h->mu);
            remember_tile(h->tile, tile);
        }
        std::vector<plp_result*> res;
        if (s == PLP_OK) res = collect(b, now_seconds() - t0);
        const std::string msg = s == PLP_OK ? "" : g_err;
        {
            std::lock_guard<std::mutex> lk(h->mu);
            const double t = now_seconds();
            for (size_t i = 0; i < wave.size(); i++) {
                Request* r = wave[i];
                r->running = false;
                r->t_done = t;
                if (s == PLP_OK) {
                    r->result = res[i];
                    r->status = r->cancelled ? PLP_E_CANCELLED : PLP_OK;
                } else {
                    r->status = s;
                    r->err = msg;
                }
            }
            h->in_use -= wave_bytes;
            h->busy_workers--;
        }
        h->cv.notify_all();
        h->cv_sched.notify_all();
    }
}

// ===========================================================================
// serving engine: one persistent decoder launch that requests join while it
// runs (continuous batching)
// ===========================================================================
// A request is eligible when it runs the extreme-point decoder for one pass
// with every restart's result kept (engine 0, passes 1, no time budget, not
// best-only); the others go to the wave workers above. An eligible request:
//   1. is admitted when its tables and results fit the serving arena (a ring
//      of device memory reserved from the handle's budget: half of it, at
//      most PLP_SERVE_ARENA_MB, default 4096) and a completion record is free;
//   2. has, in one stream pass on the upload stream, its descriptor, step
//      types and orientations copied into its arena region, its restarts
//      appended to the device work ring, and then the ring's tail advanced
//      (stream order puts the tables in memory before the tail moves);
//   3. is decoded by whichever decoders of the running launch claim its items;
//      the decoder that finishes its last restart selects the best restart and
//      writes it, with the request's sequence number, to the request's
//      host-mapped completion record;
//   4. has its slot heads and placements copied out once the record shows its
//      sequence number, and completes; its arena region is then free.
// The launch keeps running while requests arrive. The host stops it after
// SERVE_IDLE_STOP_S without requests and starts it again for the next one; a
// decoder that finds no work for about a second exits by itself as well
// (bounded polling). A request that the running launch's configuration cannot
// take (a container taller than its top-z index covers, or footprints too
// large for its 16-bit contact areas) waits until the launch has drained, and
// the next launch takes the merged configuration. Restarts that overflow the
// serving tile (P = 256 boxes, C = 768 live points; rare) make their request
// run again on the wave path's code, which retries with deeper tiles.
constexpr int SERVE_RING = 1 << 20;            // work items in flight at most
constexpr int SERVE_RECORDS = 1 << 16;         // requests in flight at most
constexpr double SERVE_IDLE_STOP_S = 0.05;
constexpr int SERVE_IDLE_POLLS = 250000;       // about 1 s of empty polls per decoder
constexpr int SERVE_DEEP_IDLE_POLLS = 8000000; // about a minute for an overflow decoder
constexpr int SERVE_DEEP = 32;                 // overflow decoders per launch (PLP_SERVE_DEEP overrides)
constexpr size_t SERVE_UP_STAGE = (size_t)32 << 20;     // pinned staging of uploads
constexpr size_t SERVE_DOWN_STAGE = (size_t)256 << 20;  // pinned staging of results

// Regions of one block freed in allocation order (the oldest first): a ring.
// Free space is [newest end, cap) + [0, oldest start) until the newest region
// lies before the oldest, then [newest end, oldest start).
struct RegionRing {
    struct R {
        size_t off, end;
        bool freed;
    };
    std::deque<R> live;
    long long base = 0;                // id of live.front()
    size_t cap = 0;
    // first fit after the newest region (or from 0); -1 when it does not fit
    long long place(size_t n, size_t* off, const std::function<bool(size_t, size_t)>& fits) {
        if (live.empty()) {
            if (!fits(0, cap)) return -1;
            *off = 0;
        } else {
            const size_t oldest = live.front().off, newest_end = live.back().end;
            const bool wrapped = live.back().off < oldest;
            if (!wrapped && fits(newest_end, cap)) *off = newest_end;
            else if (!wrapped && fits(0, oldest)) *off = 0;
            else if (wrapped && fits(newest_end, oldest)) *off = newest_end;
            else return -1;
        }
        (void)n;
        return 0;
    }
    long long push(size_t off, size_t end) {
        live.push_back({off, end, false});
        return base + (long long)live.size() - 1;
    }
    void release(long long id) {
        live[(size_t)(id - base)].freed = true;
        while (!live.empty() && live.front().freed) {
            live.pop_front();
            base++;
        }
    }
    void drop_newest() {
        if (!live.empty()) live.pop_back();
    }
    void clear() {
        base += (long long)live.size();
        live.clear();
    }
};

// A pinned block used as a RegionRing of 256-byte aligned chunks.
struct PinnedRing {
    char* p = nullptr;
    RegionRing ring;
    cudaError_t init(size_t cap) {
        ring.cap = cap;
        return cudaMallocHost(&p, cap);
    }
    ~PinnedRing() {
        if (p) cudaFreeHost(p);
    }
    char* take(size_t n, long long* id) {
        n = (n + 255) & ~(size_t)255;
        size_t off = 0;
        if (ring.place(n, &off, [&](size_t a, size_t b) { return a + n <= b; }) < 0) return nullptr;
        *id = ring.push(off, off + n);
        return p + off;
    }
};

// PLP_SERVE_TRACE=1: one stderr line per launch, stop and launch end
bool serve_trace() {
    static const bool on = [] {
        const char* v = std::getenv("PLP_SERVE_TRACE");
        return v && v[0] == '1';
    }();
    return on;
}

size_t serve_align(size_t x, size_t unit) {    // a multiple of unit and of 128 bytes
    size_t q = unit;
    while (q % 128) q += unit;
    return (x + q - 1) / q * q;
}

struct ServeConfig {
    int P = 256, C = 512, D = 1, M = 12, Hz = 0, sup16 = 0;
    int deep_P = 512, deep_C = 2048;   // the overflow decoders' tile (global memory)
    bool valid = false;
};

// absolute arena offsets of one request's tables and results
struct ServeRegion {
    size_t off = 0, end = 0;
    size_t desc = 0, steps = 0, types = 0, heads = 0, places = 0;
};

bool serve_layout(const Batch& b, size_t pos, size_t limit, ServeRegion& g) {
    const InstDesc& d = b.desc[0];
    g.off = pos;
    g.desc = serve_align(pos, sizeof(InstDesc));
    g.steps = serve_align(g.desc + sizeof(InstDesc) + sizeof(ServeTail), sizeof(int));
    g.types = serve_align(g.steps + std::max<size_t>(1, b.steps.size()) * sizeof(int), sizeof(TypeOrs));
    g.heads = serve_align(g.types + std::max<size_t>(1, b.types.size()) * sizeof(TypeOrs), sizeof(SlotHead));
    g.places = serve_align(g.heads + (size_t)d.restarts * sizeof(SlotHead), 8);
    g.end = g.places + (size_t)d.restarts * d.place_stride * 8;
    return g.end <= limit;
}

struct ServeJob {
    int64_t id = 0;
    Instance inst;                 // copies: the request may be cancelled and taken before admission
    plp_run_opts opts{};
    Request* r = nullptr;          // set at admission, when the request can no longer be taken
    Batch b;
    bool built = false;
    int state = 0;                 // 1 published, 2 copying results out
    ServeRegion g;
    long long region = -1;         // id of its arena region
    long long seq = 0;
    int slot = -1;
    cudaEvent_t ev_up = nullptr, ev = nullptr;
    long long up_id = -1, down_id = -1;   // staging regions
    char* down = nullptr;                 // pinned staging of [heads | places]
    size_t up_bytes = 0, heads_bytes = 0, places_bytes = 0;
    double t0 = 0;
};

struct ServeEngine {
    plp_handle* h;
    int device = 0, sms = 148;
    // device
    char* arena = nullptr;
    size_t cap = 0;
    // ctl: [0] head, [1] tail, [2] stop, [3] error flag, [4] abort, [5] overflow
    // head, [6] overflow reservations, [7] main decoders alive
    int* ctl = nullptr;
    int2* ring = nullptr;
    int4* dring = nullptr;
    unsigned char* deep_scratch = nullptr;
    // host
    long long* m_done_seq = nullptr;   // host-mapped completion records
    int2* m_done_best = nullptr;
    int* h_word = nullptr;         // pinned: [0] head and [3..4] overflow head and reservations after a
                                   // launch, [2] main decoders, [5] 1 and [6] 0 (stop), [8 ..] tail values
    PinnedRing up_stage, down_stage;
    ServeArgs args{};
    cudaStream_t up = nullptr, kern = nullptr, down = nullptr;
    cudaEvent_t ev_kern = nullptr, ev_go = nullptr;
    bool running = false, broken = false, stop_sent = false;
    int n_deep = 0;                       // overflow decoders per launch
    std::atomic<bool> yield_req{false};   // a synchronous call on the handle wants the SMs
    ServeConfig cfg;
    const uint32_t* mt_init = nullptr;
    RegionRing arena_ring;             // request regions of the arena
    std::deque<ServeJob*> pending;     // submitted, not yet taken by the engine (h->mu)
    std::deque<ServeJob*> fresh;       // taken, not yet admitted (engine thread)
    std::deque<ServeJob*> active;      // admitted (engine thread)
    std::condition_variable cv;        // new pending requests (h->mu)
    long long next_seq = 1;
    long long published = 0, restarts_done = 0;
    int tail = 0, tail_copies = 0;
    std::atomic<long long> n_launches{0}, n_served{0}, n_fallbacks{0}, n_waved{0};
    bool quit = false;                 // h->mu
    double last_busy = 0;
    std::thread th;
    Pinned pin;                        // the fallback's staging

    explicit ServeEngine(plp_handle* hh) : h(hh) {}

    static bool eligible(const plp_run_opts& o) {
        return o.engine == 0 && o.passes == 1 && o.time_limit_s < 0 && !o.best_only;
    }

    int deep_bytes() const { return decoder_smem_bytes(cfg.deep_P, cfg.deep_C, 4096, 1, 0); }

    int init(size_t arena_bytes) {
        device = h->device;
        sms = h->sms;
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return set_cuda_error("serving engine device", e);
        int status = PLP_OK;
        mt_init = device_mt_init(&status);
        if (!mt_init) return status;
        cap = arena_bytes;
        arena_ring.cap = cap;
        e = cudaMalloc(&arena, cap);
        if (e == cudaSuccess) e = cudaMalloc(&ctl, 64);
        if (e == cudaSuccess) e = cudaMemset(ctl, 0, 64);
        if (e == cudaSuccess) e = cudaMalloc(&ring, sizeof(int2) * SERVE_RING);
        if (e == cudaSuccess) e = cudaMalloc(&dring, sizeof(int4) * SERVE_RING);
        if (e == cudaSuccess) e = cudaMemset(dring, 0, sizeof(int4) * SERVE_RING);
        // PLP_SERVE_TILE=P,C,M: the main decoders' tile (M 1 or 12); taken
        // only if it fits one CTA's shared memory with the largest top-z
        // index and 32-bit contact areas, so no later launch can fail on it
        if (const char* v = std::getenv("PLP_SERVE_TILE")) {
            int p = 0, c = 0, m = 0;
            if (std::sscanf(v, "%d,%d,%d", &p, &c, &m) == 3 && p >= 16 && p <= P_MAX && c >= 32 && c <= C_MAX &&
                c % 32 == 0 && serve_config_supported(1, m) && decoder_smem_bytes(p, c, 4096, 1, 0) <= 227 * 1024) {
                cfg.P = p;
                cfg.C = c;
                cfg.M = m;
            }
        }
        n_deep = SERVE_DEEP;
        if (const char* v = std::getenv("PLP_SERVE_DEEP")) {
            char* end = nullptr;
            const long x = std::strtol(v, &end, 10);
            if (end != v && x >= 0 && x <= 1024) n_deep = (int)x;
        }
        if (e == cudaSuccess) e = cudaMalloc(&deep_scratch, (size_t)std::max(1, n_deep) * deep_bytes());
        if (e == cudaSuccess)
            e = cudaHostAlloc(&m_done_seq, sizeof(long long) * SERVE_RECORDS, cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaHostAlloc(&m_done_best, sizeof(int2) * SERVE_RECORDS, cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaMallocHost(&h_word, sizeof(int) * (8 + SERVE_RECORDS));
        if (e == cudaSuccess) e = up_stage.init(SERVE_UP_STAGE);
        if (e == cudaSuccess) e = down_stage.init(SERVE_DOWN_STAGE);
        for (cudaStream_t* s : {&up, &kern, &down})
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_kern, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_go, cudaEventDisableTiming);
        void* p = nullptr;
        if (e == cudaSuccess) {
            for (int i = 0; i < SERVE_RECORDS; i++) m_done_seq[i] = -1;
            std::memset(m_done_best, 0, sizeof(int2) * SERVE_RECORDS);
            std::memset(h_word, 0, sizeof(int) * 8);
            h_word[5] = 1;                 // stop word sources (never written again)
            h_word[6] = 0;
            e = cudaHostGetDevicePointer(&p, m_done_seq, 0);
        }
        args.done_seq = static_cast<volatile long long*>(p);
        if (e == cudaSuccess) e = cudaHostGetDevicePointer(&p, m_done_best, 0);
        args.done_best = static_cast<int2*>(p);
        if (e != cudaSuccess) return set_cuda_error("serving engine set-up", e);
        args.head = ctl;
        args.tail = ctl + 1;
        args.stop = ctl + 2;
        args.ring = ring;
        args.ring_mask = SERVE_RING - 1;
        args.idle_polls = SERVE_IDLE_POLLS;
        args.dring = dring;
        args.dhead = ctl + 5;
        args.dtail = ctl + 6;
        args.alive = ctl + 7;
        args.n_deep = n_deep;
        args.deep_P = cfg.deep_P;
        args.deep_C = cfg.deep_C;
        args.deep_bytes = deep_bytes();
        args.deep_scratch = deep_scratch;
        args.deep_idle_polls = SERVE_DEEP_IDLE_POLLS;
        th = std::thread([this] { loop(); });
        return PLP_OK;
    }

    ~ServeEngine() {
        {
            std::lock_guard<std::mutex> lk(h->mu);
            quit = true;
        }
        cv.notify_all();
        if (th.joinable()) th.join();
        cudaSetDevice(device);
        if (serve_trace()) std::fprintf(stderr, "[serve %.6f] teardown running=%d\n", now_seconds(), (int)running);
        if (running) {
            send_stop(1);
            cudaStreamSynchronize(up);       // the stop word is in device memory
            cudaEventSynchronize(ev_kern);   // decoders finish their items and leave
        }
        if (serve_trace()) std::fprintf(stderr, "[serve %.6f] teardown launch ended\n", now_seconds());
        for (cudaStream_t s : {up, kern, down})
            if (s) cudaStreamSynchronize(s);
        for (ServeJob* j : active) drop(j);
        for (ServeJob* j : fresh) delete j;
        for (ServeJob* j : pending) delete j;
        for (cudaStream_t s : {up, kern, down})
            if (s) cudaStreamDestroy(s);
        for (cudaEvent_t v : {ev_kern, ev_go})
            if (v) cudaEventDestroy(v);
        for (void* q : {(void*)m_done_seq, (void*)m_done_best, (void*)h_word})
            if (q) cudaFreeHost(q);
        for (void* q : {(void*)arena, (void*)ctl, (void*)ring, (void*)dring, (void*)deep_scratch})
            if (q) cudaFree(q);
    }

    void drop(ServeJob* j) {
        for (cudaEvent_t v : {j->ev_up, j->ev})
            if (v) cudaEventDestroy(v);
        delete j;
    }

    // The stop word, in stream order on the upload stream, as a copy from a
    // pinned constant: a copy runs on a copy engine while the serving launch
    // holds every SM, where a memset (which may run as a kernel) would wait
    // for the launch to end.
    // The query submits the copy at once: work enqueued on a stream can wait
    // in the driver until something flushes that stream, and a caller that
    // then waits on the launch's stream alone would wait for the decoders'
    // idle bound instead.
    void send_stop(int v) {
        const cudaError_t e = cudaMemcpyAsync(ctl + 2, h_word + (v ? 5 : 6), sizeof(int), cudaMemcpyHostToDevice, up);
        (void)cudaStreamQuery(up);
        stop_sent = v != 0;
        if (serve_trace())
            std::fprintf(stderr, "[serve %.6f] stop=%d (%s) running=%d\n", now_seconds(), v, cudaGetErrorString(e),
                         (int)running);
    }

    bool allocate(ServeJob& j) {
        size_t off = 0;
        if (arena_ring.place(0, &off, [&](size_t a, size_t b) { return serve_layout(j.b, a, b, j.g); }) < 0)
            return false;
        serve_layout(j.b, off, cap, j.g);
        j.region = arena_ring.push(j.g.off, j.g.end);
        return true;
    }

    bool compatible(const Batch& b) const {
        if (!cfg.valid) return true;
        if (cfg.sup16 && !b.sup16_ok) return false;
        if (cfg.Hz == 0) return true;
        return b.Hz != 0 && b.Hz <= cfg.Hz;
    }

    void merge_config(const Batch& b) {
        if (!cfg.valid) {
            cfg.Hz = b.Hz;
            cfg.sup16 = b.sup16_ok;
            cfg.valid = true;
            return;
        }
        cfg.Hz = (cfg.Hz == 0 || b.Hz == 0) ? 0 : std::max(cfg.Hz, b.Hz);
        cfg.sup16 = cfg.sup16 && b.sup16_ok;
    }

    void complete(ServeJob& j, int status, plp_result* res, const std::string& err) {
        {
            std::lock_guard<std::mutex> lk(h->mu);
            Request* r = j.r;
            r->running = false;
            r->t_done = now_seconds();
            if (status == PLP_OK) {
                r->result = res;
                r->status = r->cancelled ? PLP_E_CANCELLED : PLP_OK;
                if (r->cancelled) r->err = "request was cancelled";
            } else {
                r->status = status;
                r->err = err;
            }
        }
        h->cv.notify_all();
    }

    cudaError_t launch() {
        DecodeLaunch L{};
        L.inst = reinterpret_cast<const InstDesc*>(arena);
        L.step_type = reinterpret_cast<const int*>(arena);
        L.types = reinterpret_cast<const TypeOrs*>(arena);
        L.heads = reinterpret_cast<SlotHead*>(arena);
        L.places = reinterpret_cast<unsigned long long*>(arena);
        L.err_flag = ctl + 3;
        L.abort = ctl + 4;
        L.mt_init = mt_init;
        L.P = cfg.P;
        L.C = cfg.C;
        L.Hz = cfg.Hz;
        L.sup16 = cfg.sup16;
        L.engine = 0;
        L.warps_per_decoder = 1;
        L.decoders_per_cta = cfg.D;
        L.min_blocks = cfg.M;
        int occ = 0;
        cudaError_t e = serve_occupancy(cfg.P, cfg.C, cfg.Hz, cfg.D, cfg.M, cfg.sup16, &occ);
        if (e != cudaSuccess) return e;
        if (occ < 1) return cudaErrorInvalidConfiguration;
        L.ctas = std::max(sms * occ, n_deep / cfg.D + 1);
        // the overflow decoders' tile must hold this launch's top-z index
        args.deep_bytes = decoder_smem_bytes(cfg.deep_P, cfg.deep_C, cfg.Hz, 1, cfg.sup16);
        if (args.deep_bytes > deep_bytes()) return cudaErrorInvalidConfiguration;
        h_word[2] = L.ctas * cfg.D - n_deep;                      // main decoders
        send_stop(0);
        e = cudaMemcpyAsync(ctl + 7, h_word + 2, sizeof(int), cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess) e = cudaEventRecord(ev_go, up);     // the launch follows every upload so far
        if (e == cudaSuccess) e = cudaStreamWaitEvent(kern, ev_go, 0);
        if (e == cudaSuccess) e = launch_serve(L, args, kern);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_word, ctl, sizeof(int), cudaMemcpyDeviceToHost, kern);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_word + 3, ctl + 5, 2 * sizeof(int), cudaMemcpyDeviceToHost, kern);
        if (e == cudaSuccess) e = cudaEventRecord(ev_kern, kern);
        if (e == cudaSuccess) {
            running = true;
            n_launches++;
        }
        if (serve_trace())
            std::fprintf(stderr, "[serve %.6f] launch ctas=%d P=%d C=%d Hz=%d sup16=%d deep=%d tail=%d (%s)\n",
                         now_seconds(), L.ctas, cfg.P, cfg.C, cfg.Hz, cfg.sup16, n_deep, tail, cudaGetErrorString(e));
        return e;
    }

    // unclaimed work after the last launch ended: main items or overflow items
    bool work_left() const {
        const volatile int* w = h_word;
        return w[0] < tail || w[3] < w[4];
    }

    // tables, work items and the new tail of an admitted request, in one
    // stream pass on the upload stream; false when the staging is full
    int publish(ServeJob& j) {
        const InstDesc& d0 = j.b.desc[0];
        const int R = d0.restarts;
        const size_t tab = j.g.heads - j.g.desc;
        j.up_bytes = tab + (size_t)R * sizeof(int2);
        j.heads_bytes = (size_t)R * sizeof(SlotHead);
        j.places_bytes = (size_t)R * d0.place_stride * 8;
        char* img = up_stage.take(j.up_bytes, &j.up_id);
        if (!img) return PLP_E_PENDING;
        std::memset(img, 0, tab);
        InstDesc d = d0;
        d.step_off = (int)(j.g.steps / sizeof(int));
        d.type_off = (int)(j.g.types / sizeof(TypeOrs));
        d.slot_base = (int)(j.g.heads / sizeof(SlotHead));
        d.place_off = (long long)(j.g.places / 8);
        std::memcpy(img, &d, sizeof d);
        ServeTail tl{};
        tl.done_slot = j.slot;
        tl.seq = j.seq;
        std::memcpy(img + sizeof(InstDesc), &tl, sizeof tl);
        std::memcpy(img + (j.g.steps - j.g.desc), j.b.steps.data(), j.b.steps.size() * sizeof(int));
        std::memcpy(img + (j.g.types - j.g.desc), j.b.types.data(), j.b.types.size() * sizeof(TypeOrs));
        int2* items = reinterpret_cast<int2*>(img + tab);
        const int di = (int)(j.g.desc / sizeof(InstDesc));
        for (int k = 0; k < R; k++) items[k] = make_int2(di, k);
        cudaError_t e = cudaMemcpyAsync(arena + j.g.desc, img, tab, cudaMemcpyHostToDevice, up);
        const int pos = tail & (SERVE_RING - 1);
        const int first = std::min(R, SERVE_RING - pos);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ring + pos, items, first * sizeof(int2), cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess && first < R)
            e = cudaMemcpyAsync(ring, items + first, (R - first) * sizeof(int2), cudaMemcpyHostToDevice, up);
        tail += R;
        int* src = h_word + 8 + (tail_copies++ % SERVE_RECORDS);
        *src = tail;
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctl + 1, src, sizeof(int), cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j.ev_up, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(j.ev_up, up);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j.ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return set_cuda_error("serving upload", e);
        (void)cudaStreamQuery(up);     // submit now: the running launch is waiting for the tail
        published += R;
        return PLP_OK;
    }

    // the wave path's code, for a request whose restarts outgrew even the
    // overflow decoders' tile
    void fallback(ServeJob& j) {
        if (running) {                 // the serving launch holds the SMs: let it finish its items
            send_stop(1);
            cudaStreamSynchronize(up);
            cudaEventSynchronize(ev_kern);
            running = false;
        }
        TileConfig tile;
        {
            std::lock_guard<std::mutex> lk(h->mu);
            tile = h->tile;
        }
        Batch b;
        const double t0 = now_seconds();
        int s = b.build({&j.inst}, {j.opts});
        if (s == PLP_OK) s = run_batch(b, down, pin, sms, tile, &h->pool);
        std::vector<plp_result*> res;
        if (s == PLP_OK) res = collect(b, now_seconds() - t0);
        complete(j, s, s == PLP_OK ? res[0] : nullptr, s == PLP_OK ? "" : g_err);
    }

    // the result, in ordinary host memory that it owns (the pinned staging is reused)
    plp_result* result_of(ServeJob& j) {
        const InstDesc& d = j.b.desc[0];
        const size_t n = j.heads_bytes + j.places_bytes;
        char* mem = static_cast<char*>(std::malloc(std::max<size_t>(n, 1)));
        if (!mem) return nullptr;
        std::memcpy(mem, j.down, n);
        auto* r = new plp_result;
        r->restarts = d.restarts;
        r->stride = d.place_stride;
        r->ors = j.b.inst_ors[0];
        r->L = d.L; r->W = d.W; r->H = d.H;
        r->steps = j.b.steps;
        r->block = std::shared_ptr<const char>(mem, [](const char* q) { std::free(const_cast<char*>(q)); });
        r->heads = reinterpret_cast<const SlotHead*>(mem);
        r->seed0 = d.seed;
        r->time_s = now_seconds() - j.t0;
        const int2 best = m_done_best[j.slot];
        r->best = best.x;
        r->best_fallback = best.y;
        r->kept_all = true;
        r->packed = reinterpret_cast<const unsigned long long*>(mem + j.heads_bytes);
        return r;
    }

    void route_to_waves(ServeJob* j) {
        n_waved++;
        {
            std::lock_guard<std::mutex> lk(h->mu);
            h->queue.push_back(j->id);
        }
        h->cv_sched.notify_all();
        drop(j);
    }

    void fail_all(const std::string& why) {
        broken = true;
        for (ServeJob* j : active) {
            complete(*j, PLP_E_CUDA, nullptr, why);
            drop(j);
        }
        active.clear();
        arena_ring.clear();
        for (ServeJob* j : fresh) route_to_waves(j);
        fresh.clear();
    }

    // admission, in arrival order; true when a request moved
    bool admit() {
        bool progress = false;
        while (!fresh.empty()) {
            ServeJob* j = fresh.front();
            bool gone = false;
            {
                // plp_cancel marks a request cancelled before admission itself
                std::lock_guard<std::mutex> lk(h->mu);
                auto it = h->reqs.find(j->id);
                gone = it == h->reqs.end() || it->second->status != PLP_E_PENDING || it->second->cancelled;
            }
            if (gone) {
                fresh.pop_front();
                h->cv.notify_all();
                drop(j);
                progress = true;
                continue;
            }
            if (broken) {
                fresh.pop_front();
                route_to_waves(j);
                progress = true;
                continue;
            }
            if (!j->built) {
                const int s = j->b.build({&j->inst}, {j->opts});
                j->built = true;
                ServeRegion whole;
                if (s != PLP_OK || !serve_layout(j->b, 0, cap, whole) || j->b.desc[0].restarts > SERVE_RING / 4 ||
                    (size_t)j->b.desc[0].restarts * (sizeof(SlotHead) + (size_t)j->b.desc[0].place_stride * 8) >
                        SERVE_DOWN_STAGE / 2 ||
                    whole.heads - whole.desc + (size_t)j->b.desc[0].restarts * sizeof(int2) > SERVE_UP_STAGE / 2) {
                    fresh.pop_front();               // errors and oversized requests: the wave path
                    route_to_waves(j);
                    progress = true;
                    continue;
                }
            }
            if (!compatible(j->b)) {
                if (!active.empty()) break;            // drain first
                if (running) {
                    if (!stop_sent) send_stop(1);
                    break;
                }
                cfg.valid = false;                     // the next launch takes the merged configuration
            }
            if (active.size() >= SERVE_RECORDS / 2 ||
                published - restarts_done + j->b.desc[0].restarts > SERVE_RING / 2 || !allocate(*j))
                break;                                 // wait for requests to finish
            j->t0 = now_seconds();
            {
                std::lock_guard<std::mutex> lk(h->mu);
                auto it = h->reqs.find(j->id);
                if (it == h->reqs.end() || it->second->status != PLP_E_PENDING || it->second->cancelled) {
                    gone = true;
                } else {
                    j->r = it->second.get();
                    j->r->running = true;
                    j->r->t_start = j->t0;
                }
            }
            if (gone) {                                // cancelled meanwhile: give the region back
                fresh.pop_front();
                arena_ring.drop_newest();
                drop(j);
                progress = true;
                continue;
            }
            const int save_tail = tail;
            const long long save_seq = next_seq;
            j->seq = next_seq++;
            j->slot = (int)(j->seq % SERVE_RECORDS);
            const int s = publish(*j);
            if (s == PLP_E_PENDING) {                  // upload staging full: try again later
                next_seq = save_seq;
                tail = save_tail;
                arena_ring.drop_newest();
                std::lock_guard<std::mutex> lk(h->mu);
                j->r->running = false;
                break;
            }
            fresh.pop_front();
            if (s != PLP_OK) {
                arena_ring.drop_newest();
                complete(*j, s, nullptr, g_err);
                drop(j);
                progress = true;
                continue;
            }
            merge_config(j->b);
            j->state = 1;
            active.push_back(j);
            progress = true;
        }
        return progress;
    }

    // one pass of the scheduler; true when something changed
    bool step() {
        bool progress = admit();
        // upload staging comes back once its copies have run
        for (ServeJob* j : active)
            if (j->up_id >= 0 && cudaEventQuery(j->ev_up) == cudaSuccess) {
                up_stage.ring.release(j->up_id);
                j->up_id = -1;
            }
        // the launch: started again whenever published work is unclaimed
        if (running && cudaEventQuery(ev_kern) == cudaSuccess) {
            running = false;
            progress = true;
            if (serve_trace())
                std::fprintf(stderr, "[serve %.6f] launch ended head=%d overflow=%d/%d tail=%d\n", now_seconds(),
                             h_word[0], h_word[3], h_word[4], tail);
        }
        if (!running && !broken && work_left()) {
            const cudaError_t e = launch();
            if (e != cudaSuccess) {
                cudaGetLastError();
                fail_all(std::string("serving launch failed: ") + cudaGetErrorString(e));
                return true;
            }
            progress = true;
        }
        // completions: copy out the results of finished requests
        for (ServeJob* j : active) {
            if (j->state != 1) continue;
            if (__atomic_load_n(&m_done_seq[j->slot], __ATOMIC_ACQUIRE) != j->seq) continue;
            j->down = down_stage.take(j->heads_bytes + j->places_bytes, &j->down_id);
            if (!j->down) break;                       // staging full: later
            cudaError_t e = cudaMemcpyAsync(j->down, arena + j->g.heads, j->heads_bytes,
                                            cudaMemcpyDeviceToHost, down);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(j->down + j->heads_bytes, arena + j->g.places, j->places_bytes,
                                    cudaMemcpyDeviceToHost, down);
            if (e == cudaSuccess) e = cudaEventRecord(j->ev, down);
            if (e != cudaSuccess) {
                cudaGetLastError();
                fail_all("serving result copy failed");
                return true;
            }
            restarts_done += j->b.desc[0].restarts;
            j->state = 2;
            progress = true;
        }
        for (auto it = active.begin(); it != active.end();) {
            ServeJob* j = *it;
            if (j->state != 2 || j->up_id >= 0 || cudaEventQuery(j->ev) != cudaSuccess) {
                ++it;
                continue;
            }
            const SlotHead* hd = reinterpret_cast<const SlotHead*>(j->down);
            bool overflow = false;
            for (int k = 0; k < j->b.desc[0].restarts; k++) overflow = overflow || hd[k].err != ERR_NONE;
            arena_ring.release(j->region);
            if (overflow) {
                down_stage.ring.release(j->down_id);
                n_fallbacks++;
                fallback(*j);
            } else {
                plp_result* res = result_of(*j);
                down_stage.ring.release(j->down_id);
                n_served++;
                if (res) complete(*j, PLP_OK, res, "");
                else complete(*j, PLP_E_CAPACITY, nullptr, "serving: no host memory for a result");
            }
            drop(j);
            it = active.erase(it);
            progress = true;
        }
        // idle: stop the launch; with nothing in flight the counters restart at 0
        const double now = now_seconds();
        if (progress || !active.empty() || !fresh.empty()) last_busy = now;
        const bool idle = active.empty() && fresh.empty();
        if (running && !stop_sent && idle && (now - last_busy > SERVE_IDLE_STOP_S || yield_req.load()))
            send_stop(1);
        if (!running) yield_req = false;
        if (!running && idle && (tail > (1 << 30) || h_word[4] > (1 << 30)) && !work_left()) {
            cudaMemsetAsync(ctl, 0, 2 * sizeof(int), up);        // head, tail
            cudaMemsetAsync(ctl + 5, 0, 2 * sizeof(int), up);    // overflow head, reservations
            cudaStreamSynchronize(up);
            tail = 0;
            h_word[0] = h_word[3] = h_word[4] = 0;
        }
        return progress;
    }

    void loop() {
        cudaSetDevice(device);
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(h->mu);
                if (quit) break;
                if (active.empty() && fresh.empty() && pending.empty() && !running)
                    cv.wait_for(lk, std::chrono::milliseconds(50), [&] { return quit || !pending.empty(); });
                if (quit) break;
                while (!pending.empty()) {
                    fresh.push_back(pending.front());
                    pending.pop_front();
                }
            }
            if (!step()) {
                if (active.empty() && fresh.empty()) std::this_thread::sleep_for(std::chrono::microseconds(200));
                else std::this_thread::yield();
            }
        }
    }
};

// A synchronous call on the handle is about to launch: an idle serving
// launch stops now instead of after SERVE_IDLE_STOP_S, so the SMs free up.
void serve_yield(plp_handle* h) {
    std::lock_guard<std::mutex> g(h->serve_mu);
    if (h->serve) h->serve->yield_req = true;
}

// The handle's serving engine, made on first use. Its arena is half the
// budget, at most PLP_SERVE_ARENA_MB (default 4096 MiB), reserved from the
// budget that the wave path admits by. Null when serving is off (PLP_SERVE=0)
// or could not be set up; eligible requests then take the wave path.
ServeEngine* serve_engine(plp_handle* h) {
    std::lock_guard<std::mutex> g(h->serve_mu);
    if (h->serve || h->serve_off) return h->serve;
    const char* v = std::getenv("PLP_SERVE");
    if (v && std::string(v) == "0") {
        h->serve_off = true;
        return nullptr;
    }
    size_t arena = (size_t)4096 << 20;
    if (const char* a = std::getenv("PLP_SERVE_ARENA_MB")) {
        char* end = nullptr;
        const unsigned long long mb = std::strtoull(a, &end, 10);
        if (end != a && mb > 0) arena = (size_t)mb << 20;
    }
    arena = std::min(arena, h->budget / 2);
    if (arena < ((size_t)1 << 16)) {
        h->serve_off = true;
        return nullptr;
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        if (h->in_use + arena > h->budget) {
            h->serve_off = true;
            return nullptr;
        }
        h->in_use += arena;
    }
    auto* eng = new ServeEngine(h);
    if (eng->init(arena) != PLP_OK) {
        cudaGetLastError();
        delete eng;
        std::lock_guard<std::mutex> lk(h->mu);
        h->in_use -= arena;
        h->serve_off = true;
        return nullptr;
    }
    h->serve = eng;
    return eng;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* plp_last_error(const plp_handle* h) {
    if (h) return h->err.c_str();
    return g_err.c_str();
}

void plp_free(void* p) { free(p); }

void plp_default_opts(plp_run_opts* o) {
    if (!o) return;
    o->seed = 0;
    o->restarts = 1;
    o->passes = 1;
    o->eps = 0.3;
    o->theta = 0.9;
    o->order = 0;
    o->first_fit = 0;
    o->mu = 0.2;
    o->time_limit_s = -1.0;
    o->best_only = 0;
    o->engine = 0;
    o->blk_amax = 3;
    o->blk_bmax = 3;
    o->blk_kmax = 4;
    o->blk_topk = 8;
    o->blk_pick = 0;
}

// ---- instances -----------------------------------------------------------
int plp_instance_parse_multi(const char* text, size_t len, plp_instance*** out, int32_t* n) {
    if (!text || !out || !n) return set_error(PLP_E_INVALID, "plp_instance_parse_multi: null argument");
    try {
        auto v = parse_thpack(std::string(text, len));
        auto** arr = (plp_instance**)malloc(sizeof(plp_instance*) * v.size());
        for (size_t i = 0; i < v.size(); i++) arr[i] = new plp_instance{std::move(v[i])};
        *out = arr;
        *n = (int32_t)v.size();
        return PLP_OK;
    } catch (const FormatError& e) {
        return set_error(PLP_E_FORMAT, e.what());
    }
}

int plp_instance_parse(const char* text, size_t len, plp_instance** out) {
    if (!text || !out) return set_error(PLP_E_INVALID, "plp_instance_parse: null argument");
    try {
        auto v = parse_thpack(std::string(text, len));
        if (v.size() != 1)
            return set_error(PLP_E_FORMAT, "expected exactly 1 instance, got " + std::to_string(v.size()));
        *out = new plp_instance{std::move(v[0])};
        return PLP_OK;
    } catch (const FormatError& e) {
        return set_error(PLP_E_FORMAT, e.what());
    }
}

int plp_instance_load(const char* path, plp_instance** out) {
    if (!path || !out) return set_error(PLP_E_INVALID, "plp_instance_load: null argument");
    try {
        *out = new plp_instance{load_single(path)};
        return PLP_OK;
    } catch (const FormatError& e) {
        return set_error(PLP_E_FORMAT, e.what());
    }
}

int plp_instance_from_types(int32_t L, int32_t W, int32_t H, int32_t n_types, const int32_t* t7,
                            plp_instance** out) {
    if (!out || n_types < 0 || (n_types && !t7))
        return set_error(PLP_E_INVALID, "plp_instance_from_types: bad argument");
    if (L <= 0 || W <= 0 || H <= 0) return set_error(PLP_E_FORMAT, "container dimensions must be positive");
    Instance I;
    I.L = L; I.W = W; I.H = H;
    for (int i = 0; i < n_types; i++) {
        const int32_t* r = t7 + 7 * i;
        if (r[0] <= 0 || r[2] <= 0 || r[4] <= 0)
            return set_error(PLP_E_FORMAT, "item dimensions must be positive");
        if ((r[1] | r[3] | r[5]) & ~1) return set_error(PLP_E_FORMAT, "orientation flags must be 0/1");
        if (r[6] < 0) return set_error(PLP_E_FORMAT, "item qty must be >= 0");
        BoxType b;
        b.l = r[0]; b.lf = r[1]; b.w = r[2]; b.wf = r[3]; b.h = r[4]; b.hf = r[5]; b.qty = r[6];
        I.types.push_back(b);
    }
    *out = new plp_instance{std::move(I)};
    return PLP_OK;
}

void plp_instance_free(plp_instance* inst) { delete inst; }

int plp_instance_info(const plp_instance* in, int32_t* LWH, int32_t* n_types, int32_t* n_items) {
    if (!in) return set_error(PLP_E_INVALID, "plp_instance_info: null instance");
    if (LWH) { LWH[0] = in->inst.L; LWH[1] = in->inst.W; LWH[2] = in->inst.H; }
    if (n_types) *n_types = (int32_t)in->inst.types.size();
    if (n_items) *n_items = in->inst.n_items();
    return PLP_OK;
}

int plp_orientations(const plp_instance* in, int32_t type, int32_t* wdh, int32_t* n) {
    if (!in || !wdh || !n) return set_error(PLP_E_INVALID, "plp_orientations: null argument");
    if (type < 0 || type >= (int)in->inst.types.size())
        return set_error(PLP_E_INVALID, "plp_orientations: type out of range");
    const auto v = orientations(in->inst.types[type]);
    for (size_t i = 0; i < v.size(); i++)
        for (int k = 0; k < 3; k++) wdh[3 * i + k] = v[i][k];
    *n = (int32_t)v.size();
    return PLP_OK;
}

int plp_item_sequence(const plp_instance* in, int32_t order, int32_t* ti, int32_t* copy) {
    if (!in || !ti) return set_error(PLP_E_INVALID, "plp_item_sequence: null argument");
    if (order != 0 && order != 1) return set_error(PLP_E_INVALID, "unknown order");
    const auto seq = item_sequence(in->inst, order);
    std::vector<int> seen(in->inst.types.size(), 0);
    for (size_t i = 0; i < seq.size(); i++) {
        ti[i] = seq[i];
        if (copy) copy[i] = seen[seq[i]]++;
    }
    return PLP_OK;
}

// ---- results --------------------------------------------------------------
int32_t plp_result_restarts(const plp_result* r) { return r ? r->restarts : 0; }

int plp_result_summary(const plp_result* r, int32_t k, plp_summary* out) {
    if (!r || !out) return set_error(PLP_E_INVALID, "plp_result_summary: null argument");
    if (k < 0 || k >= r->restarts) return set_error(PLP_E_INVALID, "restart out of range");
    *out = r->summary(k);
    return PLP_OK;
}

static int expand(const plp_result* r, int k, std::vector<Placement>& v) {
    v.clear();
    if (!r->row_off.empty()) {
        v.assign(r->rows.begin() + r->row_off[k], r->rows.begin() + r->row_off[k + 1]);
        return PLP_OK;
    }
    const int slot = r->packed_slot(k);
    if (slot < 0) return set_error(PLP_E_NOT_FOUND, "placements of this restart were not kept (best_only)");
    const int n = r->heads[k].n_boxes;
    for (int i = 0; i < n; i++) {
        int x, y, z, oi, t;
        unpack_place(r->packed[(size_t)slot * r->stride + i], x, y, z, oi, t);
        const TypeOrs& o = r->ors[t];
        v.push_back({t, x, y, z, o.w[oi], o.d[oi], o.h[oi]});
    }
    return PLP_OK;
}

int plp_result_placements(const plp_result* r, int32_t k, int32_t* rows7, int32_t cap, int32_t* n_out) {
    if (!r || !n_out) return set_error(PLP_E_INVALID, "plp_result_placements: null argument");
    if (k < 0 || k >= r->restarts) return set_error(PLP_E_INVALID, "restart out of range");
    std::vector<Placement> v;
    int s = expand(r, k, v);
    if (s != PLP_OK) return s;
    *n_out = (int32_t)v.size();
    if (!rows7) return PLP_OK;
    if (cap < (int)v.size()) return set_error(PLP_E_INVALID, "plp_result_placements: buffer too small");
    for (size_t i = 0; i < v.size(); i++) {
        int32_t* q = rows7 + 7 * i;
        q[0] = v[i].type; q[1] = v[i].x; q[2] = v[i].y; q[3] = v[i].z;
        q[4] = v[i].w; q[5] = v[i].d; q[6] = v[i].h;
    }
    return PLP_OK;
}

int plp_result_best(const plp_result* r, int32_t* restart, int32_t* fallback) {
    if (!r) return set_error(PLP_E_INVALID, "plp_result_best: null result");
    if (restart) *restart = r->best;
    if (fallback) *fallback = r->best_fallback;
    return PLP_OK;
}

int plp_result_json(const plp_result* r, int32_t k, char* buf, size_t cap, size_t* needed) {
    if (!r) return set_error(PLP_E_INVALID, "plp_result_json: null result");
    if (k < 0 || k >= r->restarts) return set_error(PLP_E_INVALID, "restart out of range");
    std::vector<Placement> v;
    int s = expand(r, k, v);
    if (s != PLP_OK) return s;
    const plp_summary S = r->summary(k);
    RunSummary rs;
    rs.n_boxes = S.n_boxes;
    rs.volume = S.volume;
    rs.score = S.score;
    rs.fallback = S.fallback != 0;
    rs.n_passes = S.n_passes;
    rs.time_s = S.time_s;
    rs.seed = S.seed;
    const std::string js = to_json(rs, v);
    if (needed) *needed = js.size();
    if (buf && cap) {
        const size_t n = std::min(cap - 1, js.size());
        std::memcpy(buf, js.data(), n);
        buf[n] = '\0';
    }
    return PLP_OK;
}

void plp_result_free(plp_result* r) { delete r; }

// ---- plain path -----------------------------------------------------------
int plp_run_plain(const plp_instance* inst, const plp_run_opts* opts, plp_result** out) {
    if (!inst || !opts || !out) return set_error(PLP_E_INVALID, "plp_run_plain: null argument");
    if (opts->restarts < 1 || (opts->time_limit_s < 0 && opts->passes < 1))
        return set_error(PLP_E_INVALID, "restarts and passes must be >= 1");
    if (opts->order != 0 && opts->order != 1) return set_error(PLP_E_INVALID, "order must be 0 or 1");
    std::vector<RunSummary> summ;
    std::vector<std::vector<Placement>> pl;
    int s = run_plain(inst->inst, *opts, summ, pl);
    if (s != PLP_OK) return s;
    auto* r = new plp_result;
    r->restarts = opts->restarts;
    r->row_off.push_back(0);
    r->L = inst->inst.L; r->W = inst->inst.W; r->H = inst->inst.H;
    r->steps = item_sequence(inst->inst, opts->order);
    for (const auto& t : inst->inst.types) {
        TypeOrs to{};
        const auto v = orientations(t);
        to.n = (int)v.size();
        for (int k = 0; k < to.n; k++) { to.w[k] = v[k][0]; to.d[k] = v[k][1]; to.h[k] = v[k][2]; }
        r->ors.push_back(to);
    }
    for (int k = 0; k < opts->restarts; k++) {
        plp_summary ps{};
        ps.n_boxes = summ[k].n_boxes;
        ps.fallback = summ[k].fallback;
        ps.volume = summ[k].volume;
        ps.score = summ[k].score;
        ps.n_passes = summ[k].n_passes;
        ps.seed = summ[k].seed;
        ps.time_s = summ[k].time_s;
        r->summ.push_back(ps);
        r->rows.insert(r->rows.end(), pl[k].begin(), pl[k].end());
        r->row_off.push_back((long long)r->rows.size());
    }
    // best restart: accepted first, max (volume, n), earliest on ties
    for (int k = 0; k < r->restarts; k++) {
        const plp_summary& a = r->summ[k];
        if (r->best < 0) { r->best = k; continue; }
        const plp_summary& b = r->summ[r->best];
        const int aa = !a.fallback, ba = !b.fallback;
        if (aa != ba ? aa > ba : (a.volume != b.volume ? a.volume > b.volume : a.n_boxes > b.n_boxes))
            r->best = k;
    }
    r->best_fallback = r->best >= 0 ? r->summ[r->best].fallback : 1;
    *out = r;
    return PLP_OK;
}

// ---- handle ---------------------------------------------------------------
int plp_create(size_t budget_bytes, int32_t device, plp_handle** out) {
    if (!out) return set_error(PLP_E_INVALID, "plp_create: null argument");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return set_cuda_error("cudaGetDeviceCount", e);
    if (device < 0 || device >= n) return set_error(PLP_E_INVALID, "plp_create: no such device");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return set_cuda_error("cudaSetDevice", e);
    auto* h = new plp_handle;
    h->device = device;
    h->budget = budget_bytes ? budget_bytes : (size_t)100 << 30;
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
    // keep freed batch memory cached in the stream-ordered pool
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = h->budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    e = cudaStreamCreateWithFlags(&h->sync_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete h; return set_cuda_error("stream creation", e); }
    int status = PLP_OK;
    if (!device_mt_init(&status)) { cudaStreamDestroy(h->sync_stream); delete h; return status; }
    h->streams.resize(h->n_workers);
    for (int i = 0; i < h->n_workers; i++) {
        e = cudaStreamCreateWithFlags(&h->streams[i], cudaStreamNonBlocking);
        if (e != cudaSuccess) return set_cuda_error("stream creation", e);
    }
    for (int i = 0; i < h->n_workers; i++) h->workers.emplace_back(worker_main, h, i);
    {
        std::unique_lock<std::mutex> lk(h->mu);
        h->cv.wait_for(lk, std::chrono::seconds(10), [&] { return h->workers_ready == h->n_workers; });
    }
    *out = h;
    return PLP_OK;
}

void plp_destroy(plp_handle* h) {
    if (!h) return;
    // The serving launch goes first: a worker frees its pinned buffers as it
    // exits, and a pinned free waits for every kernel on the device, the
    // serving launch included, which would run on to its idle bound.
    {
        std::lock_guard<std::mutex> g(h->serve_mu);
        delete h->serve;          // stops its launch and thread
        h->serve = nullptr;
        h->serve_off = true;
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->stop = true;
    }
    h->cv_sched.notify_all();
    for (auto& t : h->workers) t.join();
    for (auto& kv : h->reqs) delete kv.second->result;
    for (auto s : h->streams) cudaStreamDestroy(s);
    if (h->sync_stream) cudaStreamDestroy(h->sync_stream);
    delete h;
}

int plp_serve_counters(plp_handle* h, int64_t* launches, int64_t* served, int64_t* fallbacks,
                       int64_t* waved) {
    if (!h) return set_error(PLP_E_INVALID, "plp_serve_counters: null handle");
    std::lock_guard<std::mutex> g(h->serve_mu);
    const ServeEngine* e = h->serve;
    if (launches) *launches = e ? e->n_launches.load() : 0;
    if (served) *served = e ? e->n_served.load() : 0;
    if (fallbacks) *fallbacks = e ? e->n_fallbacks.load() : 0;
    if (waved) *waved = e ? e->n_waved.load() : 0;
    return PLP_OK;
}

int plp_debug_sync_bound(plp_handle* h, int32_t wait_limit, int32_t skip_warp) {
    if (!h) return set_error(PLP_E_INVALID, "plp_debug_sync_bound: null handle");
    if (wait_limit < 0 || skip_warp < -1 || skip_warp >= 8)
        return set_error(PLP_E_INVALID, "plp_debug_sync_bound: out of range");
    std::lock_guard<std::mutex> g(h->sync_mu);
    std::lock_guard<std::mutex> lk(h->mu);
    h->tile.sync_limit = wait_limit;
    h->tile.sync_skip = skip_warp + 1;
    return PLP_OK;
}

int plp_set_tile(plp_handle* h, int32_t P, int32_t C, int32_t G, int32_t D, int32_t M) {
    if (!h) return set_error(PLP_E_INVALID, "plp_set_tile: null handle");
    if (P < 0 || C < 0 || G < 0 || D < 0 || M < 0 || P > P_MAX || C > C_MAX || (C && C % 32)) {
        int s = set_error(PLP_E_INVALID, "plp_set_tile: out of range");
        record(h, s);
        return s;
    }
    std::lock_guard<std::mutex> g(h->sync_mu);
    std::lock_guard<std::mutex> lk(h->mu);
    TileConfig t = h->tile;
    if (P) t.P = P;
    if (C) t.C = C;
    if (G) t.G = G;
    if (D) t.D = D;
    if (M) t.M = M;
    if (!decoder_config_supported(t.G, t.D, t.M)) {
        int s = set_error(PLP_E_INVALID,
                          "plp_set_tile: unsupported (warps per decoder, decoders per CTA, min CTAs per SM)");
        record(h, s);
        return s;
    }
    if (decoder_smem_bytes(t.P, t.C, 0, t.G) * t.D > 227 * 1024) {   // a batch's z index may lower D
        int s = set_error(PLP_E_CAPACITY, "plp_set_tile: tile exceeds shared memory");
        record(h, s);
        return s;
    }
    h->tile = t;
    return PLP_OK;
}

int plp_autotune(plp_handle* h, const plp_instance* const* insts, int32_t n_inst, const plp_run_opts* opts,
                 int32_t n_opts, int32_t max_decodes, int32_t* tile_out) {
    if (!h || !insts || !opts || n_inst < 1 || (n_opts != 1 && n_opts != n_inst) || max_decodes < 0) {
        int s = set_error(PLP_E_INVALID, "plp_autotune: bad argument");
        record(h, s);
        return s;
    }
    serve_yield(h);
    std::vector<const Instance*> in;
    std::vector<plp_run_opts> op;
    for (int i = 0; i < n_inst; i++) {
        if (!insts[i]) {
            int s = set_error(PLP_E_INVALID, "plp_autotune: null instance");
            record(h, s);
            return s;
        }
        in.push_back(&insts[i]->inst);
        op.push_back(opts[n_opts == 1 ? 0 : i]);
    }
    std::lock_guard<std::mutex> g(h->sync_mu);
    cudaSetDevice(h->device);
    Batch full;
    int s = full.build(in, op);
    if (s != PLP_OK) {
        record(h, s);
        return s;
    }
    // strided sample of the longest-first work list keeps its mix of lengths
    const size_t n = full.work.size();
    const size_t m = std::min(n, (size_t)(max_decodes ? max_decodes : 32768));
    std::vector<int2> sample(m);
    for (size_t k = 0; k < m; k++) sample[k] = full.work[k * n / m];
    // candidate tiles: one warp per decoder; depths around the instance sizes
    int max_steps = 1;
    for (const auto& d : full.desc) max_steps = std::max(max_steps, d.n_steps);
    std::vector<int> Ps, Cs;
    for (int p : {64, 128, 256})
        if (p <= P_MAX && (p >= std::min(max_steps, 64) || p == 128)) Ps.push_back(p);
    for (int c : {256, 384, 512, 768}) Cs.push_back(c);
    const int dm[][2] = {{1, 1}, {1, 12}, {1, 16}, {2, 1}, {4, 1}, {8, 1}, {8, 2}};
    std::vector<TileConfig> cand;
    for (int p : Ps)
        for (int c : Cs)
            for (const auto& x : dm) {
                TileConfig t;
                t.P = p; t.C = c; t.G = 1; t.D = x[0]; t.M = x[1];
                fit_tile(t, full);
                if (tile_smem(full, t) * t.D > 227 * 1024) continue;
                bool dup = false;
                for (const auto& u : cand) dup = dup || same_tile(u, t);
                if (!dup) cand.push_back(t);
            }
    double best_ms = 1e30;
    TileConfig best;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        best = h->tile;
    }
    // The estimate for the whole workload scales the sample's first decoder
    // launch by n / m. What follows it (the retry stage, selection) is mostly
    // the latency of the longest re-run restart, the same for the whole
    // workload as for the sample, so it is added once, or once per wave of the
    // retry tile that the scaled re-run count fills.
    const double scale = (double)n / (double)std::max<size_t>(m, 1);
    for (const TileConfig& t0 : cand) {
        Batch b;
        s = b.build(in, op);
        if (s != PLP_OK) break;
        b.work = sample;
        b.stage_slots = n;   // the retry stage as the whole workload would run it
        TileConfig t = t0;
        s = batch_prepare(b, h->sync_stream, h->sync_pin, h->sms, t, true);
        if (s != PLP_OK) break;
        double ms = 1e30;
        for (int rep = 0; rep < 3 && s == PLP_OK; rep++) {
            ExecStats x;
            TileConfig u = t0;
            s = batch_execute(b, h->sync_stream, h->sms, u, &x, false);
            if (s == PLP_OK && rep > 0) {
                const double waves = x.redo_wave > 0 ? std::max(1.0, x.redo * scale / (double)x.redo_wave) : 1.0;
                ms = std::min(ms, x.decoder_ms * scale + (x.device_ms - x.decoder_ms) * waves);
            }
        }
        if (s != PLP_OK) break;   // batch_execute released the batch
        batch_release(b, h->sync_stream);
        if (ms < best_ms) {
            best_ms = ms;
            best = t0;
        }
    }
    if (s != PLP_OK) {
        record(h, s);
        return s;
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->tile = best;
    }
    if (tile_out) {
        tile_out[0] = best.P; tile_out[1] = best.C; tile_out[2] = best.G; tile_out[3] = best.D; tile_out[4] = best.M;
    }
    return PLP_OK;
}

int plp_solve(plp_handle* h, const plp_instance* const* insts, int32_t n_inst,
              const plp_run_opts* opts, int32_t n_opts, plp_result** results) {
    if (!h || !insts || !opts || !results || n_inst < 1 || (n_opts != 1 && n_opts != n_inst)) {
        int s = set_error(PLP_E_INVALID, "plp_solve: bad argument");
        record(h, s);
        return s;
    }
    serve_yield(h);
    std::lock_guard<std::mutex> g(h->sync_mu);
    cudaSetDevice(h->device);
    std::vector<const Instance*> in;
    std::vector<plp_run_opts> op;
    for (int i = 0; i < n_inst; i++) {
        if (!insts[i]) {
            int s = set_error(PLP_E_INVALID, "plp_solve: null instance");
            record(h, s);
            return s;
        }
        in.push_back(&insts[i]->inst);
        op.push_back(opts[n_opts == 1 ? 0 : i]);
    }
    const double t0 = now_seconds();
    Batch b;
    int s = b.build(in, op);
    TileConfig tile;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        tile = h->tile;
    }
    if (s == PLP_OK) s = run_batch(b, h->sync_stream, h->sync_pin, h->sms, tile, &h->pool);
    if (s == PLP_OK) {
        std::lock_guard<std::mutex> lk(h->mu);
        remember_tile(h->tile, tile);
    }
    if (s != PLP_OK) {
        record(h, s);
        return s;
    }
    auto res = collect(b, now_seconds() - t0);
    for (int i = 0; i < n_inst; i++) results[i] = res[i];
    return PLP_OK;
}

int plp_submit(plp_handle* h, const plp_instance* inst, const plp_run_opts* opts, int64_t* id) {
    if (!h || !inst || !opts || !id) {
        int s = set_error(PLP_E_INVALID, "plp_submit: null argument");
        record(h, s);
        return s;
    }
    if (opts->restarts < 1 || opts->passes < 0 || (opts->time_limit_s < 0 && opts->passes < 1) ||
        (opts->order != 0 && opts->order != 1)) {
        int s = set_error(PLP_E_INVALID, "plp_submit: bad options");
        record(h, s);
        return s;
    }
    auto r = std::make_unique<Request>();
    r->inst = inst->inst;
    r->opts = *opts;
    r->bytes = request_bytes(r->inst, r->opts);
    if (r->bytes > h->budget) {
        int s = set_error(PLP_E_BUDGET, "request needs " + std::to_string(r->bytes) +
                                            " device bytes, more than the handle's budget");
        record(h, s);
        return s;
    }
    r->t_submit = now_seconds();
    ServeEngine* eng = ServeEngine::eligible(*opts) ? serve_engine(h) : nullptr;
    ServeJob* job = nullptr;
    if (eng) {
        job = new ServeJob;
        job->inst = inst->inst;
        job->opts = *opts;
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        r->id = h->next_id++;
        *id = r->id;
        if (job) {
            job->id = r->id;
            eng->pending.push_back(job);
        } else {
            h->queue.push_back(r->id);
        }
        h->reqs[r->id] = std::move(r);
    }
    if (job) eng->cv.notify_one();
    else h->cv_sched.notify_one();
    return PLP_OK;
}

int plp_poll(plp_handle* h, int64_t id) {
    if (!h) return set_error(PLP_E_INVALID, "plp_poll: null handle");
    std::lock_guard<std::mutex> lk(h->mu);
    auto it = h->reqs.find(id);
    if (it == h->reqs.end()) {
        int s = set_error(PLP_E_NOT_FOUND, "unknown request id");
        h->err = g_err;
        return s;
    }
    if (it->second->status != PLP_OK && it->second->status != PLP_E_PENDING) {
        g_err = it->second->err;
        h->err = g_err;
    }
    return it->second->status;
}

int plp_wait(plp_handle* h, int64_t id, int64_t timeout_ms) {
    if (!h) return set_error(PLP_E_INVALID, "plp_wait: null handle");
    std::unique_lock<std::mutex> lk(h->mu);
    auto it = h->reqs.find(id);
    if (it == h->reqs.end()) {
        int s = set_error(PLP_E_NOT_FOUND, "unknown request id");
        h->err = g_err;
        return s;
    }
    Request* r = it->second.get();
    auto done = [&] { return r->status != PLP_E_PENDING; };
    if (timeout_ms < 0) h->cv.wait(lk, done);
    else if (!h->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
        int s = set_error(PLP_E_TIMEOUT, "request still running");
        h->err = g_err;
        return s;
    }
    if (r->status != PLP_OK) {
        g_err = r->err.empty() ? "request failed" : r->err;
        h->err = g_err;
    }
    return r->status;
}

int plp_take_result(plp_handle* h, int64_t id, plp_result** out) {
    if (!h || !out) return set_error(PLP_E_INVALID, "plp_take_result: null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    auto it = h->reqs.find(id);
    if (it == h->reqs.end()) return set_error(PLP_E_NOT_FOUND, "unknown request id");
    Request* r = it->second.get();
    if (r->status == PLP_E_PENDING) return set_error(PLP_E_PENDING, "request not finished");
    const int s = r->status;
    if (s != PLP_OK) {
        g_err = r->err.empty() ? "request failed" : r->err;
        h->reqs.erase(it);
        return s;
    }
    *out = r->result;
    r->result = nullptr;
    h->reqs.erase(it);
    return PLP_OK;
}

int plp_cancel(plp_handle* h, int64_t id) {
    if (!h) return set_error(PLP_E_INVALID, "plp_cancel: null handle");
    {
        std::lock_guard<std::mutex> lk(h->mu);
        auto it = h->reqs.find(id);
        if (it == h->reqs.end()) return set_error(PLP_E_NOT_FOUND, "unknown request id");
        Request* r = it->second.get();
        if (r->status != PLP_E_PENDING) return PLP_OK;   // already finished
        r->cancelled = true;
        if (!r->running) {
            r->status = PLP_E_CANCELLED;
            r->err = "request was cancelled";
            r->t_done = now_seconds();
        }
    }
    h->cv.notify_all();
    h->cv_sched.notify_all();
    return PLP_OK;
}

int plp_request_times(plp_handle* h, int64_t id, double* queued_s, double* total_s) {
    if (!h) return set_error(PLP_E_INVALID, "plp_request_times: null handle");
    std::lock_guard<std::mutex> lk(h->mu);
    auto it = h->reqs.find(id);
    if (it == h->reqs.end()) return set_error(PLP_E_NOT_FOUND, "unknown request id");
    const Request* r = it->second.get();
    if (queued_s) *queued_s = r->t_start > 0 ? r->t_start - r->t_submit : -1.0;
    if (total_s) *total_s = r->t_done > 0 ? r->t_done - r->t_submit : -1.0;
    return PLP_OK;
}

// ---- prepared batches ------------------------------------------------------
}  // extern "C"

struct plp_batch {
    plp_handle* h = nullptr;
    Batch b;
    bool executed = false;
};

extern "C" {

int plp_batch_prepare(plp_handle* h, const plp_instance* const* insts, int32_t n_inst,
                      const plp_run_opts* opts, int32_t n_opts, plp_batch** out) {
    if (!h || !insts || !opts || !out || n_inst < 1 || (n_opts != 1 && n_opts != n_inst)) {
        int s = set_error(PLP_E_INVALID, "plp_batch_prepare: bad argument");
        record(h, s);
        return s;
    }
    std::lock_guard<std::mutex> g(h->sync_mu);
    cudaSetDevice(h->device);
    auto pb = std::make_unique<plp_batch>();
    pb->h = h;
    std::vector<const Instance*> in;
    std::vector<plp_run_opts> op;
    for (int i = 0; i < n_inst; i++) {
        if (!insts[i]) {
            int s = set_error(PLP_E_INVALID, "plp_batch_prepare: null instance");
            record(h, s);
            return s;
        }
        in.push_back(&insts[i]->inst);
        op.push_back(opts[n_opts == 1 ? 0 : i]);
    }
    int s = pb->b.build(in, op);
    TileConfig tile;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        tile = h->tile;
    }
    if (s == PLP_OK) s = batch_prepare(pb->b, h->sync_stream, h->sync_pin, h->sms, tile, false);
    if (s != PLP_OK) {
        record(h, s);
        return s;
    }
    *out = pb.release();
    return PLP_OK;
}

int plp_batch_run(plp_batch* pb, double* device_ms, double* decoder_ms, int32_t* launches) {
    if (!pb) return set_error(PLP_E_INVALID, "plp_batch_run: null batch");
    plp_handle* h = pb->h;
    serve_yield(h);
    std::lock_guard<std::mutex> g(h->sync_mu);
    cudaSetDevice(h->device);
    TileConfig tile;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        tile = h->tile;
    }
    ExecStats x;
    int s = batch_execute(pb->b, h->sync_stream, h->sms, tile, &x, true);
    if (s != PLP_OK) {
        record(h, s);
        return s;
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        remember_tile(h->tile, tile);
    }
    pb->executed = true;
    if (device_ms) *device_ms = x.device_ms;
    if (decoder_ms) *decoder_ms = x.decoder_ms;
    if (launches) *launches = x.launches;
    return PLP_OK;
}

int plp_batch_fetch(plp_batch* pb, plp_result** results) {
    if (!pb || !results) return set_error(PLP_E_INVALID, "plp_batch_fetch: null argument");
    if (!pb->executed) return set_error(PLP_E_INVALID, "plp_batch_fetch: batch has not run");
    plp_handle* h = pb->h;
    std::lock_guard<std::mutex> g(h->sync_mu);
    cudaSetDevice(h->device);
    const double t0 = now_seconds();
    int s = batch_fetch(pb->b, h->sync_stream, nullptr, &h->pool);
    if (s != PLP_OK) {
        record(h, s);
        return s;
    }
    auto res = collect(pb->b, now_seconds() - t0);
    for (size_t i = 0; i < res.size(); i++) results[i] = res[i];
    return PLP_OK;
}

int plp_batch_io_bytes(const plp_batch* pb, int64_t* h2d, int64_t* d2h) {
    if (!pb) return set_error(PLP_E_INVALID, "plp_batch_io_bytes: null batch");
    if (h2d) *h2d = (int64_t)batch_h2d_bytes(pb->b);
    if (d2h) *d2h = (int64_t)batch_d2h_bytes(pb->b);
    return PLP_OK;
}

int plp_batch_graph(const plp_batch* pb) { return pb && pb->b.gexec ? 1 : 0; }

void plp_batch_free(plp_batch* pb) {
    if (!pb) return;
    {
        std::lock_guard<std::mutex> g(pb->h->sync_mu);
        batch_release(pb->b, pb->h->sync_stream);
    }
    delete pb;
}

// ---- allocation-free decode --------------------------------------------------
int plp_decode_noalloc(const plp_instance* inst, const plp_run_opts* opts, void* d_heads,
                       void* d_places, void* stream) {
    if (!inst || !opts || !d_heads || !d_places)
        return set_error(PLP_E_INVALID, "plp_decode_noalloc: null argument");
    if (opts->restarts < 1 || opts->passes < 1 || (opts->order != 0 && opts->order != 1))
        return set_error(PLP_E_INVALID, "plp_decode_noalloc: bad options");
    if (opts->engine != 0)
        return set_error(PLP_E_INVALID, "plp_decode_noalloc: extreme-point decoder only (engine 0)");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // The tables go in with a copy from ordinary host memory that lives only
    // for this call: a capture would record that address, so capture is refused.
    cudaStreamCaptureStatus cap_status = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(st, &cap_status);
    if (ce != cudaSuccess) return set_cuda_error("plp_decode_noalloc: stream query", ce);
    if (cap_status != cudaStreamCaptureStatusNone)
        return set_error(PLP_E_INVALID, "plp_decode_noalloc: not callable during stream capture");
    Batch b;
    int s = b.build({&inst->inst}, {*opts});
    if (s != PLP_OK) return s;
    // Tile deep enough that no restart can outgrow it: every placement adds
    // at most 7 live points (its 8 corners minus the one it covers), and at
    // most one box is placed per step.
    const int steps = std::max(1, b.desc[0].n_steps);
    TileConfig t;
    t.P = (steps + 15) & ~15;
    t.C = std::min(C_MAX, ((1 + 7 * steps) + 31) & ~31);
    t.G = 1;
    t.M = 1;
    t.D = 8;
    while (t.D > 1 && decoder_smem_bytes(t.P, t.C, b.Hz, t.G) * t.D > 200 * 1024) t.D >>= 1;
    if (t.P > P_MAX || decoder_smem_bytes(t.P, t.C, b.Hz, t.G) * t.D > 227 * 1024 || 1 + 7 * steps > C_MAX)
        return set_error(PLP_E_CAPACITY, "plp_decode_noalloc: instance too large for the shared-memory tile");
    // scratch: the address is set up on the first call on each device
    void* scr = nullptr;
    size_t cap = 0;
    cudaError_t e = noalloc_scratch(&scr, &cap);
    if (e != cudaSuccess) return set_cuda_error("plp_decode_noalloc: scratch address", e);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = decoder_occupancy(t.P, t.C, b.Hz, t.G, t.D, t.M, &occ);
    if (e != cudaSuccess) return set_cuda_error("plp_decode_noalloc: occupancy", e);
    occ = std::max(occ, 1);
    long long ctas = std::max<long long>(1, std::min<long long>((b.n_slots + t.D - 1) / t.D, (long long)sms * occ));
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t o_mt = 0;
    const size_t o_desc = al(o_mt + 624 * 4);
    const size_t o_steps = al(o_desc + sizeof(InstDesc));
    const size_t o_types = al(o_steps + std::max<size_t>(1, b.steps.size()) * sizeof(int));
    const size_t o_work = al(o_types + std::max<size_t>(1, b.types.size()) * sizeof(TypeOrs));
    const size_t o_flags = al(o_work + b.work.size() * sizeof(int2));
    const size_t o_rows = al(o_flags + 16);
    const size_t row_bytes = (size_t)t.D * b.max_stride * 8;   // multi-pass rows of one CTA
    if (o_rows > cap || (b.multi_pass && o_rows + row_bytes > cap))
        return set_error(PLP_E_CAPACITY, "plp_decode_noalloc: tables exceed the 8 MiB fixed scratch "
                                         "(fewer restarts, steps or types per call)");
    if (b.multi_pass) ctas = std::min<long long>(ctas, (long long)((cap - o_rows) / row_bytes));
    // tables staged in host memory and copied in one transfer; the counters
    // and flags that must start at zero are zero in the staged bytes
    std::vector<unsigned char> host(o_rows, 0);
    mt_init_table(reinterpret_cast<uint32_t*>(host.data() + o_mt));
    std::memcpy(host.data() + o_desc, b.desc.data(), sizeof(InstDesc));
    std::memcpy(host.data() + o_steps, b.steps.data(), b.steps.size() * sizeof(int));
    std::memcpy(host.data() + o_types, b.types.data(), b.types.size() * sizeof(TypeOrs));
    std::memcpy(host.data() + o_work, b.work.data(), b.work.size() * sizeof(int2));
    char* d = static_cast<char*>(scr);
    e = cudaMemcpyAsync(d, host.data(), host.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return set_cuda_error("plp_decode_noalloc: table copy", e);
    DecodeLaunch L{};
    L.inst = reinterpret_cast<const InstDesc*>(d + o_desc);
    L.step_type = reinterpret_cast<const int*>(d + o_steps);
    L.types = reinterpret_cast<const TypeOrs*>(d + o_types);
    L.work = reinterpret_cast<const int2*>(d + o_work);
    L.n_work = (int)b.work.size();
    L.work_next = reinterpret_cast<int*>(d + o_flags);
    L.err_flag = reinterpret_cast<int*>(d + o_flags + 8);
    L.abort = reinterpret_cast<int*>(d + o_flags + 12);
    L.heads = static_cast<SlotHead*>(d_heads);
    L.places = static_cast<unsigned long long*>(d_places);
    L.scratch = reinterpret_cast<unsigned long long*>(d + o_rows);
    L.mt_init = reinterpret_cast<const uint32_t*>(d + o_mt);
    L.P = t.P;
    L.C = t.C;
    L.Hz = b.Hz;
    L.warps_per_decoder = t.G;
    L.decoders_per_cta = t.D;
    L.min_blocks = t.M;
    L.ctas = (int)ctas;
    e = launch_decoder(L, st);
    if (e != cudaSuccess) return set_cuda_error("plp_decode_noalloc: decoder launch", e);
    return PLP_OK;
}

// ---- reference work accounting ---------------------------------------------
int plp_result_work(const plp_result* r, int32_t k, int64_t* aabb_tests, int64_t* pairs) {
    if (!r) return set_error(PLP_E_INVALID, "plp_result_work: null result");
    if (k < 0 || k >= r->restarts) return set_error(PLP_E_INVALID, "restart out of range");
    std::vector<Placement> pl;
    int s = expand(r, k, pl);
    if (s != PLP_OK) return s;
    // Replays the reference candidate list (origin + corners of placed boxes,
    // minus points strictly inside one) step by step. The step at which each
    // box was placed is recovered greedily: a step whose type differs from the
    // next placed box was skipped; a skipped step of type t leaves the state
    // unchanged, so the next step of type t would fail too -- hence the next
    // box of type t is always placed at the first step of type t that comes.
    std::vector<std::array<int, 3>> cand{{0, 0, 0}};   // (z, y, x), sorted, unique
    long long T = 0, Pn = 0;
    size_t idx = 0;
    for (int t : r->steps) {
        const TypeOrs& o = r->ors[t];
        if (o.n == 0) continue;
        long long c2 = 0;
        for (const auto& p : cand)
            for (int q = 0; q < o.n; q++)
                c2 += (p[2] + o.w[q] <= r->L && p[1] + o.d[q] <= r->W && p[0] + o.h[q] <= r->H);
        T += 2LL * (long long)idx * c2;
        Pn += (long long)cand.size() * o.n;
        if (idx < pl.size() && pl[idx].type == t) {
            const Placement& b = pl[idx++];
            std::vector<std::array<int, 3>> nc;
            nc.reserve(cand.size() + 8);
            for (const auto& p : cand)
                if (!(b.x < p[2] && p[2] < b.x + b.w && b.y < p[1] && p[1] < b.y + b.d && b.z < p[0] &&
                      p[0] < b.z + b.h))
                    nc.push_back(p);
            for (int c = 0; c < 8; c++)
                nc.push_back({b.z + ((c & 4) ? b.h : 0), b.y + ((c & 2) ? b.d : 0), b.x + ((c & 1) ? b.w : 0)});
            std::sort(nc.begin(), nc.end());
            nc.erase(std::unique(nc.begin(), nc.end()), nc.end());
            cand.swap(nc);
        }
    }
    if (aabb_tests) *aabb_tests = T;
    if (pairs) *pairs = Pn;
    return PLP_OK;
}

// ---- kernel hooks -----------------------------------------------------------
int plp_rng_dump(const int64_t* seeds, int32_t n_seeds, int32_t n_random, int32_t n_bits,
                 int32_t k_bits, double* out_random, uint32_t* out_bits) {
    if (!seeds || n_seeds < 0 || n_random < 0 || n_bits < 0 || k_bits < 1 || k_bits > 32 ||
        (n_random && !out_random) || (n_bits && !out_bits))
        return set_error(PLP_E_INVALID, "plp_rng_dump: bad argument");
    if (n_seeds == 0) return PLP_OK;
    int status = PLP_OK;
    const uint32_t* mt_init = device_mt_init(&status);
    if (!mt_init) return status;
    const size_t sb = (size_t)n_seeds * 8, rb = (size_t)n_seeds * n_random * 8,
                 bb = (size_t)n_seeds * n_bits * 4;
    char* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sb + rb + bb + 64);
    if (e != cudaSuccess) return set_cuda_error("plp_rng_dump: allocation", e);
    e = cudaMemcpy(d, seeds, sb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch_rng_dump(reinterpret_cast<const long long*>(d), n_seeds, n_random, n_bits, k_bits,
                            mt_init, reinterpret_cast<double*>(d + sb),
                            reinterpret_cast<uint32_t*>(d + sb + rb), nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && rb) e = cudaMemcpy(out_random, d + sb, rb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && bb) e = cudaMemcpy(out_bits, d + sb + rb, bb, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_cuda_error("plp_rng_dump", e);
    return PLP_OK;
}

int plp_rng_dump_host(const int64_t* seeds, int32_t n_seeds, int32_t n_random, int32_t n_bits,
                      int32_t k_bits, double* out_random, uint32_t* out_bits) {
    if (!seeds || n_seeds < 0 || n_random < 0 || n_bits < 0 || k_bits < 1 || k_bits > 32 ||
        (n_random && !out_random) || (n_bits && !out_bits))
        return set_error(PLP_E_INVALID, "plp_rng_dump_host: bad argument");
    for (int s = 0; s < n_seeds; s++) {
        const int64_t v = seeds[s];
        PyRng rng((uint64_t)(v < 0 ? -v : v));
        for (int i = 0; i < n_random; i++) out_random[(size_t)s * n_random + i] = rng.random();
        for (int i = 0; i < n_bits; i++) out_bits[(size_t)s * n_bits + i] = rng.getrandbits(k_bits);
    }
    return PLP_OK;
}

int plp_fsr_score(const int32_t* rows7, const int32_t* offsets, int32_t n_pack, double mu,
                  double* out_score, double* out_fsr) {
    if (!offsets || n_pack < 0 || !out_score) return set_error(PLP_E_INVALID, "plp_fsr_score: bad argument");
    if (n_pack == 0) return PLP_OK;
    const int total = offsets[n_pack];
    int cap = 32;
    for (int i = 0; i < n_pack; i++) {
        const int n = offsets[i + 1] - offsets[i];
        if (n < 0) return set_error(PLP_E_INVALID, "plp_fsr_score: offsets must be nondecreasing");
        while (cap < n) cap += 32;
    }
    if (total && !rows7) return set_error(PLP_E_INVALID, "plp_fsr_score: null rows");
    if (fsr_smem_per_warp(cap) * 4 > 227 * 1024)
        return set_error(PLP_E_CAPACITY, "plp_fsr_score: packing larger than the shared-memory tile");
    const size_t rb = (size_t)total * 28, ob = (size_t)(n_pack + 1) * 4, scb = (size_t)n_pack * 8,
                 fb = (size_t)total * 8;
    const size_t o_off = (rb + 255) & ~size_t(255), o_sc = o_off + ((ob + 255) & ~size_t(255)),
                 o_f = o_sc + ((scb + 255) & ~size_t(255));
    char* d = nullptr;
    cudaError_t e = cudaMalloc(&d, o_f + fb + 64);
    if (e != cudaSuccess) return set_cuda_error("plp_fsr_score: allocation", e);
    if (rb) e = cudaMemcpy(d, rows7, rb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_off, offsets, ob, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch_fsr(reinterpret_cast<const int*>(d), reinterpret_cast<const int*>(d + o_off), n_pack,
                       cap, mu, reinterpret_cast<double*>(d + o_sc),
                       out_fsr ? reinterpret_cast<double*>(d + o_f) : nullptr, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out_score, d + o_sc, scb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && out_fsr && fb) e = cudaMemcpy(out_fsr, d + o_f, fb, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_cuda_error("plp_fsr_score", e);
    return PLP_OK;
}

int plp_item_order(const plp_instance* const* insts, int32_t n_inst, int32_t order,
                   int32_t* out_types, int64_t* out_offsets) {
    if (!insts || n_inst < 0 || !out_offsets || (order != 0 && order != 1))
        return set_error(PLP_E_INVALID, "plp_item_order: bad argument");
    std::vector<long long> vols;
    std::vector<int> qty, toff, nt;
    std::vector<long long> soff{0};
    int maxn = 1;
    for (int i = 0; i < n_inst; i++) {
        const Instance& I = insts[i]->inst;
        if (I.types.size() >= 65536) return set_error(PLP_E_CAPACITY, "plp_item_order: too many types");
        toff.push_back((int)vols.size());
        nt.push_back((int)I.types.size());
        for (const auto& t : I.types) {
            if (t.volume() >= 0x7fffffffLL || t.qty >= 65536)
                return set_error(PLP_E_CAPACITY, "plp_item_order: volume or quantity beyond the sort key");
            vols.push_back(t.volume());
            qty.push_back(t.qty);
        }
        soff.push_back(soff.back() + I.n_items());
        maxn = std::max(maxn, I.n_items());
    }
    int cap = 1;
    while (cap < maxn) cap <<= 1;
    if (8 * cap > 227 * 1024) return set_error(PLP_E_CAPACITY, "plp_item_order: instance too large");
    for (int i = 0; i <= n_inst; i++) out_offsets[i] = soff[i];
    if (n_inst == 0 || soff.back() == 0) return PLP_OK;
    if (!out_types) return set_error(PLP_E_INVALID, "plp_item_order: null output");
    const size_t vb = vols.size() * 8 + 8, qb = qty.size() * 4 + 4, tb = (size_t)n_inst * 4,
                 ob = soff.size() * 8, outb = (size_t)soff.back() * 4;
    size_t o = 0;
    auto take = [&](size_t n) { size_t r = o; o += (n + 255) & ~size_t(255); return r; };
    const size_t o_v = take(vb), o_q = take(qb), o_t = take(tb), o_n = take(tb), o_s = take(ob),
                 o_out = take(outb);
    char* d = nullptr;
    cudaError_t e = cudaMalloc(&d, o);
    if (e != cudaSuccess) return set_cuda_error("plp_item_order: allocation", e);
    if (!vols.empty()) e = cudaMemcpy(d + o_v, vols.data(), vols.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !qty.empty()) e = cudaMemcpy(d + o_q, qty.data(), qty.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_t, toff.data(), tb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_n, nt.data(), tb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_s, soff.data(), ob, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch_item_order(reinterpret_cast<const long long*>(d + o_v),
                              reinterpret_cast<const int*>(d + o_q), reinterpret_cast<const int*>(d + o_t),
                              reinterpret_cast<const int*>(d + o_n),
                              reinterpret_cast<const long long*>(d + o_s), n_inst, order,
                              reinterpret_cast<int*>(d + o_out), cap, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out_types, d + o_out, outb, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_cuda_error("plp_item_order", e);
    return PLP_OK;
}

// ---- formatting -------------------------------------------------------------
int plp_py_repr(double x, char* buf, size_t cap) {
    if (!buf || !cap) return set_error(PLP_E_INVALID, "plp_py_repr: null buffer");
    const std::string s = py_repr(x);
    if (s.size() + 1 > cap) return set_error(PLP_E_INVALID, "plp_py_repr: buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return PLP_OK;
}

int plp_selftest(char* buf, size_t cap, size_t* needed) {
    std::string o;
    char line[64];
    for (unsigned s : {0u, 1u, 7u, 123456789u}) {
        PyRng rng(s);
        o += "SEED " + std::to_string(s) + "\n";
        for (int i = 0; i < 16; i++) {
            const double v = rng.random();
            unsigned long long bits;
            std::memcpy(&bits, &v, 8);
            std::snprintf(line, sizeof line, "%016llx\n", bits);
            o += line;
        }
        for (int i = 0; i < 16; i++) o += std::to_string(rng.getrandbits(13)) + "\n";
    }
    const double vals[] = {0.0, 1.0, 0.5, 0.1, 2.0 / 3.0, 0.5785123966942148,
                           0.6132075471698113, 0.6595744680851063, 1e-05, 1e-04,
                           1e15, 1e16, 0.001, 123456789.5, 1.0 / 121.0, 1.0 / 106.0};
    for (double v : vals) o += "REPR " + py_repr(v) + "\n";
    if (needed) *needed = o.size();
    if (buf && cap) {
        const size_t n = std::min(cap - 1, o.size());
        std::memcpy(buf, o.data(), n);
        buf[n] = '\0';
    }
    return PLP_OK;
}

}  // extern "C"

// ---- plain-path scorer -----------------------------------------------------
namespace plpb {

int device_fsr_score(const std::vector<Placement>& p, double mu, double* score) {
    std::vector<int32_t> rows;
    rows.reserve(p.size() * 7);
    for (const auto& q : p) rows.insert(rows.end(), {q.type, q.x, q.y, q.z, q.w, q.d, q.h});
    const int32_t off[2] = {0, (int32_t)p.size()};
    return plp_fsr_score(rows.data(), off, 1, mu, score, nullptr);
}

}  // namespace plpb
