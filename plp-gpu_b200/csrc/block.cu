// block.cu -- the block-building engine (blockproof/plp_block.cpp) as a
// persistent kernel: one warp per restart, every restart of every instance in
// one launch, like the extreme-point decoder.
//
// Reference semantics:
//   catalogue, shape precedence   blockproof/plp_block.cpp:29-47,237-262
//   block pass (plan, placement)  blockproof/plp_block.cpp:95-223
//   contact pick rules            blockproof/plp_block.cpp:55-84,188-200
//   run loop and selection        blockproof/plp_block.cpp:228-304
//   C1/C2/C3, EP update, FSR      gpu/plp_common.hpp (check_feasible_one,
//                                 sort_dedup_pt, compute_fsr)
//
// The catalogue and its orderings are computed on the host per instance (the
// shapes, each type's shapes in precedence order, the first fitting shape for
// every remaining count, the placement rank of every shape). Per sweep a warp
// builds the plan with the reference's RNG draws, sorts the plan's placement
// ranks with a bitonic sort in shared memory, and places the blocks: a
// single-orientation feasibility scan over the live extreme points (lockstep,
// one lane per point), the pick (first feasible point, a uniform random one,
// or the best bottom/side contact) and the extreme-point update. A placed
// block is written out at once as its a x b x k item boxes in the
// reference's decomposition order; the pass is scored by FSR over them.
//
// Exactness: points covered by a placed box (half-open) are infeasible for
// every block and are dropped, which leaves every feasible list -- and so
// every pick, count and RNG draw -- unchanged; C3 is the exact integer form
// 2 s >= w d of the reference's FP64 ratio test (see decoder.cu).
#include "device_common.cuh"
#include "engine.hpp"
#include "feas_eval.cuh"
#include "fsr_warp.cuh"

#include <climits>

namespace plpb {

struct BlockArgs {
    const InstDesc* __restrict__ inst;
    const TypeOrs* __restrict__ types;
    const BlkShape* __restrict__ cat;
    const int* __restrict__ tab;
    const int2* __restrict__ work;
    int n_work;
    const int* n_work_dev;         // set: the work count, written by an earlier launch
    int* work_next;
    int* err_flag;
    int* abort;
    SlotHead* heads;
    unsigned long long* places;
    unsigned long long* scratch;
    const uint32_t* __restrict__ mt_init;
    int P, C, N, T, Hz;   // blocks, live points, items, types (tile), top-z index
};

__host__ __device__ inline int pow2_at_least(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

struct BlkLayout {
    int off_bx, off_bz, off_z2, off_bi, off_key, off_w, off_wi, off_wm, off_rem, off_types, off_plan, off_zt,
        bytes;
    // FSR overlay of the point region at the end of a pass (relative to off_key)
    int f_bx, f_bz, f_z2, f_bi, f_scr;
};

__host__ __device__ inline BlkLayout blk_layout(int P, int C, int N, int T, int Hz) {
    BlkLayout l;
    int o = 624 * 4;                        // MT state
    o = (o + 15) & ~15;
    l.off_bx = o;  o += 16 * P;             // placed blocks sorted by top: {x, y, x2, y2}
    l.off_bz = o;  o += 4 * P;              // bottom z
    l.off_z2 = o;  o += 4 * P;              // top z
    l.off_bi = o;  o += 2 * P;              // placement index
    o = (o + 15) & ~15;
    // live points (keys), items {key, jlo | jsup << 16}, their point index and
    // feasibility; the item tables of the pass's FSR overlay them afterwards
    l.off_key = o;
    l.off_w = o + 4 * C;
    l.off_wi = o + 12 * C;
    l.off_wm = o + 14 * C;
    int pts = 15 * C;
    const int n = N > 0 ? N : 1;
    int f = 0;
    l.f_bx = f;  f += 16 * n;
    l.f_bz = f;  f += 4 * n;
    l.f_z2 = f;  f += 4 * n;
    l.f_bi = f;  f += 2 * n;
    f = (f + 15) & ~15;
    l.f_scr = f;
    int scr = 18 * n + 32;
    if (scr < 4 * pow2_at_least(n)) scr = 4 * pow2_at_least(n);   // item sort keys, used before the FSR
    f += scr;
    o += pts > f ? pts : f;
    o = (o + 15) & ~15;
    l.off_rem = o;    o += 4 * (T > 0 ? T : 1);   // copies left per type
    l.off_types = o;  o += 4 * (T > 0 ? T : 1);   // this sweep's type order
    l.off_plan = o;   o += 4 * pow2_at_least(n);  // plan ranks (bitonic width)
    o = (o + 15) & ~15;
    l.off_zt = o;     o += 2 * Hz;                // u16: boxes with top < z
    o = (o + 15) & ~15;
    l.bytes = o;
    return l;
}

int block_smem_bytes(int P, int C, int N, int T, int Hz) { return blk_layout(P, C, N, T, Hz).bytes; }

// Ascending bitonic sort of a[0, n) in shared memory by one warp; a holds
// room for the next power of two (padded with UINT_MAX).
__device__ __forceinline__ void warp_sort_u32(uint32_t* a, int n, int lane) {
    const int npad = pow2_at_least(n);
    for (int i = n + lane; i < npad; i += 32) a[i] = 0xffffffffu;
    __syncwarp();
    for (int k = 2; k <= npad; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < npad; i += 32) {
                const int l = i ^ j;
                if (l > i) {
                    const uint32_t x = a[i], y = a[l];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        a[i] = y;
                        a[l] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Evaluates items W[w0, w1) for one block (bw, bd, bh), one lane per item, all
// lanes walking the top-sorted boxes in lockstep: the C3 contact sum over the
// boxes whose top is z, then C1 over the boxes above z. Feasibility goes to
// wm[]. With first_only, stops after the first chunk holding a feasible item.
// Returns the first feasible item index in the range, or INT_MAX.
__device__ __forceinline__ int blk_eval(const uint2* W, unsigned char* wm, int w0, int w1, bool first_only,
                                        const int4* bx, const int* bzs, int nb, int bw, int bd, int bh,
                                        uint32_t xmask, uint32_t ymask, int xb, int xyb, int lane) {
    int first = INT_MAX;
    const long long need = (long long)bw * bd;
    for (int cb = w0; cb < w1; cb += 32) {
        const int w = cb + lane;
        const bool has = w < w1;
        const uint2 e = has ? W[w] : make_uint2(0, 0);
        const int jlo = (int)(e.y & 0xffffu), jsup = (int)(e.y >> 16);
        const int x = (int)(e.x & xmask), y = (int)((e.x >> xb) & ymask), z = (int)(e.x >> xyb);
        bool alive = has;
        const bool supz = has && z > 0;
        // C3: contact with the boxes whose top is z (2 s >= w d, exact)
        const int slo = __reduce_min_sync(FULL, supz ? jlo : INT_MAX);
        const int shi = __reduce_max_sync(FULL, supz ? jsup : 0);
        long long s = 0;
        for (int j = slo; j < shi; j++) {
            const int4 b = bx[j];
            if (supz && j >= jlo && j < jsup) {
                const int ox = min(x + bw, b.z) - max(x, b.x);
                const int oy = min(y + bd, b.w) - max(y, b.y);
                if (ox > 0 && oy > 0) s += (long long)ox * oy;
            }
        }
        if (supz && 2 * s < need) alive = false;
        // C1: boxes above z, 4 per round
        const int clo = __reduce_min_sync(FULL, alive ? jsup : INT_MAX);
        for (int j0 = clo; j0 < nb; j0 += 4) {
            int4 bb[4];
            int bz[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const bool in = j0 + u < nb;
                bb[u] = in ? bx[j0 + u] : make_int4(0, 0, 0, 0);
                bz[u] = in ? bzs[j0 + u] : 0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int4 b = bb[u];
                if (alive && j0 + u >= jsup && b.x < x + bw && x < b.z && b.y < y + bd && y < b.w &&
                    bz[u] < z + bh)
                    alive = false;
            }
            if (!__any_sync(FULL, alive)) break;
        }
        if (has) wm[w] = alive ? 1 : 0;
        const unsigned bal = __ballot_sync(FULL, alive);
        if (bal && first == INT_MAX) {
            first = cb + __ffs(bal) - 1;
            if (first_only) break;
        }
    }
    __syncwarp();
    return first;
}

// Bottom support and flush side contact of a block at (x, y, z) against the
// placed boxes (blockproof/plp_block.cpp:68-84), 64-bit areas.
__device__ __forceinline__ void blk_contact(int x0, int y0, int z0, int bw, int bd, int bh, const int4* bx,
                                            const int* bzs, const int* z2s, int nb, long long& bottom,
                                            long long& side) {
    const long long x = x0, y = y0, z = z0;
    long long bo = z == 0 ? (long long)bw * bd : 0, si = 0;
    for (int j = 0; j < nb; j++) {
        const int4 b = bx[j];
        const long long bz = bzs[j], bt = z2s[j];
        const long long ox = min(x + bw, (long long)b.z) - max(x, (long long)b.x);
        const long long oy = min(y + bd, (long long)b.w) - max(y, (long long)b.y);
        const long long oz = min(z + bh, bt) - max(z, bz);
        if (bt == z && ox > 0 && oy > 0) bo += ox * oy;
        if (oy > 0 && oz > 0 && (b.z == x || b.x == x + bw)) si += oy * oz;
        if (ox > 0 && oz > 0 && (b.w == y || b.y == y + bd)) si += ox * oz;
    }
    bottom = bo;
    side = si;
}

// Places a block at live point pc: box tables (top-sorted insert), top-z
// index, points covered by the block dropped, its uncovered corners merged in.
__device__ __forceinline__ int blk_place(int pc, int bw, int bd, int bh, uint32_t* keys, int4* bx, int* bzs,
                                         int* z2s, unsigned short* bis, unsigned short* zt, int Hz, int& nc,
                                         int& nb, int P, int C, uint32_t xmask, uint32_t ymask, int xb, int xyb,
                                         int lane) {
    const uint32_t pkey = keys[pc];
    const int px = (int)(pkey & xmask), py = (int)((pkey >> xb) & ymask), pz = (int)(pkey >> xyb);
    const int px2 = px + bw, py2 = py + bd, pz2 = pz + bh;
    if (nb >= P) return ERR_BOX_CAP;
    // box tables from the top: covered corners, boxes above the new top move up
    unsigned cov = 1u;   // corner 0 = the point itself
    int nabove = 0;
    for (int hi = nb; hi > 0; hi -= 32) {
        const int jj = hi - 1 - lane;
        const bool in = jj >= 0;
        int4 b = make_int4(0, 0, 0, 0);
        int bzb = 0, bzt = 0;
        unsigned short bi = 0;
        if (in) {
            b = bx[jj];
            bzb = bzs[jj];
            bzt = z2s[jj];
            bi = bis[jj];
            const unsigned xin = (b.x <= px && px < b.z ? 1u : 0u) | (b.x <= px2 && px2 < b.z ? 2u : 0u);
            const unsigned yin = (b.y <= py && py < b.w ? 1u : 0u) | (b.y <= py2 && py2 < b.w ? 2u : 0u);
            const unsigned zin = (bzb <= pz && pz < bzt ? 1u : 0u) | (bzb <= pz2 && pz2 < bzt ? 2u : 0u);
#pragma unroll
            for (int c = 0; c < 8; c++)
                if (((xin >> (c & 1)) & (yin >> ((c >> 1) & 1)) & (zin >> (c >> 2))) & 1u) cov |= 1u << c;
        }
        const bool up = in && bzt > pz2;
        nabove += __popc(__ballot_sync(FULL, up));
        __syncwarp();
        if (up) {
            bx[jj + 1] = b;
            bzs[jj + 1] = bzb;
            z2s[jj + 1] = bzt;
            bis[jj + 1] = bi;
        }
    }
    cov = __reduce_or_sync(FULL, cov);
    {
        const int ip = nb - nabove;
        __syncwarp();
        if (lane == 0) {
            bx[ip] = make_int4(px, py, px2, py2);
            bzs[ip] = pz;
            z2s[ip] = pz2;
            bis[ip] = (unsigned short)nb;
        }
    }
    if (zt)
        for (int zz = pz2 + 1 + lane; zz < Hz; zz += 32) zt[zz]++;
    nb++;
    // covered points have keys >= the pick's: survivors of [pc, nc) move down
    int ns = pc;
    for (int cb = pc; cb < nc; cb += 32) {
        const int i = cb + lane;
        bool keep = false;
        uint32_t key = 0;
        if (i < nc) {
            key = keys[i];
            const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask), z = (int)(key >> xyb);
            keep = !(px <= x && x < px2 && py <= y && y < py2 && pz <= z && z < pz2);
        }
        const unsigned bal = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep) keys[ns + __popc(bal & lanemask_lt())] = key;
        ns += __popc(bal);
    }
    __syncwarp();
    // uncovered corners (index order = (z, y, x) order), ranked among the survivors
    uint32_t ck = 0;
    int rank = 0;
    bool isnew = false;
    if (lane < 8 && !((cov >> lane) & 1u)) {
        const int cx = (lane & 1) ? px2 : px, cy = (lane & 2) ? py2 : py, cz = (lane & 4) ? pz2 : pz;
        ck = ((uint32_t)cz << xyb) | ((uint32_t)cy << xb) | (uint32_t)cx;
        int lo = pc, n = ns - pc;
        while (n > 0) {
            const int half = n >> 1;
            if (keys[lo + half] < ck) { lo += half + 1; n -= half + 1; }
            else n = half;
        }
        rank = lo;
        isnew = !(lo < ns && keys[lo] == ck);
    }
    const unsigned newm = __ballot_sync(FULL, isnew);
    const int nnew = ns + __popc(newm);
    if (nnew > C) return ERR_CAND_CAP;
    if (newm) {
        const int first_ins = __reduce_min_sync(FULL, isnew ? rank : INT_MAX);
        uint32_t ckk[8];
#pragma unroll
        for (int c = 0; c < 8; c++) ckk[c] = __shfl_sync(FULL, ck, c);
        for (int hi = ns; hi > first_ins; hi -= 32) {
            const int i = hi - 1 - lane;
            const bool in = i >= first_ins;
            uint32_t key = 0;
            int off = 0;
            if (in) {
                key = keys[i];
#pragma unroll
                for (int c = 0; c < 8; c++) off += ((newm >> c) & 1u) && ckk[c] < key;
            }
            __syncwarp();
            if (in && off) keys[i + off] = key;
            __syncwarp();
        }
        if (isnew) keys[rank + __popc(newm & ((1u << lane) - 1u))] = ck;
    }
    nc = nnew;
    __syncwarp();
    return ERR_NONE;
}

__device__ __forceinline__ void block_body(const BlockArgs& a, unsigned char* base, int gdec) {
    const int lane = threadIdx.x & 31;
    const BlkLayout lay = blk_layout(a.P, a.C, a.N, a.T, a.Hz);
    uint32_t* mt = reinterpret_cast<uint32_t*>(base);
    int4* bx = reinterpret_cast<int4*>(base + lay.off_bx);
    int* bzs = reinterpret_cast<int*>(base + lay.off_bz);
    int* z2s = reinterpret_cast<int*>(base + lay.off_z2);
    unsigned short* bis = reinterpret_cast<unsigned short*>(base + lay.off_bi);
    uint32_t* keys = reinterpret_cast<uint32_t*>(base + lay.off_key);
    uint2* Wl = reinterpret_cast<uint2*>(base + lay.off_w);
    unsigned short* wi = reinterpret_cast<unsigned short*>(base + lay.off_wi);
    unsigned char* wm = base + lay.off_wm;
    int* rem = reinterpret_cast<int*>(base + lay.off_rem);
    int* tys = reinterpret_cast<int*>(base + lay.off_types);
    uint32_t* plan = reinterpret_cast<uint32_t*>(base + lay.off_plan);
    unsigned short* zt = a.Hz ? reinterpret_cast<unsigned short*>(base + lay.off_zt) : nullptr;
    unsigned char* fsr_base = base + lay.off_key;

    const int n_work = a.n_work_dev ? *a.n_work_dev : a.n_work;
    for (;;) {
        if (*reinterpret_cast<volatile int*>(a.abort)) return;
        int item = 0;
        if (lane == 0) item = atomicAdd(a.work_next, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= n_work) break;
        const int2 wk = a.work[item];
        const InstDesc I = a.inst[wk.x];
        const int restart = wk.y;
        const int slot = I.slot_base + restart;
        const int L = I.L, W = I.W, H = I.H;
        const uint32_t xmask = (1u << I.xb) - 1u, ymask = (1u << I.yb) - 1u;
        const int xb = I.xb, xyb = I.xb + I.yb;
        const bool randomized = I.eps > 0.0;
        const int* tab = a.tab;
        const BlkShape* cat = a.cat + I.cat_off;
        const TypeOrs* tors = a.types + I.type_off;
        unsigned long long* best_out = a.places + I.place_off + (long long)restart * I.place_stride;
        unsigned long long* pass_out =
            I.passes > 1 ? a.scratch + (long long)gdec * I.place_stride : best_out;
        int mpos = 624;
        {
            const long long sd = I.seed + restart;
            mt_seed_warp(mt, (unsigned long long)(sd < 0 ? -sd : sd), a.mt_init, lane);
        }
        const long long t0 = global_ns();
        int npass = 0;
        int err = ERR_NONE;
        bool have_acc = false, have_any = false;
        long long best_vol = 0;
        int best_n = 0;
        double best_score = 0.0;

        for (int pass = 0; pass < I.passes && err == ERR_NONE; pass++) {
            int nb = 0, nc = 1, n_items = 0;
            long long vol = 0;
            if (zt)
                for (int i = lane; i < a.Hz; i += 32) zt[i] = 0;
            for (int t = lane; t < I.n_types; t += 32) rem[t] = tab[I.bo_qty + t];
            if (lane == 0) keys[0] = 0u;
            __syncwarp();
            for (;;) {   // sweeps: plan, then placement (blockproof/plp_block.cpp:129-207)
                // types with copies left, by (volume desc, index)
                int nty = 0;
                for (int q0 = 0; q0 < I.n_types; q0 += 32) {
                    const int q = q0 + lane;
                    const int t = q < I.n_types ? tab[I.bo_order + q] : 0;
                    const bool ok = q < I.n_types && rem[t] > 0 && tors[t].n > 0;
                    const unsigned bal = __ballot_sync(FULL, ok);
                    if (ok) tys[nty + __popc(bal & lanemask_lt())] = t;
                    nty += __popc(bal);
                }
                __syncwarp();
                if (nty == 0) break;
                if (randomized && mt_random(mt, mpos, lane) >= 1.0 - I.eps) {   // shuffle the type order
                    for (int i = nty - 1; i > 0; i--) {
                        const int j = mt_randrange(mt, mpos, lane, i + 1);
                        if (j < 0) { err = ERR_RNG; break; }
                        if (lane == 0) {
                            const int tmp = tys[i];
                            tys[i] = tys[j];
                            tys[j] = tmp;
                        }
                        __syncwarp();
                    }
                    if (err != ERR_NONE) break;
                }
                // plan: per type, the largest fitting shapes (eps: one of the top-k)
                int nplan = 0;
                for (int q = 0; q < nty && err == ERR_NONE; q++) {
                    const int t = tys[q];
                    int r = rem[t];
                    const int l0 = tab[I.bo_list_off + t], ns = tab[I.bo_list_off + t + 1] - l0;
                    const int s0 = tab[I.bo_start_off + t], nst = tab[I.bo_start_off + t + 1] - s0;
                    while (r > 0 && ns > 0) {
                        // first shape with cnt <= r (the table covers r below the largest count)
                        const int start = r > nst ? 0 : tab[I.bo_start + s0 + r - 1];
                        if (start >= ns) break;
                        const int tk = min(I.blk_topk, ns - start);
                        int pick = 0;
                        if (randomized && mt_random(mt, mpos, lane) >= 1.0 - I.eps) {
                            pick = mt_randrange(mt, mpos, lane, tk);
                            if (pick < 0) { err = ERR_RNG; break; }
                        }
                        const BlkShape S = cat[tab[I.bo_list + l0 + start + pick]];
                        if (lane == 0) plan[nplan] = (uint32_t)S.rank;
                        nplan++;
                        r -= S.cnt;
                    }
                }
                if (err != ERR_NONE || nplan == 0) break;
                __syncwarp();
                warp_sort_u32(plan, nplan, lane);   // placement order
                bool any = false;
                for (int e = 0; e < nplan && err == ERR_NONE; e++) {
                    const BlkShape S = cat[tab[I.bo_shape_of_rank + (int)plan[e]]];
                    if (rem[S.ti] < S.cnt) continue;   // planned before, stale
                    // points with the block inside the container and, above the
                    // floor, a box top at their height
                    int nW = 0;
                    for (int cb = 0; cb < nc; cb += 32) {
                        const int i = cb + lane;
                        bool ok = false;
                        uint2 it = make_uint2(0, 0);
                        if (i < nc) {
                            const uint32_t key = keys[i];
                            const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask), z = (int)(key >> xyb);
                            if (x + S.bw <= L && y + S.bd <= W && z + S.bh <= H) {
                                const int jlo = box_start(zt, z2s, nb, z);
                                const int jsup = z > 0 ? box_start(zt, z2s, nb, z + 1) : jlo;
                                ok = z == 0 || jsup > jlo;
                                it = make_uint2(key, (unsigned)jlo | ((unsigned)jsup << 16));
                            }
                        }
                        const unsigned bal = __ballot_sync(FULL, ok);
                        if (ok) {
                            const int d = nW + __popc(bal & lanemask_lt());
                            Wl[d] = it;
                            wi[d] = (unsigned short)i;
                        }
                        nW += __popc(bal);
                    }
                    __syncwarp();
                    const int first = blk_eval(Wl, wm, 0, nW, true, bx, bzs, nb, S.bw, S.bd, S.bh, xmask, ymask,
                                               xb, xyb, lane);
                    if (first == INT_MAX) continue;   // this block stays out (for now): no draw
                    int pw = first;
                    const bool full = randomized && mt_random(mt, mpos, lane) >= 1.0 - I.eps;
                    if (full || I.blk_pick != 0) {
                        const int end = (first & ~31) + 32;   // chunks up to first's are evaluated
                        if (end < nW)
                            blk_eval(Wl, wm, end, nW, false, bx, bzs, nb, S.bw, S.bd, S.bh, xmask, ymask, xb, xyb,
                                     lane);
                    }
                    if (full) {
                        int count = 0;
                        for (int w = first + lane; w < nW; w += 32) count += wm[w];
                        count = __reduce_add_sync(FULL, count);
                        const int idx = mt_randrange(mt, mpos, lane, count);
                        if (idx < 0) { err = ERR_RNG; break; }
                        int run = 0;
                        for (int cb = first; cb < nW; cb += 32) {
                            const int w = cb + lane;
                            const bool f = w < nW && wm[w];
                            const unsigned bal = __ballot_sync(FULL, f);
                            const int c = __popc(bal);
                            if (idx < run + c) {
                                pw = cb + __fns(bal, 0, idx - run + 1);
                                break;
                            }
                            run += c;
                        }
                    } else if (I.blk_pick != 0) {
                        // best (primary, secondary) contact; the earliest point on ties
                        long long k0 = -1, k1 = -1;
                        int bi = INT_MAX;
                        for (int cb = first; cb < nW; cb += 32) {
                            const int w = cb + lane;
                            if (w < nW && wm[w]) {
                                const uint32_t key = Wl[w].x;
                                long long sup, side;
                                blk_contact((int)(key & xmask), (int)((key >> xb) & ymask), (int)(key >> xyb), S.bw,
                                            S.bd, S.bh, bx, bzs, z2s, nb, sup, side);
                                const long long p0 = I.blk_pick == 1 ? sup : sup + side;
                                const long long p1 = I.blk_pick == 1 ? side : sup;
                                if (p0 > k0 || (p0 == k0 && p1 > k1)) { k0 = p0; k1 = p1; bi = w; }
                            }
                        }
#pragma unroll
                        for (int d = 16; d > 0; d >>= 1) {
                            const long long o0 = __shfl_xor_sync(FULL, k0, d);
                            const long long o1 = __shfl_xor_sync(FULL, k1, d);
                            const int ob = __shfl_xor_sync(FULL, bi, d);
                            if (o0 > k0 || (o0 == k0 && (o1 > k1 || (o1 == k1 && ob < bi)))) {
                                k0 = o0; k1 = o1; bi = ob;
                            }
                        }
                        pw = bi;
                    }
                    const int pc = wi[pw];
                    const uint32_t pkey = keys[pc];
                    const int px = (int)(pkey & xmask), py = (int)((pkey >> xb) & ymask), pz = (int)(pkey >> xyb);
                    if (n_items + S.cnt > I.place_stride) { err = ERR_BOX_CAP; break; }
                    // the block's item boxes, in the reference's (a, b, k) order
                    const int iw = S.bw / S.a, id = S.bd / S.b, ih = S.bh / S.k;
                    for (int q = lane; q < S.cnt; q += 32) {
                        const int i = q / (S.b * S.k), j = (q / S.k) % S.b, t = q % S.k;
                        pass_out[n_items + q] = pack_place(px + i * iw, py + j * id, pz + t * ih, S.oi, S.ti);
                    }
                    n_items += S.cnt;
                    vol += (long long)S.cnt * iw * id * ih;
                    err = blk_place(pc, S.bw, S.bd, S.bh, keys, bx, bzs, z2s, bis, zt, a.Hz, nc, nb, a.P, a.C, xmask,
                                    ymask, xb, xyb, lane);
                    if (lane == 0) rem[S.ti] -= S.cnt;
                    __syncwarp();
                    any = true;
                }
                if (err != ERR_NONE || !any) break;
            }
            if (err != ERR_NONE) break;
            // FSR over the item boxes: top-sorted tables rebuilt from the pass's items
            {
                int4* fbx = reinterpret_cast<int4*>(fsr_base + lay.f_bx);
                int* fbz = reinterpret_cast<int*>(fsr_base + lay.f_bz);
                int* fz2 = reinterpret_cast<int*>(fsr_base + lay.f_z2);
                unsigned short* fbi = reinterpret_cast<unsigned short*>(fsr_base + lay.f_bi);
                uint32_t* sk = reinterpret_cast<uint32_t*>(fsr_base + lay.f_scr);
                __syncwarp();
                for (int q = lane; q < n_items; q += 32) {
                    int x, y, z, oi, ty;
                    unpack_place(pass_out[q], x, y, z, oi, ty);
                    sk[q] = ((uint32_t)(z + tors[ty].h[oi]) << 16) | (uint32_t)q;
                }
                warp_sort_u32(sk, n_items, lane);
                for (int p = lane; p < n_items; p += 32) {
                    const int q = (int)(sk[p] & 0xffffu);
                    int x, y, z, oi, ty;
                    unpack_place(pass_out[q], x, y, z, oi, ty);
                    fbx[p] = make_int4(x, y, x + tors[ty].w[oi], y + tors[ty].d[oi]);
                    fbz[p] = z;
                    fz2[p] = z + tors[ty].h[oi];
                    fbi[p] = (unsigned short)q;
                }
                __syncwarp();
                const double score = fsr_score_warp(fbx, fbz, fz2, fbi, n_items, I.mu,
                                                    reinterpret_cast<char*>(fsr_base + lay.f_scr), lane, nullptr);
                const bool acc = !I.has_theta || score >= I.theta;
                bool take;
                if (acc) take = !have_acc || vol > best_vol || (vol == best_vol && n_items > best_n);
                else take = !have_acc && (!have_any || vol > best_vol || (vol == best_vol && n_items > best_n));
                if (take) {
                    best_vol = vol;
                    best_n = n_items;
                    best_score = score;
                    if (pass_out != best_out)
                        for (int i = lane; i < n_items; i += 32) best_out[i] = pass_out[i];
                }
                have_any = true;
                have_acc = have_acc || acc;
                npass = pass + 1;
                __syncwarp();
            }
            if (I.budget_ns >= 0 && __shfl_sync(FULL, global_ns() - t0, 0) >= I.budget_ns) break;
        }
        if (lane == 0) {
            if (err) atomicOr(a.err_flag, 1 << err);
            SlotHead h;
            h.n_boxes = err ? 0 : best_n;
            h.err = err;
            h.volume = err ? 0 : best_vol;
            h.score = err ? 0.0 : best_score;
            h.n_passes = npass;
            h.fallback = have_acc ? 0 : 1;
            a.heads[slot] = h;
        }
        __syncwarp();
    }
}

template <int D, int M>
__global__ void __launch_bounds__(32 * D, M) block_kernel(BlockArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dec = threadIdx.x >> 5;
    const BlkLayout lay = blk_layout(a.P, a.C, a.N, a.T, a.Hz);
    block_body(a, smem_raw + (size_t)dec * lay.bytes, blockIdx.x * D + dec);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
#define PLP_BLOCK_CONFIGS(X) X(1, 1) X(2, 1) X(4, 1) X(8, 1)

using BlockFn = void (*)(BlockArgs);

static BlockFn block_fn(int D, int M) {
#define PLP_PICK(d, m) \
    if (D == d && M == m) return block_kernel<d, m>;
    PLP_BLOCK_CONFIGS(PLP_PICK)
#undef PLP_PICK
    return nullptr;
}

bool block_config_supported(int D, int M) { return block_fn(D, M) != nullptr; }

static int block_launch_smem(const DecodeLaunch& L) {
    return block_smem_bytes(L.P, L.C, L.N, L.T, L.Hz) * L.decoders_per_cta;
}

cudaError_t block_occupancy(int P, int C, int N, int T, int Hz, int D, int M, int* ctas_per_sm) {
    BlockFn fn = block_fn(D, M);
    if (!fn) return cudaErrorInvalidConfiguration;
    const int smem = block_smem_bytes(P, C, N, T, Hz) * D;
    return cached_occupancy(reinterpret_cast<const void*>(fn), 32 * D, smem, ctas_per_sm);
}

cudaError_t configure_block(const DecodeLaunch& L) {
    BlockFn fn = block_fn(L.decoders_per_cta, L.min_blocks);
    if (!fn) return cudaErrorInvalidConfiguration;
    return ensure_dyn_smem(reinterpret_cast<const void*>(fn), block_launch_smem(L));
}

cudaError_t enqueue_block(const DecodeLaunch& L, cudaStream_t st) {
    BlockFn fn = block_fn(L.decoders_per_cta, L.min_blocks);
    if (!fn) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaMemsetAsync(L.work_next, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(L.abort, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    BlockArgs a;
    a.inst = L.inst;
    a.types = L.types;
    a.cat = L.bcat;
    a.tab = L.btab;
    a.work = L.work;
    a.n_work = L.n_work;
    a.n_work_dev = L.n_work_dev;
    a.work_next = L.work_next;
    a.err_flag = L.err_flag;
    a.abort = L.abort;
    a.heads = L.heads;
    a.places = L.places;
    a.scratch = L.scratch;
    a.mt_init = L.mt_init;
    a.P = L.P;
    a.C = L.C;
    a.N = L.N;
    a.T = L.T;
    a.Hz = L.Hz;
    fn<<<L.ctas, 32 * L.decoders_per_cta, block_launch_smem(L), st>>>(a);
    return cudaGetLastError();
}

}  // namespace plpb
