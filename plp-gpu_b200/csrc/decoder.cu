// decoder.cu -- the persistent multi-restart extreme-point decoder (one warp
// per restart), device FSR, per-instance best-of selection, and the device
// MT19937 / FSR / item-order hooks.
//
// Reference semantics (pqant/plp-gpu):
//   decode pass        plp/solver.py:180-240, gpu/plp_common.hpp:404-456
//   feasibility        plp/solver.py:196-218, gpu/plp_common.hpp:297-321
//   pick + RNG draws   gpu/plp_common.hpp:426-435 (no draw when no pair is
//                      feasible; random() only when eps > 0 and not first-fit;
//                      randrange(len(feas)) only on the random branch)
//   FSR / score        plp/solver.py:109-148, gpu/plp_common.hpp:356-399
//   selection          plp/solver.py:156-166, gpu/plp_common.hpp:493-511
//   rows               gpu/plp_gpu.cu:350 (restart k = PyRng(seed + k))
//
// Two persistent decoders share the work list and result layout:
//   decoder1_kernel<D, M>    one warp per restart, incremental per-point
//                            evaluation (the default; see its section)
//   decoder_kernel<G, D, M>  G warps per restart, lockstep scan of the
//                            filtered points every step (multi-warp variant)
//
// Layout of one decoder in shared memory (both kernels):
//   MT19937 state       624 x u32
//   placed boxes        sorted by top z (ascending): {x, y, x2, y2} int4,
//                       bottom z, top z, placement index
//   live points         sorted unique keys (z, y, x) (+ per-point state and
//                       contact areas in decoder1_kernel)
//   item list           the points to evaluate this step
// FSR reuses the point buffers as scratch once the pass is done.
//
// Exactness notes (why the device results equal the reference's):
//  * A point covered by a placed box in the half-open sense
//    (b.x <= x < b.x2, same for y and z) is infeasible for every orientation
//    and stays infeasible (boxes are never removed). The reference keeps such
//    points in its candidate list; they never produce a feasible pair, so the
//    ordered list of feasible pairs -- the only thing the pick reads -- is the
//    same when they are dropped. The live list is exactly the reference's
//    candidate set minus covered points, in the same (z, y, x) order.
//  * C1/C2/C3 are evaluated per point for all orientations at once. C2 is the
//    same integer test; C3 sums the same integer overlap areas (the ratio
//    test is the reference's FP64 form in decoder_kernel and its exact
//    integer equivalent in decoder1_kernel); C1 only visits boxes whose top
//    lies above z (a box with top <= z cannot overlap a box starting at z),
//    which does not change the boolean.
//  * The first feasible pair (greedy branch) is found by scanning points in
//    order; random() is drawn only after one feasible pair exists, and the
//    full count / idx-th selection runs only on the random branch.
#include "device_common.cuh"
#include "engine.hpp"
#include "feas_eval.cuh"
#include "fsr_warp.cuh"

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

namespace plpb {

// ---------------------------------------------------------------------------
// shared-memory layout of one decoder
// ---------------------------------------------------------------------------
// Scalars one decoder's warps exchange through shared memory.
struct DecShared {
    unsigned long long bar;   // mbarrier of the decoder's warps (G > 1)
    int item;      // current work item
    int nW;        // items in the filtered point list
    int wnext;     // multi-warp decoder: warp 0's end-of-pass-loop decision
    int best_w;    // smallest feasible item found so far
    int full;      // random branch: every feasible pair is needed
    int err;
    int nc;        // live points
    int nb;        // placed boxes
    int pad[6];
};
static_assert(sizeof(DecShared) == 64, "DecShared layout");

struct DecLayout {
    int off_bx, off_bz, off_z2, off_bi, off_ca, off_cb, off_cm, off_zt, off_sh, bytes;
    __host__ __device__ int off_cc(int C) const { return off_cm + C; }   // chunk counts (int)
};

// P: placed-box depth, C: live-point depth, Hz: entries of the top-z index
// (container height + 2; 0 = use binary search instead)
__host__ __device__ inline DecLayout dec_layout(int P, int C, int Hz) {
    DecLayout l;
    int o = 624 * 4;                       // MT state
    o = (o + 15) & ~15;
    l.off_bx = o;  o += 16 * P;            // int4 {x, y, x2, y2}
    l.off_bz = o;  o += 4 * P;             // bottom z
    l.off_z2 = o;  o += 4 * P;             // top z
    l.off_bi = o;  o += 2 * P;             // placement index
    o = (o + 15) & ~15;
    l.off_ca = o;
    // live points (4C), item list / survivor scratch (8C), item masks (C),
    // per-chunk item counts (C / 8); FSR overlays 18 bytes per box
    int region = 13 * C + C / 8 + 16;
    if (region < 18 * P + 32) region = 18 * P + 32;
    l.off_cb = o + 4 * C;
    l.off_cm = o + 12 * C;
    o += region;
    o = (o + 15) & ~15;
    l.off_zt = o;  o += 2 * Hz;            // u16: boxes with top < z
    o = (o + 15) & ~15;
    l.off_sh = o;  o += (int)sizeof(DecShared);
    l.bytes = o;
    return l;
}

// Layout of one single-warp (incremental) decoder: as above, but every live
// point also carries its evaluation state and six contact areas.
struct Dec1Layout {
    int off_bx, off_bz, off_z2, off_bi, off_key, off_st, off_sup, off_w, off_wi, off_zt, off_sh, bytes;
};

// sb: bytes per stored contact area (4, or 2 when every orientation's
// footprint area is below 65536; an area never exceeds its footprint, since
// boxes sharing a top cannot overlap below it)
__host__ __device__ inline Dec1Layout dec1_layout(int P, int C, int Hz, int sb) {
    Dec1Layout l;
    int o = 624 * 4;                       // MT state
    o = (o + 15) & ~15;
    l.off_bx = o;  o += 16 * P;            // int4 {x, y, x2, y2}
    l.off_bz = o;  o += 4 * P;             // bottom z
    l.off_z2 = o;  o += 4 * P;             // top z
    l.off_bi = o;  o += 2 * P;             // placement index
    o = (o + 15) & ~15;
    // live points: key, state, 6 contact areas; FSR overlays 18 bytes per box
    l.off_key = o;
    l.off_st = o + 4 * C;
    l.off_sup = o + 8 * C;
    int region = (8 + 6 * sb) * C;
    if (region < 18 * P + 32) region = 18 * P + 32;
    o += region;
    o = (o + 15) & ~15;
    l.off_w = o;   o += 8 * C;             // items to evaluate {key, m2 | jlo << 8 | jsup << 20}
    l.off_wi = o;  o += 2 * C;             // their point index
    o = (o + 15) & ~15;
    l.off_zt = o;  o += 2 * Hz;            // u16: boxes with top < z
    o = (o + 15) & ~15;
    l.off_sh = o;  o += (int)sizeof(DecShared);
    l.bytes = o;
    return l;
}

#ifndef PLP_SERVE_TU
int decoder_smem_bytes(int P, int C, int Hz, int G, int sup16) {
    return G == 1 ? dec1_layout(P, C, Hz, sup16 ? 2 : 4).bytes : dec_layout(P, C, Hz).bytes;
}
#endif

struct DecoderArgs {
    const InstDesc* __restrict__ inst;
    const int* __restrict__ step_type;
    const TypeOrs* __restrict__ types;
    const int2* __restrict__ work;
    int n_work;
    const int* n_work_dev;         // set: the work count, written by an earlier launch
    int* work_next;
    int* err_flag;
    int* abort;
    SlotHead* heads;
    unsigned long long* places;
    unsigned long long* scratch;   // per resident warp: passes > 1
    const uint32_t* __restrict__ mt_init;
    int P, C, Hz;
    int sync_limit;                // tries per barrier wait (0 = SYNC_WAIT_LIMIT)
    int sync_skip;                 // test hook: 1 + the warp that skips its first arrive
    const uint32_t* seed_tab;      // seeded MT states of seeds seed_lo .. seed_lo + seed_n - 1 (or null)
    long long seed_lo;
    int seed_n;
};


// ---------------------------------------------------------------------------
// the persistent decoder kernel: D decoders per CTA, G warps per decoder
// ---------------------------------------------------------------------------
// Barrier of one decoder's G warps: an mbarrier in shared memory that
// completes a phase when each warp has arrived once. Every wait is bounded:
// if it gives up, or another warp of the launch already gave up, the
// launch-wide abort flag is set and the caller unwinds, so a broken
// synchronisation ends the launch with ERR_SYNC instead of hanging the GPU.
constexpr int SYNC_WAIT_LIMIT = 1 << 18;   // tries of up to ~10 us each: bounded near 3 s

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}

// The waiting thread may be suspended until the phase completes or about
// 10 us pass (suspend-time hint), so waiting warps do not spin on issue slots.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(10000u)
        : "memory");
    return ok != 0;
}

template <int G>
struct GroupSync {
    unsigned long long* bar;
    int* abort;
    unsigned phase;
    int limit;          // tries before a wait gives up
    bool skip_arrive;   // test hook: this warp's next arrive is left out
    // returns false when the launch is aborting (the caller must return)
    __device__ __forceinline__ bool operator()(int lane) {
        __syncwarp();
        if (G == 1) return true;
        if (lane == 0 && !skip_arrive) mbar_arrive(bar);
        skip_arrive = false;
        bool ok = true;
        for (int k = 0; !mbar_try_wait(bar, phase); k++) {
            if (k >= limit || ((k & 63) == 63 && *reinterpret_cast<volatile int*>(abort))) {
                ok = false;
                break;
            }
        }
        phase ^= 1u;
        ok = __all_sync(FULL, ok);
        if (!ok && lane == 0) atomicExch(abort, 1);
        return ok;
    }
};


// Per-step orientation data (identical in every warp of a decoder).
struct StepOrs {
    int no;
    int ow[6], od[6], oh[6], wd[6];
    int wmax, dmax, hmax;   // largest edge along x, y, z over the orientations
};

// One decoder's G warps evaluate the filtered points W[start .. nW): warp g
// takes points start + g, start + g + G, ...; inside a warp each lane tests
// one placed box, so a point's boxes are checked 32 at a time with coalesced
// loads and the per-box results are combined with warp reductions.
//   C3 (z > 0): integer contact areas of the boxes whose top is z, summed
//               with __reduce_add_sync; lane o then applies the FP64 ratio
//               test of orientation o.
//   C1:         boxes whose top is above z; an orientation is blocked when a
//               box overlaps it; blocked sets are OR-reduced per 32 boxes and
//               the scan stops once every orientation is blocked.
// Greedy mode stops at the smallest feasible item (sh->best_w); the mask of
// every evaluated item goes to wmask.
// Item of the filtered point list: x = point key, y = orientation mask
// (bits 0-5) | first box with top >= z (bits 8-19) | first box with top > z
// (bits 20-31). Box indices refer to the top-sorted tables of this step.
__device__ __forceinline__ uint2 make_item(uint32_t key, unsigned m, int jlo, int jsup) {
    return make_uint2(key, m | ((unsigned)jlo << 8) | ((unsigned)jsup << 20));
}

// One decoder's G warps evaluate the filtered points W[start .. nW) in
// chunks of 32 (chunk k by warp k % G), one lane per point. All lanes walk the
// top-sorted boxes in lockstep, so every box is one shared-memory broadcast:
//   support loop: boxes whose top is the height of some lane's point; each
//                 lane adds the integer contact areas of the boxes with top ==
//                 its z, then applies the FP64 ratio test (C3);
//   C1 loop:      boxes above, from the lowest start of the chunk, until every
//                 lane's orientations are blocked.
// Greedy mode stops at the first chunk with a feasible point and records the
// smallest feasible item in sh->best_w; every evaluated item's mask goes to
// wmask.
template <int G, bool GREEDY>
__device__ __forceinline__ void scan_points(DecShared* sh, const uint2* W, unsigned char* wmask,
                                            const int4* bx, const int* bzs, int nb, const StepOrs& S,
                                            uint32_t xmask, uint32_t ymask, int xb, int xyb, int g,
                                            int lane, int start) {
    const int nW = sh->nW;
    for (int cb = start + 32 * g; cb < nW; cb += 32 * G) {
        if (GREEDY && G > 1 && cb > *reinterpret_cast<volatile int*>(&sh->best_w)) break;
        const int w = cb + lane;
        const uint2 e = w < nW ? W[w] : make_uint2(0, 0);
        unsigned alive = e.y & 0x3fu;
        const int jlo = (int)((e.y >> 8) & 0xfffu), jsup = (int)(e.y >> 20);
        const int x = (int)(e.x & xmask), y = (int)((e.x >> xb) & ymask), z = (int)(e.x >> xyb);
        const bool sup = alive && jsup > jlo;                            // z > 0
        const int slo = __reduce_min_sync(FULL, sup ? jlo : INT_MAX);
        const int shi = __reduce_max_sync(FULL, sup ? jsup : 0);
        if (slo < shi) {                                                 // C3 support
            int a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0;
            for (int j0 = slo; j0 < shi; j0 += 4) {
                int4 bb[4];
#pragma unroll
                for (int u = 0; u < 4; u++) bb[u] = j0 + u < shi ? bx[j0 + u] : make_int4(0, 0, 0, 0);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int j = j0 + u;
                    const int4 b = bb[u];
                    if (sup && j >= jlo && j < jsup) {
#define PLP_ACC(o, av)                                                   \
    {                                                                    \
        const int ox = min(x + S.ow[o], b.z) - max(x, b.x);              \
        const int oy = min(y + S.od[o], b.w) - max(y, b.y);              \
        if (ox > 0 && oy > 0) av += ox * oy;                             \
    }
                        PLP_ACC(0, a0) PLP_ACC(1, a1) PLP_ACC(2, a2) PLP_ACC(3, a3) PLP_ACC(4, a4) PLP_ACC(5, a5)
#undef PLP_ACC
                    }
                }
            }
            if (sup) {
                // (double)s / (double)(w*d) < 0.5 fails the orientation
                const int av[6] = {a0, a1, a2, a3, a4, a5};
#pragma unroll
                for (int o = 0; o < 6; o++)
                    if (((alive >> o) & 1u) && (double)av[o] / (double)S.wd[o] < 0.5) alive &= ~(1u << o);
            }
        }
        const int clo = __reduce_min_sync(FULL, alive ? jsup : INT_MAX);
        // C1 overlap, 4 boxes per round: loads first, then a cheap "near"
        // test per box (ahead of the point and within the largest edge on each
        // axis); only boxes near some lane get the per-orientation test. Boxes
        // past nb read as {0,0,0,0}, which is never near (x >= 0).
        for (int j0 = clo; j0 < nb; j0 += 4) {
            int4 bb[4];
            int bz[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const bool in = j0 + u < nb;
                bb[u] = in ? bx[j0 + u] : make_int4(0, 0, 0, 0);
                bz[u] = in ? bzs[j0 + u] : 0;
            }
            unsigned near = 0;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int4 b = bb[u];
                const bool nu = alive && j0 + u >= jsup && x < b.z && y < b.w && b.x < x + S.wmax &&
                                b.y < y + S.dmax && bz[u] < z + S.hmax;
                near |= (nu ? 1u : 0u) << u;
            }
            const unsigned todo = __reduce_or_sync(FULL, near);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if ((todo >> u) & 1u) {                 // uniform: some lane is near box u
                    if ((near >> u) & 1u) {
                        // offsets from the point (coordinates are below 2^16)
                        const int dx = bb[u].x - x, dy = bb[u].y - y, dz = bz[u] - z;
#pragma unroll
                        for (int o = 0; o < 6; o++)
                            if (dx < S.ow[o] && dy < S.od[o] && dz < S.oh[o]) alive &= ~(1u << o);
                    }
                }
            }
            if (!__any_sync(FULL, alive != 0)) break;
        }
        if (w < nW) wmask[w] = (unsigned char)alive;
        if (GREEDY) {
            const unsigned bal = __ballot_sync(FULL, alive != 0);
            if (bal) {
                if (lane == 0) atomicMin(&sh->best_w, cb + __ffs(bal) - 1);
                break;
            }
        }
    }
}

// Filtered item of one live point (C2 mask, and above the floor at least one
// box top at its height), or m = 0.
__device__ __forceinline__ uint2 filter_point(uint32_t key, const StepOrs& S, int L, int W, int H,
                                              uint32_t xmask, uint32_t ymask, int xb, int xyb,
                                              const unsigned short* zt, const int* z2s, int nb) {
    const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask), z = (int)(key >> xyb);
    unsigned m = 0;
#pragma unroll
    for (int o = 0; o < 6; o++)
        if (o < S.no && x + S.ow[o] <= L && y + S.od[o] <= W && z + S.oh[o] <= H) m |= 1u << o;
    if (!m) return make_uint2(0, 0);
    const int jlo = box_start(zt, z2s, nb, z);
    const int jsup = z > 0 ? box_start(zt, z2s, nb, z + 1) : jlo;
    if (z > 0 && jsup == jlo) return make_uint2(0, 0);   // nothing supports a box at this height
    return make_item(key, m, jlo, jsup);
}

// Warp 0 of a decoder: pick the pair, place the box, update the live points,
// the top-sorted box tables and the top-z index. Returns a DecodeErr.
__device__ __forceinline__ int place_step(DecShared* sh, const StepOrs& S, int t, int best, bool full,
                                          uint32_t* mt, int& mpos, uint32_t* candA, uint32_t* candB,
                                          const uint2* W,
                                          const unsigned char* cmask, int4* bx, int* bzs, int* z2s,
                                          unsigned short* bis, unsigned short* zt, int Hz, int& nc,
                                          int& nb, int P, int C, uint32_t xmask, uint32_t ymask, int xb,
                                          int xyb, unsigned long long* pass_out, long long& vol, int lane) {
    int pick_w = best;
    int pick_oi = __ffs(cmask[best]) - 1;
    if (full) {
        const int nW = sh->nW;
        int count = 0;
        for (int i = best + lane; i < nW; i += 32) count += __popc(cmask[i]);
        count = __reduce_add_sync(FULL, count);
        const int idx = mt_randrange(mt, mpos, lane, count);
        if (idx < 0) return ERR_RNG;
        // idx-th feasible pair in (point, orientation) order
        int run = 0;
        for (int cb = best; cb < nW; cb += 32) {
            const int i = cb + lane;
            const unsigned m = i < nW ? cmask[i] : 0u;
            const int c = __popc(m);
            int inc = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(FULL, inc, d);
                if (lane >= d) inc += v;
            }
            const int tot = __shfl_sync(FULL, inc, 31);
            if (idx < run + tot) {
                const unsigned hit = __ballot_sync(FULL, idx < run + inc);
                const int l = __ffs(hit) - 1;
                const int excl = __shfl_sync(FULL, inc - c, l);
                const unsigned ml = __shfl_sync(FULL, m, l);
                pick_w = cb + l;
                pick_oi = __fns(ml, 0, idx - run - excl + 1);
                break;
            }
            run += tot;
        }
    }
    const uint32_t pkey = W[pick_w].x;
    __syncwarp();   // every lane has read the item list before candB is overwritten
    const int px = (int)(pkey & xmask), py = (int)((pkey >> xb) & ymask), pz = (int)(pkey >> xyb);
    int pw = 0, pd = 0, ph = 0;
#pragma unroll
    for (int o = 0; o < 6; o++)
        if (o == pick_oi) { pw = S.ow[o]; pd = S.od[o]; ph = S.oh[o]; }
    const int px2 = px + pw, py2 = py + pd, pz2 = pz + ph;
    if (nb >= P) return ERR_BOX_CAP;
    if (lane == 0) pass_out[nb] = pack_place(px, py, pz, pick_oi, t);
    vol += 1LL * pw * pd * ph;
    // corners of the new box covered by an already placed box
    unsigned cov = 1u;   // corner 0 = (px, py, pz): covered by the new box
    for (int jj = lane; jj < nb; jj += 32) {
        const int4 b = bx[jj];
        const int bzb = bzs[jj], bzt = z2s[jj];
        const unsigned xin = (b.x <= px && px < b.z ? 1u : 0u) | (b.x <= px2 && px2 < b.z ? 2u : 0u);
        const unsigned yin = (b.y <= py && py < b.w ? 1u : 0u) | (b.y <= py2 && py2 < b.w ? 2u : 0u);
        const unsigned zin = (bzb <= pz && pz < bzt ? 1u : 0u) | (bzb <= pz2 && pz2 < bzt ? 2u : 0u);
#pragma unroll
        for (int c = 0; c < 8; c++)
            if (((xin >> (c & 1)) & (yin >> ((c >> 1) & 1)) & (zin >> (c >> 2))) & 1u) cov |= 1u << c;
    }
    cov = __reduce_or_sync(FULL, cov);
    // survivors (points not covered by the new box), compacted into candB
    // (the item list it held is no longer read: the pick was taken above)
    int ns = 0;
    for (int cb = 0; cb < nc; cb += 32) {
        const int i = cb + lane;
        bool keep = false;
        uint32_t key = 0;
        if (i < nc) {
            key = candA[i];
            const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask), z = (int)(key >> xyb);
            keep = !(px <= x && x < px2 && py <= y && y < py2 && pz <= z && z < pz2);
        }
        const unsigned bal = __ballot_sync(FULL, keep);
        if (keep) candB[ns + __popc(bal & lanemask_lt())] = key;
        ns += __popc(bal);
    }
    __syncwarp();
    // new corners, in index order c = (cz << 2) | (cy << 1) | cx, which is their (z, y, x) order
    uint32_t ck = 0;
    int rank = 0;
    bool isnew = false;
    if (lane < 8 && !((cov >> lane) & 1u)) {
        const int cx = (lane & 1) ? px2 : px, cy = (lane & 2) ? py2 : py, cz = (lane & 4) ? pz2 : pz;
        ck = ((uint32_t)cz << xyb) | ((uint32_t)cy << xb) | (uint32_t)cx;
        int lo = 0, n = ns;
        while (n > 0) {
            const int half = n >> 1;
            if (candB[lo + half] < ck) { lo += half + 1; n -= half + 1; }
            else n = half;
        }
        rank = lo;
        isnew = !(lo < ns && candB[lo] == ck);
    }
    const unsigned newm = __ballot_sync(FULL, isnew);
    const int nnew = ns + __popc(newm);
    if (nnew > C) return ERR_CAND_CAP;
    uint32_t ckk[8];
#pragma unroll
    for (int c = 0; c < 8; c++) ckk[c] = __shfl_sync(FULL, ck, c);
    for (int cb = 0; cb < ns; cb += 32) {
        const int i = cb + lane;
        if (i < ns) {
            const uint32_t key = candB[i];
            int off = 0;
#pragma unroll
            for (int c = 0; c < 8; c++) off += ((newm >> c) & 1u) && ckk[c] < key;
            candA[i + off] = key;
        }
    }
    if (isnew) candA[rank + __popc(newm & ((1u << lane) - 1u))] = ck;
    nc = nnew;
    // insert the box into the top-sorted tables (after equal tops)
    int ip;
    {
        int lo = 0, n = nb;
        while (n > 0) {
            const int half = n >> 1;
            if (z2s[lo + half] <= pz2) { lo += half + 1; n -= half + 1; }
            else n = half;
        }
        ip = lo;
    }
    for (int hi = nb; hi > ip; hi -= 32) {
        const int i = hi - 1 - lane;
        int4 vb = make_int4(0, 0, 0, 0);
        int vz = 0, vt = 0;
        unsigned short vi = 0;
        const bool mv = i >= ip;
        if (mv) { vb = bx[i]; vz = bzs[i]; vt = z2s[i]; vi = bis[i]; }
        __syncwarp();
        if (mv) { bx[i + 1] = vb; bzs[i + 1] = vz; z2s[i + 1] = vt; bis[i + 1] = vi; }
        __syncwarp();
    }
    if (lane == 0) {
        bx[ip] = make_int4(px, py, px2, py2);
        bzs[ip] = pz;
        z2s[ip] = pz2;
        bis[ip] = (unsigned short)nb;
    }
    if (zt)
        for (int zz = pz2 + 1 + lane; zz < Hz; zz += 32) zt[zz]++;
    nb++;
    __syncwarp();
    return ERR_NONE;
}

template <int G>
__device__ __forceinline__ void decoder_body(const DecoderArgs& a, unsigned char* base, int dec,
                                             int gdec) {
    const int lane = threadIdx.x & 31;
    const int g = (threadIdx.x >> 5) % G;
    const DecLayout lay = dec_layout(a.P, a.C, a.Hz);
    uint32_t* mt = reinterpret_cast<uint32_t*>(base);
    int4* bx = reinterpret_cast<int4*>(base + lay.off_bx);
    int* bzs = reinterpret_cast<int*>(base + lay.off_bz);
    int* z2s = reinterpret_cast<int*>(base + lay.off_z2);
    unsigned short* bis = reinterpret_cast<unsigned short*>(base + lay.off_bi);
    uint32_t* candA = reinterpret_cast<uint32_t*>(base + lay.off_ca);
    uint32_t* candB = reinterpret_cast<uint32_t*>(base + lay.off_cb);   // survivor scratch
    uint2* Wl = reinterpret_cast<uint2*>(base + lay.off_cb);             // item list (same space)
    unsigned char* cmask = base + lay.off_cm;                             // item masks
    int* ccount = reinterpret_cast<int*>(base + lay.off_cc(a.C));         // per-chunk item counts
    unsigned short* zt = a.Hz ? reinterpret_cast<unsigned short*>(base + lay.off_zt) : nullptr;
    DecShared* sh = reinterpret_cast<DecShared*>(base + lay.off_sh);
    GroupSync<G> sync{&sh->bar, a.abort, 0u, a.sync_limit > 0 ? a.sync_limit : SYNC_WAIT_LIMIT,
                      a.sync_skip == g + 1};
#define PLP_SYNC()                        \
    if (!sync(lane)) {                    \
        if (lane == 0) atomicOr(a.err_flag, 1 << ERR_SYNC); \
        return;                           \
    }

    const int n_work = a.n_work_dev ? *a.n_work_dev : a.n_work;
    for (;;) {
        if (*reinterpret_cast<volatile int*>(a.abort)) return;
        if (g == 0 && lane == 0) sh->item = atomicAdd(a.work_next, 1);
        PLP_SYNC()
        const int item = sh->item;
        PLP_SYNC()   // everyone has the item before it can change
        if (item >= n_work) break;
        const int2 wk = a.work[item];
        const InstDesc I = a.inst[wk.x];
        const int restart = wk.y;
        const int slot = I.slot_base + restart;
        const int L = I.L, W = I.W, H = I.H;
        const uint32_t xmask = (1u << I.xb) - 1u, ymask = (1u << I.yb) - 1u;
        const int xb = I.xb, xyb = I.xb + I.yb;
        const bool randomized = !(I.first_fit || I.eps == 0.0);
        unsigned long long* best_out = a.places + I.place_off + (long long)restart * I.place_stride;
        unsigned long long* pass_out =
            I.passes > 1 ? a.scratch + (long long)gdec * I.place_stride : best_out;
        int mpos = 624;   // RNG position (warp 0)
        if (g == 0) {
            const long long sd = I.seed + restart;
            mt_seed_warp(mt, (unsigned long long)(sd < 0 ? -sd : sd), a.mt_init, lane);
        }
        const long long t0 = global_ns();   // read by warp 0 only
        int npass = 0;
        int err = ERR_NONE;
        bool have_acc = false, have_any = false;
        long long best_vol = 0;
        int best_n = 0;
        double best_score = 0.0;

        for (int pass = 0; pass < I.passes && err == ERR_NONE; pass++) {
            int nb = 0, nc = 1;   // warp 0's copies are authoritative
            long long vol = 0;
            if (zt)
                for (int i = threadIdx.x % (32 * G); i < a.Hz; i += 32 * G) zt[i] = 0;
            if (g == 0 && lane == 0) {
                candA[0] = 0u;
                sh->err = ERR_NONE;
                sh->nc = 1;
                sh->nb = 0;
            }
            for (int st = 0; st < I.n_steps; st++) {
                const int t = a.step_type[I.step_off + st];
                const TypeOrs& T = a.types[I.type_off + t];
                StepOrs S;
                S.no = T.n;
                if (S.no == 0) continue;
                S.wmax = S.dmax = S.hmax = 0;
#pragma unroll
                for (int o = 0; o < 6; o++) {
                    S.ow[o] = T.w[o];
                    S.od[o] = T.d[o];
                    S.oh[o] = T.h[o];
                    S.wd[o] = S.ow[o] * S.od[o];
                    S.wmax = max(S.wmax, S.ow[o]);
                    S.dmax = max(S.dmax, S.od[o]);
                    S.hmax = max(S.hmax, S.oh[o]);
                }
                PLP_SYNC()                 // A: previous step's tables are final
                if (sh->err != ERR_NONE) break;
                nc = sh->nc;
                nb = sh->nb;
                // filter: points with an orientation inside the container and,
                // above the floor, at least one box top at their height
                if (G == 1) {
                    int nW = 0;
                    for (int cb = 0; cb < nc; cb += 32) {
                        const int ci = cb + lane;
                        const uint2 it = ci < nc ? filter_point(candA[ci], S, L, W, H, xmask, ymask, xb,
                                                                xyb, zt, z2s, nb)
                                                 : make_uint2(0, 0);
                        const bool keep = (it.y & 0x3fu) != 0;
                        const unsigned bal = __ballot_sync(FULL, keep);
                        if (keep) Wl[nW + __popc(bal & lanemask_lt())] = it;
                        nW += __popc(bal);
                    }
                    if (lane == 0) {
                        sh->nW = nW;
                        sh->best_w = INT_MAX;
                    }
                } else {
                    // two passes over chunks of 32 points (chunk c by warp c % G):
                    // count, then write at the chunk's prefix offset
                    const int nch = (nc + 31) >> 5;
                    for (int c = g; c < nch; c += G) {
                        const int ci = c * 32 + lane;
                        const uint2 it = ci < nc ? filter_point(candA[ci], S, L, W, H, xmask, ymask, xb,
                                                                xyb, zt, z2s, nb)
                                                 : make_uint2(0, 0);
                        const unsigned bal = __ballot_sync(FULL, (it.y & 0x3fu) != 0);
                        if (lane == 0) ccount[c] = __popc(bal);
                    }
                    PLP_SYNC()
                    // pass 2: offset of chunk c = sum of the counts before it (read only)
                    for (int c = g; c < nch; c += G) {
                        int off = 0;
                        for (int k = lane; k < c; k += 32) off += ccount[k];
                        off = __reduce_add_sync(FULL, off);
                        const int ci = c * 32 + lane;
                        const uint2 it = ci < nc ? filter_point(candA[ci], S, L, W, H, xmask, ymask, xb,
                                                                xyb, zt, z2s, nb)
                                                 : make_uint2(0, 0);
                        const bool keep = (it.y & 0x3fu) != 0;
                        const unsigned bal = __ballot_sync(FULL, keep);
                        if (keep) Wl[off + __popc(bal & lanemask_lt())] = it;
                    }
                    int run = 0;
                    if (g == 0) {
                        for (int k = lane; k < nch; k += 32) run += ccount[k];
                        run = __reduce_add_sync(FULL, run);
                    }
                    if (g == 0 && lane == 0) {
                        sh->nW = run;
                        sh->best_w = INT_MAX;
                    }
                }
                PLP_SYNC()                 // B
                if (sh->nW == 0) continue;             // no feasible pair: skip this copy
                scan_points<G, true>(sh, Wl, cmask, bx, bzs, nb, S, xmask, ymask, xb, xyb, g, lane, 0);
                PLP_SYNC()                 // C
                if (g == 0) {                          // random() only once a pair is feasible
                    const int best = sh->best_w;
                    int full = 0;
                    if (best != INT_MAX && randomized) full = mt_random(mt, mpos, lane) >= 1.0 - I.eps;
                    if (lane == 0) sh->full = full;
                }
                PLP_SYNC()                 // D
                const int best = sh->best_w;
                if (best == INT_MAX) continue;
                const bool full = sh->full != 0;
                if (full) {
                    scan_points<G, false>(sh, Wl, cmask, bx, bzs, nb, S, xmask, ymask, xb, xyb, g, lane,
                                          best + 1);
                    PLP_SYNC()             // E
                }
                if (g == 0) {
                    const int e = place_step(sh, S, t, best, full, mt, mpos, candA, candB, Wl, cmask, bx, bzs,
                                             z2s, bis, zt, a.Hz, nc, nb, a.P, a.C, xmask, ymask, xb, xyb,
                                             pass_out, vol, lane);
                    if (lane == 0) {
                        sh->nc = nc;
                        sh->nb = nb;
                        if (e != ERR_NONE) sh->err = e;
                    }
                }
            }
            PLP_SYNC()
            err = sh->err;
            nb = sh->nb;
            if (err != ERR_NONE) break;
            // score the pass and keep the selected one (warp 0)
            if (g == 0) {
                const double score = fsr_score_warp(bx, bzs, z2s, bis, nb, I.mu,
                                                    reinterpret_cast<char*>(candA), lane, nullptr);
                const bool acc = !I.has_theta || score >= I.theta;
                bool take;
                if (acc) take = !have_acc || vol > best_vol || (vol == best_vol && nb > best_n);
                else take = !have_acc && (!have_any || vol > best_vol || (vol == best_vol && nb > best_n));
                if (take) {
                    best_vol = vol;
                    best_n = nb;
                    best_score = score;
                    if (pass_out != best_out)
                        for (int i = lane; i < nb; i += 32) best_out[i] = pass_out[i];
                }
                have_any = true;
                have_acc = have_acc || acc;
                // wall-clock budget (gpu/plp_common.hpp:484-492), decided by warp 0
                const bool stop = I.budget_ns >= 0 && __shfl_sync(FULL, global_ns() - t0, 0) >= I.budget_ns;
                if (lane == 0) sh->wnext = stop ? 1 : 0;
                __syncwarp();
            }
            PLP_SYNC()   // FSR scratch overlays the point buffers
            npass = pass + 1;
            const bool stop = sh->wnext != 0;
            PLP_SYNC()   // every warp has read the decision
            if (stop) break;
        }
        if (g == 0 && lane == 0) {
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
        PLP_SYNC()
    }
}

template <int G, int D, int M>
__global__ void __launch_bounds__(32 * G * D, M) decoder_kernel(DecoderArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dec = (threadIdx.x >> 5) / G;
    const DecLayout lay = dec_layout(a.P, a.C, a.Hz);
    if (G > 1 && threadIdx.x % (32 * G) == 0)
        mbar_init(&reinterpret_cast<DecShared*>(smem_raw + (size_t)dec * lay.bytes + lay.off_sh)->bar, G);
    __syncthreads();
    decoder_body<G>(a, smem_raw + (size_t)dec * lay.bytes, dec, blockIdx.x * D + dec);
}

// ---------------------------------------------------------------------------
// incremental single-warp decoder (G = 1)
// ---------------------------------------------------------------------------
// Every live point carries its evaluation for the current item type:
//   st bits 0-5   C2 mask m2 (orientation inside the container)
//   st bits 8-13  C1 blocked orientations (exact for the bits of `known`)
//   st bits 16-21 C3 support-ok orientations (all six at z = 0)
//   st bits 24-29 known = m2 & support-ok when C1 was evaluated
//   st bit  31    valid
//   sup[o]        integer contact area under orientation o (z > 0)
// Boxes are only ever added during a pass, so a blocked orientation stays
// blocked and a contact area only grows: a valid point stays exact if each
// newly placed box is applied to it once (C1 OR, C3 sum), which the next
// step's filter pass does. Consecutive items of the same type share the
// evaluation; a type change invalidates every point. A point is evaluated
// from scratch (all boxes) only while it is invalid: new corners, points the
// greedy scan has not reached yet, and points whose support grew onto an
// orientation whose C1 was never evaluated.
//
// The C3 test is the integer form of the reference's FP64 ratio:
// (double)s / (double)(w*d) < 0.5  <=>  2 s < w d. Both s and w d are
// integers below 2^52, so both doubles are exact; if s/(wd) < 1/2 then
// s/(wd) <= 1/2 - 1/(2wd) <= 1/2 - 2^-53, a double below 1/2 that bounds the
// rounded quotient from above (rounding is monotone); if s/(wd) >= 1/2 the
// rounded quotient is >= 1/2 as well.
constexpr uint32_t ST_VALID = 1u << 31;

__device__ __forceinline__ uint32_t st_pack(unsigned m2, unsigned blk, unsigned sok, unsigned known) {
    return ST_VALID | m2 | (blk << 8) | (sok << 16) | (known << 24);
}
__device__ __forceinline__ unsigned st_feasible(uint32_t s) {
    return (s & ST_VALID) ? (s & (s >> 16) & ~(s >> 8) & 0x3fu) : 0u;
}

// Evaluates items W[w0 .. w1) from scratch and stores their state. A group
// of 2^lg lanes shares one item (lanes take every 2^lg-th box), 32 >> lg
// items at a time, lg chosen so that a short item list still spreads over the
// whole warp. Greedy mode stops after the first group holding a feasible
// item. Returns {first feasible item or INT_MAX, end of the evaluated range}.
template <typename SupT>
__device__ __forceinline__ int2 eval_items(const bool GREEDY, const uint2* W, const unsigned short* wi, int w0, int w1,
                                           const int4* bx, const int* bzs, int nb, const StepOrs& S,
                                           uint32_t xmask, uint32_t ymask, int xb, int xyb,
                                           uint32_t* st, SupT* sup, int C, int lane) {
    int first = INT_MAX;
    int w = w0;
    while (w < w1) {
        const int K = min(32, w1 - w);
        const int lg = K > 16 ? 0 : K > 8 ? 1 : K > 4 ? 2 : K > 2 ? 3 : K > 1 ? 4 : 5;
        const int span = 1 << lg;
        const int q = lane >> lg, ph = lane & (span - 1);
        const bool has = q < K;
        const uint2 e = has ? W[w + q] : make_uint2(0, 0);
        const unsigned m2 = e.y & 0x3fu;
        const int jlo = (int)((e.y >> 8) & 0xfffu), jsup = (int)(e.y >> 20);
        const int x = (int)(e.x & xmask), y = (int)((e.x >> xb) & ymask), z = (int)(e.x >> xyb);
        const bool supz = has && z > 0;
        int a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0;
        // C3: boxes whose top is z
        const int slo = __reduce_min_sync(FULL, supz ? jlo : INT_MAX);
        const int shi = __reduce_max_sync(FULL, supz ? jsup : 0);
        for (int j0 = slo; j0 < shi; j0 += 4 << lg) {
            int4 bb[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = j0 + (u << lg) + ph;
                bb[u] = j < shi ? bx[j] : make_int4(0, 0, 0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = j0 + (u << lg) + ph;
                const int4 b = bb[u];
                if (supz && j >= jlo && j < jsup) {
#define PLP_ACC(o, av)                                                   \
    {                                                                    \
        const int ox = min(x + S.ow[o], b.z) - max(x, b.x);              \
        const int oy = min(y + S.od[o], b.w) - max(y, b.y);              \
        if (ox > 0 && oy > 0) av += ox * oy;                             \
    }
                    PLP_ACC(0, a0) PLP_ACC(1, a1) PLP_ACC(2, a2) PLP_ACC(3, a3) PLP_ACC(4, a4) PLP_ACC(5, a5)
#undef PLP_ACC
                }
            }
        }
        for (int m = 1; m < span; m <<= 1) {
            a0 += __shfl_xor_sync(FULL, a0, m);
            a1 += __shfl_xor_sync(FULL, a1, m);
            a2 += __shfl_xor_sync(FULL, a2, m);
            a3 += __shfl_xor_sync(FULL, a3, m);
            a4 += __shfl_xor_sync(FULL, a4, m);
            a5 += __shfl_xor_sync(FULL, a5, m);
        }
        unsigned sok = 0x3fu;
        if (z > 0) {
            const int av[6] = {a0, a1, a2, a3, a4, a5};
            sok = 0;
#pragma unroll
            for (int o = 0; o < 6; o++)
                if (2LL * av[o] >= (long long)S.wd[o]) sok |= 1u << o;
        }
        const unsigned known = m2 & sok;
        unsigned alive = has ? known : 0u;
        // C1: boxes above z, 4 per lane per round; the "near" test (ahead of
        // the point, within the largest edge on each axis) gates the
        // per-orientation test. Lanes of one item AND their alive sets.
        const int clo = __reduce_min_sync(FULL, alive ? jsup : INT_MAX);
        for (int j0 = clo; j0 < nb; j0 += 4 << lg) {
            int4 bb[4];
            int bz[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = j0 + (u << lg) + ph;
                const bool in = j < nb;
                bb[u] = in ? bx[j] : make_int4(0, 0, 0, 0);
                bz[u] = in ? bzs[j] : 0;
            }
            unsigned near = 0;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = j0 + (u << lg) + ph;
                const int4 b = bb[u];
                const bool nu = alive && j >= jsup && x < b.z && y < b.w && b.x < x + S.wmax &&
                                b.y < y + S.dmax && bz[u] < z + S.hmax;
                near |= (nu ? 1u : 0u) << u;
            }
            const unsigned todo = __reduce_or_sync(FULL, near);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if ((todo >> u) & 1u) {
                    if ((near >> u) & 1u) {
                        // offsets from the point (coordinates are below 2^16)
                        const int dx = bb[u].x - x, dy = bb[u].y - y, dz = bz[u] - z;
#pragma unroll
                        for (int o = 0; o < 6; o++)
                            if (dx < S.ow[o] && dy < S.od[o] && dz < S.oh[o]) alive &= ~(1u << o);
                    }
                }
            }
            for (int m = 1; m < span; m <<= 1) alive &= __shfl_xor_sync(FULL, alive, m);
            if (!__any_sync(FULL, alive != 0)) break;
        }
        if (has && ph == 0) {
            const int p = wi[w + q];
            st[p] = st_pack(m2, known & ~alive, sok, known);
            if (z > 0) {
                sup[p] = (SupT)a0;
                sup[C + p] = (SupT)a1;
                sup[2 * C + p] = (SupT)a2;
                sup[3 * C + p] = (SupT)a3;
                sup[4 * C + p] = (SupT)a4;
                sup[5 * C + p] = (SupT)a5;
            }
        }
        w += K;
        if (GREEDY) {
            const unsigned bal = __ballot_sync(FULL, has && ph == 0 && alive != 0);
            if (bal) {
                first = w - K + ((__ffs(bal) - 1) >> lg);
                break;
            }
        }
    }
    __syncwarp();
    return make_int2(first, w);
}

// Applies one newly placed box to a valid point's state (C1 OR, C3 contact
// areas). Returns the new state, or 0 when the support grew onto an
// orientation whose C1 was never evaluated (the point is re-evaluated).
template <typename SupT>
__device__ __forceinline__ uint32_t st_apply_box(uint32_t s, int x, int y, int z, int4 B, int Bz, int Bz2,
                                                 const StepOrs& S, SupT* sup, int C, int p) {
    const bool above = Bz2 > z && x < B.z && y < B.w;
    const bool level = z > 0 && Bz2 == z;
    if (!above && !level) return s;   // the box neither blocks nor supports the point
    const unsigned m2 = s & 0x3fu, known = (s >> 24) & 0x3fu;
    unsigned blk = (s >> 8) & 0x3fu, sok = (s >> 16) & 0x3fu;
    if (above) {
        const int dx = B.x - x, dy = B.y - y, dz = Bz - z;
#pragma unroll
        for (int o = 0; o < 6; o++)
            if (dx < S.ow[o] && dy < S.od[o] && dz < S.oh[o]) blk |= 1u << o;
    }
    if (level) {
#pragma unroll
        for (int o = 0; o < 6; o++) {
            if ((m2 >> o) & 1u) {
                const int ox = min(x + S.ow[o], B.z) - max(x, B.x);
                const int oy = min(y + S.od[o], B.w) - max(y, B.y);
                if (ox > 0 && oy > 0) {
                    const int v = (int)sup[o * C + p] + ox * oy;
                    sup[o * C + p] = (SupT)v;
                    if (2LL * v >= (long long)S.wd[o]) sok |= 1u << o;
                }
            }
        }
        if (sok & m2 & ~known) return 0u;
    }
    return st_pack(m2, blk, sok, known);
}

// Warp: pick the pair, place the box, drop the points it covers and insert
// its uncovered corners (invalid), then update the top-sorted box tables and
// the top-z index. pp is the first point holding a feasible pair.
template <typename SupT>
__device__ __forceinline__ int place1(int t, int pp, bool full, uint32_t* mt, int& mpos, uint32_t* keys,
                                      uint32_t* st, SupT* sup, int4* bx, int* bzs, int* z2s,
                                      unsigned short* bis, unsigned short* zt, int Hz, int& nc, int& nb,
                                      int P, int C, const StepOrs& S, uint32_t xmask, uint32_t ymask,
                                      int xb, int xyb, unsigned long long* pass_out, long long& vol,
                                      int4& Bo, int& Bzo, int& Bz2o, int lane) {
    int pick = pp;
    int pick_oi = __ffs(st_feasible(st[pp])) - 1;
    if (full) {
        int count = 0;
        for (int i = pp + lane; i < nc; i += 32) count += __popc(st_feasible(st[i]));
        count = __reduce_add_sync(FULL, count);
        const int idx = mt_randrange(mt, mpos, lane, count);
        if (idx < 0) return ERR_RNG;
        // idx-th feasible pair in (point, orientation) order
        int run = 0;
        for (int cb = pp; cb < nc; cb += 32) {
            const int i = cb + lane;
            const unsigned m = i < nc ? st_feasible(st[i]) : 0u;
            const int c = __popc(m);
            // lane prefix of the pair counts (each below 8) from their bits
            const unsigned b0 = __ballot_sync(FULL, c & 1), b1 = __ballot_sync(FULL, c & 2),
                           b2 = __ballot_sync(FULL, c & 4);
            const unsigned lt = lanemask_lt();
            const int excl = __popc(b0 & lt) + 2 * __popc(b1 & lt) + 4 * __popc(b2 & lt);
            const int tot = __popc(b0) + 2 * __popc(b1) + 4 * __popc(b2);
            if (idx < run + tot) {
                const unsigned hit = __ballot_sync(FULL, idx < run + excl + c);
                const int l = __ffs(hit) - 1;
                const int ex = __shfl_sync(FULL, excl, l);
                const unsigned ml = __shfl_sync(FULL, m, l);
                pick = cb + l;
                pick_oi = __fns(ml, 0, idx - run - ex + 1);
                break;
            }
            run += tot;
        }
    }
    const uint32_t pkey = keys[pick];
    const int px = (int)(pkey & xmask), py = (int)((pkey >> xb) & ymask), pz = (int)(pkey >> xyb);
    int pw = 0, pd = 0, ph = 0;
#pragma unroll
    for (int o = 0; o < 6; o++)
        if (o == pick_oi) { pw = S.ow[o]; pd = S.od[o]; ph = S.oh[o]; }
    const int px2 = px + pw, py2 = py + pd, pz2 = pz + ph;
    if (nb >= P) return ERR_BOX_CAP;
    if (lane == 0) pass_out[nb] = pack_place(px, py, pz, pick_oi, t);
    vol += 1LL * pw * pd * ph;
    // Box tables, one pass from the top: the corners of the new box that a
    // placed box covers, and the boxes whose top is above the new box's move
    // up one slot (each round reads before it writes, and writes only slots
    // it or an earlier round has read).
    unsigned cov = 1u;   // corner 0 = (px, py, pz): covered by the new box
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
        const int ip = nb - nabove;   // after the boxes with equal tops
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
    // Points covered by the new box have keys >= the pick's (z >= pz, then
    // y >= py, then x >= px), so only [pick, nc) changes. Survivors move down
    // in place: every destination is at or below its source, and each round
    // reads before it writes.
    int ns = pick;
    for (int cb = pick; cb < nc; cb += 32) {
        const int i = cb + lane;
        bool keep = false;
        uint32_t key = 0, s = 0;
        int s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
        bool mv_sup = false;
        if (i < nc) {
            // all of a point's words load at once (in bounds; used if it moves)
            key = keys[i];
            s = st[i];
            s0 = sup[i]; s1 = sup[C + i]; s2 = sup[2 * C + i];
            s3 = sup[3 * C + i]; s4 = sup[4 * C + i]; s5 = sup[5 * C + i];
            const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask), z = (int)(key >> xyb);
            keep = !(px <= x && x < px2 && py <= y && y < py2 && pz <= z && z < pz2);
            mv_sup = keep && (s & ST_VALID) && z > 0;
        }
        const unsigned bal = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep) {
            const int d = ns + __popc(bal & lanemask_lt());
            if (d != i) {
                keys[d] = key;
                st[d] = s;
                if (mv_sup) {
                    sup[d] = (SupT)s0; sup[C + d] = (SupT)s1; sup[2 * C + d] = (SupT)s2;
                    sup[3 * C + d] = (SupT)s3; sup[4 * C + d] = (SupT)s4; sup[5 * C + d] = (SupT)s5;
                }
            }
        }
        ns += __popc(bal);
    }
    __syncwarp();
    // new corners, in index order c = (cz << 2) | (cy << 1) | cx, which is
    // their (z, y, x) order; all lie after the pick
    uint32_t ck = 0;
    int rank = 0;
    bool isnew = false;
    // the lanes sample the survivors [pick, ns) at even spacing; one ballot
    // per corner brackets it between two samples, a binary search finishes
    const int nsv = ns - pick;
    const uint32_t ks = nsv > 0 ? keys[pick + ((lane * nsv) >> 5)] : 0xffffffffu;
    {
        const int cx = (lane & 1) ? px2 : px, cy = (lane & 2) ? py2 : py, cz = (lane & 4) ? pz2 : pz;
        ck = ((uint32_t)cz << xyb) | ((uint32_t)cy << xb) | (uint32_t)cx;
    }
    int below = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const uint32_t kc = __shfl_sync(FULL, ck, c);
        const int t = __popc(__ballot_sync(FULL, ks < kc));
        if (lane == c) below = t;
    }
    if (lane < 8 && !((cov >> lane) & 1u)) {
        int lo = below == 0 ? pick : pick + (((below - 1) * nsv) >> 5) + 1;
        const int hi = below == 32 ? ns : pick + ((below * nsv) >> 5);
        int n = hi - lo;
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
        // survivors at or after the first insertion move up by the number of
        // new corners below them; rounds go from the top, reading first
        for (int hi = ns; hi > first_ins; hi -= 32) {
            const int i = hi - 1 - lane;
            const bool in = i >= first_ins;
            uint32_t key = 0, s = 0;
            int s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
            bool mv_sup = false;
            int off = 0;
            if (in) {
                key = keys[i];
                s = st[i];
                s0 = sup[i]; s1 = sup[C + i]; s2 = sup[2 * C + i];
                s3 = sup[3 * C + i]; s4 = sup[4 * C + i]; s5 = sup[5 * C + i];
                mv_sup = (s & ST_VALID) && (key >> xyb) > 0;
#pragma unroll
                for (int c = 0; c < 8; c++) off += ((newm >> c) & 1u) && ckk[c] < key;
            }
            __syncwarp();
            if (in && off) {
                const int d = i + off;
                keys[d] = key;
                st[d] = s;
                if (mv_sup) {
                    sup[d] = (SupT)s0; sup[C + d] = (SupT)s1; sup[2 * C + d] = (SupT)s2;
                    sup[3 * C + d] = (SupT)s3; sup[4 * C + d] = (SupT)s4; sup[5 * C + d] = (SupT)s5;
                }
            }
            __syncwarp();
        }
        if (isnew) {
            const int d = rank + __popc(newm & ((1u << lane) - 1u));
            keys[d] = ck;
            st[d] = 0u;
        }
    }
    nc = nnew;
    Bo = make_int4(px, py, px2, py2);
    Bzo = pz;
    Bz2o = pz2;
    __syncwarp();
    return ERR_NONE;
}

// ---------------------------------------------------------------------------
// serving: work from a host-published ring, completion on the device
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int2 ld_relaxed_gpu_int2(const int2* p) {
    int x, y;
    asm volatile("ld.relaxed.gpu.global.v2.s32 {%0, %1}, [%2];" : "=r"(x), "=r"(y) : "l"(p) : "memory");
    return make_int2(x, y);
}

__device__ __forceinline__ void st_release_sys(volatile long long* p, long long v) {
    asm volatile("st.release.sys.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Lane 0 of an overflow decoder: the next overflow item (ticket), or -1 once
// the host asked the launch to stop and every main decoder has exited with
// nothing left, or after deep_idle_polls empty polls.
__device__ __forceinline__ int serve_claim_deep(const ServeArgs& s) {
    unsigned ns = 64;
    for (int k = 0; k < s.deep_idle_polls; k++) {
        const int t = ld_acquire_gpu(s.dtail);
        int h = *reinterpret_cast<volatile int*>(s.dhead);
        while (h < t) {
            const int prev = atomicCAS(s.dhead, h, h + 1);
            if (prev == h) return h;
            h = prev;
        }
        // main decoders push before they leave, so once none is left the
        // reservation count seen after that is final
        if (ld_acquire_gpu(s.stop) && ld_acquire_gpu(s.alive) == 0 && ld_acquire_gpu(s.dtail) <= h) return -1;
        __nanosleep(ns);
        if (ns < 8192) ns <<= 1;
    }
    return -1;
}

// Lane 0: waits (bounded) until the producer of ticket t has written it.
__device__ __forceinline__ bool serve_deep_item(const ServeArgs& s, int t, int2* w) {
    int4* e = s.dring + (t & s.ring_mask);
    for (int k = 0; k < (1 << 22); k++) {
        if (ld_acquire_gpu(&e->z) == t + 1) {
            *w = make_int2(*reinterpret_cast<volatile int*>(&e->x), *reinterpret_cast<volatile int*>(&e->y));
            return true;
        }
        __nanosleep(32);
    }
    return false;
}

// A main decoder hands a restart that outgrew its tile to the overflow ring.
__device__ __forceinline__ void serve_push_deep(const ServeArgs& s, int2 wk, int lane) {
    if (lane == 0) {
        const int t = atomicAdd(s.dtail, 1);
        int4* e = s.dring + (t & s.ring_mask);
        *reinterpret_cast<volatile int*>(&e->x) = wk.x;
        *reinterpret_cast<volatile int*>(&e->y) = wk.y;
        st_release_gpu(&e->z, t + 1);
    }
    __syncwarp();
}

// Lane 0: claims the next published work item, or returns -1 once the host
// has asked the launch to stop (and nothing is left) or after idle_polls
// empty polls. The host publishes by stream-ordered copies into device
// memory (items first, then the tail), so the polls stay on this GPU's L2.
// Every loop is bounded: the inner one by the items published, the outer
// one by idle_polls.
__device__ __forceinline__ int serve_claim(const ServeArgs& s) {
    unsigned ns = 32;
    for (int k = 0; k < s.idle_polls; k++) {
        const int t = ld_acquire_gpu(s.tail);
        int h = *reinterpret_cast<volatile int*>(s.head);
        while (h < t) {
            const int prev = atomicCAS(s.head, h, h + 1);
            if (prev == h) return h;
            h = prev;
        }
        if (ld_acquire_gpu(s.stop)) return -1;
        __nanosleep(ns);
        if (ns < 4096) ns <<= 1;
    }
    return -1;
}

// A request descriptor read through L2 (serving arenas reuse addresses while
// the launch runs, so no table may come from a stale L1 line).
__device__ __forceinline__ InstDesc load_desc_cg(const InstDesc* p) {
    static_assert(sizeof(InstDesc) % 8 == 0, "InstDesc is copied in 8-byte words");
    InstDesc d;
    const long long* src = reinterpret_cast<const long long*>(p);
    long long* dst = reinterpret_cast<long long*>(&d);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(InstDesc) / 8); i++) dst[i] = __ldcg(src + i);
    return d;
}

template <bool CG>
__device__ __forceinline__ int ld_table(const int* p) { return CG ? __ldcg(p) : *p; }

// Best restart of one instance, one warp: accepted first, then max (volume,
// n_boxes), the earliest restart on ties (the strict > of
// gpu/plp_common.hpp:507-511). CG: the heads are read through L2.
template <bool CG>
__device__ __forceinline__ int2 select_best_warp(const InstDesc& I, const SlotHead* heads, int lane) {
    int br = -1, bacc = 0, bn = 0;
    long long bv = -1;
    for (int r = lane; r < I.restarts; r += 32) {
        const SlotHead* hp = heads + I.slot_base + r;
        const int fb = CG ? __ldcg(&hp->fallback) : hp->fallback;
        const long long vol = CG ? __ldcg(&hp->volume) : hp->volume;
        const int nbx = CG ? __ldcg(&hp->n_boxes) : hp->n_boxes;
        const int acc = fb ? 0 : 1;
        const bool better = br < 0 || acc > bacc || (acc == bacc && (vol > bv || (vol == bv && nbx > bn)));
        if (better) { br = r; bacc = acc; bv = vol; bn = nbx; }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const int r2 = __shfl_down_sync(FULL, br, d);
        const int a2 = __shfl_down_sync(FULL, bacc, d);
        const long long v2 = __shfl_down_sync(FULL, bv, d);
        const int n2 = __shfl_down_sync(FULL, bn, d);
        bool better;
        if (r2 < 0) better = false;
        else if (br < 0) better = true;
        else if (a2 != bacc) better = a2 > bacc;
        else if (v2 != bv) better = v2 > bv;
        else if (n2 != bn) better = n2 > bn;
        else better = r2 < br;
        if (better) { br = r2; bacc = a2; bv = v2; bn = n2; }
    }
    return make_int2(__shfl_sync(FULL, br, 0), __shfl_sync(FULL, bacc, 0) ? 0 : 1);
}

// After a restart's head is written: the warp that finishes the request's
// last restart selects its best restart and publishes it, with the request's
// sequence number, in the host-mapped completion record.
__device__ __forceinline__ void serve_finish(const DecoderArgs& a, const ServeArgs& s, int di, const InstDesc& I,
                                             int lane) {
    ServeTail* tl = reinterpret_cast<ServeTail*>(const_cast<InstDesc*>(a.inst) + di + 1);
    int last = 0;
    if (lane == 0) {
        __threadfence();
        last = atomicAdd(&tl->done_count, 1) == I.restarts - 1;
    }
    last = __shfl_sync(FULL, last, 0);
    if (!last) return;
    __threadfence();
    const int2 b = select_best_warp<true>(I, a.heads, lane);
    if (lane == 0) {
        const int slot = __ldcg(&tl->done_slot);
        const long long seq = __ldcg(&tl->seq);
        s.done_best[slot] = b;
        __threadfence_system();
        st_release_sys(s.done_seq + slot, seq);
    }
    __syncwarp();
}

// MODE 0: batch launch; 1: serving launch, main decoder (pushes restarts
// that outgrow its tile to the overflow ring); 2: serving launch, overflow
// decoder (deeper tile in global memory, takes the overflow ring).
template <typename SupT, int MODE>
__device__ __forceinline__ void decoder1_body(const DecoderArgs& a, unsigned char* base, int gdec,
                                              const ServeArgs& sv) {
    const int lane = threadIdx.x & 31;
    const Dec1Layout lay = dec1_layout(a.P, a.C, a.Hz, (int)sizeof(SupT));
    const int C = a.C;
    uint32_t* mt = reinterpret_cast<uint32_t*>(base);
    int4* bx = reinterpret_cast<int4*>(base + lay.off_bx);
    int* bzs = reinterpret_cast<int*>(base + lay.off_bz);
    int* z2s = reinterpret_cast<int*>(base + lay.off_z2);
    unsigned short* bis = reinterpret_cast<unsigned short*>(base + lay.off_bi);
    uint32_t* keys = reinterpret_cast<uint32_t*>(base + lay.off_key);
    uint32_t* st = reinterpret_cast<uint32_t*>(base + lay.off_st);
    SupT* sup = reinterpret_cast<SupT*>(base + lay.off_sup);
    uint2* Wl = reinterpret_cast<uint2*>(base + lay.off_w);
    unsigned short* wi = reinterpret_cast<unsigned short*>(base + lay.off_wi);
    unsigned short* zt = a.Hz ? reinterpret_cast<unsigned short*>(base + lay.off_zt) : nullptr;

    constexpr bool SERVE = MODE != 0;
    const int n_work = SERVE ? 0 : (a.n_work_dev ? *a.n_work_dev : a.n_work);
    for (;;) {
        if (*reinterpret_cast<volatile int*>(a.abort)) break;
        int2 wk;
        if constexpr (SERVE) {
            int item = -1, wx = 0, wy = 0;
            if (lane == 0) {
                if constexpr (MODE == 1) {
                    item = serve_claim(sv);
                    if (item >= 0) {
                        const int2 w = ld_relaxed_gpu_int2(sv.ring + (item & sv.ring_mask));
                        wx = w.x;
                        wy = w.y;
                    }
                } else {
                    item = serve_claim_deep(sv);
                    int2 w = make_int2(0, 0);
                    if (item >= 0 && !serve_deep_item(sv, item, &w)) {
                        atomicOr(a.err_flag, 1 << ERR_SYNC);   // a producer never finished its item
                        item = -1;
                    }
                    wx = w.x;
                    wy = w.y;
                }
            }
            if (__shfl_sync(FULL, item, 0) < 0) break;
            wk = make_int2(__shfl_sync(FULL, wx, 0), __shfl_sync(FULL, wy, 0));
        } else {
            int item = 0;
            if (lane == 0) item = atomicAdd(a.work_next, 1);
            item = __shfl_sync(FULL, item, 0);
            if (item >= n_work) break;
            wk = a.work[item];
        }
        const InstDesc I = SERVE ? load_desc_cg(a.inst + wk.x) : a.inst[wk.x];
        const int restart = wk.y;
        const int slot = I.slot_base + restart;
        const int L = I.L, W = I.W, H = I.H;
        const uint32_t xmask = (1u << I.xb) - 1u, ymask = (1u << I.yb) - 1u;
        const int xb = I.xb, xyb = I.xb + I.yb;
        const bool randomized = !(I.first_fit || I.eps == 0.0);
        unsigned long long* best_out = a.places + I.place_off + (long long)restart * I.place_stride;
        unsigned long long* pass_out =
            I.passes > 1 ? a.scratch + (long long)gdec * I.place_stride : best_out;
        int mpos = 624;
        {
            const long long sd = I.seed + restart;
            if (!SERVE && a.seed_tab && sd >= a.seed_lo && sd - a.seed_lo < a.seed_n) {
                // the seeded state, computed once for every restart of the batch with this seed
                const uint4* src = reinterpret_cast<const uint4*>(a.seed_tab + (sd - a.seed_lo) * 624);
                uint4* dst = reinterpret_cast<uint4*>(mt);
                for (int i = lane; i < 156; i += 32) dst[i] = __ldg(src + i);
                __syncwarp();
            } else {
                mt_seed_warp(mt, (unsigned long long)(sd < 0 ? -sd : sd), a.mt_init, lane);
            }
        }
        const long long t0 = global_ns();   // the reference's run() clock starts after seeding
        int npass = 0;
        int err = ERR_NONE;
        bool have_acc = false, have_any = false;
        long long best_vol = 0;
        int best_n = 0;
        double best_score = 0.0;

        for (int pass = 0; pass < I.passes && err == ERR_NONE; pass++) {
            int nb = 0, nc = 1;
            long long vol = 0;
            if (zt)
                for (int i = lane; i < a.Hz; i += 32) zt[i] = 0;
            if (lane == 0) {
                keys[0] = 0u;
                st[0] = 0u;
            }
            __syncwarp();
            int state_type = -1;
            bool pending = false;   // a placed box not yet applied to the valid states
            bool stuck = false;     // the last step of state_type found no feasible pair
            int4 B = make_int4(0, 0, 0, 0);
            int Bz = 0, Bz2 = 0;
            int t_next = I.n_steps > 0 ? ld_table<SERVE>(a.step_type + I.step_off) : 0;
            for (int sti = 0; sti < I.n_steps; sti++) {
                const int t = t_next;
                if (sti + 1 < I.n_steps) t_next = ld_table<SERVE>(a.step_type + I.step_off + sti + 1);
                // With no box placed since, another item of that type meets the
                // same states and finds no pair either; it draws no random
                // number, so the step is skipped without changing the result.
                if (stuck && t == state_type) continue;
                const TypeOrs& T = a.types[I.type_off + t];
                StepOrs S;
                S.no = ld_table<SERVE>(&T.n);
                if (S.no == 0) continue;
                S.wmax = S.dmax = S.hmax = 0;
#pragma unroll
                for (int o = 0; o < 6; o++) {
                    S.ow[o] = ld_table<SERVE>(&T.w[o]);
                    S.od[o] = ld_table<SERVE>(&T.d[o]);
                    S.oh[o] = ld_table<SERVE>(&T.h[o]);
                    S.wd[o] = S.ow[o] * S.od[o];
                    S.wmax = max(S.wmax, S.ow[o]);
                    S.dmax = max(S.dmax, S.od[o]);
                    S.hmax = max(S.hmax, S.oh[o]);
                }
                const bool fresh = t != state_type;
                state_type = t;
                const bool apply = pending && !fresh;
                pending = false;
                // filter: bring valid states up to date with the last box and
                // read their feasible sets; list the invalid points that have an
                // orientation inside the container and, above the floor, a box
                // top at their height. v = first valid point with a feasible pair.
                int nW = 0, v = INT_MAX, nWg = -1;
                for (int cb = 0; cb < nc; cb += 32) {
                    const int i = cb + lane;
                    unsigned f = 0;
                    bool cand = false;
                    uint2 it = make_uint2(0, 0);
                    if (i < nc) {
                        const uint32_t key = keys[i];
                        const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask), z = (int)(key >> xyb);
                        uint32_t s = fresh ? 0u : st[i];
                        const uint32_t s_in = s;
                        if ((s & ST_VALID) && apply) s = st_apply_box(s, x, y, z, B, Bz, Bz2, S, sup, C, i);
                        if (s & ST_VALID) {
                            f = st_feasible(s);
                        } else {
                            unsigned m = 0;
#pragma unroll
                            for (int o = 0; o < 6; o++)
                                if (o < S.no && x + S.ow[o] <= L && y + S.od[o] <= W && z + S.oh[o] <= H) m |= 1u << o;
                            if (!m) {
                                s = ST_VALID;   // nothing fits: infeasible for the rest of the run
                            } else {
                                s = 0u;
                                const int jlo = box_start(zt, z2s, nb, z);
                                const int jsup = z > 0 ? box_start(zt, z2s, nb, z + 1) : jlo;
                                if (z == 0 || jsup > jlo) {
                                    cand = true;
                                    it = make_item(key, m, jlo, jsup);
                                }
                            }
                        }
                        if (s != s_in || fresh) st[i] = s;
                    }
                    const unsigned bal = __ballot_sync(FULL, cand);
                    if (v == INT_MAX) {
                        const unsigned bf = __ballot_sync(FULL, f != 0);
                        if (bf) {
                            v = cb + __ffs(bf) - 1;
                            nWg = nW + __popc(bal & ((1u << (v - cb)) - 1u));
                        }
                    }
                    if (cand) {
                        const int d = nW + __popc(bal & lanemask_lt());
                        Wl[d] = it;
                        wi[d] = (unsigned short)i;
                    }
                    nW += __popc(bal);
                }
                if (nWg < 0) nWg = nW;
                __syncwarp();
                // greedy: the invalid points before v, in order; then, on the
                // random branch, every item left (one evaluation site)
                int pp = v, lo = 0, hi = nWg;
                bool greedy = true, full = false;
                for (;;) {
                    if (lo < hi) {
                        const int2 r = eval_items(greedy, Wl, wi, lo, hi, bx, bzs, nb, S, xmask, ymask, xb, xyb,
                                                  st, sup, C, lane);
                        if (greedy) {
                            if (r.x != INT_MAX) pp = wi[r.x];
                            lo = r.y;
                        }
                    }
                    if (!greedy || pp == INT_MAX) break;
                    full = randomized && mt_random(mt, mpos, lane) >= 1.0 - I.eps;
                    if (!full || lo >= nW) break;
                    greedy = false;   // every feasible pair is needed
                    hi = nW;
                }
                stuck = pp == INT_MAX;
                if (stuck) continue;                     // no feasible pair: no draw
                err = place1(t, pp, full, mt, mpos, keys, st, sup, bx, bzs, z2s, bis, zt, a.Hz, nc, nb, a.P,
                             C, S, xmask, ymask, xb, xyb, pass_out, vol, B, Bz, Bz2, lane);
                if (err != ERR_NONE) break;
                pending = true;
            }
            if (err != ERR_NONE) break;
            const double score =
                fsr_score_warp(bx, bzs, z2s, bis, nb, I.mu, reinterpret_cast<char*>(keys), lane, nullptr, zt);
            const bool acc = !I.has_theta || score >= I.theta;
            bool take;
            if (acc) take = !have_acc || vol > best_vol || (vol == best_vol && nb > best_n);
            else take = !have_acc && (!have_any || vol > best_vol || (vol == best_vol && nb > best_n));
            if (take) {
                best_vol = vol;
                best_n = nb;
                best_score = score;
                if (pass_out != best_out)
                    for (int i = lane; i < nb; i += 32) best_out[i] = pass_out[i];
            }
            have_any = true;
            have_acc = have_acc || acc;
            npass = pass + 1;
            __syncwarp();
            // wall-clock budget (gpu/plp_common.hpp:484-492): stop once it is spent
            if (I.budget_ns >= 0 && __shfl_sync(FULL, global_ns() - t0, 0) >= I.budget_ns) break;
        }
        // a serving main decoder hands a restart that outgrew its tile to the
        // launch's overflow decoders instead of reporting it
        bool to_deep = false;
        if constexpr (MODE == 1) to_deep = sv.n_deep > 0 && (err == ERR_BOX_CAP || err == ERR_CAND_CAP);
        if (lane == 0 && !to_deep) {
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
        if constexpr (SERVE) {
            if (to_deep) serve_push_deep(sv, wk, lane);
            else serve_finish(a, sv, wk.x, I, lane);
        }
    }
    if constexpr (MODE == 1) {
        if (lane == 0) {   // pushes above are visible before the count drops
            __threadfence();
            atomicSub(sv.alive, 1);
        }
    }
}

static DecoderArgs decoder_args(const DecodeLaunch& L) {
    DecoderArgs a;
    a.inst = L.inst;
    a.step_type = L.step_type;
    a.types = L.types;
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
    a.Hz = L.Hz;
    a.sync_limit = L.sync_limit;
    a.sync_skip = L.sync_skip;
    a.seed_tab = L.seed_tab;
    a.seed_lo = L.seed_lo;
    a.seed_n = L.seed_n;
    return a;
}

#ifndef PLP_SERVE_TU
// S16: contact areas stored as 16-bit (every footprint area < 65536)
template <int D, int M, int S16>
__global__ void __launch_bounds__(32 * D, M) decoder1_kernel(DecoderArgs a) {
    using SupT = typename std::conditional<S16 != 0, unsigned short, int>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dec = threadIdx.x >> 5;
    const Dec1Layout lay = dec1_layout(a.P, a.C, a.Hz, (int)sizeof(SupT));
    decoder1_body<SupT, 0>(a, smem_raw + (size_t)dec * lay.bytes, blockIdx.x * D + dec, ServeArgs{});
}


// ---------------------------------------------------------------------------
// per-instance best restart: accepted first, then max (volume, n_boxes),
// earliest restart on ties (the strict > of gpu/plp_common.hpp:507-511)
// ---------------------------------------------------------------------------
__global__ void select_best_kernel(const InstDesc* __restrict__ inst, int n_inst,
                                   const SlotHead* __restrict__ heads, int2* __restrict__ best) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= n_inst) return;
    const InstDesc I = inst[i];
    const int2 b = select_best_warp<false>(I, heads, lane);
    if (lane == 0) best[i] = b;
}

// ---------------------------------------------------------------------------
// seeded MT19937 states of a range of seeds (one warp per seed), shared by
// every restart of a batch that uses the same seed
// ---------------------------------------------------------------------------
__global__ void seed_table_kernel(long long lo, int n, const uint32_t* __restrict__ mt_init,
                                  uint32_t* __restrict__ out) {
    __shared__ uint32_t mts[4][624];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * 4 + w;
    if (i >= n) return;
    const long long sd = lo + i;
    mt_seed_warp(mts[w], (unsigned long long)(sd < 0 ? -sd : sd), mt_init, lane);
    for (int k = lane; k < 624; k += 32) out[(long long)i * 624 + k] = mts[w][k];
}

// ---------------------------------------------------------------------------
// device MT19937 dump (kernel test hook, like --rngdump): one warp per seed
// ---------------------------------------------------------------------------
__global__ void rng_dump_kernel(const long long* __restrict__ seeds, int n_seeds, int n_random,
                                int n_bits, int k_bits, const uint32_t* __restrict__ mt_init,
                                double* __restrict__ out_r, uint32_t* __restrict__ out_b) {
    __shared__ uint32_t mts[4][624];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int s = blockIdx.x * 4 + wid;
    if (s >= n_seeds) return;
    uint32_t* mt = mts[wid];
    const long long sv = seeds[s];
    mt_seed_warp(mt, (unsigned long long)(sv < 0 ? -sv : sv), mt_init, lane);
    int pos = 624;
    for (int i = 0; i < n_random; i++) {
        const double r = mt_random(mt, pos, lane);
        if (lane == 0) out_r[(long long)s * n_random + i] = r;
    }
    for (int i = 0; i < n_bits; i++) {
        const uint32_t b = mt_next(mt, pos, lane) >> (32 - k_bits);
        if (lane == 0) out_b[(long long)s * n_bits + i] = b;
    }
}

// ---------------------------------------------------------------------------
// standalone FSR over packings given as placement rows (kernel test hook and
// the plain path's scorer): one warp per packing, boxes sorted by top first
// ---------------------------------------------------------------------------
__global__ void fsr_kernel(const int* __restrict__ rows7, const int* __restrict__ offsets,
                           int n_pack, int cap, double mu, double* __restrict__ out_score,
                           double* __restrict__ out_fsr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int pk = blockIdx.x * (blockDim.x >> 5) + wid;
    const int per = 16 * cap + 4 * cap + 4 * cap + 2 * cap + 18 * cap + 64;
    unsigned char* base = smem_raw + (size_t)wid * ((per + 15) & ~15);
    if (pk >= n_pack) return;
    int4* bx = reinterpret_cast<int4*>(base);
    int* bz = reinterpret_cast<int*>(base + 16 * cap);
    int* z2 = reinterpret_cast<int*>(base + 20 * cap);
    unsigned short* bi = reinterpret_cast<unsigned short*>(base + 24 * cap);
    char* scratch = reinterpret_cast<char*>(base + ((26 * cap + 15) & ~15));
    const int o0 = offsets[pk];
    const int n = offsets[pk + 1] - o0;
    // insertion by rank on top z (ties by index) gives the sorted order
    for (int i = lane; i < n; i += 32) {
        const int* r = rows7 + 7 * (o0 + i);
        const int t = r[3] + r[6];
        int rank = 0;
        for (int j = 0; j < n; j++) {
            const int* q = rows7 + 7 * (o0 + j);
            const int tj = q[3] + q[6];
            rank += tj < t || (tj == t && j < i);
        }
        bx[rank] = make_int4(r[1], r[2], r[1] + r[4], r[2] + r[5]);
        bz[rank] = r[3];
        z2[rank] = t;
        bi[rank] = (unsigned short)i;
    }
    __syncwarp();
    const double sc = fsr_score_warp(bx, bz, z2, bi, n, mu, scratch, lane,
                                     out_fsr ? out_fsr + o0 : nullptr);
    if (lane == 0) out_score[pk] = sc;
}

// ---------------------------------------------------------------------------
// item order on the device (kernel d): one block per instance expands the
// (type, copy) list and bitonic-sorts the keys (-volume, type, copy), packed
// as  (maxvol - volume) << 32 | type << 16 | copy  into 64-bit words.
// ---------------------------------------------------------------------------
__global__ void item_order_kernel(const long long* __restrict__ vols, const int* __restrict__ qty,
                                  const int* __restrict__ type_off, const int* __restrict__ n_types,
                                  const long long* __restrict__ step_off, int order,
                                  int* __restrict__ out_types, int sort_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* key = reinterpret_cast<unsigned long long*>(smem_raw);
    __shared__ int s_n;
    const int inst = blockIdx.x;
    const int t0 = type_off[inst], nt = n_types[inst];
    const long long o0 = step_off[inst];
    const int n = (int)(step_off[inst + 1] - o0);
    if (threadIdx.x == 0) s_n = n;
    int npad = 1;
    while (npad < n) npad <<= 1;
    // expand: thread per type writes its copies (prefix over qty by scan of types)
    if (threadIdx.x == 0) {
        int p = 0;
        for (int t = 0; t < nt; t++) {
            const int q = qty[t0 + t];
            const long long v = vols[t0 + t];
            for (int c = 0; c < q; c++, p++)
                key[p] = (order == 0 ? ((unsigned long long)(0x7fffffffLL - v) << 32) : 0ull) |
                         ((unsigned long long)t << 16) | (unsigned long long)c;
        }
        for (; p < npad; p++) key[p] = ~0ull;
    }
    __syncthreads();
    if (order == 0 && npad <= sort_cap) {
        for (int k = 2; k <= npad; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < npad; i += blockDim.x) {
                    const int l = i ^ j;
                    if (l > i) {
                        const unsigned long long x = key[i], y = key[l];
                        const bool up = (i & k) == 0;
                        if ((x > y) == up) { key[i] = y; key[l] = x; }
                    }
                }
                __syncthreads();
            }
        }
    }
    for (int i = threadIdx.x; i < s_n; i += blockDim.x)
        out_types[o0 + i] = (int)((key[i] >> 16) & 0xffff);
}

// ---------------------------------------------------------------------------
// copy each instance's best restart placements into a compact buffer (one
// warp per instance) so best-only results need a single small copy back
// ---------------------------------------------------------------------------
__global__ void gather_best_kernel(const InstDesc* __restrict__ inst, int n_inst,
                                   const int2* __restrict__ best,
                                   const unsigned long long* __restrict__ places,
                                   unsigned long long* __restrict__ out, int out_stride) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= n_inst) return;
    const InstDesc I = inst[i];
    const int r = best[i].x;
    if (r < 0) return;
    const unsigned long long* src = places + I.place_off + (long long)r * I.place_stride;
    for (int k = lane; k < I.place_stride; k += 32) out[(long long)i * out_stride + k] = src[k];
}

// ---------------------------------------------------------------------------
// host launchers (engine.hpp)
// ---------------------------------------------------------------------------
// (G warps per decoder, D decoders per CTA, M minimum resident CTAs per SM:
// a register cap of 65536 / (32 G D M) per thread) instantiations
#define PLP_DECODER_CONFIGS(X)                                                                 \
    X(1, 1, 1) X(1, 1, 12) X(1, 1, 16) X(1, 2, 1) X(1, 4, 1) X(1, 4, 4) X(1, 8, 1) X(1, 8, 2) X(2, 1, 1) X(2, 2, 1) X(2, 2, 5) \
    X(2, 4, 1) X(2, 4, 3) X(4, 1, 1) X(4, 1, 5) X(4, 1, 6) X(4, 2, 1) X(4, 2, 3) X(4, 4, 1)   \
    X(8, 1, 1) X(8, 1, 3) X(8, 2, 1)

using DecoderFn = void (*)(DecoderArgs);

// G = 1: the incremental single-warp decoder (16- or 32-bit contact areas);
// G > 1: the multi-warp decoder
template <int G, int D, int M>
static DecoderFn pick_kernel(int sup16) {
    if constexpr (G == 1) return sup16 ? decoder1_kernel<D, M, 1> : decoder1_kernel<D, M, 0>;
    else return decoder_kernel<G, D, M>;
}

static DecoderFn decoder_fn(int G, int D, int M, int sup16 = 0) {
#define PLP_PICK(g, d, m) \
    if (G == g && D == d && M == m) return pick_kernel<g, d, m>(sup16);
    PLP_DECODER_CONFIGS(PLP_PICK)
#undef PLP_PICK
    return nullptr;
}

bool decoder_config_supported(int G, int D, int M) { return decoder_fn(G, D, M) != nullptr; }

namespace {
std::mutex g_attr_mu;
std::map<std::pair<const void*, int>, int> g_dyn_smem;                 // (kernel, device) -> limit set
std::map<std::tuple<const void*, int, int, int>, int> g_occupancy;    // (kernel, device, threads, smem)
}  // namespace

cudaError_t ensure_dyn_smem(const void* fn, int smem) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    int& cur = g_dyn_smem[{fn, dev}];
    if (smem <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) cur = smem;
    return e;
}

cudaError_t cached_occupancy(const void* fn, int threads, int smem, int* ctas_per_sm) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        auto it = g_occupancy.find(std::make_tuple(fn, dev, threads, smem));
        if (it != g_occupancy.end()) {
            *ctas_per_sm = it->second;
            return cudaSuccess;
        }
    }
    e = ensure_dyn_smem(fn, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, threads, (size_t)smem);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    g_occupancy[std::make_tuple(fn, dev, threads, smem)] = *ctas_per_sm;
    return cudaSuccess;
}


static int decoder_launch_smem(const DecodeLaunch& L) {
    return decoder_smem_bytes(L.P, L.C, L.Hz, L.warps_per_decoder, L.sup16) * L.decoders_per_cta;
}

// Function attributes (dynamic shared memory) for a launch; not a stream
// operation, so it is done before any capture.
cudaError_t configure_decoder(const DecodeLaunch& L) {
    if (L.engine == 1) return configure_block(L);
    DecoderFn fn = decoder_fn(L.warps_per_decoder, L.decoders_per_cta, L.min_blocks, L.sup16);
    if (!fn) return cudaErrorInvalidConfiguration;
    return ensure_dyn_smem(reinterpret_cast<const void*>(fn), decoder_launch_smem(L));
}

// Stream operations only (counter resets and the launch): capturable.
cudaError_t enqueue_decoder(const DecodeLaunch& L, cudaStream_t st) {
    if (L.engine == 1) return enqueue_block(L, st);
    DecoderFn fn = decoder_fn(L.warps_per_decoder, L.decoders_per_cta, L.min_blocks, L.sup16);
    if (!fn) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaMemsetAsync(L.work_next, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(L.abort, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    fn<<<L.ctas, 32 * L.warps_per_decoder * L.decoders_per_cta, decoder_launch_smem(L), st>>>(decoder_args(L));
    return cudaGetLastError();
}

cudaError_t launch_decoder(const DecodeLaunch& L, cudaStream_t st) {
    cudaError_t e = configure_decoder(L);
    if (e != cudaSuccess) return e;
    return enqueue_decoder(L, st);
}

cudaError_t launch_seed_table(long long lo, int n, const uint32_t* mt_init, uint32_t* out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    seed_table_kernel<<<(n + 3) / 4, 128, 0, st>>>(lo, n, mt_init, out);
    return cudaGetLastError();
}

cudaError_t decoder_occupancy(int P, int C, int Hz, int G, int D, int M, int* ctas_per_sm, int sup16) {
    DecoderFn fn = decoder_fn(G, D, M, sup16);
    if (!fn) return cudaErrorInvalidConfiguration;
    const int smem = decoder_smem_bytes(P, C, Hz, G, sup16) * D;
    return cached_occupancy(reinterpret_cast<const void*>(fn), 32 * G * D, smem, ctas_per_sm);
}

// Appends the work items whose restart overflowed its tile (box or live-point
// capacity) to `redo`; `count` is zero on entry. The list's order does not
// matter: each restart's results land in its own slot.
__global__ void redo_collect_kernel(const int2* __restrict__ work, int n_work, const InstDesc* __restrict__ inst,
                                    const SlotHead* __restrict__ heads, int2* __restrict__ redo,
                                    int* __restrict__ count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_work; i += gridDim.x * blockDim.x) {
        const int2 w = work[i];
        const int err = heads[inst[w.x].slot_base + w.y].err;
        if (err == ERR_BOX_CAP || err == ERR_CAND_CAP) redo[atomicAdd(count, 1)] = w;
    }
}

cudaError_t launch_redo_collect(const int2* work, int n_work, const InstDesc* inst, const SlotHead* heads,
                                int2* redo, int* count, int sms, cudaStream_t st) {
    const int blocks = std::max(1, std::min((n_work + 255) / 256, sms * 8));
    redo_collect_kernel<<<blocks, 256, 0, st>>>(work, n_work, inst, heads, redo, count);
    return cudaGetLastError();
}

cudaError_t launch_select_best(const InstDesc* inst, int n_inst, const SlotHead* heads, int2* best,
                               cudaStream_t st) {
    const int wpb = 8;
    select_best_kernel<<<(n_inst + wpb - 1) / wpb, 32 * wpb, 0, st>>>(inst, n_inst, heads, best);
    return cudaGetLastError();
}

cudaError_t launch_rng_dump(const long long* seeds, int n_seeds, int n_random, int n_bits,
                            int k_bits, const uint32_t* mt_init, double* out_r, uint32_t* out_b,
                            cudaStream_t st) {
    rng_dump_kernel<<<(n_seeds + 3) / 4, 128, 0, st>>>(seeds, n_seeds, n_random, n_bits, k_bits,
                                                       mt_init, out_r, out_b);
    return cudaGetLastError();
}

int fsr_smem_per_warp(int cap) {
    const int per = 16 * cap + 4 * cap + 4 * cap + 2 * cap + 18 * cap + 64;
    return (per + 15) & ~15;
}

cudaError_t launch_fsr(const int* rows7, const int* offsets, int n_pack, int cap, double mu,
                       double* out_score, double* out_fsr, cudaStream_t st) {
    const int wpb = 4;
    const int smem = fsr_smem_per_warp(cap) * wpb;
    cudaError_t e = ensure_dyn_smem(reinterpret_cast<const void*>(fsr_kernel), smem);
    if (e != cudaSuccess) return e;
    fsr_kernel<<<(n_pack + wpb - 1) / wpb, 32 * wpb, smem, st>>>(rows7, offsets, n_pack, cap, mu,
                                                                 out_score, out_fsr);
    return cudaGetLastError();
}

cudaError_t launch_item_order(const long long* vols, const int* qty, const int* type_off,
                              const int* n_types, const long long* step_off, int n_inst, int order,
                              int* out_types, int sort_cap, cudaStream_t st) {
    const int smem = 8 * sort_cap;
    cudaError_t e = ensure_dyn_smem(reinterpret_cast<const void*>(item_order_kernel), smem);
    if (e != cudaSuccess) return e;
    item_order_kernel<<<n_inst, 256, smem, st>>>(vols, qty, type_off, n_types, step_off, order,
                                                 out_types, sort_cap);
    return cudaGetLastError();
}

cudaError_t launch_gather_best(const InstDesc* inst, int n_inst, const int2* best,
                               const unsigned long long* places, unsigned long long* out,
                               int out_stride, cudaStream_t st) {
    const int wpb = 8;
    gather_best_kernel<<<(n_inst + wpb - 1) / wpb, 32 * wpb, 0, st>>>(inst, n_inst, best, places, out,
                                                                     out_stride);
    return cudaGetLastError();
}

#endif  // PLP_SERVE_TU

#ifdef PLP_SERVE_TU
// The serving launch: the single-warp decoder over the host-published ring.
template <int D, int M, int S16>
__global__ void __launch_bounds__(32 * D, M) serve_kernel(DecoderArgs a, ServeArgs s) {
    using SupT = typename std::conditional<S16 != 0, unsigned short, int>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dec = threadIdx.x >> 5;
    const int gdec = blockIdx.x * D + dec;
    if (gdec < s.n_deep) {
        DecoderArgs ad = a;
        ad.P = s.deep_P;
        ad.C = s.deep_C;
        decoder1_body<SupT, 2>(ad, s.deep_scratch + (size_t)gdec * s.deep_bytes, gdec, s);
    } else {
        const Dec1Layout lay = dec1_layout(a.P, a.C, a.Hz, (int)sizeof(SupT));
        decoder1_body<SupT, 1>(a, smem_raw + (size_t)dec * lay.bytes, gdec, s);
    }
}

// ---- serving launches ------------------------------------------------------
using ServeFn = void (*)(DecoderArgs, ServeArgs);
#define PLP_SERVE_CONFIGS(X) X(1, 1) X(1, 12)

static ServeFn serve_fn(int D, int M, int sup16) {
#define PLP_PICK_SERVE(d, m) \
    if (D == d && M == m) return sup16 ? serve_kernel<d, m, 1> : serve_kernel<d, m, 0>;
    PLP_SERVE_CONFIGS(PLP_PICK_SERVE)
#undef PLP_PICK_SERVE
    return nullptr;
}

bool serve_config_supported(int D, int M) { return serve_fn(D, M, 0) != nullptr; }

cudaError_t serve_occupancy(int P, int C, int Hz, int D, int M, int sup16, int* ctas_per_sm) {
    ServeFn fn = serve_fn(D, M, sup16);
    if (!fn) return cudaErrorInvalidConfiguration;
    const int smem = decoder_smem_bytes(P, C, Hz, 1, sup16) * D;
    cudaError_t e = ensure_dyn_smem(reinterpret_cast<const void*>(fn), smem);
    if (e != cudaSuccess) return e;
    return cached_occupancy(reinterpret_cast<const void*>(fn), 32 * D, smem, ctas_per_sm);
}

cudaError_t launch_serve(const DecodeLaunch& L, const ServeArgs& s, cudaStream_t st) {
    ServeFn fn = serve_fn(L.decoders_per_cta, L.min_blocks, L.sup16);
    if (!fn || L.warps_per_decoder != 1 || L.engine != 0) return cudaErrorInvalidConfiguration;
    const int smem = decoder_smem_bytes(L.P, L.C, L.Hz, 1, L.sup16) * L.decoders_per_cta;
    cudaError_t e = ensure_dyn_smem(reinterpret_cast<const void*>(fn), smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(L.abort, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    fn<<<L.ctas, 32 * L.decoders_per_cta, smem, st>>>(decoder_args(L), s);
    return cudaGetLastError();
}

#endif  // PLP_SERVE_TU

}  // namespace plpb
