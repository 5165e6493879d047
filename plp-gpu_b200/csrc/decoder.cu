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
// Layout of one decoder (a warp) in shared memory:
//   MT19937 state       624 x u32
//   placed boxes        sorted by top z (ascending): {x, y, x2, y2} int4,
//                       bottom z, top z, placement index
//   live points         sorted unique keys (z, y, x), double buffer
//   point masks         one byte per live point (random branch)
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
//    same integer test; C3 sums the same integer overlap areas and keeps the
//    reference's FP64 ratio test (double)s / (double)(w*d) < 0.5; C1 only
//    visits boxes whose top lies above z (a box with top <= z cannot overlap
//    a box starting at z), which does not change the boolean.
//  * The first feasible pair (greedy branch) is found by scanning points in
//    order; random() is drawn only after one feasible pair exists, and the
//    full count / idx-th selection runs only on the random branch.
#include "device_common.cuh"
#include "engine.hpp"
#include "feas_eval.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace plpb {

// ---------------------------------------------------------------------------
// shared-memory layout of one decoder
// ---------------------------------------------------------------------------
struct DecLayout {
    int off_bx, off_bz, off_z2, off_bi, off_ca, off_cb, off_cm, bytes;
};

__host__ __device__ inline DecLayout dec_layout(int P, int C) {
    DecLayout l;
    int o = 624 * 4;                       // MT state
    o = (o + 15) & ~15;
    l.off_bx = o;  o += 16 * P;            // int4 {x, y, x2, y2}
    l.off_bz = o;  o += 4 * P;             // bottom z
    l.off_z2 = o;  o += 4 * P;             // top z
    l.off_bi = o;  o += 2 * P;             // placement index
    o = (o + 15) & ~15;
    l.off_ca = o;
    // point buffers: 2 x C keys + C mask bytes; FSR overlays 18 bytes per box
    int region = 9 * C;
    if (region < 18 * P + 32) region = 18 * P + 32;
    l.off_cb = o + 4 * C;
    l.off_cm = o + 8 * C;
    o += region;
    o = (o + 15) & ~15;
    l.bytes = o;
    return l;
}

int decoder_smem_bytes(int P, int C) { return dec_layout(P, C).bytes; }

struct DecoderArgs {
    const InstDesc* __restrict__ inst;
    const int* __restrict__ step_type;
    const TypeOrs* __restrict__ types;
    const int2* __restrict__ work;
    int n_work;
    int* work_next;
    int* err_flag;
    SlotHead* heads;
    unsigned long long* places;
    unsigned long long* scratch;   // per resident warp: passes > 1
    const uint32_t* __restrict__ mt_init;
    int P, C;
    int dec_bytes;
    int decoders_per_cta;
};

// ---------------------------------------------------------------------------
// FSR of the packing held in the box tables (warp). Load flows from each box
// k, taken in (z desc, placement index asc) order, to the boxes whose top is
// k's bottom, proportionally to the integer contact area. Levels are handled
// in descending z; inside a level the boxes k are taken in index order and
// the supports j are updated in parallel (each j by one lane), so every
// load[j] receives its additions in the reference order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fsr_score_warp(const int4* bx, const int* bz, const int* z2,
                                 const unsigned short* bi, int n, double mu, char* scratch,
                                 int lane, double* fsr_out) {
    if (n == 0) return 0.0;
    double* load = reinterpret_cast<double*>(scratch);               // by sorted position
    uint32_t* key = reinterpret_cast<uint32_t*>(scratch + 8 * n);    // sort keys
    int* tot = reinterpret_cast<int*>(scratch + 12 * n);             // contact total per box
    unsigned short* pos = reinterpret_cast<unsigned short*>(scratch + 16 * n);  // idx -> pos
    int npad = 1;
    while (npad < n) npad <<= 1;
    // sort keys: (0xffff - z) << 16 | idx  ->  ascending = z desc, idx asc.
    // npad may exceed n; the tail lives in the tot[] area, which is filled after.
    for (int p = lane; p < npad; p += 32) {
        key[p] = p < n ? ((uint32_t)(0xffff - bz[p]) << 16) | bi[p] : 0xffffffffu;
        if (p < n) pos[bi[p]] = (unsigned short)p;
    }
    __syncwarp();
    // bitonic sort in shared memory (ascending)
    for (int k = 2; k <= npad; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < npad; i += 32) {
                const int l = i ^ j;
                if (l > i) {
                    const uint32_t a = key[i], b = key[l];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        key[i] = b;
                        key[l] = a;
                    }
                }
            }
            __syncwarp();
        }
    }
    // masses and contact totals
    for (int p = lane; p < n; p += 32) {
        const int4 b = bx[p];
        const int h = z2[p] - bz[p];
        const long long vol = 1LL * (b.z - b.x) * (b.w - b.y) * h;
        load[p] = 50.0 * (double)vol / 1e6;
    }
    __syncwarp();
    for (int p = lane; p < n; p += 32) {
        const int4 b = bx[p];
        const int zb = bz[p];
        int t = 0;
        if (zb > 0) {
            for (int j = lower_bound_top(z2, n, zb); j < n && z2[j] == zb; j++) {
                const int4 c = bx[j];
                const int ox = min(b.z, c.z) - max(b.x, c.x);
                if (ox <= 0) continue;
                const int oy = min(b.w, c.w) - max(b.y, c.y);
                if (oy > 0) t += ox * oy;
            }
        }
        tot[p] = t;   // overwrites the sort padding, which is no longer read
    }
    __syncwarp();
    // propagate, level by level in (z desc, index asc) order
    int q = 0;
    while (q < n) {
        const int k0 = pos[key[q] & 0xffff];
        const int zl = bz[k0];
        int qe = q;
        while (qe < n && (int)(0xffff - (key[qe] >> 16)) == zl) qe++;
        if (zl > 0) {
            const int jlo = lower_bound_top(z2, n, zl);
            int jhi = jlo;
            while (jhi < n && z2[jhi] == zl) jhi++;
            for (int jb = jlo; jb < jhi; jb += 32) {
                const int j = jb + lane;
                if (j < jhi) {
                    const int4 c = bx[j];
                    double lj = load[j];
                    for (int qq = q; qq < qe; qq++) {
                        const int k = pos[key[qq] & 0xffff];
                        const int total = tot[k];
                        if (total <= 0) continue;
                        const int4 b = bx[k];
                        const int ox = min(b.z, c.z) - max(b.x, c.x);
                        if (ox <= 0) continue;
                        const int oy = min(b.w, c.w) - max(b.y, c.y);
                        if (oy <= 0) continue;
                        lj += load[k] * (double)(ox * oy) / (double)total;
                    }
                    load[j] = lj;
                }
            }
        }
        __syncwarp();
        q = qe;
    }
    int cnt = 0;
    for (int p = lane; p < n; p += 32) {
        const int4 b = bx[p];
        const long long vol = 1LL * (b.z - b.x) * (b.w - b.y) * (z2[p] - bz[p]);
        const double m = 50.0 * (double)vol / 1e6;
        const double f = (mu / 0.3) * load[p] / m;
        if (fsr_out) fsr_out[bi[p]] = f;
        cnt += f >= 1.0;
    }
    cnt = __reduce_add_sync(FULL, cnt);
    return (double)cnt / (double)n;
}

// ---------------------------------------------------------------------------
// the persistent decoder kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) decoder_kernel(DecoderArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const DecLayout lay = dec_layout(a.P, a.C);
    unsigned char* base = smem_raw + (size_t)wid * a.dec_bytes;
    uint32_t* mt = reinterpret_cast<uint32_t*>(base);
    int4* bx = reinterpret_cast<int4*>(base + lay.off_bx);
    int* bzs = reinterpret_cast<int*>(base + lay.off_bz);
    int* z2s = reinterpret_cast<int*>(base + lay.off_z2);
    unsigned short* bis = reinterpret_cast<unsigned short*>(base + lay.off_bi);
    uint32_t* candA = reinterpret_cast<uint32_t*>(base + lay.off_ca);
    uint32_t* candB = reinterpret_cast<uint32_t*>(base + lay.off_cb);
    unsigned char* cmask = base + lay.off_cm;
    const int gwarp = blockIdx.x * a.decoders_per_cta + wid;

    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.work_next, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.n_work) break;
        const int2 w = a.work[item];
        const InstDesc I = a.inst[w.x];
        const int restart = w.y;
        const int slot = I.slot_base + restart;
        const int L = I.L, W = I.W, H = I.H;
        const uint32_t xmask = (1u << I.xb) - 1u, ymask = (1u << I.yb) - 1u;
        const int xb = I.xb, xyb = I.xb + I.yb;
        const bool randomized = !(I.first_fit || I.eps == 0.0);
        unsigned long long* best_out = a.places + I.place_off + (long long)restart * I.place_stride;
        unsigned long long* pass_out =
            I.passes > 1 ? a.scratch + (long long)gwarp * I.place_stride : best_out;

        long long s = I.seed + restart;
        const unsigned long long sabs = (unsigned long long)(s < 0 ? -s : s);
        mt_seed_warp(mt, sabs, a.mt_init, lane);
        int mpos = 624;

        int err = ERR_NONE;
        bool have_acc = false, have_any = false;
        long long best_vol = 0;
        int best_n = 0;
        double best_score = 0.0;

        for (int pass = 0; pass < I.passes && err == ERR_NONE; pass++) {
            int nb = 0, nc = 1;
            long long vol = 0;
            if (lane == 0) candA[0] = 0u;
            __syncwarp();
            for (int st = 0; st < I.n_steps; st++) {
                const int t = a.step_type[I.step_off + st];
                const TypeOrs& T = a.types[I.type_off + t];
                const int no = T.n;
                if (no == 0) continue;
                int ow[6], od[6], oh[6];
#pragma unroll
                for (int o = 0; o < 6; o++) {
                    ow[o] = T.w[o];
                    od[o] = T.d[o];
                    oh[o] = T.h[o];
                }
                const Boxes B{bx, bzs, z2s, nb};
                // scan live points in order: greedy stops at the first chunk
                // holding a feasible pair; the random branch scans on and
                // records every point's mask
                int first_ci = -1, first_oi = 0, count = 0;
                bool full = false;
                for (int cb = 0; cb < nc; cb += 32) {
                    const int ci = cb + lane;
                    unsigned m = 0;
                    if (ci < nc) {
                        const uint32_t key = candA[ci];
                        m = eval_point<int>((int)(key & xmask), (int)((key >> xb) & ymask),
                                       (int)(key >> xyb), ow, od, oh, no, L, W, H, B);
                    }
                    if (!full) {
                        const unsigned bal = __ballot_sync(FULL, m != 0);
                        if (!bal) continue;
                        const int l = __ffs(bal) - 1;
                        first_ci = cb + l;
                        first_oi = __ffs(__shfl_sync(FULL, m, l)) - 1;
                        if (!randomized) break;
                        const double u = mt_random(mt, mpos, lane);
                        if (u < 1.0 - I.eps) break;
                        full = true;
                    }
                    if (ci < nc) cmask[ci] = (unsigned char)m;
                    count += __reduce_add_sync(FULL, __popc(m));
                }
                if (first_ci < 0) continue;               // no feasible pair: skip this copy
                int pick_ci = first_ci, pick_oi = first_oi;
                if (full) {
                    __syncwarp();
                    const int idx = mt_randrange(mt, mpos, lane, count);
                    if (idx < 0) { err = ERR_RNG; break; }
                    // idx-th feasible pair in (point, orientation) order
                    int run = 0;
                    const int cb0 = first_ci & ~31;
                    for (int cb = cb0; cb < nc; cb += 32) {
                        const int ci = cb + lane;
                        const unsigned m = ci < nc && ci >= first_ci ? cmask[ci] : 0u;
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
                            pick_ci = cb + l;
                            pick_oi = __fns(ml, 0, idx - run - excl + 1);
                            break;
                        }
                        run += tot;
                    }
                }
                // ---- place the box ----
                const uint32_t pkey = candA[pick_ci];
                const int px = (int)(pkey & xmask), py = (int)((pkey >> xb) & ymask),
                          pz = (int)(pkey >> xyb);
                int pw = 0, pd = 0, ph = 0;
#pragma unroll
                for (int o = 0; o < 6; o++)
                    if (o == pick_oi) { pw = ow[o]; pd = od[o]; ph = oh[o]; }
                const int px2 = px + pw, py2 = py + pd, pz2 = pz + ph;
                if (nb >= a.P) { err = ERR_BOX_CAP; break; }
                if (lane == 0) pass_out[nb] = pack_place(px, py, pz, pick_oi, t);
                vol += 1LL * pw * pd * ph;

                // ---- live-point update ----
                // corners of the new box covered by an already placed box
                unsigned cov = 1u;   // corner 0 = (px, py, pz) is covered by the new box
                for (int j = lane; j < nb; j += 32) {
                    const int4 b = bx[j];
                    const int bzb = bzs[j], bzt = z2s[j];
                    const unsigned xin = (b.x <= px && px < b.z ? 1u : 0u) | (b.x <= px2 && px2 < b.z ? 2u : 0u);
                    const unsigned yin = (b.y <= py && py < b.w ? 1u : 0u) | (b.y <= py2 && py2 < b.w ? 2u : 0u);
                    const unsigned zin = (bzb <= pz && pz < bzt ? 1u : 0u) | (bzb <= pz2 && pz2 < bzt ? 2u : 0u);
#pragma unroll
                    for (int c = 0; c < 8; c++)
                        if (((xin >> (c & 1)) & (yin >> ((c >> 1) & 1)) & (zin >> (c >> 2))) & 1u)
                            cov |= 1u << c;
                }
                cov = __reduce_or_sync(FULL, cov);
                // survivors: points not covered by the new box, compacted into candB
                int ns = 0;
                for (int cb = 0; cb < nc; cb += 32) {
                    const int i = cb + lane;
                    bool keep = false;
                    uint32_t key = 0;
                    if (i < nc) {
                        key = candA[i];
                        const int x = (int)(key & xmask), y = (int)((key >> xb) & ymask),
                                  z = (int)(key >> xyb);
                        keep = !(px <= x && x < px2 && py <= y && y < py2 && pz <= z && z < pz2);
                    }
                    const unsigned bal = __ballot_sync(FULL, keep);
                    if (keep) candB[ns + __popc(bal & lanemask_lt())] = key;
                    ns += __popc(bal);
                }
                __syncwarp();
                // new corners: sorted by index c = (cz << 2) | (cy << 1) | cx,
                // which is also their (z, y, x) order
                uint32_t ck = 0;
                int rank = 0;
                bool isnew = false;
                if (lane < 8 && !((cov >> lane) & 1u)) {
                    const int cx = (lane & 1) ? px2 : px, cy = (lane & 2) ? py2 : py,
                              cz = (lane & 4) ? pz2 : pz;
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
                if (nnew > a.C) { err = ERR_CAND_CAP; break; }
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
                // insert the box into the top-z-sorted tables (after equal tops)
                int ip = 0;
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
                nb++;
                __syncwarp();
            }
            if (err != ERR_NONE) break;
            // ---- score the pass and keep the selected one ----
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
            __syncwarp();
        }
        if (lane == 0) {
            if (err) atomicOr(a.err_flag, 1 << err);
            SlotHead h;
            h.n_boxes = err ? 0 : best_n;
            h.err = err;
            h.volume = err ? 0 : best_vol;
            h.score = err ? 0.0 : best_score;
            h.n_passes = I.passes;
            h.fallback = have_acc ? 0 : 1;
            a.heads[slot] = h;
        }
        __syncwarp();
    }
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
    // key: accepted, volume, n_boxes, then the smallest restart wins
    int br = -1, bacc = 0, bn = 0;
    long long bv = -1;
    for (int r = lane; r < I.restarts; r += 32) {
        const SlotHead h = heads[I.slot_base + r];
        const int acc = h.fallback ? 0 : 1;
        const bool better = br < 0 || acc > bacc ||
                            (acc == bacc && (h.volume > bv || (h.volume == bv && h.n_boxes > bn)));
        if (better) { br = r; bacc = acc; bv = h.volume; bn = h.n_boxes; }
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
    if (lane == 0) best[i] = make_int2(br, bacc ? 0 : 1);
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
cudaError_t launch_decoder(const DecodeLaunch& L, cudaStream_t st) {
    DecoderArgs a;
    a.inst = L.inst;
    a.step_type = L.step_type;
    a.types = L.types;
    a.work = L.work;
    a.n_work = L.n_work;
    a.work_next = L.work_next;
    a.err_flag = L.err_flag;
    a.heads = L.heads;
    a.places = L.places;
    a.scratch = L.scratch;
    a.mt_init = L.mt_init;
    a.P = L.P;
    a.C = L.C;
    a.dec_bytes = decoder_smem_bytes(L.P, L.C);
    a.decoders_per_cta = L.decoders_per_cta;
    const int smem = a.dec_bytes * L.decoders_per_cta;
    cudaError_t e = cudaFuncSetAttribute(decoder_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(L.work_next, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    decoder_kernel<<<L.ctas, 32 * L.decoders_per_cta, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t decoder_occupancy(int P, int C, int decoders_per_cta, int* ctas_per_sm) {
    const int smem = decoder_smem_bytes(P, C) * decoders_per_cta;
    cudaError_t e = cudaFuncSetAttribute(decoder_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, decoder_kernel,
                                                         32 * decoders_per_cta, smem);
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
    cudaError_t e = cudaFuncSetAttribute(fsr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    fsr_kernel<<<(n_pack + wpb - 1) / wpb, 32 * wpb, smem, st>>>(rows7, offsets, n_pack, cap, mu,
                                                                 out_score, out_fsr);
    return cudaGetLastError();
}

cudaError_t launch_item_order(const long long* vols, const int* qty, const int* type_off,
                              const int* n_types, const long long* step_off, int n_inst, int order,
                              int* out_types, int sort_cap, cudaStream_t st) {
    const int smem = 8 * sort_cap;
    cudaError_t e = cudaFuncSetAttribute(item_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
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

}  // namespace plpb
