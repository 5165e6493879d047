// fsr_warp.cuh -- FSR stability score of one packing by one warp, over the
// packing's boxes held sorted by top z in shared memory. Shared by the
// extreme-point decoder (decoder.cu), the block engine (block.cu) and the
// standalone fsr_kernel.
#pragma once

#include "device_common.cuh"
#include "feas_eval.cuh"

namespace plpb {

// ---------------------------------------------------------------------------
// FSR of the packing held in the box tables (warp). Load flows from each box
// k, taken in (z desc, placement index asc) order, to the boxes whose top is
// k's bottom, proportionally to the integer contact area. Levels are handled
// in descending z; inside a level the boxes k are taken in index order and
// the supports j are updated in parallel (each j by one lane), so every
// load[j] receives its additions in the reference order.
// ---------------------------------------------------------------------------
// zt (may be null): the top-z index zt[z] = number of boxes with top < z, so
// the boxes with top exactly z are [zt[z], zt[z + 1]) without a search.
static __device__ __noinline__ double fsr_score_warp(const int4* bx, const int* bz, const int* z2,
                                 const unsigned short* bi, int n, double mu, char* scratch,
                                 int lane, double* fsr_out, const unsigned short* zt = nullptr) {
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
            const int j0 = zt ? (int)zt[zb] : lower_bound_top(z2, n, zb);
            for (int j = j0; j < n && z2[j] == zb; j++) {
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
            int jlo, jhi;
            if (zt) {
                jlo = zt[zl];
                jhi = zt[zl + 1];
            } else {
                jlo = lower_bound_top(z2, n, zl);
                jhi = jlo;
                while (jhi < n && z2[jhi] == zl) jhi++;
            }
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

}  // namespace plpb
