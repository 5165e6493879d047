// feas_eval.cuh -- C1/C2/C3 of one candidate point against all orientations
// of an item type, over placed boxes held sorted by top z. Shared by the
// one-step kernel (feas.cu) and the persistent decoder (decoder.cu).
//
// Reference: check_feasible_one, gpu/plp_common.hpp:297-321 (C2, then C3 with
// the FP64 ratio (double)s / (double)(w*d) < 0.5, then C1); the boolean per
// (point, orientation) is identical:
//  * C2 is the same integer test per orientation;
//  * C3 (z > 0) sums the same integer overlap areas over the boxes whose top
//    is exactly z (the only ones the reference adds) and applies the same
//    FP64 ratio test;
//  * C1 visits only boxes whose top is above z: a box with top <= z fails the
//    reference's `z < b.z2` term and can never overlap.
#pragma once

#include "device_common.cuh"

namespace plpb {

struct Boxes {
    const int4* bx;   // {x, y, x2, y2}
    const int* bz;    // bottom z
    const int* z2;    // top z, ascending
    int n;
};

__device__ __forceinline__ int lower_bound_top(const int* z2, int n, int z) {
    int lo = 0;
    while (n > 0) {
        const int half = n >> 1;
        if (z2[lo + half] < z) {
            lo += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return lo;
}

// First box with top >= z from the top-z index zt (zt[z] = boxes with top
// < z), or by binary search when there is no index.
__device__ __forceinline__ int box_start(const unsigned short* zt, const int* z2, int nb, int z) {
    return zt ? (int)zt[z] : lower_bound_top(z2, nb, z);
}

// Bit o of the result: orientation o (w = ow[o], d = od[o], h = oh[o]) at
// point (x, y, z) is feasible. Acc is the support-area accumulator type
// (int when the container area is known to fit, long long otherwise).
template <typename Acc>
__device__ __forceinline__ unsigned eval_point(int x, int y, int z, const int (&ow)[6],
                                               const int (&od)[6], const int (&oh)[6], int no,
                                               int L, int W, int H, const Boxes& B) {
    unsigned alive = 0;
#pragma unroll
    for (int o = 0; o < 6; o++)
        if (o < no && !(x + ow[o] > L || y + od[o] > W || z + oh[o] > H)) alive |= 1u << o;   // C2
    if (!alive) return 0;
    int j = lower_bound_top(B.z2, B.n, z);
    if (z > 0) {                                                                             // C3
        Acc s[6] = {0, 0, 0, 0, 0, 0};
        for (; j < B.n && B.z2[j] == z; j++) {
            const int4 b = B.bx[j];
#pragma unroll
            for (int o = 0; o < 6; o++) {
                const Acc ox = (Acc)min(x + ow[o], b.z) - (Acc)max(x, b.x);
                const Acc oy = (Acc)min(y + od[o], b.w) - (Acc)max(y, b.y);
                if (ox > 0 && oy > 0) s[o] += ox * oy;
            }
        }
#pragma unroll
        for (int o = 0; o < 6; o++)
            if (((alive >> o) & 1u) && (double)s[o] / (double)(ow[o] * od[o]) < 0.5)
                alive &= ~(1u << o);
        if (!alive) return 0;
    } else {
        while (j < B.n && B.z2[j] == z) j++;   // top == z: cannot overlap
    }
    for (; j < B.n; j++) {                                                                   // C1
        const int4 b = B.bx[j];
        if (x < b.z && y < b.w) {
            const int bz = B.bz[j];
#pragma unroll
            for (int o = 0; o < 6; o++)
                if (b.x < x + ow[o] && b.y < y + od[o] && bz < z + oh[o]) alive &= ~(1u << o);
            if (!alive) break;
        }
    }
    return alive;
}

}  // namespace plpb
