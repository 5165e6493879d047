// device_common.cuh -- tables shared by host and device, and device helpers
// (CPython-exact MT19937 with a warp-cooperative twist, point keys).
//
// All device code is compiled with --fmad=false so no double expression is
// contracted; every FP64 expression keeps the reference operand order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace plpb {

constexpr unsigned FULL = 0xffffffffu;

// One instance of a batched solve (device copy). Points (x, y, z) are packed
// into 32-bit keys z << (xb + yb) | y << xb | x, whose numeric order is the
// reference candidate order (z, y, x) (gpu/plp_common.hpp:282-291).
struct InstDesc {
    int L, W, H;
    int n_steps;         // decode steps (items in sequence order)
    int step_off;        // first entry in the step-type table
    int type_off;        // first entry in the orientation table
    int xb, yb;          // key field widths (bit length of L and W)
    int restarts;
    int slot_base;       // result slot of restart 0
    int place_stride;    // placement capacity per slot (= n_steps)
    int passes;
    long long place_off; // first placement of restart 0
    long long seed;      // restart k is seeded with |seed + k|
    double eps, theta, mu;
    int has_theta, first_fit;
    long long budget_ns; // >= 0: passes (at most `passes`) until this much
                         // global-timer time has passed since the restart began
    // block-building engine (engine == 1): offsets of this instance's tables
    // in the launch's block table (ints) and shape catalogue
    int engine;          // 0 extreme-point decoder, 1 block-building engine
    int n_types;
    int blk_topk, blk_pick;
    int bo_order;        // types by (volume desc, index)
    int bo_qty;          // copies per type
    int bo_list;         // per type: catalogue indices in shape precedence order
    int bo_list_off;     // n_types + 1 offsets into that list
    int bo_start;        // per type: first fitting list index for r < max count
    int bo_start_off;    // n_types + 1 offsets into that table
    int bo_shape_of_rank;
    int cat_off, n_cat;
};

// Block shape of the block-building engine (blockproof/plp_block.cpp:29-37):
// cnt = a*b*k copies of type ti in orientation oi as a bw x bd x bh stack;
// rank = its position in the placement order (block volume desc, type,
// orientation, k desc, a desc, b desc; blockproof/plp_block.cpp:165-175).
struct BlkShape {
    int ti, oi, a, b, k, cnt, bw, bd, bh, rank;
};

// Nanoseconds of the GPU's global timer (one clock for all SMs).
__device__ __forceinline__ long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (long long)t;
}

// Orientation table entry of one box type: up to 6 (w, d, h), dedup'd in the
// reference's parser order (gpu/plp_common.hpp:269-280); unused slots are 0.
struct TypeOrs {
    int n;
    int w[6], d[6], h[6];
    int pad[3];
};
static_assert(sizeof(TypeOrs) == 88, "TypeOrs layout");

// Per-restart result head. The placements of the selected pass follow in the
// placement table, one packed 64-bit word each (see pack_place).
struct SlotHead {
    int n_boxes;
    int err;             // 0 or a DecodeErr value
    long long volume;
    double score;
    int n_passes;
    int fallback;        // 1: no pass reached theta (reference D4' flag)
};
static_assert(sizeof(SlotHead) == 32, "SlotHead layout");

enum DecodeErr : int {
    ERR_NONE = 0,
    ERR_BOX_CAP = 1,     // more placed boxes than the shared-memory tile holds
    ERR_CAND_CAP = 2,    // more live extreme points than the tile holds
    ERR_RNG = 3,         // randrange rejection loop exceeded its bound
    ERR_SYNC = 4,        // a decoder's warps stopped meeting at a barrier (wait bound hit)
};

// placement word: x | y << 16 | z << 32 | orientation << 48 | type << 51
__host__ __device__ inline unsigned long long pack_place(int x, int y, int z, int oi, int type) {
    return (unsigned long long)(unsigned)x | ((unsigned long long)(unsigned)y << 16) |
           ((unsigned long long)(unsigned)z << 32) | ((unsigned long long)(unsigned)oi << 48) |
           ((unsigned long long)(unsigned)type << 51);
}
__host__ __device__ inline void unpack_place(unsigned long long v, int& x, int& y, int& z,
                                             int& oi, int& type) {
    x = (int)(v & 0xffff);
    y = (int)((v >> 16) & 0xffff);
    z = (int)((v >> 32) & 0xffff);
    oi = (int)((v >> 48) & 7);
    type = (int)(v >> 51);
}

#ifdef __CUDACC__

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// MT19937 (Matsumoto & Nishimura), CPython seeding and draws.
// State lives in shared memory, the read position in a warp-uniform register;
// every lane of the warp calls the draw functions with identical arguments.
// ---------------------------------------------------------------------------

// init_by_array on |seed| (one or two 32-bit key words), starting from the
// seed-independent init_genrand(19650218) table `init`. The recurrence is
// serial: lane 0 runs it, the warp then syncs.
static __device__ __noinline__ void mt_seed_warp(uint32_t* mt, unsigned long long seed_abs,
                                    const uint32_t* __restrict__ init, int lane) {
    for (int i = lane; i < 624; i += 32) mt[i] = init[i];
    __syncwarp();
    if (lane == 0) {
        // Key word j of step k is k mod nkey; its addend is key[j] + j.
        const uint32_t k0 = (uint32_t)seed_abs;
        const uint32_t k1 = (uint32_t)(seed_abs >> 32);
        const uint32_t add0 = k0, add1 = k1 ? k1 + 1u : k0;
        // First loop: 624 steps over i = 1 .. 623, then i = 1 again. Blocks
        // of 8 with their old words loaded up front keep the load latency
        // off the serial chain.
        uint32_t prev = mt[0];
        for (int i = 1; i < 624; i += 8) {
            uint32_t o[8];
#pragma unroll
            for (int u = 0; u < 8; u++) o[u] = i + u < 624 ? mt[i + u] : 0u;
#pragma unroll
            for (int u = 0; u < 8; u++) {
                if (i + u < 624) {
                    const uint32_t t = prev ^ (prev >> 30);
                    prev = (o[u] ^ (t * 1664525u)) + (((i + u - 1) & 1) ? add1 : add0);
                    mt[i + u] = prev;
                }
            }
        }
        {
            const uint32_t t = prev ^ (prev >> 30);
            prev = (mt[1] ^ (t * 1664525u)) + add1;   // step 623 (odd)
            mt[1] = prev;
        }
        // Second loop: 623 steps over i = 2 .. 623, then i = 1.
        for (int i = 2; i < 624; i += 8) {
            uint32_t o[8];
#pragma unroll
            for (int u = 0; u < 8; u++) o[u] = i + u < 624 ? mt[i + u] : 0u;
#pragma unroll
            for (int u = 0; u < 8; u++) {
                if (i + u < 624) {
                    const uint32_t t = prev ^ (prev >> 30);
                    prev = (o[u] ^ (t * 1566083941u)) - (uint32_t)(i + u);
                    mt[i + u] = prev;
                }
            }
        }
        {
            const uint32_t t = prev ^ (prev >> 30);
            mt[1] = (mt[1] ^ (t * 1566083941u)) - 1u;
        }
        mt[0] = 0x80000000u;
    }
    __syncwarp();
}

// Regenerates all 624 words. Word i needs old words i, i+1 and word
// (i + 397) mod 624, which is still old for i < 227 and already new for
// i >= 227. Chunks of 32 in increasing i therefore only read finished or
// untouched words; inside a chunk all lanes read before any lane writes.
static __device__ __noinline__ void mt_twist_warp(uint32_t* mt, int lane) {
    for (int base = 0; base < 623; base += 32) {
        const int i = base + lane;
        uint32_t nv = 0;
        if (i < 623) {
            const uint32_t y = (mt[i] & 0x80000000u) | (mt[i + 1] & 0x7fffffffu);
            const int k = i < 227 ? i + 397 : i - 227;
            nv = mt[k] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        __syncwarp();
        if (i < 623) mt[i] = nv;
        __syncwarp();
    }
    if (lane == 0) {
        const uint32_t y = (mt[623] & 0x80000000u) | (mt[0] & 0x7fffffffu);
        mt[623] = mt[396] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    __syncwarp();
}

__device__ __forceinline__ uint32_t mt_next(uint32_t* mt, int& pos, int lane) {
    if (pos >= 624) {
        mt_twist_warp(mt, lane);
        pos = 0;
    }
    uint32_t y = mt[pos++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

// CPython random(): (a * 2^26 + b) / 2^53 with a = 27 bits, b = 26 bits.
__device__ __forceinline__ double mt_random(uint32_t* mt, int& pos, int lane) {
    const uint32_t a = mt_next(mt, pos, lane) >> 5;
    const uint32_t b = mt_next(mt, pos, lane) >> 6;
    return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

// CPython randrange(n), n >= 1: getrandbits(bit_length(n)) until < n.
// Returns -1 if the (astronomically unlikely) rejection bound is hit.
__device__ __forceinline__ int mt_randrange(uint32_t* mt, int& pos, int lane, int n) {
    const int k = 32 - __clz(n);
    for (int tries = 0; tries < 4096; tries++) {
        const uint32_t r = mt_next(mt, pos, lane) >> (32 - k);
        if (r < (uint32_t)n) return (int)r;
    }
    return -1;
}

#endif  // __CUDACC__

}  // namespace plpb
