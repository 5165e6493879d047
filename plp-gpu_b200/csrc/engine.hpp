// engine.hpp -- host-side launchers of the device kernels (internal).
#pragma once

#include <cuda_runtime.h>

#include "device_common.cuh"

namespace plpb {

struct DecodeLaunch {
    const InstDesc* inst;
    const int* step_type;
    const TypeOrs* types;
    const int2* work;
    int n_work;
    const int* n_work_dev;    // set: the work count is read here at kernel start (n_work bounds it)
    int* work_next;
    int* err_flag;            // OR of (1 << err) over restarts that failed
    int* abort;               // set when a bounded barrier wait gives up
    SlotHead* heads;
    unsigned long long* places;
    unsigned long long* scratch;
    const uint32_t* mt_init;
    int P, C;                 // shared-memory tile: boxes and live points per decoder
    int Hz;                   // entries of the top-z index (max height + 2), 0 = none
    int engine;               // 0 extreme-point decoder, 1 block-building engine
    int sup16;                // decoder: contact areas stored as 16-bit
    const BlkShape* bcat;     // block engine: shape catalogue of the batch
    const int* btab;          // block engine: per-instance orderings (ints)
    int N, T;                 // block engine tile: items, types per decoder
    int warps_per_decoder;    // G
    int decoders_per_cta;     // D
    int min_blocks;           // M (register cap through the launch bounds)
    int ctas;
    int sync_limit;           // test hook: tries per barrier wait (0 = the kernel's bound)
    int sync_skip;            // test hook: 1 + the warp that skips its first arrive (0 = none)
    const uint32_t* seed_tab; // seeded MT states of seeds seed_lo .. seed_lo + seed_n - 1 (null: seed in place)
    long long seed_lo;
    int seed_n;
};
// seeded MT states of seeds lo .. lo + n - 1, 624 words each
cudaError_t launch_seed_table(long long lo, int n, const uint32_t* mt_init, uint32_t* out, cudaStream_t st);

int decoder_smem_bytes(int P, int C, int Hz, int G, int sup16 = 0);   // sup16: 16-bit contact areas
bool decoder_config_supported(int G, int D, int M);
cudaError_t decoder_occupancy(int P, int C, int Hz, int G, int D, int M, int* ctas_per_sm, int sup16 = 0);
cudaError_t launch_decoder(const DecodeLaunch& L, cudaStream_t st);     // configure + enqueue
cudaError_t configure_decoder(const DecodeLaunch& L);                    // function attributes
cudaError_t enqueue_decoder(const DecodeLaunch& L, cudaStream_t st);     // stream operations only
// block-building engine (block.cu); one warp per restart, D decoders per CTA
int block_smem_bytes(int P, int C, int N, int T, int Hz);
bool block_config_supported(int D, int M);
cudaError_t block_occupancy(int P, int C, int N, int T, int Hz, int D, int M, int* ctas_per_sm);
cudaError_t configure_block(const DecodeLaunch& L);
cudaError_t enqueue_block(const DecodeLaunch& L, cudaStream_t st);
// Per-device caches of kernel launch attributes: the dynamic shared-memory
// limit is raised only when a launch needs more than every earlier launch of
// the kernel on the device, and occupancy is queried once per (kernel,
// device, block size, shared memory). Both calls change or read per-kernel
// driver state, and made per solve they cost more than a small solve's host side.
cudaError_t ensure_dyn_smem(const void* fn, int smem);
cudaError_t cached_occupancy(const void* fn, int threads, int smem, int* ctas_per_sm);

// work items whose restart overflowed its tile, appended to redo (count zeroed by the caller)
// Serving: one persistent launch of the single-warp decoder takes its work
// from a ring of (request descriptor, restart) items that the host publishes
// while it runs, and the decoder that finishes a request's last restart
// selects its best restart and reports it in host-mapped memory.
//
// A request's descriptor is followed in device memory by a ServeTail; the
// launch's tables (descriptors, step types, orientations, slot heads,
// placements) all live in one arena whose regions are reused while the
// launch runs, so the serving kernel reads every table through L2.
struct ServeTail {
    int done_count;       // restarts finished (device atomics)
    int done_slot;        // index of the request's host-mapped completion record
    long long seq;        // the request's sequence number, written to that record
};
struct ServeArgs {
    int* head;                      // device: work items claimed
    const int* tail;                // device: work items published (written by stream-ordered copies)
    const int* stop;                // device: nonzero = exit once no work is left
    const int2* ring;               // device: work items (descriptor index, restart)
    int ring_mask;                  // ring entries - 1 (a power of two)
    volatile long long* done_seq;   // host-mapped: per completion record, the finished request's seq
    int2* done_best;                // host-mapped: per completion record, (best restart, fallback)
    int idle_polls;                 // empty polls before a decoder exits (about 4 us each)
    // Restarts that outgrow the launch's tile are pushed by their decoder onto
    // the overflow ring and decoded again by the launch's first n_deep
    // decoders, whose deeper tile (deep_P, deep_C) lives in global memory.
    int4* dring;                    // device: {descriptor, restart, ticket + 1, 0}, ring_mask + 1 entries
    int* dhead;                     // device: overflow items claimed
    int* dtail;                     // device: overflow items reserved
    int* alive;                     // device: main decoders of the launch not yet exited
    int n_deep, deep_P, deep_C, deep_bytes;
    unsigned char* deep_scratch;    // device: n_deep x deep_bytes
    int deep_idle_polls;            // empty polls before an overflow decoder exits
};
bool serve_config_supported(int D, int M);
cudaError_t serve_occupancy(int P, int C, int Hz, int D, int M, int sup16, int* ctas_per_sm);
cudaError_t launch_serve(const DecodeLaunch& L, const ServeArgs& s, cudaStream_t st);

cudaError_t launch_redo_collect(const int2* work, int n_work, const InstDesc* inst, const SlotHead* heads,
                                int2* redo, int* count, int sms, cudaStream_t st);
cudaError_t launch_select_best(const InstDesc* inst, int n_inst, const SlotHead* heads, int2* best,
                               cudaStream_t st);
cudaError_t launch_rng_dump(const long long* seeds, int n_seeds, int n_random, int n_bits,
                            int k_bits, const uint32_t* mt_init, double* out_r, uint32_t* out_b,
                            cudaStream_t st);
int fsr_smem_per_warp(int cap);
cudaError_t launch_fsr(const int* rows7, const int* offsets, int n_pack, int cap, double mu,
                       double* out_score, double* out_fsr, cudaStream_t st);
cudaError_t launch_item_order(const long long* vols, const int* qty, const int* type_off,
                              const int* n_types, const long long* step_off, int n_inst, int order,
                              int* out_types, int sort_cap, cudaStream_t st);
// one-step feasibility (kernel a); first_out (optional) receives the smallest
// feasible pair index (atomicMin; caller initialises it to INT_MAX)
cudaError_t launch_feas(const int* cand, int n_cand, const int* ors, int n_ors, const int* fast6,
                        int n_fast, int L, int W, int H, unsigned char* bits, int* first_out,
                        cudaStream_t st);

}  // namespace plpb
