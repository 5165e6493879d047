/* plp_capi.h -- C ABI of the B200 extreme-point decoder (libplp_b200.so).
 *
 * Plain C types only (pointers, sizes, status codes); no exceptions, no exit().
 * Every entry point returns a plp_status (0 = PLP_OK). The last error message
 * of the calling thread is available from plp_last_error(NULL); handle-bound
 * calls also record it on the handle (plp_last_error(handle)).
 *
 * Reference interfaces each group replaces (pqant/plp-gpu):
 *   plp_feas_check_all   FeasibilityBackend::check_all, gpu/plp_common.hpp:326-332
 *                        (CUDA impl CudaBackend::check_all, gpu/plp_gpu.cu:443-495)
 *   plp_instance_*       plp::parse / plp::load_instance, gpu/plp_common.hpp:68-151
 *   plp_run_plain        plp::run with CudaBackend, gpu/plp_gpu.cu:1684-1686 and
 *                        gpu/plp_common.hpp:471-523 (one feasibility launch per step)
 *   plp_solve            run_device / run_batch, gpu/plp_gpu.cu:343-412,1395-1474
 *                        (row k = PyRng(seed + k)), generalised to many instances
 *   plp_create/submit/.. no reference counterpart: the serving loop
 *   plp_rng_dump         --rngdump N, gpu/plp_gpu.cu:1479-1536
 *   plp_fsr_score        plp::stability_score, gpu/plp_common.hpp:393-399
 *   plp_item_order       plp::item_sequence, gpu/plp_common.hpp:335-351
 *   plp_to_json / plp_py_repr   plp::to_json / plp::py_repr, gpu/plp_common.hpp:535-610
 *   plp_selftest         --selftest, gpu/plp_gpu.cpp:43-66
 */
#ifndef PLP_CAPI_H
#define PLP_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PLP_OK = 0,
    PLP_E_INVALID = 1,      /* bad argument (null pointer, negative size, bad option) */
    PLP_E_FORMAT = 2,       /* instance text violates the thpack format */
    PLP_E_CUDA = 3,         /* a CUDA call failed (message names it) */
    PLP_E_CAPACITY = 4,     /* a size limit of this build was exceeded */
    PLP_E_BUDGET = 5,       /* request larger than the handle's device-memory budget */
    PLP_E_TIMEOUT = 6,      /* plp_wait timed out (request still running) */
    PLP_E_NOT_FOUND = 7,    /* unknown request id */
    PLP_E_CANCELLED = 8,    /* request was cancelled */
    PLP_E_PENDING = 9,      /* plp_poll: not finished yet */
    PLP_E_DEVICE = 10       /* a kernel reported an internal error status */
} plp_status;

/* ------------------------------------------------------------------------ */
/* errors                                                                    */
/* ------------------------------------------------------------------------ */
typedef struct plp_handle plp_handle;
/* Message of the last failed call: of the handle when h != NULL, else of the
 * calling thread. Valid until the next call on the same handle / thread. */
const char* plp_last_error(const plp_handle* h);

/* ------------------------------------------------------------------------ */
/* one-step feasibility (the drop-in for FeasibilityBackend::check_all)      */
/* ------------------------------------------------------------------------ */
/* Host buffers in and out. bits_out[ci * n_ors + oi] = 1 iff placing
 * orientation oi = (w, d, h) at candidate ci = (x, y, z) satisfies C2 (inside
 * L x W x H), C3 (>= 50 % bottom support, FP64 ratio) and C1 (no overlap with
 * the n_fast placed boxes (x, y, z, x2, y2, z2)). Runs on the calling thread's
 * CUDA stream and device buffers; thread-safe across threads. */
int plp_feas_check_all(const int32_t* cand_xyz, int32_t n_cand,
                       const int32_t* ors_wdh, int32_t n_ors,
                       const int32_t* fast6, int32_t n_fast,
                       int32_t L, int32_t W, int32_t H, uint8_t* bits_out);

/* The same on device buffers, enqueued on `stream` (a cudaStream_t, or NULL
 * for the legacy default stream); no synchronisation. */
int plp_feas_check_all_dev(const int32_t* d_cand_xyz, int32_t n_cand,
                           const int32_t* d_ors_wdh, int32_t n_ors,
                           const int32_t* d_fast6, int32_t n_fast,
                           int32_t L, int32_t W, int32_t H, uint8_t* d_bits_out,
                           void* stream);

/* ------------------------------------------------------------------------ */
/* instances                                                                 */
/* ------------------------------------------------------------------------ */
typedef struct plp_instance plp_instance;

/* Parse thpack text holding exactly one instance (P == 1).
 * PLP_E_FORMAT with the reference parser's message on a violation. */
int plp_instance_parse(const char* text, size_t len, plp_instance** out);
/* Parse thpack text with P >= 1 instances; *out receives n instance handles
 * (free each with plp_instance_free and the array with plp_free). */
int plp_instance_parse_multi(const char* text, size_t len, plp_instance*** out, int32_t* n);
int plp_instance_load(const char* path, plp_instance** out);
/* types7: n_types rows (l, lf, w, wf, h, hf, qty). */
int plp_instance_from_types(int32_t L, int32_t W, int32_t H, int32_t n_types,
                            const int32_t* types7, plp_instance** out);
void plp_instance_free(plp_instance* inst);
/* L, W, H, n_types, total item count */
int plp_instance_info(const plp_instance* inst, int32_t* LWH, int32_t* n_types,
                      int32_t* n_items);
/* orientation table of one type: up to 6 (w, d, h), dedup'd in parser order */
int plp_orientations(const plp_instance* inst, int32_t type, int32_t* wdh6x3, int32_t* n);
/* item sequence on the host: order 0 = volume, 1 = input; ti/copy hold n_items */
int plp_item_sequence(const plp_instance* inst, int32_t order, int32_t* ti, int32_t* copy);
void plp_free(void* p);

/* ------------------------------------------------------------------------ */
/* run options and results                                                   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t seed;         /* restart k uses PyRng(|seed + k|) */
    int32_t restarts;     /* >= 1 */
    int32_t passes;       /* >= 1 fixed passes per restart (RNG carried over); with a
                             time limit, the most passes to run (0 = no cap) */
    double eps;           /* eps-greedy probability */
    double theta;         /* acceptance threshold; NaN = no threshold (--no-theta) */
    int32_t order;        /* 0 = volume, 1 = input */
    int32_t first_fit;    /* 1 = always the first feasible pair */
    double mu;            /* friction coefficient (reference default 0.2) */
    double time_limit_s;  /* < 0: exactly `passes` passes; >= 0: passes until this
                             much time has passed since the restart began (at
                             least one; gpu/plp_common.hpp:484-492). The device
                             decoders read the GPU's global timer after each pass;
                             the summary's n_passes is the count run. */
    int32_t best_only;    /* 1: copy back the placements of the best restart only
                             (summaries of every restart are always returned) */
    /* engine 1 is the block-building engine (blockproof/plp_block.cpp): items
     * grouped into a x b x k blocks of one type and orientation, placed at
     * extreme points; order and first_fit do not apply to it. */
    int32_t engine;       /* 0 extreme-point decoder, 1 block-building engine */
    int32_t blk_amax, blk_bmax, blk_kmax;   /* block limits (reference defaults 3, 3, 4) */
    int32_t blk_topk;     /* eps pick among the top-k fitting shapes (default 8) */
    int32_t blk_pick;     /* point rule: 0 first, 1 support, 2 contact */
} plp_run_opts;

void plp_default_opts(plp_run_opts* o);   /* reference CLI defaults */

typedef struct {
    int32_t n_boxes;
    int32_t fallback;
    int64_t volume;
    double score;
    int32_t n_passes;
    int32_t err;          /* 0, or a device status for this restart */
    int64_t seed;
    double time_s;
} plp_summary;

typedef struct plp_result plp_result;   /* results of one instance's restarts */

int32_t plp_result_restarts(const plp_result* r);
int plp_result_summary(const plp_result* r, int32_t restart, plp_summary* out);
/* placements as rows (type, x, y, z, w, d, h); n_out receives the count */
int plp_result_placements(const plp_result* r, int32_t restart, int32_t* rows7,
                          int32_t cap, int32_t* n_out);
/* best restart (accepted first, max (volume, n_boxes), earliest on ties) */
int plp_result_best(const plp_result* r, int32_t* restart, int32_t* fallback);
/* reference JSON of one restart (plp/solver.py:297-307 layout). Writes at most
 * cap bytes incl. NUL; *needed receives the full length excl. NUL. */
int plp_result_json(const plp_result* r, int32_t restart, char* buf, size_t cap, size_t* needed);
void plp_result_free(plp_result* r);
/* Reference work of one restart's reported pass, the roofline's algorithmic
 * unit: aabb_tests = sum over steps of 2 * n_placed * (C2-surviving pairs of
 * the reference candidate list), pairs = sum of n_cand * n_ors. */
int plp_result_work(const plp_result* r, int32_t restart, int64_t* aabb_tests, int64_t* pairs);

/* ------------------------------------------------------------------------ */
/* plain path: host decode loop, one feasibility launch per item step        */
/* ------------------------------------------------------------------------ */
int plp_run_plain(const plp_instance* inst, const plp_run_opts* opts, plp_result** out);

/* ------------------------------------------------------------------------ */
/* handle: device arena, stream, persistent batched solver, serving loop     */
/* ------------------------------------------------------------------------ */
/* budget_bytes: device memory the handle may hold for admitted requests
 * (0 = 100 GB). device: CUDA ordinal. */
int plp_create(size_t budget_bytes, int32_t device, plp_handle** out);
void plp_destroy(plp_handle* h);

/* Decoder tile for later solves on this handle: placed-box depth P and
 * live-point depth C (per decoder, in shared memory; C a multiple of 32),
 * warps per decoder G, decoders per CTA D and minimum resident CTAs per SM M
 * (which caps registers per thread at 65536 / (32 G D M)). (G, D, M) must be
 * one of (1,1,1) (1,1,12) (1,2,1) (1,4,1) (1,4,4) (1,8,1) (1,8,2) (2,1,1) (2,2,1) (2,2,5)
 * (2,4,1) (2,4,3) (4,1,1) (4,1,5) (4,1,6) (4,2,1) (4,2,3) (4,4,1) (8,1,1)
 * (8,1,3) (8,2,1); 0 keeps the current value. (1,1,12) holds the decoder to
 * 160 registers, so three warps fit in each SM partition's register file
 * where 185 allow two. Restarts that outgrow the tile
 * are re-run with a deeper one, so the tile affects speed only, never results.
 * A new handle starts at P = 256, C = 512, G = 1, D = 1, M = 1. */
int plp_set_tile(plp_handle* h, int32_t P, int32_t C, int32_t G, int32_t D, int32_t M);

/* Autotuner (no reference counterpart): times candidate tiles -- one warp per
 * decoder with placed-box depth P, live-point depth C, decoders per CTA D and
 * minimum CTAs per SM M -- on a strided sample of at most max_decodes of the
 * workload's decodes (0 = 32768), each after a warm-up run, and keeps the
 * fastest as the handle's tile. A candidate's estimate scales the sample's
 * decoder launch to the whole workload and adds the retry stage (restarts that
 * outgrew the tile, re-run at a deeper one) at its latency, which does not
 * shrink with the sample. tile_out (may be NULL) receives {P, C, G, D, M}.
 * The tile never changes results. */
int plp_autotune(plp_handle* h, const plp_instance* const* insts, int32_t n_inst,
                 const plp_run_opts* opts, int32_t n_opts, int32_t max_decodes, int32_t* tile_out);

/* Synchronous batched solve: every restart of every instance in one
 * persistent decoder launch (plus a FSR/selection launch), results copied to
 * the host. opts holds n_inst entries (or 1 entry shared by all). A batch
 * whose restarts take more than one wave of resident decoders re-runs the
 * restarts that outgrew the tile at a deeper tile in the same stream pass.
 * The results of one call share a pinned host block from the handle's pool,
 * which the device writes once and the results read in place. It returns to
 * the pool when the last of them is freed, so results may outlive the
 * handle. The pool pins at most a quarter of host memory, or the environment
 * variable PLP_PINNED_POOL_MB (read at plp_create; 0 turns it off); beyond
 * that results go to pageable memory. */
int plp_solve(plp_handle* h, const plp_instance* const* insts, int32_t n_inst,
              const plp_run_opts* opts, int32_t n_opts, plp_result** results);

/* Prepared batch: the tables of a solve uploaded once and kept resident, so a
 * caller can run the device part repeatedly (timing) and fetch results when
 * it wants them. plp_batch_run is synchronous; device_ms is the CUDA-event
 * time of all device work of the run, decoder_ms that of the decoder kernel
 * alone, launches the number of kernels launched. A run that needed no
 * host-side capacity retry is captured as one CUDA graph (error-flag reset,
 * decoder, the device retry stage where it applies, flag copy, selection,
 * gather) and later runs with the same tile replay it with a single graph
 * launch and a single synchronisation. */
typedef struct plp_batch plp_batch;
int plp_batch_prepare(plp_handle* h, const plp_instance* const* insts, int32_t n_inst,
                      const plp_run_opts* opts, int32_t n_opts, plp_batch** out);
int plp_batch_run(plp_batch* b, double* device_ms, double* decoder_ms, int32_t* launches);
/* results of the last run (n_inst result objects) */
int plp_batch_fetch(plp_batch* b, plp_result** results);
/* bytes the batch copies host->device (tables) and device->host (results) */
int plp_batch_io_bytes(const plp_batch* b, int64_t* h2d, int64_t* d2h);
/* 1 when the batch's next run replays its captured CUDA graph, else 0 (no
 * reference counterpart). */
int plp_batch_graph(const plp_batch* b);
void plp_batch_free(plp_batch* b);

/* Serving: admit a request; it starts as soon as the memory budget allows and
 * runs concurrently with other admitted requests. */
int plp_submit(plp_handle* h, const plp_instance* inst, const plp_run_opts* opts,
               int64_t* request_id);
/* PLP_OK when finished, PLP_E_PENDING while queued or running */
int plp_poll(plp_handle* h, int64_t request_id);
/* block until finished or timeout_ms elapses (< 0: no timeout) */
int plp_wait(plp_handle* h, int64_t request_id, int64_t timeout_ms);
/* take the finished result (ownership passes to the caller) */
int plp_take_result(plp_handle* h, int64_t request_id, plp_result** out);
int plp_cancel(plp_handle* h, int64_t request_id);
/* seconds from submit to finish, and to start on the device */
int plp_request_times(plp_handle* h, int64_t request_id, double* queued_s, double* total_s);

/* No counterpart in the reference. Requests that run the extreme-point decoder
 * for one pass with every restart kept (engine 0, passes 1, no time limit,
 * not best_only) are served by one persistent decoder launch that they join
 * while it runs: each request's tables go into a device arena (half the
 * budget, at most PLP_SERVE_ARENA_MB, default 4096 MiB, reserved from the
 * budget on the first such request), its restarts into a device work ring,
 * and the decoder that finishes its last restart selects its best restart on
 * the device. Other requests run in waves on worker streams. PLP_SERVE=0 in
 * the environment when the first request arrives sends every request to the
 * waves. A restart that outgrows the launch's tile is decoded again, inside
 * the same launch, by one of its overflow decoders (a deeper tile in global
 * memory). While the serving launch runs it holds the SMs: plp_solve,
 * plp_batch_run and plp_autotune on this handle ask an idle launch to stop at
 * once; other work on the GPU runs once it has stopped (50 ms after the last
 * request finished). This call reports the handle's serving launches,
 * requests served by them, requests re-run on the wave path's code after a
 * restart outgrew even the overflow tile, and eligible requests sent to the
 * waves (larger than the arena or its staging). */
int plp_serve_counters(plp_handle* h, int64_t* launches, int64_t* served, int64_t* fallbacks,
                       int64_t* waved);

/* ------------------------------------------------------------------------ */
/* allocation-free decode                                                    */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference. For callers that cannot allocate device
 * memory -- a process whose device memory is owned by another framework's
 * caching allocator, a plugin hosted by a runtime that forbids allocation on
 * its request path, a latency-critical loop that must not enter the
 * allocator: decodes every restart of one instance like plp_solve, but the
 * decoder's scratch (tables, work list, counters, multi-pass rows) is a fixed
 * 8 MiB array inside the library, so the call allocates no device memory.
 *   d_heads:  opts->restarts records of 32 bytes {int32 n_boxes, int32 err,
 *             int64 volume, double score, int32 n_passes, int32 fallback}
 *   d_places: opts->restarts rows of max(n_items, 1) uint64 words, placement i
 *             = x | y << 16 | z << 32 | orientation index << 48 | type << 51
 * Both are caller-owned device buffers. The work is enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream); synchronise it before
 * reading the outputs. The first call on each device looks up the scratch's
 * device address (cudaGetSymbolAddress) and keeps it for the process, so the
 * entry point cannot be used on a device after cudaDeviceReset.
 * Host side: the call builds the tables in ordinary (pageable) host memory
 * that it allocates and frees, and copies them in with cudaMemcpyAsync; a
 * pageable copy makes the host wait until the bytes are staged, so the call
 * can block. It is therefore refused (PLP_E_INVALID) while `stream` is being
 * captured. Every call shares the scratch, so calls that overlap on the
 * GPU race: serialise them (one stream, or wait between calls). Instances
 * whose tables do not fit the scratch (about 8 MiB of restarts x 8 bytes,
 * types x 88 bytes and steps x 4 bytes) return PLP_E_CAPACITY.
 * Errors per restart: err != 0 in a record marks a restart that failed, and
 * no retry runs (plp_solve reruns such restarts, this call does not): 1 or 2
 * = tile overflow (not reached: the tile is sized for the instance's step
 * count), 3 = the randrange rejection bound was hit. Check err in every
 * record. */
int plp_decode_noalloc(const plp_instance* inst, const plp_run_opts* opts, void* d_heads,
                       void* d_places, void* stream);

/* ------------------------------------------------------------------------ */
/* kernel-level hooks (parity tests of the individual device kernels)        */
/* ------------------------------------------------------------------------ */
/* device MT19937 (kernel c): for each seed, n_random random() doubles then
 * n_bits getrandbits(k_bits) values, CPython-exact. */
int plp_rng_dump(const int64_t* seeds, int32_t n_seeds, int32_t n_random,
                 int32_t n_bits, int32_t k_bits, double* out_random, uint32_t* out_bits);
/* the same stream from the host MT19937 (the plain path's generator) */
int plp_rng_dump_host(const int64_t* seeds, int32_t n_seeds, int32_t n_random,
                      int32_t n_bits, int32_t k_bits, double* out_random, uint32_t* out_bits);
/* No counterpart in the reference. Test hook of the bounded barrier wait of
 * the multi-warp decoders (tile G > 1): later launches of this handle give
 * each wait wait_limit tries of about 10 us (0 = the kernel's own bound, near
 * 3 s) and, when skip_warp >= 0, warp skip_warp of every decoder leaves out
 * its first arrive, so that wait runs out. The launch then ends early with
 * the barrier error and the solve returns PLP_E_DEVICE; the handle stays
 * usable. plp_debug_sync_bound(h, 0, -1) restores normal launches. */
int plp_debug_sync_bound(plp_handle* h, int32_t wait_limit, int32_t skip_warp);
/* device FSR (kernel e): packings given as rows (type, x, y, z, w, d, h);
 * offsets[n_pack + 1] delimit packings. */
int plp_fsr_score(const int32_t* rows7, const int32_t* offsets, int32_t n_pack, double mu,
                  double* out_score, double* out_fsr);
/* device item-order sort (kernel d): per instance sequence of types. */
int plp_item_order(const plp_instance* const* insts, int32_t n_inst, int32_t order,
                   int32_t* out_types, int64_t* out_offsets);

/* ------------------------------------------------------------------------ */
/* host formatting                                                           */
/* ------------------------------------------------------------------------ */
int plp_py_repr(double x, char* buf, size_t cap);
/* the reference --selftest text (RNG + repr blocks); *needed as in plp_result_json */
int plp_selftest(char* buf, size_t cap, size_t* needed);

#ifdef __cplusplus
}
#endif
#endif /* PLP_CAPI_H */
