/* plp_oracle.h -- CPU oracle for the extreme-point decoder (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference decoder (pqant/plp-gpu), used only
 * by tests/, the smoke check and bench.py's CPU-baseline leg as the checker.
 * Nothing in the product links or calls it.
 *
 * Semantics followed (reference file:line):
 *   parser          plp/parser.py:67-139, gpu/plp_common.hpp:68-151
 *   orientations    plp/parser.py:142-156 + plp/solver.py:75-83,
 *                   gpu/plp_common.hpp:269-280
 *   item sequence   plp/solver.py:169-177, gpu/plp_common.hpp:335-351
 *   PyRng           gpu/plp_common.hpp:164-250 (CPython random.Random(int))
 *   feasibility     plp/solver.py:196-218, gpu/plp_common.hpp:297-321
 *   decode pass     plp/solver.py:180-240, gpu/plp_common.hpp:404-456
 *   FSR / score     plp/solver.py:104-148, gpu/plp_common.hpp:356-399
 *   run / select    plp/solver.py:156-166,243-271, gpu/plp_common.hpp:471-523
 *   JSON / repr     plp/solver.py:297-307, gpu/plp_common.hpp:535-610
 *
 * Pinned against: the reference's checked-in parity JSONs
 * (parity/ref_cpu/ BR1..BR3, SYN1), its --selftest vectors (gpu/make_selftest_ref.py,
 * regenerated with CPython into tests/golden/selftest_ref.txt), the FSR /
 * geometry known answers of tests/test_solver.py and tests/test_geometry.py,
 * and outputs of the reference's own g++ build run on synthetic instances
 * (tests/golden/, made by tests/golden/make_golden.py).
 */
#ifndef PLP_ORACLE_H
#define PLP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int l, w, h;        /* box edges, cm */
    int lf, wf, hf;     /* 0/1: that edge may be vertical */
    int qty;
} orc_item;

typedef struct {
    int L, W, H;
    int n_types;
    orc_item* items;    /* n_types entries, owned */
} orc_instance;

typedef struct {
    uint32_t mt[624];
    int pos;
} orc_rng;

/* one placed box, in placement order */
typedef struct {
    int type, x, y, z, w, d, h;
} orc_place;

/* work counters of one decode pass (filled when non-NULL) */
typedef struct {
    int64_t steps;          /* item steps with >= 1 orientation */
    int64_t pairs;          /* sum over steps of n_cand * n_ors */
    int64_t c2_pairs;       /* pairs that pass C2 */
    int64_t aabb_full;      /* T: sum over C2-surviving pairs of 2 * n_placed */
    int64_t max_cand;       /* largest candidate list seen */
    int64_t pairs_to_first; /* pairs up to and including the first feasible */
    int64_t random_steps;   /* steps that took the uniform-random branch */
} orc_stats;

typedef struct {
    int n_boxes;
    int64_t volume;
    double score;
    int fallback;
    int n_passes;
    double time_s;
    int64_t seed;
    orc_place* placements;  /* n_boxes entries, owned */
} orc_result;

/* ---- instance I/O ------------------------------------------------------ */
/* Parses thpack text. Returns the number of instances (>= 1) and sets *out,
 * or returns -1 and writes a message to err. */
int orc_parse(const char* text, orc_instance** out, char* err, int errlen);
void orc_free_instances(orc_instance* v, int n);

int orc_orientations(const orc_item* it, int out[6][3]);
/* fills ti[] (and copy[] when non-NULL); order 0 = volume, 1 = input.
 * Returns the number of steps. ti must hold sum(qty) entries. */
int orc_item_sequence(const orc_instance* inst, int order, int* ti, int* copy);

/* ---- CPython-compatible MT19937 ---------------------------------------- */
void orc_rng_seed(orc_rng* r, uint64_t seed);
uint32_t orc_rng_next32(orc_rng* r);
double orc_rng_random(orc_rng* r);
uint32_t orc_rng_getrandbits(orc_rng* r, int k);
int orc_rng_randrange(orc_rng* r, int n);

/* ---- feasibility ------------------------------------------------------- */
/* fast6: n_fast boxes as (x, y, z, x2, y2, z2) */
int orc_feasible_one(int x, int y, int z, int w, int d, int h,
                     const int32_t* fast6, int n_fast, int L, int W, int H);
/* bits[ci * n_ors + oi]; cand_xyz: n_cand (x, y, z); ors_wdh: n_ors (w, d, h) */
void orc_check_all(const int32_t* cand_xyz, int n_cand, const int32_t* ors_wdh,
                   int n_ors, const int32_t* fast6, int n_fast, int L, int W,
                   int H, uint8_t* bits);

/* ---- decoder ----------------------------------------------------------- */
/* One decode pass. out must hold sum(qty) entries. Returns n placed. */
int orc_decode_pass(const orc_instance* inst, int order, int first_fit,
                    double eps, orc_rng* rng, orc_place* out, orc_stats* st);

void orc_compute_fsr(const orc_place* p, int n, double mu, double* fsr);
double orc_stability_score(const orc_place* p, int n, double mu);

/* One run: exactly n_passes passes (time_limit_s < 0) or passes until the
 * wall-clock budget runs out. has_theta = 0 accepts every packing. */
void orc_run(const orc_instance* inst, int64_t seed, int n_passes,
             double time_limit_s, double eps, int has_theta, double theta,
             int order, int first_fit, double mu, orc_result* res,
             orc_stats* st);
void orc_free_result(orc_result* r);

/* ---- block-building engine (blockproof/plp_block.cpp) -------------------- */
/* Block limits a x b x k, the top-k shape pick width and the pick rule among
 * feasible points: 0 first, 1 support (bottom, then side contact), 2 contact
 * (bottom + side, then bottom). */
typedef struct {
    int amax, bmax, kmax, topk, pick;
} orc_block_cfg;

/* One block pass; the placed blocks decomposed into item boxes (block order,
 * then a, b, k loops). out must hold sum(qty) entries. Returns n items. */
int orc_block_pass(const orc_instance* inst, const orc_block_cfg* cfg, double eps,
                   orc_rng* rng, orc_place* out);
/* run_block: passes with online best-of selection (theta, fallback). */
void orc_block_run(const orc_instance* inst, int64_t seed, int n_passes, double time_limit_s,
                   double eps, int has_theta, double theta, double mu,
                   const orc_block_cfg* cfg, orc_result* res);

/* ---- output ------------------------------------------------------------ */
/* CPython float repr; buf >= 32 bytes. Returns strlen. */
int orc_py_repr(double x, char* buf);
/* json.dumps layout of plp.solver --json. Returns needed length (excluding
 * NUL); writes at most cap bytes. */
int orc_to_json(const orc_result* r, char* buf, int cap);

#ifdef __cplusplus
}
#endif
#endif
