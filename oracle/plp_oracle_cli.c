/* plp_oracle_cli.c -- command-line front end of the CPU oracle (TEST
 * INFRASTRUCTURE). Flags follow the reference CLI (gpu/plp_gpu.cpp:80-117):
 *
 *   plp_oracle <instance> [--seed N] [--time S] [--eps F] [--theta F | --no-theta]
 *              [--order volume|input] [--first-fit] [--mu F] [--single-pass] [--json]
 *   extensions used by the test suite:
 *              [--passes N]    fixed pass count instead of a wall-clock budget
 *              [--restarts R]  one JSON line per restart, seeds seed..seed+R-1
 *              [--stats]       print work counters (pairs, AABB tests) as JSON
 *              [--block [--amax A] [--bmax B] [--kmax K] [--topk N]
 *                       [--pick first|support|contact]]
 *                              the block-building engine (blockproof/plp_block.cpp
 *                              flags and defaults: 3, 3, 4, 8, first; mu 0.2)
 *   plp_oracle --selftest      RNG + repr blocks (gpu/plp_gpu.cpp:43-66 layout)
 */
#include "plp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char* read_file(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* b = (char*)malloc((size_t)n + 1);
    size_t got = fread(b, 1, (size_t)n, f);
    b[got] = '\0';
    fclose(f);
    return b;
}

static void selftest(void) {
    const unsigned seeds[] = {0u, 1u, 7u, 123456789u};
    for (int s = 0; s < 4; s++) {
        orc_rng r;
        orc_rng_seed(&r, seeds[s]);
        printf("SEED %u\n", seeds[s]);
        for (int i = 0; i < 16; i++) {
            double v = orc_rng_random(&r);
            unsigned long long bits;
            memcpy(&bits, &v, 8);
            printf("%016llx\n", bits);
        }
        for (int i = 0; i < 16; i++) printf("%u\n", orc_rng_getrandbits(&r, 13));
    }
    const double vals[] = {0.0, 1.0, 0.5, 0.1, 2.0 / 3.0, 0.5785123966942148,
                           0.6132075471698113, 0.6595744680851063, 1e-05, 1e-04,
                           1e15, 1e16, 0.001, 123456789.5, 1.0 / 121.0, 1.0 / 106.0};
    char buf[48];
    for (int i = 0; i < 16; i++) {
        orc_py_repr(vals[i], buf);
        printf("REPR %s\n", buf);
    }
}

int main(int argc, char** argv) {
    const char* path = NULL;
    long long seed = 0;
    double time_s = 300.0, eps = 0.3, theta = 0.9, mu = 0.2;
    int has_theta = 1, order = 0, first_fit = 0, single = 0, as_json = 0;
    int passes = 0, restarts = 1, stats = 0, block = 0;
    orc_block_cfg bc = {3, 3, 4, 8, 0};
    const char* e = getenv("PLP_MU");
    if (e) mu = strtod(e, NULL);
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
#define NEXT() (i + 1 < argc ? argv[++i] : (fprintf(stderr, "missing value for %s\n", a), exit(2), ""))
        if (!strcmp(a, "--selftest")) { selftest(); return 0; }
        else if (!strcmp(a, "--seed")) seed = atoll(NEXT());
        else if (!strcmp(a, "--time")) time_s = strtod(NEXT(), NULL);
        else if (!strcmp(a, "--eps")) eps = strtod(NEXT(), NULL);
        else if (!strcmp(a, "--mu")) mu = strtod(NEXT(), NULL);
        else if (!strcmp(a, "--theta")) theta = strtod(NEXT(), NULL);
        else if (!strcmp(a, "--no-theta")) has_theta = 0;
        else if (!strcmp(a, "--order")) {
            const char* o = NEXT();
            if (!strcmp(o, "volume")) order = 0;
            else if (!strcmp(o, "input")) order = 1;
            else { fprintf(stderr, "unknown order %s\n", o); return 2; }
        }
        else if (!strcmp(a, "--first-fit")) first_fit = 1;
        else if (!strcmp(a, "--single-pass")) single = 1;
        else if (!strcmp(a, "--json")) as_json = 1;
        else if (!strcmp(a, "--passes")) passes = atoi(NEXT());
        else if (!strcmp(a, "--restarts")) restarts = atoi(NEXT());
        else if (!strcmp(a, "--stats")) stats = 1;
        else if (!strcmp(a, "--block")) block = 1;
        else if (!strcmp(a, "--amax")) bc.amax = atoi(NEXT());
        else if (!strcmp(a, "--bmax")) bc.bmax = atoi(NEXT());
        else if (!strcmp(a, "--kmax")) bc.kmax = atoi(NEXT());
        else if (!strcmp(a, "--topk")) bc.topk = atoi(NEXT());
        else if (!strcmp(a, "--pick")) {
            const char* v = NEXT();
            if (!strcmp(v, "first")) bc.pick = 0;
            else if (!strcmp(v, "support")) bc.pick = 1;
            else if (!strcmp(v, "contact")) bc.pick = 2;
            else { fprintf(stderr, "bad --pick: %s (first|support|contact)\n", v); return 2; }
        }
        else if (a[0] != '-') path = a;
        else { fprintf(stderr, "unknown flag: %s\n", a); return 2; }
    }
    if (!path) { fprintf(stderr, "usage: plp_oracle <instance> [flags]\n"); return 2; }
    char* text = read_file(path);
    if (!text) { fprintf(stderr, "instance error: cannot open %s\n", path); return 1; }
    orc_instance* insts = NULL;
    char err[256];
    int n = orc_parse(text, &insts, err, sizeof err);
    free(text);
    if (n < 0) { fprintf(stderr, "instance error: %s\n", err); return 1; }
    if (n != 1) {
        fprintf(stderr, "instance error: expected exactly 1 instance, got %d\n", n);
        orc_free_instances(insts, n);
        return 1;
    }
    const int fixed = single ? 1 : passes;
    int cap = 1 << 20;
    char* buf = (char*)malloc((size_t)cap);
    for (int r = 0; r < restarts; r++) {
        orc_result res;
        orc_stats st;
        memset(&st, 0, sizeof st);
        if (block) {
            orc_block_cfg c = bc;
            if (c.amax < 1) c.amax = 1;
            if (c.bmax < 1) c.bmax = 1;
            if (c.kmax < 1) c.kmax = 1;
            if (c.topk < 1) c.topk = 1;
            orc_block_run(&insts[0], seed + r, fixed > 0 ? fixed : 1, fixed > 0 ? -1.0 : time_s, eps,
                          has_theta, theta, mu, &c, &res);
        } else {
            orc_run(&insts[0], seed + r, fixed > 0 ? fixed : 1, fixed > 0 ? -1.0 : time_s, eps,
                    has_theta, theta, order, first_fit, mu, &res, stats ? &st : NULL);
        }
        if (stats) {
            printf("{\"seed\": %lld, \"steps\": %lld, \"pairs\": %lld, \"c2_pairs\": %lld, "
                   "\"aabb_full\": %lld, \"max_cand\": %lld, \"pairs_to_first\": %lld, "
                   "\"random_steps\": %lld, \"n_boxes\": %d}\n",
                   seed + r, (long long)st.steps, (long long)st.pairs, (long long)st.c2_pairs,
                   (long long)st.aabb_full, (long long)st.max_cand,
                   (long long)st.pairs_to_first, (long long)st.random_steps, res.n_boxes);
        } else if (as_json) {
            orc_to_json(&res, buf, cap);
            printf("%s\n", buf);
        } else {
            printf("n_boxes=%d volume_cm3=%lld stability_score=%.4f fallback=%s n_passes=%d "
                   "time_s=%.3f\n", res.n_boxes, (long long)res.volume, res.score,
                   res.fallback ? "true" : "false", res.n_passes, res.time_s);
        }
        orc_free_result(&res);
    }
    free(buf);
    orc_free_instances(insts, n);
    return 0;
}
