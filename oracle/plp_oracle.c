/* plp_oracle.c -- CPU oracle for the extreme-point decoder (TEST INFRASTRUCTURE).
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg use this file,
 * and only as the checker. The reference file:line each part follows is
 * cited in plp_oracle.h and at each function below.
 *
 * Build: gcc -O2 -std=c11 -ffp-contract=off (contraction off keeps every
 * double expression in the reference's operand order).
 */
#define _POSIX_C_SOURCE 200809L
#include "plp_oracle.h"

#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* parser: gpu/plp_common.hpp:68-141 (token rules), plp/parser.py:67-131      */
/* ------------------------------------------------------------------------ */

typedef struct {
    char** tok;     /* all tokens, flattened */
    int* line_of;   /* token -> line ordinal (among non-blank lines) */
    int* line_start;/* line ordinal -> first token */
    int* line_len;  /* line ordinal -> token count */
    int n_tok, n_lines;
    char* buf;
} tokens_t;

static void tok_free(tokens_t* t) {
    free(t->tok); free(t->line_of); free(t->line_start); free(t->line_len);
    free(t->buf);
}

static int is_ws(char c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
}

static void tokenize(const char* text, tokens_t* t) {
    size_t n = strlen(text);
    t->buf = (char*)malloc(n + 1);
    memcpy(t->buf, text, n + 1);
    int cap_tok = 64, cap_line = 16;
    t->tok = (char**)malloc(sizeof(char*) * cap_tok);
    t->line_of = (int*)malloc(sizeof(int) * cap_tok);
    t->line_start = (int*)malloc(sizeof(int) * cap_line);
    t->line_len = (int*)malloc(sizeof(int) * cap_line);
    t->n_tok = 0;
    t->n_lines = 0;
    char* p = t->buf;
    while (*p) {
        char* eol = strchr(p, '\n');
        char* next = eol ? eol + 1 : p + strlen(p);
        if (eol) *eol = '\0';
        int first = t->n_tok;
        char* q = p;
        while (*q) {
            while (*q && is_ws(*q)) *q++ = '\0';
            if (!*q) break;
            if (t->n_tok == cap_tok) {
                cap_tok *= 2;
                t->tok = (char**)realloc(t->tok, sizeof(char*) * cap_tok);
                t->line_of = (int*)realloc(t->line_of, sizeof(int) * cap_tok);
            }
            t->tok[t->n_tok] = q;
            t->line_of[t->n_tok] = t->n_lines;
            t->n_tok++;
            while (*q && !is_ws(*q)) q++;
        }
        if (t->n_tok > first) {
            if (t->n_lines == cap_line) {
                cap_line *= 2;
                t->line_start = (int*)realloc(t->line_start, sizeof(int) * cap_line);
                t->line_len = (int*)realloc(t->line_len, sizeof(int) * cap_line);
            }
            t->line_start[t->n_lines] = first;
            t->line_len[t->n_lines] = t->n_tok - first;
            t->n_lines++;
        }
        p = next;
    }
}

static int to_ll(const char* s, long long* v) {
    char* end = NULL;
    errno = 0;
    long long r = strtoll(s, &end, 10);
    if (end == s || *end != '\0') return 0;
    *v = r;
    return 1;
}

#define PARSE_FAIL(...)                                   \
    do {                                                  \
        if (err && errlen > 0) snprintf(err, (size_t)errlen, __VA_ARGS__); \
        goto fail;                                        \
    } while (0)

int orc_parse(const char* text, orc_instance** out, char* err, int errlen) {
    tokens_t t;
    tokenize(text, &t);
    orc_instance* v = NULL;
    long long P = 0;
    int made = 0;
    if (t.n_lines == 0) PARSE_FAIL("empty file");
    if (!to_ll(t.tok[t.line_start[0]], &P))
        PARSE_FAIL("not an integer: %s (instance count)", t.tok[t.line_start[0]]);
    if (P <= 0 || t.n_lines < 2) PARSE_FAIL("instance count must be >= 1");
    v = (orc_instance*)calloc((size_t)P, sizeof(orc_instance));
    int ln = 1;
    for (long long p = 0; p < P; p++) {
        if (ln >= t.n_lines || t.line_len[ln] > 2) PARSE_FAIL("malformed problem line");
        ln++;
        if (ln >= t.n_lines || t.line_len[ln] != 3)
            PARSE_FAIL("container line must have 3 dimensions");
        long long dims[3];
        for (int i = 0; i < 3; i++) {
            const char* s = t.tok[t.line_start[ln] + i];
            if (!to_ll(s, &dims[i])) PARSE_FAIL("not an integer: %s (container dimension)", s);
        }
        if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
            PARSE_FAIL("container dimensions must be positive");
        ln++;
        if (ln >= t.n_lines || t.line_len[ln] != 1)
            PARSE_FAIL("type-count line must be a single integer");
        long long n;
        if (!to_ll(t.tok[t.line_start[ln]], &n))
            PARSE_FAIL("not an integer: %s (type count)", t.tok[t.line_start[ln]]);
        ln++;
        orc_instance* in = &v[p];
        in->L = (int)dims[0]; in->W = (int)dims[1]; in->H = (int)dims[2];
        in->n_types = n > 0 ? (int)n : 0;
        in->items = (orc_item*)calloc(in->n_types > 0 ? (size_t)in->n_types : 1, sizeof(orc_item));
        made = (int)p + 1;
        for (long long k = 1; k <= n; k++) {
            if (ln >= t.n_lines) PARSE_FAIL("instance truncated");
            char** tk = &t.tok[t.line_start[ln]];
            int cnt = t.line_len[ln];
            ln++;
            if (cnt != 8) PARSE_FAIL("item line must have 8 tokens");
            long long idx, dl, dw, dh, q;
            if (!to_ll(tk[0], &idx)) PARSE_FAIL("not an integer: %s (item index)", tk[0]);
            if (idx != k) PARSE_FAIL("item index must be sequential");
            if (!to_ll(tk[1], &dl)) PARSE_FAIL("not an integer: %s (item dimension)", tk[1]);
            if (!to_ll(tk[3], &dw)) PARSE_FAIL("not an integer: %s (item dimension)", tk[3]);
            if (!to_ll(tk[5], &dh)) PARSE_FAIL("not an integer: %s (item dimension)", tk[5]);
            if (dl <= 0 || dw <= 0 || dh <= 0) PARSE_FAIL("item dimensions must be positive");
            for (int f = 2; f <= 6; f += 2)
                if (strcmp(tk[f], "0") != 0 && strcmp(tk[f], "1") != 0)
                    PARSE_FAIL("orientation flags must be 0/1");
            if (!to_ll(tk[7], &q)) PARSE_FAIL("not an integer: %s (item qty)", tk[7]);
            if (q < 0) PARSE_FAIL("item qty must be >= 0");
            orc_item* it = &in->items[k - 1];
            it->l = (int)dl; it->w = (int)dw; it->h = (int)dh;
            it->lf = tk[2][0] == '1'; it->wf = tk[4][0] == '1'; it->hf = tk[6][0] == '1';
            it->qty = (int)q;
        }
    }
    if (ln != t.n_lines) PARSE_FAIL("trailing data after last instance");
    tok_free(&t);
    *out = v;
    return (int)P;
fail:
    if (v) orc_free_instances(v, made);
    tok_free(&t);
    return -1;
}

void orc_free_instances(orc_instance* v, int n) {
    if (!v) return;
    for (int i = 0; i < n; i++) free(v[i].items);
    free(v);
}

/* ------------------------------------------------------------------------ */
/* orientations: plp/parser.py:142-156 (order) + plp/solver.py:75-83 (dedup) */
/* ------------------------------------------------------------------------ */

static int add_or(int out[6][3], int n, int w, int d, int h) {
    for (int i = 0; i < n; i++)
        if (out[i][0] == w && out[i][1] == d && out[i][2] == h) return n;
    out[n][0] = w; out[n][1] = d; out[n][2] = h;
    return n + 1;
}

int orc_orientations(const orc_item* it, int out[6][3]) {
    int n = 0;
    if (it->lf) { n = add_or(out, n, it->w, it->h, it->l); n = add_or(out, n, it->h, it->w, it->l); }
    if (it->wf) { n = add_or(out, n, it->l, it->h, it->w); n = add_or(out, n, it->h, it->l, it->w); }
    if (it->hf) { n = add_or(out, n, it->l, it->w, it->h); n = add_or(out, n, it->w, it->l, it->h); }
    return n;
}

/* ------------------------------------------------------------------------ */
/* item sequence: plp/solver.py:169-177 -- key (-volume, type, copy)        */
/* ------------------------------------------------------------------------ */

typedef struct { long long vol; int ti, c; } seq_t;

static int seq_cmp(const void* a, const void* b) {
    const seq_t* x = (const seq_t*)a;
    const seq_t* y = (const seq_t*)b;
    if (x->vol != y->vol) return x->vol > y->vol ? -1 : 1;
    if (x->ti != y->ti) return x->ti < y->ti ? -1 : 1;
    return (x->c > y->c) - (x->c < y->c);
}

int orc_item_sequence(const orc_instance* inst, int order, int* ti, int* copy) {
    int n = 0;
    for (int t = 0; t < inst->n_types; t++) n += inst->items[t].qty;
    seq_t* s = (seq_t*)malloc(sizeof(seq_t) * (size_t)(n > 0 ? n : 1));
    int k = 0;
    for (int t = 0; t < inst->n_types; t++) {
        const orc_item* it = &inst->items[t];
        for (int c = 0; c < it->qty; c++) {
            s[k].vol = (long long)it->l * it->w * it->h;
            s[k].ti = t;
            s[k].c = c;
            k++;
        }
    }
    if (order == 0) qsort(s, (size_t)n, sizeof(seq_t), seq_cmp);
    for (int i = 0; i < n; i++) {
        ti[i] = s[i].ti;
        if (copy) copy[i] = s[i].c;
    }
    free(s);
    return n;
}

/* ------------------------------------------------------------------------ */
/* MT19937 as CPython's random.Random(int): gpu/plp_common.hpp:164-250.     */
/* Matsumoto & Nishimura's init_genrand / init_by_array / genrand_int32,    */
/* seeded with the little-endian 32-bit words of |seed|.                     */
/* ------------------------------------------------------------------------ */

static void mt_init_scalar(uint32_t* mt, uint32_t s) {
    mt[0] = s;
    for (uint32_t i = 1; i < 624; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i;
}

void orc_rng_seed(orc_rng* r, uint64_t seed) {
    uint32_t key[2];
    int nkey = 0;
    uint64_t v = seed;
    do {
        key[nkey++] = (uint32_t)v;
        v >>= 32;
    } while (v);
    uint32_t* mt = r->mt;
    mt_init_scalar(mt, 19650218u);
    int i = 1, j = 0;
    for (int k = (624 > nkey ? 624 : nkey); k > 0; k--) {
        uint32_t prev = mt[i - 1] ^ (mt[i - 1] >> 30);
        mt[i] = (mt[i] ^ (prev * 1664525u)) + key[j] + (uint32_t)j;
        if (++i >= 624) { mt[0] = mt[623]; i = 1; }
        if (++j >= nkey) j = 0;
    }
    for (int k = 623; k > 0; k--) {
        uint32_t prev = mt[i - 1] ^ (mt[i - 1] >> 30);
        mt[i] = (mt[i] ^ (prev * 1566083941u)) - (uint32_t)i;
        if (++i >= 624) { mt[0] = mt[623]; i = 1; }
    }
    mt[0] = 0x80000000u;
    r->pos = 624;
}

static void mt_twist(uint32_t* mt) {
    for (int i = 0; i < 624; i++) {
        uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
        uint32_t v = mt[(i + 397) % 624] ^ (y >> 1);
        mt[i] = (y & 1u) ? (v ^ 0x9908b0dfu) : v;
    }
}

uint32_t orc_rng_next32(orc_rng* r) {
    if (r->pos >= 624) {
        mt_twist(r->mt);
        r->pos = 0;
    }
    uint32_t y = r->mt[r->pos++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* CPython random(): 53-bit double from two words (27 + 26 bits). */
double orc_rng_random(orc_rng* r) {
    uint32_t a = orc_rng_next32(r) >> 5;
    uint32_t b = orc_rng_next32(r) >> 6;
    return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

uint32_t orc_rng_getrandbits(orc_rng* r, int k) { return orc_rng_next32(r) >> (32 - k); }

/* CPython randrange(n) = _randbelow_with_getrandbits(n), n >= 1. */
int orc_rng_randrange(orc_rng* r, int n) {
    int k = 0;
    for (unsigned v = (unsigned)n; v; v >>= 1) k++;
    uint32_t x;
    do {
        x = orc_rng_getrandbits(r, k);
    } while (x >= (uint32_t)n);
    return (int)x;
}

/* ------------------------------------------------------------------------ */
/* feasibility: C2 -> C3 -> C1, plp/solver.py:199-218                       */
/* ------------------------------------------------------------------------ */

int orc_feasible_one(int x, int y, int z, int w, int d, int h,
                     const int32_t* fast6, int n_fast, int L, int W, int H) {
    if (x + w > L || y + d > W || z + h > H) return 0;               /* C2 */
    if (z > 0) {                                                       /* C3 */
        long long s = 0;
        for (int j = 0; j < n_fast; j++) {
            const int32_t* b = fast6 + 6 * j;
            if (b[5] != z) continue;
            long long ox = (long long)(x + w < b[3] ? x + w : b[3]) - (x > b[0] ? x : b[0]);
            if (ox <= 0) continue;
            long long oy = (long long)(y + d < b[4] ? y + d : b[4]) - (y > b[1] ? y : b[1]);
            if (oy > 0) s += ox * oy;
        }
        if ((double)s / (double)(w * d) < 0.5) return 0;
    }
    for (int j = 0; j < n_fast; j++) {                                 /* C1 */
        const int32_t* b = fast6 + 6 * j;
        if (x < b[3] && b[0] < x + w && y < b[4] && b[1] < y + d && z < b[5] && b[2] < z + h)
            return 0;
    }
    return 1;
}

void orc_check_all(const int32_t* cand_xyz, int n_cand, const int32_t* ors_wdh,
                   int n_ors, const int32_t* fast6, int n_fast, int L, int W,
                   int H, uint8_t* bits) {
    for (int ci = 0; ci < n_cand; ci++)
        for (int oi = 0; oi < n_ors; oi++)
            bits[ci * n_ors + oi] = (uint8_t)orc_feasible_one(
                cand_xyz[3 * ci], cand_xyz[3 * ci + 1], cand_xyz[3 * ci + 2],
                ors_wdh[3 * oi], ors_wdh[3 * oi + 1], ors_wdh[3 * oi + 2],
                fast6, n_fast, L, W, H);
}

/* ------------------------------------------------------------------------ */
/* decode pass: plp/solver.py:180-240                                        */
/* ------------------------------------------------------------------------ */

static int pt_cmp(const void* a, const void* b) {
    const int32_t* p = (const int32_t*)a;
    const int32_t* q = (const int32_t*)b;
    if (p[2] != q[2]) return p[2] < q[2] ? -1 : 1;
    if (p[1] != q[1]) return p[1] < q[1] ? -1 : 1;
    return (p[0] > q[0]) - (p[0] < q[0]);
}

int orc_decode_pass(const orc_instance* inst, int order, int first_fit,
                    double eps, orc_rng* rng, orc_place* out, orc_stats* st) {
    const int L = inst->L, W = inst->W, H = inst->H;
    int n_steps = 0;
    for (int t = 0; t < inst->n_types; t++) n_steps += inst->items[t].qty;
    int* seq = (int*)malloc(sizeof(int) * (size_t)(n_steps > 0 ? n_steps : 1));
    orc_item_sequence(inst, order, seq, NULL);
    int (*ors)[6][3] = malloc(sizeof(int[6][3]) * (size_t)(inst->n_types > 0 ? inst->n_types : 1));
    int* n_ors = (int*)malloc(sizeof(int) * (size_t)(inst->n_types > 0 ? inst->n_types : 1));
    for (int t = 0; t < inst->n_types; t++) n_ors[t] = orc_orientations(&inst->items[t], ors[t]);

    int cap = 8 * n_steps + 16;
    int32_t* cand = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)cap);
    int32_t* fast = (int32_t*)malloc(sizeof(int32_t) * 6 * (size_t)(n_steps > 0 ? n_steps : 1));
    uint8_t* bits = (uint8_t*)malloc((size_t)cap * 6);
    int n_cand = 1, n_fast = 0, n_out = 0;
    cand[0] = cand[1] = cand[2] = 0;

    for (int s = 0; s < n_steps; s++) {
        const int ti = seq[s];
        const int no = n_ors[ti];
        if (no == 0) continue;
        if (st) {
            st->steps++;
            st->pairs += (int64_t)n_cand * no;
            if (n_cand > st->max_cand) st->max_cand = n_cand;
        }
        int cnt = 0, first = -1;
        for (int ci = 0; ci < n_cand; ci++) {
            const int x = cand[3 * ci], y = cand[3 * ci + 1], z = cand[3 * ci + 2];
            for (int oi = 0; oi < no; oi++) {
                const int w = ors[ti][oi][0], d = ors[ti][oi][1], h = ors[ti][oi][2];
                if (st && !(x + w > L || y + d > W || z + h > H)) {
                    st->c2_pairs++;
                    st->aabb_full += 2 * (int64_t)n_fast;
                }
                uint8_t b = (uint8_t)orc_feasible_one(x, y, z, w, d, h, fast, n_fast, L, W, H);
                bits[ci * no + oi] = b;
                if (b) {
                    if (first < 0) first = ci * no + oi;
                    cnt++;
                }
            }
        }
        if (st) st->pairs_to_first += first >= 0 ? first + 1 : (int64_t)n_cand * no;
        if (cnt == 0) continue;                      /* no feasible pair: skip copy */
        int pick = first;
        if (!(first_fit || eps == 0.0 || rng == NULL)) {
            if (orc_rng_random(rng) >= 1.0 - eps) {
                if (st) st->random_steps++;
                int idx = orc_rng_randrange(rng, cnt);
                for (int p = 0; p < n_cand * no; p++)
                    if (bits[p] && idx-- == 0) { pick = p; break; }
            }
        }
        const int ci = pick / no, oi = pick % no;
        const int x = cand[3 * ci], y = cand[3 * ci + 1], z = cand[3 * ci + 2];
        const int w = ors[ti][oi][0], d = ors[ti][oi][1], h = ors[ti][oi][2];
        out[n_out].type = ti;
        out[n_out].x = x; out[n_out].y = y; out[n_out].z = z;
        out[n_out].w = w; out[n_out].d = d; out[n_out].h = h;
        n_out++;
        int32_t* f = fast + 6 * n_fast++;
        f[0] = x; f[1] = y; f[2] = z; f[3] = x + w; f[4] = y + d; f[5] = z + h;
        /* extreme points: drop those strictly inside the new box, add its 8
         * corners, keep the list sorted by (z, y, x) and unique */
        int m = 0;
        for (int i = 0; i < n_cand; i++) {
            const int px = cand[3 * i], py = cand[3 * i + 1], pz = cand[3 * i + 2];
            if (x < px && px < x + w && y < py && py < y + d && z < pz && pz < z + h) continue;
            cand[3 * m] = px; cand[3 * m + 1] = py; cand[3 * m + 2] = pz;
            m++;
        }
        for (int c = 0; c < 8; c++) {
            cand[3 * m] = x + ((c & 1) ? w : 0);
            cand[3 * m + 1] = y + ((c & 2) ? d : 0);
            cand[3 * m + 2] = z + ((c & 4) ? h : 0);
            m++;
        }
        qsort(cand, (size_t)m, sizeof(int32_t) * 3, pt_cmp);
        int u = 0;
        for (int i = 0; i < m; i++) {
            if (u > 0 && pt_cmp(cand + 3 * (u - 1), cand + 3 * i) == 0) continue;
            if (u != i) memmove(cand + 3 * u, cand + 3 * i, sizeof(int32_t) * 3);
            u++;
        }
        n_cand = u;
    }
    free(seq); free(ors); free(n_ors); free(cand); free(fast); free(bits);
    return n_out;
}

/* ------------------------------------------------------------------------ */
/* FSR: plp/solver.py:109-148                                                */
/* ------------------------------------------------------------------------ */

typedef struct { int z, i; } zord_t;

static int zord_cmp(const void* a, const void* b) {
    const zord_t* p = (const zord_t*)a;
    const zord_t* q = (const zord_t*)b;
    if (p->z != q->z) return p->z > q->z ? -1 : 1;   /* z descending */
    return (p->i > q->i) - (p->i < q->i);            /* stable: index ascending */
}

void orc_compute_fsr(const orc_place* p, int n, double mu, double* fsr) {
    double* m = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double* load = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    zord_t* ord = (zord_t*)malloc(sizeof(zord_t) * (size_t)(n > 0 ? n : 1));
    int* aj = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    long long* aa = (long long*)malloc(sizeof(long long) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        m[i] = 50.0 * (double)((long long)p[i].w * p[i].d * p[i].h) / 1e6;
        load[i] = m[i];
        ord[i].z = p[i].z;
        ord[i].i = i;
    }
    qsort(ord, (size_t)n, sizeof(zord_t), zord_cmp);
    for (int kk = 0; kk < n; kk++) {
        const int k = ord[kk].i;
        const orc_place* bk = &p[k];
        int na = 0;
        long long total = 0;
        for (int j = 0; j < n; j++) {
            if (j == k || p[j].z + p[j].h != bk->z) continue;
            long long hx = (long long)bk->x + bk->w, jx = (long long)p[j].x + p[j].w;
            long long ox = (hx < jx ? hx : jx) - (bk->x > p[j].x ? bk->x : p[j].x);
            if (ox <= 0) continue;
            long long hy = (long long)bk->y + bk->d, jy = (long long)p[j].y + p[j].d;
            long long oy = (hy < jy ? hy : jy) - (bk->y > p[j].y ? bk->y : p[j].y);
            if (oy > 0) {
                aj[na] = j;
                aa[na] = ox * oy;
                total += ox * oy;
                na++;
            }
        }
        if (total > 0)
            for (int a = 0; a < na; a++)
                load[aj[a]] += load[k] * (double)aa[a] / (double)total;
    }
    for (int i = 0; i < n; i++) fsr[i] = (mu / 0.3) * load[i] / m[i];
    free(m); free(load); free(ord); free(aj); free(aa);
}

double orc_stability_score(const orc_place* p, int n, double mu) {
    if (n == 0) return 0.0;
    double* f = (double*)malloc(sizeof(double) * (size_t)n);
    orc_compute_fsr(p, n, mu, f);
    int c = 0;
    for (int i = 0; i < n; i++) c += f[i] >= 1.0;
    free(f);
    return (double)c / (double)n;
}

/* ------------------------------------------------------------------------ */
/* run + D4' selection: plp/solver.py:156-166,243-271                       */
/* ------------------------------------------------------------------------ */

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

void orc_run(const orc_instance* inst, int64_t seed, int n_passes,
             double time_limit_s, double eps, int has_theta, double theta,
             int order, int first_fit, double mu, orc_result* res,
             orc_stats* st) {
    orc_rng rng;
    orc_rng_seed(&rng, (uint64_t)(seed < 0 ? -seed : seed));
    int n_steps = 0;
    for (int t = 0; t < inst->n_types; t++) n_steps += inst->items[t].qty;
    size_t cap = (size_t)(n_steps > 0 ? n_steps : 1);
    orc_place* cur = (orc_place*)malloc(sizeof(orc_place) * cap);
    orc_place* best_acc = (orc_place*)malloc(sizeof(orc_place) * cap);
    orc_place* best_all = (orc_place*)malloc(sizeof(orc_place) * cap);
    int n_acc = -1, n_all = -1;            /* -1: none yet */
    long long v_acc = 0, v_all = 0;
    double s_acc = 0, s_all = 0;
    double t0 = now_s();
    int k = 0;
    for (;;) {
        int n = orc_decode_pass(inst, order, first_fit, eps, &rng, cur, st);
        k++;
        long long vol = 0;
        for (int i = 0; i < n; i++) vol += (long long)cur[i].w * cur[i].d * cur[i].h;
        double sc = orc_stability_score(cur, n, mu);
        if (n_all < 0 || vol > v_all || (vol == v_all && n > n_all)) {
            n_all = n; v_all = vol; s_all = sc;
            memcpy(best_all, cur, sizeof(orc_place) * (size_t)n);
        }
        if ((!has_theta || sc >= theta) &&
            (n_acc < 0 || vol > v_acc || (vol == v_acc && n > n_acc))) {
            n_acc = n; v_acc = vol; s_acc = sc;
            memcpy(best_acc, cur, sizeof(orc_place) * (size_t)n);
        }
        if (time_limit_s < 0 ? k >= n_passes : (now_s() - t0) >= time_limit_s) break;
    }
    const int use_acc = n_acc >= 0;
    res->n_boxes = use_acc ? n_acc : n_all;
    res->volume = use_acc ? v_acc : v_all;
    res->score = use_acc ? s_acc : s_all;
    res->fallback = !use_acc;
    res->n_passes = k;
    res->seed = seed;
    res->placements = (orc_place*)malloc(sizeof(orc_place) * (size_t)(res->n_boxes > 0 ? res->n_boxes : 1));
    memcpy(res->placements, use_acc ? best_acc : best_all, sizeof(orc_place) * (size_t)res->n_boxes);
    res->time_s = now_s() - t0;
    free(cur); free(best_acc); free(best_all);
}

/* ------------------------------------------------------------------------ */
/* Block-building engine: blockproof/plp_block.cpp:29-304                    */
/* ------------------------------------------------------------------------ */

/* one block shape: cnt = a*b*k copies of type ti in orientation oi as a
 * bw x bd x bh stack (blockproof/plp_block.cpp:29-37) */
typedef struct {
    int ti, oi, a, b, k;
    long long cnt;
    int bw, bd, bh;
} blk_shape;

typedef struct {
    blk_shape* cat;
    int n_cat;
    int** by_type;     /* per type: catalogue indices, shape precedence order */
    int* n_by_type;
    int (*ors)[6][3];
    int* n_ors;
} blk_tables;

static const blk_shape* g_cmp_cat;   /* qsort context (single-threaded oracle) */

/* most copies, tallest stack, widest base, then orientation index
 * (blockproof/plp_block.cpp:41-47) */
static int blk_prec_cmp(const void* pa, const void* pb) {
    const blk_shape* x = &g_cmp_cat[*(const int*)pa];
    const blk_shape* y = &g_cmp_cat[*(const int*)pb];
    if (x->cnt != y->cnt) return x->cnt > y->cnt ? -1 : 1;
    if (x->bh != y->bh) return x->bh > y->bh ? -1 : 1;
    if (x->a != y->a) return x->a > y->a ? -1 : 1;
    if (x->b != y->b) return x->b > y->b ? -1 : 1;
    return x->oi < y->oi ? -1 : (x->oi > y->oi ? 1 : 0);
}

/* placement order: block volume desc, type, orientation, k, a, b
 * (blockproof/plp_block.cpp:165-175) */
static int blk_place_cmp(const void* pa, const void* pb) {
    const blk_shape* s = &g_cmp_cat[*(const int*)pa];
    const blk_shape* t = &g_cmp_cat[*(const int*)pb];
    const long long vs = (long long)s->bw * s->bd * s->bh, vt = (long long)t->bw * t->bd * t->bh;
    if (vs != vt) return vs > vt ? -1 : 1;
    if (s->ti != t->ti) return s->ti < t->ti ? -1 : 1;
    if (s->oi != t->oi) return s->oi < t->oi ? -1 : 1;
    if (s->k != t->k) return s->k > t->k ? -1 : 1;
    if (s->a != t->a) return s->a > t->a ? -1 : 1;
    if (s->b != t->b) return s->b > t->b ? -1 : (s->b < t->b ? 1 : 0);
    return 0;
}

static const orc_instance* g_cmp_inst;
/* types: item volume desc, then index (blockproof/plp_block.cpp:135-139) */
static int blk_type_cmp(const void* pa, const void* pb) {
    const int x = *(const int*)pa, y = *(const int*)pb;
    const orc_item* a = &g_cmp_inst->items[x];
    const orc_item* b = &g_cmp_inst->items[y];
    const long long vx = (long long)a->l * a->w * a->h, vy = (long long)b->l * b->w * b->h;
    if (vx != vy) return vx > vy ? -1 : 1;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* catalogue bounded by amax/bmax/kmax, the pallet and the quantity
 * (blockproof/plp_block.cpp:237-256) */
static void blk_build(const orc_instance* inst, const orc_block_cfg* cfg, blk_tables* T) {
    const int nt = inst->n_types;
    T->ors = malloc(sizeof(int[6][3]) * (size_t)(nt > 0 ? nt : 1));
    T->n_ors = malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    int cap = 64;
    T->cat = malloc(sizeof(blk_shape) * (size_t)cap);
    T->n_cat = 0;
    for (int ti = 0; ti < nt; ti++) {
        T->n_ors[ti] = orc_orientations(&inst->items[ti], T->ors[ti]);
        for (int oi = 0; oi < T->n_ors[ti]; oi++) {
            const int w = T->ors[ti][oi][0], d = T->ors[ti][oi][1], h = T->ors[ti][oi][2];
            for (int a = 1; a <= cfg->amax; a++) {
                if (a * w > inst->L) break;
                for (int b = 1; b <= cfg->bmax; b++) {
                    if (b * d > inst->W) break;
                    for (int k = 1; k <= cfg->kmax; k++) {
                        if (k * h > inst->H) break;
                        const long long cnt = (long long)a * b * k;
                        if (cnt > inst->items[ti].qty) break;
                        if (T->n_cat == cap) {
                            cap *= 2;
                            T->cat = realloc(T->cat, sizeof(blk_shape) * (size_t)cap);
                        }
                        blk_shape* s = &T->cat[T->n_cat++];
                        s->ti = ti; s->oi = oi; s->a = a; s->b = b; s->k = k; s->cnt = cnt;
                        s->bw = a * w; s->bd = b * d; s->bh = k * h;
                    }
                }
            }
        }
    }
    T->by_type = malloc(sizeof(int*) * (size_t)(nt > 0 ? nt : 1));
    T->n_by_type = calloc((size_t)(nt > 0 ? nt : 1), sizeof(int));
    for (int i = 0; i < T->n_cat; i++) T->n_by_type[T->cat[i].ti]++;
    for (int ti = 0; ti < nt; ti++) {
        T->by_type[ti] = malloc(sizeof(int) * (size_t)(T->n_by_type[ti] > 0 ? T->n_by_type[ti] : 1));
        T->n_by_type[ti] = 0;
    }
    for (int i = 0; i < T->n_cat; i++) {
        const int ti = T->cat[i].ti;
        T->by_type[ti][T->n_by_type[ti]++] = i;
    }
    g_cmp_cat = T->cat;
    for (int ti = 0; ti < nt; ti++)
        if (T->n_by_type[ti] > 1)
            qsort(T->by_type[ti], (size_t)T->n_by_type[ti], sizeof(int), blk_prec_cmp);
}

static void blk_free(const orc_instance* inst, blk_tables* T) {
    for (int ti = 0; ti < inst->n_types; ti++) free(T->by_type[ti]);
    free(T->by_type); free(T->n_by_type); free(T->cat); free(T->ors); free(T->n_ors);
}

/* bottom support and flush side contact of shape s at point p
 * (blockproof/plp_block.cpp:68-84) */
static void blk_contact(int x0, int y0, int z0, const blk_shape* s, const int32_t* fast, int n_fast,
                        long long* bottom, long long* side) {
    const long long x = x0, y = y0, z = z0, bw = s->bw, bd = s->bd, bh = s->bh;
    long long bo = 0, si = 0;
    if (z == 0) bo = bw * bd;
    for (int j = 0; j < n_fast; j++) {
        const int32_t* b = fast + 6 * j;
        const long long ox = (x + bw < b[3] ? x + bw : b[3]) - (x > b[0] ? x : b[0]);
        const long long oy = (y + bd < b[4] ? y + bd : b[4]) - (y > b[1] ? y : b[1]);
        const long long oz = (z + bh < b[5] ? z + bh : b[5]) - (z > b[2] ? z : b[2]);
        if (b[5] == z && ox > 0 && oy > 0) bo += ox * oy;
        if (oy > 0 && oz > 0 && (b[3] == x || b[0] == x + bw)) si += oy * oz;
        if (ox > 0 && oz > 0 && (b[4] == y || b[1] == y + bd)) si += ox * oz;
    }
    *bottom = bo;
    *side = si;
}

static int blk_pass_t(const orc_instance* inst, const blk_tables* T, const orc_block_cfg* cfg,
                      double eps, orc_rng* rng, orc_place* out) {
    const int L = inst->L, W = inst->W, H = inst->H, nt = inst->n_types;
    int total = 0;
    for (int t = 0; t < nt; t++) total += inst->items[t].qty;
    int* rem = malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    for (int t = 0; t < nt; t++) rem[t] = inst->items[t].qty;
    int cap = 8 * total + 16;
    int32_t* cand = malloc(sizeof(int32_t) * 3 * (size_t)cap);
    int32_t* fast = malloc(sizeof(int32_t) * 6 * (size_t)(total > 0 ? total : 1));
    int* bshape = malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));   /* placed block shapes */
    int* feas = malloc(sizeof(int) * (size_t)cap);
    int* types = malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    int* plan = malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    int n_cand = 1, n_fast = 0;
    cand[0] = cand[1] = cand[2] = 0;
    for (;;) {
        /* plan: every type with copies left, block decomposition per type */
        int n_types = 0;
        for (int ti = 0; ti < nt; ti++)
            if (rem[ti] > 0 && T->n_ors[ti] > 0) types[n_types++] = ti;
        if (n_types == 0) break;
        g_cmp_inst = inst;
        qsort(types, (size_t)n_types, sizeof(int), blk_type_cmp);
        if (eps > 0.0 && orc_rng_random(rng) >= 1.0 - eps)
            for (int i = n_types - 1; i > 0; i--) {
                const int j = orc_rng_randrange(rng, i + 1);
                const int tmp = types[i]; types[i] = types[j]; types[j] = tmp;
            }
        int n_plan = 0;
        for (int q = 0; q < n_types; q++) {
            const int ti = types[q];
            int r = rem[ti];
            const int* shp = T->by_type[ti];
            const int ns = T->n_by_type[ti];
            while (r > 0) {
                int start = ns;
                while (start > 0 && T->cat[shp[start - 1]].cnt <= r) start--;
                if (start == ns) break;
                const int tk = cfg->topk < ns - start ? cfg->topk : ns - start;
                int pick = 0;
                if (eps > 0.0 && orc_rng_random(rng) >= 1.0 - eps) pick = orc_rng_randrange(rng, tk);
                plan[n_plan++] = shp[start + pick];
                r -= (int)T->cat[shp[start + pick]].cnt;
            }
        }
        if (n_plan == 0) break;
        g_cmp_cat = T->cat;
        qsort(plan, (size_t)n_plan, sizeof(int), blk_place_cmp);
        /* placement: extreme-point insertion at block granularity */
        int any = 0;
        for (int q = 0; q < n_plan; q++) {
            const blk_shape* s = &T->cat[plan[q]];
            if (rem[s->ti] < s->cnt) continue;
            int nf = 0;
            for (int ci = 0; ci < n_cand; ci++)
                if (orc_feasible_one(cand[3 * ci], cand[3 * ci + 1], cand[3 * ci + 2], s->bw, s->bd, s->bh,
                                     fast, n_fast, L, W, H))
                    feas[nf++] = ci;
            if (nf == 0) continue;
            int pc;
            if (eps > 0.0 && orc_rng_random(rng) >= 1.0 - eps) {
                pc = feas[orc_rng_randrange(rng, nf)];
            } else if (cfg->pick == 0) {
                pc = feas[0];
            } else {
                long long k0 = -1, k1 = -1;
                int bi = 0;
                for (int i = 0; i < nf; i++) {
                    long long sup, side;
                    blk_contact(cand[3 * feas[i]], cand[3 * feas[i] + 1], cand[3 * feas[i] + 2], s, fast,
                                n_fast, &sup, &side);
                    const long long p0 = cfg->pick == 1 ? sup : sup + side;
                    const long long p1 = cfg->pick == 1 ? side : sup;
                    if (p0 > k0 || (p0 == k0 && p1 > k1)) { k0 = p0; k1 = p1; bi = i; }
                }
                pc = feas[bi];
            }
            const int x = cand[3 * pc], y = cand[3 * pc + 1], z = cand[3 * pc + 2];
            bshape[n_fast] = plan[q];
            int32_t* f = fast + 6 * n_fast++;
            f[0] = x; f[1] = y; f[2] = z; f[3] = x + s->bw; f[4] = y + s->bd; f[5] = z + s->bh;
            /* extreme points: drop the strictly interior ones, add the 8 corners */
            int m = 0;
            for (int i = 0; i < n_cand; i++) {
                const int px = cand[3 * i], py = cand[3 * i + 1], pz = cand[3 * i + 2];
                if (x < px && px < x + s->bw && y < py && py < y + s->bd && z < pz && pz < z + s->bh) continue;
                cand[3 * m] = px; cand[3 * m + 1] = py; cand[3 * m + 2] = pz;
                m++;
            }
            for (int c = 0; c < 8; c++) {
                cand[3 * m] = x + ((c & 1) ? s->bw : 0);
                cand[3 * m + 1] = y + ((c & 2) ? s->bd : 0);
                cand[3 * m + 2] = z + ((c & 4) ? s->bh : 0);
                m++;
            }
            qsort(cand, (size_t)m, sizeof(int32_t) * 3, pt_cmp);
            int u = 0;
            for (int i = 0; i < m; i++) {
                if (u > 0 && pt_cmp(cand + 3 * (u - 1), cand + 3 * i) == 0) continue;
                if (u != i) memmove(cand + 3 * u, cand + 3 * i, sizeof(int32_t) * 3);
                u++;
            }
            n_cand = u;
            rem[s->ti] -= (int)s->cnt;
            any = 1;
        }
        if (!any) break;
    }
    /* decompose the blocks into item boxes (blockproof/plp_block.cpp:210-222) */
    int n = 0;
    for (int j = 0; j < n_fast; j++) {
        const blk_shape* s = &T->cat[bshape[j]];
        const int iw = s->bw / s->a, id = s->bd / s->b, ih = s->bh / s->k;
        for (int i = 0; i < s->a; i++)
            for (int jj = 0; jj < s->b; jj++)
                for (int t = 0; t < s->k; t++) {
                    orc_place* o = &out[n++];
                    o->type = s->ti;
                    o->x = fast[6 * j] + i * iw; o->y = fast[6 * j + 1] + jj * id; o->z = fast[6 * j + 2] + t * ih;
                    o->w = iw; o->d = id; o->h = ih;
                }
    }
    free(rem); free(cand); free(fast); free(bshape); free(feas); free(types); free(plan);
    return n;
}

int orc_block_pass(const orc_instance* inst, const orc_block_cfg* cfg, double eps, orc_rng* rng,
                   orc_place* out) {
    blk_tables T;
    blk_build(inst, cfg, &T);
    const int n = blk_pass_t(inst, &T, cfg, eps, rng, out);
    blk_free(inst, &T);
    return n;
}

/* run_block: blockproof/plp_block.cpp:228-304 (online best-of; the same
 * outcome as run()'s stored packings) */
void orc_block_run(const orc_instance* inst, int64_t seed, int n_passes, double time_limit_s,
                   double eps, int has_theta, double theta, double mu, const orc_block_cfg* cfg,
                   orc_result* res) {
    orc_rng rng;
    orc_rng_seed(&rng, (uint64_t)(seed < 0 ? -seed : seed));
    blk_tables T;
    blk_build(inst, cfg, &T);
    int total = 0;
    for (int t = 0; t < inst->n_types; t++) total += inst->items[t].qty;
    const size_t cap = (size_t)(total > 0 ? total : 1);
    orc_place* cur = malloc(sizeof(orc_place) * cap);
    orc_place* best_acc = malloc(sizeof(orc_place) * cap);
    orc_place* best_all = malloc(sizeof(orc_place) * cap);
    int n_acc = -1, n_all = -1;
    long long v_acc = -1, v_all = -1;
    double s_acc = 0, s_all = 0;
    const double t0 = now_s();
    int k = 0;
    for (;;) {
        const int n = blk_pass_t(inst, &T, cfg, eps, &rng, cur);
        k++;
        long long vol = 0;
        for (int i = 0; i < n; i++) vol += (long long)cur[i].w * cur[i].d * cur[i].h;
        const double sc = orc_stability_score(cur, n, mu);
        const int upd_all = vol > v_all || (vol == v_all && n > n_all);
        const int upd_acc = (!has_theta || sc >= theta) && (n_acc < 0 || vol > v_acc || (vol == v_acc && n > n_acc));
        if (upd_acc) {
            n_acc = n; v_acc = vol; s_acc = sc;
            memcpy(best_acc, cur, sizeof(orc_place) * (size_t)n);
        }
        if (upd_all) {
            n_all = n; v_all = vol; s_all = sc;
            memcpy(best_all, cur, sizeof(orc_place) * (size_t)n);
        }
        if (time_limit_s < 0 ? k >= n_passes : (now_s() - t0) >= time_limit_s) break;
    }
    const int use_acc = n_acc >= 0;
    res->n_boxes = use_acc ? n_acc : n_all;
    res->volume = use_acc ? v_acc : v_all;
    res->score = use_acc ? s_acc : s_all;
    res->fallback = !use_acc;
    res->n_passes = k;
    res->seed = seed;
    res->placements = malloc(sizeof(orc_place) * (size_t)(res->n_boxes > 0 ? res->n_boxes : 1));
    memcpy(res->placements, use_acc ? best_acc : best_all, sizeof(orc_place) * (size_t)res->n_boxes);
    res->time_s = now_s() - t0;
    free(cur); free(best_acc); free(best_all);
    blk_free(inst, &T);
}

void orc_free_result(orc_result* r) {
    free(r->placements);
    r->placements = NULL;
}

/* ------------------------------------------------------------------------ */
/* CPython float repr (shortest round-trip digits; fixed iff -4 < exp10 <= 16)
 * and json.dumps layout: plp/solver.py:297-307                             */
/* ------------------------------------------------------------------------ */

int orc_py_repr(double x, char* buf) {
    if (isnan(x)) return sprintf(buf, "nan");
    if (isinf(x)) return sprintf(buf, x < 0 ? "-inf" : "inf");
    if (x == 0.0) return sprintf(buf, signbit(x) ? "-0.0" : "0.0");
    const double a = fabs(x);
    char tmp[40];
    int prec = 1;
    for (; prec <= 17; prec++) {
        snprintf(tmp, sizeof tmp, "%.*e", prec - 1, a);
        if (strtod(tmp, NULL) == a) break;
    }
    char digits[24];
    int nd = 0;
    const char* e = strchr(tmp, 'e');
    for (const char* c = tmp; c < e; c++)
        if (*c != '.') digits[nd++] = *c;
    while (nd > 1 && digits[nd - 1] == '0') nd--;
    digits[nd] = '\0';
    const int decpt = atoi(e + 1) + 1;            /* a = 0.DIGITS * 10^decpt */
    char* o = buf;
    if (x < 0) *o++ = '-';
    if (decpt > -4 && decpt <= 16) {
        if (decpt <= 0) {
            o += sprintf(o, "0.");
            for (int i = 0; i < -decpt; i++) *o++ = '0';
            o += sprintf(o, "%s", digits);
        } else if (decpt >= nd) {
            o += sprintf(o, "%s", digits);
            for (int i = nd; i < decpt; i++) *o++ = '0';
            o += sprintf(o, ".0");
        } else {
            memcpy(o, digits, (size_t)decpt);
            o += decpt;
            *o++ = '.';
            o += sprintf(o, "%s", digits + decpt);
        }
    } else {
        *o++ = digits[0];
        if (nd > 1) {
            *o++ = '.';
            o += sprintf(o, "%s", digits + 1);
        }
        const int ex = decpt - 1;
        o += sprintf(o, "e%c%02d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    }
    *o = '\0';
    return (int)(o - buf);
}

typedef struct { char* p; int len, cap; } sbuf_t;

static void sb_put(sbuf_t* s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
#include <stdarg.h>
static void sb_put(sbuf_t* s, const char* fmt, ...) {
    char tmp[128];
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(tmp, sizeof tmp, fmt, ap);
    va_end(ap);
    for (int i = 0; i < n; i++) {
        if (s->len < s->cap) s->p[s->len] = tmp[i];
        s->len++;
    }
}

int orc_to_json(const orc_result* r, char* buf, int cap) {
    sbuf_t s = {buf, 0, cap > 0 ? cap - 1 : 0};
    char a[40], b[40];
    orc_py_repr(r->score, a);
    orc_py_repr(r->time_s, b);
    sb_put(&s, "{\"n_boxes\": %d, \"volume_cm3\": %lld, \"stability_score\": %s", r->n_boxes,
           (long long)r->volume, a);
    sb_put(&s, ", \"fallback\": %s, \"n_passes\": %d, \"time_s\": %s, \"seed\": %lld",
           r->fallback ? "true" : "false", r->n_passes, b, (long long)r->seed);
    sb_put(&s, ", \"placements\": [");
    for (int i = 0; i < r->n_boxes; i++) {
        const orc_place* p = &r->placements[i];
        sb_put(&s, "%s[%d, %d, %d, %d, %d, %d, %d]", i ? ", " : "", p->type, p->x, p->y, p->z,
               p->w, p->d, p->h);
    }
    sb_put(&s, "]}");
    if (cap > 0) buf[s.len < cap ? s.len : cap - 1] = '\0';
    return s.len;
}
