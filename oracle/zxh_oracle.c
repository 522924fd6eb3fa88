/*
 * zxh_oracle.c -- TEST INFRASTRUCTURE ONLY (see zxh_oracle.h).
 *
 * CPU restatement of the reference path, ZXH-Sim (AxEquals-b/ZXH_ADAE), paths below
 * relative to src/zxh/ of that project:
 *   - gate recording and lowering ........ src/core/zxh.cpp:234-310
 *   - execute() scheduler ................ src/core/zxh.cpp:312-553
 *   - U3 fusion, identity drop ........... src/core/zxh.cpp:101-172,363-428
 *   - GF(2) affine map, solve, selectors . src/core/bitmat.cpp:34-161, selector.cpp:20-49
 *   - lazy expansion, calc_mem ........... src/core/zxh.cpp:648-719, src/sv/sv_common.cpp:330-349
 *   - gate kernels (serial semantics) .... src/kernel/kernel_general.cpp:72-356
 *   - diagonal-window bucket order ....... src/kernel/kernel_general.cpp:72-113,288-330
 *   - GPU multinomial sampler ............ src/measure/measure_cuda.cu:250-286,387-516,642-691
 *   - seeds ............................... src/measure/measure_cuda.cu:103-109,1026-1035
 *   - result mapping ...................... src/measure/measure_cuda.cu:315-338
 *   - get_state ordering .................. src/core/zxh.cpp:579-636
 * Complex arithmetic uses C99 double complex, which GCC evaluates with the same
 * expressions as libstdc++'s std::complex<double>, so the state is bit-identical to
 * the reference's serial CPU backend on the same gate list.
 */
#include "zxh_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

enum { G_NONE = 0, G_BARRIER, G_Z, G_RZ, G_P, G_CRZ, G_CP, G_X, G_CX, G_H, G_U3, G_RX };

typedef struct {
    uint32_t type, cq, q, reserved;
    double theta, lambda, phi;
} rec_t;

static const double PI_ = 3.14159265358979323846;

typedef struct {
    uint64_t alpha;
    int beta;
} sel_t;

typedef struct {
    sel_t s0, s1;
    double theta;
} diag_t;

typedef struct {
    diag_t *v;
    size_t n, cap;
} dvec_t;

typedef struct {
    int active;
    cplx u00, u01, u10, u11;
} acc_t;

struct zxo_sim {
    int N, disable_x, eager;
    rec_t *gates;
    size_t ngates, cap;
    /* execution state */
    uint64_t rows[64];
    int m;     /* columns of A */
    uint64_t b;
    cplx *sv;  /* 2^M */
    int M, msv;
    cplx gphase;
    int executed;
    dvec_t p_l, p_h, p_x, cp_ll, cp_hh, cp_hl;
};

/* ---- GF(2) affine map (bitmat.cpp) ---------------------------------------- */

static int parity64(uint64_t x) { return __builtin_popcountll(x) & 1; }

/* solve A x = e_q by Gaussian elimination; A has full column rank so x is unique
 * (bitmat.cpp:46-122). */
static int solve_eq(const uint64_t *rows, int N, int m, int q, uint64_t *x)
{
    uint64_t r[64];
    int rhs[64], pivot[64];
    for (int i = 0; i < N; i++) {
        r[i] = rows[i];
        rhs[i] = (i == q);
    }
    if (m == 0) {
        *x = 0;
        return rhs[q] ? 0 : 1;
    }
    int row = 0;
    for (int col = 0; col < m; col++) {
        pivot[col] = -1;
        if (row >= N) continue;
        int piv = row;
        while (piv < N && !((r[piv] >> col) & 1)) piv++;
        if (piv == N) continue;
        if (piv != row) {
            uint64_t t = r[piv]; r[piv] = r[row]; r[row] = t;
            int tb = rhs[piv]; rhs[piv] = rhs[row]; rhs[row] = tb;
        }
        for (int i = 0; i < N; i++)
            if (i != row && ((r[i] >> col) & 1)) {
                r[i] ^= r[row];
                rhs[i] ^= rhs[row];
            }
        pivot[col] = row;
        row++;
    }
    for (int i = 0; i < N; i++)
        if (r[i] == 0 && rhs[i]) return 0;
    uint64_t sol = 0;
    for (int col = 0; col < m; col++)
        if (pivot[col] >= 0 && rhs[pivot[col]]) sol |= (uint64_t)1 << col;
    *x = sol;
    return 1;
}

static sel_t make_sel(const zxo_sim *s, int q)
{
    sel_t r;
    /* make_local_selector with block_start 0 keeps alpha & low_bits(m) and beta
     * (zxh.cpp:55-60); alpha never has bits >= m. */
    r.alpha = s->rows[q] & (s->msv >= 64 ? ~0ULL : ((1ULL << s->msv) - 1));
    r.beta = (int)((s->b >> q) & 1);
    return r;
}

static int sel_eval(sel_t sl, uint64_t x) { return parity64(x & sl.alpha) ^ sl.beta; }

/* ---- diag window (kernel_general.cpp:41-113,278-345) ---------------------- */

static void dpush(dvec_t *d, sel_t a, sel_t b, double th)
{
    if (d->n == d->cap) {
        d->cap = d->cap ? d->cap * 2 : 64;
        d->v = (diag_t *)realloc(d->v, d->cap * sizeof(diag_t));
    }
    d->v[d->n].s0 = a;
    d->v[d->n].s1 = b;
    d->v[d->n].theta = th;
    d->n++;
}

enum { C_LOW, C_HIGH, C_CROSS };
static int classify(sel_t sl)
{
    if ((sl.alpha >> 8) == 0) return C_LOW;
    if ((sl.alpha & 0xffULL) == 0) return C_HIGH;
    return C_CROSS;
}

static int diag_empty(const zxo_sim *s)
{
    return !(s->p_l.n || s->p_h.n || s->p_x.n || s->cp_ll.n || s->cp_hh.n || s->cp_hl.n);
}

static void diag_reset(zxo_sim *s)
{
    s->p_l.n = s->p_h.n = s->p_x.n = s->cp_ll.n = s->cp_hh.n = s->cp_hl.n = 0;
}

static void diag_push_p(zxo_sim *s, sel_t sl, double th)
{
    sel_t none = {0, 0};
    switch (classify(sl)) {
    case C_LOW: dpush(&s->p_l, sl, none, th); break;
    case C_HIGH: dpush(&s->p_h, sl, none, th); break;
    default: dpush(&s->p_x, sl, none, th); break;
    }
}

static int diag_try_push_cp(zxo_sim *s, sel_t a, sel_t b, double th)
{
    int ca = classify(a), cb = classify(b);
    if (ca == C_LOW && cb == C_LOW) { dpush(&s->cp_ll, a, b, th); return 1; }
    if (ca == C_HIGH && cb == C_HIGH) { dpush(&s->cp_hh, a, b, th); return 1; }
    if (ca == C_LOW && cb == C_HIGH) { dpush(&s->cp_hl, a, b, th); return 1; }
    if (ca == C_HIGH && cb == C_LOW) { dpush(&s->cp_hl, b, a, th); return 1; }
    return 0;
}

static cplx phase_of(double a) { return cexp(CMPLX(0.0, a)); }

static void diag_flush(zxo_sim *s)
{
    if (diag_empty(s)) return;
    const uint64_t n = 1ULL << s->msv;
    for (uint64_t x = 0; x < n; x++) {
        const uint64_t lane = x & 0xffULL, slice = x & ~0xffULL;
        double t = 0.0;
        for (size_t i = 0; i < s->p_l.n; i++) if (sel_eval(s->p_l.v[i].s0, lane)) t += s->p_l.v[i].theta;
        for (size_t i = 0; i < s->p_h.n; i++) if (sel_eval(s->p_h.v[i].s0, slice)) t += s->p_h.v[i].theta;
        for (size_t i = 0; i < s->p_x.n; i++) if (sel_eval(s->p_x.v[i].s0, x)) t += s->p_x.v[i].theta;
        for (size_t i = 0; i < s->cp_ll.n; i++)
            if (sel_eval(s->cp_ll.v[i].s0, lane) && sel_eval(s->cp_ll.v[i].s1, lane)) t += s->cp_ll.v[i].theta;
        for (size_t i = 0; i < s->cp_hh.n; i++)
            if (sel_eval(s->cp_hh.v[i].s0, slice) && sel_eval(s->cp_hh.v[i].s1, slice)) t += s->cp_hh.v[i].theta;
        for (size_t i = 0; i < s->cp_hl.n; i++)
            if (sel_eval(s->cp_hl.v[i].s0, lane) && sel_eval(s->cp_hl.v[i].s1, slice)) t += s->cp_hl.v[i].theta;
        if (t != 0.0) s->sv[x] *= phase_of(t);
    }
    diag_reset(s);
}

/* ---- state and kernels ----------------------------------------------------- */

static void expand(zxo_sim *s) { s->msv++; } /* new half is already zero (sv_common.cpp:330-349) */

/* u3_block_kernel (kernel_general.cpp:121-141) */
static void u3_block(zxo_sim *s, uint64_t delta, sel_t sl, cplx u00, cplx u01, cplx u10, cplx u11)
{
    const uint64_t n = 1ULL << s->msv;
    for (uint64_t i = 0; i < n; i++) {
        if (sel_eval(sl, i)) continue;
        const uint64_t j = i ^ delta;
        if (j >= n) continue;
        const cplx ev = s->sv[i], od = s->sv[j];
        s->sv[i] = u00 * ev + u01 * od;
        s->sv[j] = u10 * ev + u11 * od;
    }
}

static void build_u3(double th, double la, double ph, cplx *u00, cplx *u01, cplx *u10, cplx *u11)
{
    /* zxh.cpp:101-113 */
    const double c = cos(th / 2.0), sn = sin(th / 2.0);
    const cplx el = phase_of(la), ep = phase_of(ph), epl = phase_of(ph + la);
    *u00 = CMPLX(c, 0.0);
    *u01 = -el * sn;
    *u10 = ep * sn;
    *u11 = epl * c;
}

static uint64_t solve_expand(zxo_sim *s, int q)
{
    uint64_t d = 0;
    if (!solve_eq(s->rows, s->N, s->m, q, &d)) {
        expand(s);
        s->rows[q] |= 1ULL << s->m; /* append_col(e_q) */
        s->m++;
        d = 1ULL << (s->m - 1);
    }
    return d;
}

static uint64_t lowmask(int bits) { return bits >= 64 ? ~0ULL : ((1ULL << bits) - 1); }

static void apply_u3(zxo_sim *s, int q, double th, double la, double ph)
{
    /* zxh.cpp:782-825 (1 process: delta_b == 0) */
    const uint64_t d = solve_expand(s, q);
    const sel_t sl = make_sel(s, q);
    cplx u00, u01, u10, u11;
    build_u3(th, la, ph, &u00, &u01, &u10, &u11);
    u3_block(s, d & lowmask(s->msv), sl, u00, u01, u10, u11);
}

static void apply_x_explicit(zxo_sim *s, int q)
{
    /* zxh.cpp:742-759, x_block_kernel kernel_general.cpp:143-156 */
    const uint64_t d = solve_expand(s, q) & lowmask(s->msv);
    const sel_t sl = make_sel(s, q);
    const uint64_t n = 1ULL << s->msv;
    for (uint64_t i = 0; i < n; i++) {
        if (sel_eval(sl, i)) continue;
        const uint64_t j = i ^ d;
        if (j >= n) continue;
        cplx t = s->sv[i]; s->sv[i] = s->sv[j]; s->sv[j] = t;
    }
}

static void apply_cx_explicit(zxo_sim *s, int cq, int q)
{
    /* zxh.cpp:761-780, cx_block_kernel kernel_general.cpp:158-171 */
    const uint64_t d = solve_expand(s, q) & lowmask(s->msv);
    const sel_t sc = make_sel(s, cq), st = make_sel(s, q);
    const uint64_t n = 1ULL << s->msv;
    for (uint64_t i = 0; i < n; i++) {
        if (sel_eval(st, i) || !sel_eval(sc, i)) continue;
        const uint64_t j = i ^ d;
        if (j >= n) continue;
        cplx t = s->sv[i]; s->sv[i] = s->sv[j]; s->sv[j] = t;
    }
}

/* ---- U3 fusion (zxh.cpp:115-172) ------------------------------------------- */

static const double kEps = (double)1e-5f; /* kU3BatchEps = 1e-5f promoted to double */

static int close_val(cplx a, cplx b) { return cabs(a - b) <= kEps; }

static int is_identity(const acc_t *a)
{
    return close_val(a->u00, CMPLX(1.0, 0.0)) && close_val(a->u01, CMPLX(0.0, 0.0)) &&
           close_val(a->u10, CMPLX(0.0, 0.0)) && close_val(a->u11, CMPLX(1.0, 0.0));
}

static void acc_reset(acc_t *a)
{
    a->active = 0;
    a->u00 = CMPLX(1.0, 0.0); a->u01 = CMPLX(0.0, 0.0);
    a->u10 = CMPLX(0.0, 0.0); a->u11 = CMPLX(1.0, 0.0);
}

static void left_mul(acc_t *a, cplx n00, cplx n01, cplx n10, cplx n11)
{
    const cplx o00 = a->u00, o01 = a->u01, o10 = a->u10, o11 = a->u11;
    a->u00 = n00 * o00 + n01 * o10;
    a->u01 = n00 * o01 + n01 * o11;
    a->u10 = n10 * o00 + n11 * o10;
    a->u11 = n10 * o01 + n11 * o11;
    a->active = !is_identity(a);
}

/* ---- recording ------------------------------------------------------------- */

zxo_sim *zxo_create(int n, int disable_x, int eager_expand_all)
{
    if (n < 1 || n > 63) return NULL;
    zxo_sim *s = (zxo_sim *)calloc(1, sizeof(zxo_sim));
    s->N = n;
    s->disable_x = disable_x;
    s->eager = eager_expand_all;
    s->gphase = CMPLX(1.0, 0.0);
    return s;
}

void zxo_destroy(zxo_sim *s)
{
    if (!s) return;
    free(s->gates);
    free(s->sv);
    free(s->p_l.v); free(s->p_h.v); free(s->p_x.v);
    free(s->cp_ll.v); free(s->cp_hh.v); free(s->cp_hl.v);
    free(s);
}

static void add_gate(zxo_sim *s, uint32_t t, uint32_t cq, uint32_t q, double th, double la, double ph)
{
    if (s->ngates == s->cap) {
        s->cap = s->cap ? s->cap * 2 : 256;
        s->gates = (rec_t *)realloc(s->gates, s->cap * sizeof(rec_t));
    }
    rec_t r = {t, cq, q, 0, th, la, ph};
    s->gates[s->ngates++] = r;
}

int zxo_push(zxo_sim *s, const void *recs, size_t count)
{
    const rec_t *g = (const rec_t *)recs;
    for (size_t i = 0; i < count; i++) {
        const uint32_t t = g[i].type, q = g[i].q, cq = g[i].cq;
        const int two = (t == G_CRZ || t == G_CP || t == G_CX);
        if (t != G_BARRIER && (int)q >= s->N) return 1;
        if (two && (int)cq >= s->N) return 1;
        switch (t) {
        case G_BARRIER: add_gate(s, G_BARRIER, 0, 0, 0, 0, 0); break;
        case G_Z: add_gate(s, G_Z, 0, q, 0, 0, 0); break;
        case G_RZ: add_gate(s, G_RZ, 0, q, g[i].theta, 0, 0); break;
        case G_P: add_gate(s, G_P, 0, q, g[i].theta, 0, 0); break;
        case G_CRZ: /* zxh.cpp:246-252 */
            add_gate(s, G_P, 0, cq, -0.5 * g[i].theta, 0, 0);
            add_gate(s, G_CP, cq, q, g[i].theta, 0, 0);
            break;
        case G_CP: add_gate(s, G_CP, cq, q, g[i].theta, 0, 0); break;
        case G_X: add_gate(s, G_X, 0, q, 0, 0, 0); break;
        case G_CX: add_gate(s, G_CX, cq, q, 0, 0, 0); break;
        case G_H: add_gate(s, G_H, 0, q, 0, 0, 0); break;
        case G_U3: add_gate(s, G_U3, 0, q, g[i].theta, g[i].lambda, g[i].phi); break;
        case G_RX: add_gate(s, G_U3, 0, q, g[i].theta, PI_ / 2.0, -PI_ / 2.0); break; /* zxh.cpp:303-310 */
        default: return 1;
        }
    }
    return 0;
}

int zxo_clear_gates(zxo_sim *s)
{
    s->ngates = 0;
    s->gphase = CMPLX(1.0, 0.0);
    return 0;
}

size_t zxo_required_M(zxo_sim *s)
{
    /* calc_mem, zxh.cpp:648-681 */
    uint64_t rows[64] = {0};
    int m = 0;
    for (size_t i = 0; i < s->ngates; i++) {
        const rec_t *g = &s->gates[i];
        int is_exp = 0;
        if (g->type == G_X || g->type == G_CX) {
            if (!s->disable_x) {
                if (g->type == G_CX) rows[g->q] ^= rows[g->cq];
            } else {
                is_exp = 1;
            }
        } else if (g->type == G_H || g->type == G_U3) {
            is_exp = 1;
        }
        if (is_exp) {
            uint64_t d;
            if (!solve_eq(rows, s->N, m, (int)g->q, &d)) {
                rows[g->q] |= 1ULL << m;
                m++;
            }
        }
    }
    return (size_t)m;
}

/* ---- execute (zxh.cpp:312-553) --------------------------------------------- */

static int is_u3(const rec_t *g) { return g->type == G_H || g->type == G_U3; }

static void flush_u3_batch(zxo_sim *s, acc_t *pend, int *pend_count)
{
    if (*pend_count == 0) return;
    /* descriptors in qubit order, each one full sweep (kernel_general.cpp:173-202) */
    for (int q = 0; q < s->N; q++) {
        if (!pend[q].active) continue;
        uint64_t d = 0;
        solve_eq(s->rows, s->N, s->m, q, &d);
        const sel_t sl = make_sel(s, q);
        u3_block(s, d & lowmask(s->msv), sl, pend[q].u00, pend[q].u01, pend[q].u10, pend[q].u11);
    }
    for (int q = 0; q < s->N; q++) acc_reset(&pend[q]);
    *pend_count = 0;
}

int zxo_execute(zxo_sim *s)
{
    const int M = s->eager ? s->N : (int)zxo_required_M(s);
    if (M > 40) return 2; /* oracle is for small states only */
    free(s->sv);
    s->M = M;
    s->sv = (cplx *)calloc((size_t)1 << M, sizeof(cplx));
    if (!s->sv) return 3;
    s->sv[0] = CMPLX(1.0, 0.0);
    s->msv = 0;
    s->gphase = CMPLX(1.0, 0.0);
    memset(s->rows, 0, sizeof(s->rows));
    s->m = 0;
    s->b = 0;
    if (s->eager) { /* expand_all, zxh.cpp:721-729 */
        s->msv = s->N;
        for (int q = 0; q < s->N; q++) s->rows[q] = 1ULL << q;
        s->m = s->N;
    }
    diag_reset(s);
    acc_t pend[64];
    for (int q = 0; q < 64; q++) acc_reset(&pend[q]);
    int pend_count = 0;

    for (size_t gi = 0; gi < s->ngates;) {
        const rec_t *g = &s->gates[gi];
        if (is_u3(g)) {
            diag_flush(s);
            while (gi < s->ngates && is_u3(&s->gates[gi])) {
                const rec_t *u = &s->gates[gi];
                const double th = u->type == G_H ? PI_ / 2.0 : u->theta;
                const double la = u->type == G_H ? PI_ : u->lambda;
                const double ph = u->type == G_H ? 0.0 : u->phi;
                uint64_t d;
                if (!solve_eq(s->rows, s->N, s->m, (int)u->q, &d)) {
                    flush_u3_batch(s, pend, &pend_count);
                    apply_u3(s, (int)u->q, th, la, ph);
                    gi++;
                    continue;
                }
                /* absorb_u3_gate, zxh.cpp:363-388 */
                cplx u00, u01, u10, u11;
                build_u3(th, la, ph, &u00, &u01, &u10, &u11);
                acc_t *a = &pend[u->q];
                const int was = a->active;
                if (!was) {
                    a->active = 1;
                    a->u00 = CMPLX(1.0, 0.0); a->u01 = CMPLX(0.0, 0.0);
                    a->u10 = CMPLX(0.0, 0.0); a->u11 = CMPLX(1.0, 0.0);
                }
                left_mul(a, u00, u01, u10, u11);
                if (!was && a->active) pend_count++;
                else if (was && !a->active) pend_count--;
                gi++;
            }
            flush_u3_batch(s, pend, &pend_count);
            continue;
        }
        switch (g->type) {
        case G_BARRIER: diag_flush(s); break;
        case G_Z:
        case G_RZ: {
            const double th = g->type == G_Z ? PI_ : g->theta;
            diag_push_p(s, make_sel(s, (int)g->q), th);
            s->gphase *= phase_of(-0.5 * th);
            break;
        }
        case G_P: diag_push_p(s, make_sel(s, (int)g->q), g->theta); break;
        case G_X:
            if (s->disable_x) { diag_flush(s); apply_x_explicit(s, (int)g->q); }
            else s->b ^= 1ULL << g->q;
            break;
        case G_CX:
            if (s->disable_x) { diag_flush(s); apply_cx_explicit(s, (int)g->cq, (int)g->q); }
            else {
                s->rows[g->q] ^= s->rows[g->cq];
                if ((s->b >> g->cq) & 1) s->b ^= 1ULL << g->q;
            }
            break;
        case G_CP: {
            const sel_t a = make_sel(s, (int)g->cq), b = make_sel(s, (int)g->q);
            if (!diag_try_push_cp(s, a, b, g->theta)) {
                diag_flush(s);
                /* cp_kernel, kernel_general.cpp:347-356 */
                const uint64_t n = 1ULL << s->msv;
                const cplx ph = phase_of(g->theta);
                for (uint64_t x = 0; x < n; x++)
                    if (sel_eval(a, x) && sel_eval(b, x)) s->sv[x] *= ph;
            }
            break;
        }
        default: break;
        }
        gi++;
    }
    diag_flush(s);
    s->executed = 1;
    return 0;
}

static uint64_t rev_bits(uint64_t v, int n)
{
    uint64_t o = 0;
    for (int i = 0; i < n; i++) o = (o << 1) | ((v >> i) & 1);
    return o;
}

static uint64_t virt_of(const zxo_sim *s, uint64_t real)
{
    uint64_t v = 0;
    for (int q = 0; q < s->N; q++)
        if (parity64(real & s->rows[q]) ^ (int)((s->b >> q) & 1)) v |= 1ULL << q;
    return v;
}

int zxo_get_state(zxo_sim *s, double *out, int order)
{
    if (!s->executed) return 2;
    const uint64_t vsize = 1ULL << s->N, rsize = 1ULL << s->m;
    cplx *o = (cplx *)out;
    for (uint64_t i = 0; i < vsize; i++) o[i] = CMPLX(0.0, 0.0);
    for (uint64_t r = 0; r < rsize; r++) {
        const uint64_t v = virt_of(s, r);
        const uint64_t idx = order == 0 ? rev_bits(v, s->N) : v;
        o[idx] = s->sv[r] * s->gphase;
    }
    return 0;
}

int zxo_real_state(zxo_sim *s, double *out, size_t *m_out)
{
    if (!s->executed) return 2;
    memcpy(out, s->sv, ((size_t)1 << s->msv) * sizeof(cplx));
    *m_out = (size_t)s->msv;
    return 0;
}

void zxo_global_phase(zxo_sim *s, double *re, double *im)
{
    *re = creal(s->gphase);
    *im = cimag(s->gphase);
}

int zxo_affine(zxo_sim *s, uint64_t *rows, uint64_t *b, size_t *m_out)
{
    memcpy(rows, s->rows, sizeof(uint64_t) * (size_t)s->N);
    *b = s->b;
    *m_out = (size_t)s->m;
    return 0;
}

/* ---- GPU sampler restatement (measure_cuda.cu) ------------------------------ */

static uint64_t splitmix64(uint64_t x)
{
    uint64_t z = x + 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static uint64_t mix_seed(uint64_t base, uint64_t salt)
{
    uint64_t z = base + 0x9e3779b97f4a7c15ULL + salt;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static double uniform_open01(uint64_t seed)
{
    const uint64_t mant = splitmix64(seed) >> 11;
    /* (2^53 + 1.0) rounds to 2^53 in double, as on the device */
    return ((double)mant + 1.0) / ((double)(1ULL << 53) + 1.0);
}

double zxo_uniform(uint64_t seed, int stream, uint64_t idx)
{
    const uint64_t s0 = mix_seed(seed, 0);
    if (stream == 0) return uniform_open01(s0 ^ (0x510e527fade682d1ULL + idx));
    return uniform_open01(mix_seed(s0, 1) ^ (0x9b05688c2b3e6c1fULL + idx));
}

static size_t upper_search(const double *cdf, size_t n, double tau)
{
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] <= tau) lo = mid + 1;
        else hi = mid;
    }
    return lo >= n ? n - 1 : lo;
}

int zxo_sample_gpu(zxo_sim *s, uint64_t seed, size_t shots, uint64_t *words, uint64_t *real_out)
{
    if (!s->executed) return 2;
    const size_t wc = ((size_t)s->N + 63) / 64;
    memset(words, 0, shots * wc * sizeof(uint64_t));
    if (shots == 0) return 0;
    const size_t local = (size_t)1 << s->msv;
    const size_t seglen = local < 4096 ? local : 4096;
    const size_t nseg = (local + seglen - 1) / seglen;
    double *mass = (double *)malloc(nseg * sizeof(double));
    double *cdfm = (double *)malloc(nseg * sizeof(double));
    uint64_t *counts = (uint64_t *)calloc(nseg, sizeof(uint64_t));
    uint64_t *offs = (uint64_t *)malloc(nseg * sizeof(uint64_t));
    uint64_t *real = (uint64_t *)calloc(shots, sizeof(uint64_t));
    double *cdf = (double *)malloc(seglen * sizeof(double));
    double *scr = (double *)malloc(seglen * sizeof(double));
    /* segment_mass_kernel: 256 strided partial sums, then a shared-memory tree */
    for (size_t g = 0; g < nseg; g++) {
        double sh[256];
        for (int t = 0; t < 256; t++) {
            double loc = 0.0;
            for (size_t k = (size_t)t; k < seglen; k += 256) {
                const cplx v = s->sv[g * seglen + k];
                loc += creal(v) * creal(v) + cimag(v) * cimag(v);
            }
            sh[t] = loc;
        }
        for (int st = 128; st >= 1; st >>= 1)
            for (int t = 0; t < st; t++) sh[t] += sh[t + st];
        mass[g] = sh[0];
    }
    double run = 0.0;
    for (size_t g = 0; g < nseg; g++) { run += mass[g]; cdfm[g] = run; }
    const uint64_t stream = mix_seed(seed, 0);
    const double total = cdfm[nseg - 1];
    if (total > 0.0)
        for (size_t i = 0; i < shots; i++) {
            const double u = uniform_open01(stream ^ (0x510e527fade682d1ULL + (uint64_t)i));
            counts[upper_search(cdfm, nseg, u * total)]++;
        }
    uint64_t acc = 0;
    for (size_t g = 0; g < nseg; g++) { offs[g] = acc; acc += counts[g]; }
    const uint64_t stream2 = mix_seed(stream, 1);
    for (size_t g = 0; g < nseg; g++) {
        if (counts[g] == 0) continue;
        for (size_t k = 0; k < seglen; k++) {
            const cplx v = s->sv[g * seglen + k];
            cdf[k] = creal(v) * creal(v) + cimag(v) * cimag(v);
        }
        for (size_t st = 1; st < seglen; st <<= 1) { /* Hillis-Steele, measure_cuda.cu:479-487 */
            for (size_t k = 0; k < seglen; k++) scr[k] = k >= st ? cdf[k - st] : 0.0;
            for (size_t k = 0; k < seglen; k++) cdf[k] += scr[k];
        }
        const double segtot = cdf[seglen - 1];
        if (segtot <= 0.0) continue;
        for (uint64_t ls = 0; ls < counts[g]; ls++) {
            const uint64_t oi = offs[g] + ls;
            const double u = uniform_open01(stream2 ^ (0x9b05688c2b3e6c1fULL + oi));
            real[oi] = g * seglen + upper_search(cdf, seglen, u * segtot);
        }
    }
    for (size_t i = 0; i < shots; i++) {
        const uint64_t v = virt_of(s, real[i]);
        for (int q = 0; q < s->N; q++)
            if ((v >> q) & 1) words[i * wc + (q >> 6)] |= 1ULL << (q & 63);
        if (real_out) real_out[i] = real[i];
    }
    free(mass); free(cdfm); free(counts); free(offs); free(real); free(cdf); free(scr);
    return 0;
}
