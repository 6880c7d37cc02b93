/*
 * comer2_oracle.c -- CPU oracle of the COMER2 search hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never part of the product).
 * A plain-C restatement of the reference algorithm; every function cites the
 * reference file:line it follows (paths relative to the comer2 source root).
 * Built twice by oracle/Makefile: -DREAL=float and -DREAL=double.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "comer2_oracle.h"

#ifndef REAL
#define REAL float
#endif
typedef REAL real;

#define IS_FLOAT (sizeof(real) == sizeof(float))
static inline real LOG(real x) { return IS_FLOAT ? (real)logf((float)x) : (real)log((double)x); }
static inline real SQRT(real x) { return IS_FLOAT ? (real)sqrtf((float)x) : (real)sqrt((double)x); }
static inline real MAXR(real a, real b) { return a < b ? b : a; }   /* myhdmax, cucom/cucommon.h:66 */

#define NAA 20
#define NCV 19
#define NSS 3
#define LOG0 (-32768.0f)

/* transitions into position i: index i of the (len+1)-row array.
 * DP uses: MMp, MIc(i+1), MDp, IMp, IIc(i+1), DMp, DDp
 * (src/libmycu/cudp/CuBatchDP_init.cuh:132-155, CuBatchDP_com.h:87-96) */
enum { T_MM = 0, T_MI, T_MD, T_IM, T_II, T_DM, T_DD };

typedef struct { real MM, MI, MD, IM, II, DM, DD; } trn7;

static trn7 get_trn(const orc_profile* p, int i)
{
    trn7 t;
    if (i < 0 || i >= p->len) {   /* DPLocInitTrnProbs: log 0 */
        t.MM = t.MI = t.MD = t.IM = t.II = t.DM = t.DD = LOG0;
        return t;
    }
    const float* a = p->trn + (size_t)i * 7;
    const float* b = p->trn + (size_t)(i + 1) * 7;
    t.MM = a[T_MM]; t.MI = b[T_MI]; t.MD = a[T_MD];
    t.IM = a[T_IM]; t.II = b[T_II]; t.DM = a[T_DM]; t.DD = a[T_DD];
    return t;
}

/* ---------------------------------------------------------------------- */
/* Context-vector constants as _TCTXVECT computes them in float
 * (src/libpro/srcpro/TCTXVECT.cpp:26-54): DIM = 19, KAPPA0 = 0.1, NU0 = DIM. */
void orc_cv_constants(float* lokappa0, float* pownu0, float* cterm)
{
    const int dim = NCV;
    const float kappa0 = 0.1f;
    const float nu0 = (float)dim;
    float lo = 1.f / kappa0;
    float pw = -0.5f * (nu0 + 2.f);
    float ct = (0.5f * dim + pw) * (logf(kappa0) - logf(kappa0 + 2.f));
    float sum = 0.0f;
    for (int ii = 1; ii <= dim; ii++)
        sum += logf(nu0 + 1.0f - ii) - 0.69314718055994530941723212146f;
    ct += sum;
    *lokappa0 = lo; *pownu0 = pw; *cterm = ct;
}

/* ---------------------------------------------------------------------- */
/* Score of one cell (query position i, db position j).
 * aa term:  src/libmycu/cusco/CuBatchScoreMatrix_Init.cu:129-182
 *           (shift 0.002 with MAPALN, 0.0003 otherwise: _Init.cuh:14-15)
 * SS term:  src/libmycu/cusco/CuBatchScoreMatrix_ssss.cuh:48-131, index rule
 *           GetSSSSTableIndex (:25-31), table SerializedScoresSM.cuh:103-120
 * CV term:  src/libmycu/cusco/CuBatchScoreMatrix_cvs2s.cuh:47-136, map
 *           SerializedCVS2Scores.cuh:377-410
 * total:    _ssss_cvs2s.cu:250-266  S = S0 + (SS + CV), MOD = (SS + CV) - 0.5*cvswgt
 */
static real score_aa(const orc_params* P, const orc_profile* q, const orc_profile* d, int i, int j)
{
    const float* qf = q->trg + (size_t)i * NAA;
    const float* df = d->trg + (size_t)j * NAA;
    real s = 0;
    for (int a = 0; a < NAA; a++)
        s += ((real)qf[a] * (real)df[a]) / ((real)0.5f * ((real)q->bkg[a] + (real)d->bkg[a]));
    real shift = P->mapaln ? (real)0.002f : (real)0.0003f;
    return LOG(s) - shift;
}

static int ss_index(int state, float prb) { return state * 10 + (int)(prb * 9.999f); }

static real score_ss(const orc_params* P, const orc_profile* q, const orc_profile* d, int i, int j)
{
    const float* qs = q->ss + (size_t)i * NSS;
    const float* ds = d->ss + (size_t)j * NSS;
    const int card = P->ssss_card;
    real s = 0;
    for (int a = 0; a < NSS; a++) {
        real f1 = qs[a];
        int row = ss_index(a, qs[a]);
        for (int b = 0; b < NSS; b++) {
            real f2 = ds[b];
            int col = ss_index(b, ds[b]);
            s += f1 * f2 * (real)P->ssss[row * card + col];
        }
    }
    if ((real)-99.f < s) {
        real f1 = qs[NSS - 1], f2 = ds[NSS - 1];
        s += (f1 + (real)0.1f) * (f2 + (real)0.1f) * (real)0.1111111f;
        s -= (real)0.05f;
        s *= (real)P->ssswgt;
    }
    return s;
}

static real cvmap(const orc_params* P, real x)
{
    if (x <= (real)P->cvkeys[0]) return P->cvvals[0];
    if ((real)P->cvkeys[P->cvcard - 1] <= x) return P->cvvals[P->cvcard - 1];
    int idx = P->cvshift + (int)rint((double)(2 * x));
    return P->cvvals[idx];
}

static real score_cv(const orc_params* P, const orc_profile* q, const orc_profile* d, int i, int j)
{
    const float* qc = q->cv + (size_t)i * NCV;
    const float* dc = d->cv + (size_t)j * NCV;
    real s = 0;
    for (int k = 0; k < NCV; k++) s += (real)qc[k] * (real)dc[k];
    s += (real)P->cv_lokappa0;
    s = ((real)q->cvnorm2[i] + (real)1.0f + (real)P->cv_lokappa0) *
        ((real)d->cvnorm2[j] + (real)1.0f + (real)P->cv_lokappa0) - s * s;
    real qp = q->cvprior[i], dp = d->cvprior[j];
    if (!P->mapaln) { qp = (real)(int)qp; dp = (real)(int)dp; }
    s = (real)P->cv_cterm + (real)P->cv_pownu0 * LOG(s) - qp - dp;
    s = cvmap(P, s);
    return s * (real)P->cvswgt;
}

void orc_score_cell(const orc_params* P, const orc_profile* q, const orc_profile* d, int i, int j,
                    real* S, real* MOD, real* S0, real* SS, real* CV)
{
    real s0 = score_aa(P, q, d, i, j);
    real ss = P->ssswgt > 0 ? score_ss(P, q, d, i, j) : 0;
    real cv = P->cvswgt > 0 ? score_cv(P, q, d, i, j) : 0;
    real add = ss + cv;
    if (S0) *S0 = s0;
    if (SS) *SS = ss;
    if (CV) *CV = cv;
    if (S) *S = s0 + add;
    if (MOD) *MOD = add - (real)0.5f * (real)P->cvswgt;
}

void orc_score_matrix(const orc_params* P, const orc_profile* q, const orc_profile* d, real* S, real* MOD)
{
    for (int i = 0; i < q->len; i++)
        for (int j = 0; j < d->len; j++)
            orc_score_cell(P, q, d, i, j, S ? S + (size_t)i * d->len + j : NULL,
                           MOD ? MOD + (size_t)i * d->len + j : NULL, NULL, NULL, NULL);
}

/* ---------------------------------------------------------------------- */
/* Distant-corner masking (src/libmycu/cudp/CuBatchDP_init_btck.cuh:118-166):
 * cells in the two far triangles take the score -9. */
static int corner_edge(int lq, int ld)
{
    int m = lq > ld ? lq : ld;
    int e = (int)rintf(0.34f * (float)m);
    return e > 60 ? 60 : e;
}
static int in_corner(int lq, int ld, int e, int y, int x)
{
    return (lq <= y + e && x <= e + y - lq) || (ld - e + y <= x && y < e);
}

typedef struct { real MM, MI, IM, DN, ND; } st5;
static const st5 ZERO5 = {0, 0, 0, 0, 0};

/* Boundary states left of column 0 as the reference's 32x32 oblique blocks
 * produce them (src/libmycu/cudp/CuBatchDP_init_btck.cu:117-262,303-360):
 *  - rows with r%32 == 31 see all-zero states at column -1 (diagonal-buffer
 *    initialisation);
 *  - other rows see states computed from log(0) db transitions: MM = 0,
 *    MI/IM/ND near -32768, and DN a chain down column -1,
 *    DN(r) = max(MM_up + qMD(r), DN_up + qDD(r)), whose "up" is all-zero at
 *    rows r%32 == 0 (bottom-buffer initialisation);
 *  - the diagonal neighbour of (r, 0) is all-zero for r%32 in {0, 31}. */
static void colm1_states(const orc_profile* q, st5* C)
{
    for (int r = 0; r < q->len; r++) {
        trn7 t = get_trn(q, r);
        st5 U = (r % 32 == 0) ? ZERO5 : C[r - 1];
        st5 c;
        c.MM = 0;
        c.MI = MAXR((U.MM + t.MM) + (real)LOG0, (U.MI + t.MM) + (real)LOG0);
        if (r % 32 == 0)
            c.IM = MAXR(((real)0 + t.MI) + (real)LOG0, ((real)0 + t.II) + (real)LOG0);
        else
            c.IM = ((real)0 + t.MI) + (real)LOG0;
        c.DN = MAXR(U.MM + t.MD, U.DN + t.DD);
        c.ND = (real)LOG0;
        C[r] = c;
    }
}

/*
 * Phase-1 Viterbi DP of one pair (src/libmycu/cudp/CuBatchDP_init_btck.cu:303-360):
 *   MM = max(0, max{MI'+qMM+dIM, IM'+qIM+dMM, DN'+qDM+dMM, ND'+qMM+dDM, MM'+qMM+dMM} + S)  (diag)
 *   MI = max(MM^+qMM+dMI, MI^+qMM+dII)        (up)
 *   IM = max(MM<+qMI+dMM, IM<+qII+dMM)        (left)
 *   DN = max(MM^+qMD, DN^+qDD)                (up)
 *   ND = max(MM<+dMD, ND<+dDD)                (left)
 * btck: DIAG if MM != 0, then UP/LEFT for each later state that exceeds the
 * running maximum.  The best MM over all cells is returned with the
 * lexicographically smallest (row, column) among tied maxima; *nties counts
 * the cells attaining it.  S is [Lq*Ld]; btck (optional) [Lq*Ld].
 */
void orc_dp(const orc_params* P, const orc_profile* q, const orc_profile* d, const real* S,
            real* best_out, int* bx, int* by, int* nties, signed char* btck)
{
    (void)P;
    const int lq = q->len, ld = d->len;
    const int edge = corner_edge(lq, ld);
    st5* prev = (st5*)malloc(sizeof(st5) * (size_t)ld);
    st5* cur = (st5*)malloc(sizeof(st5) * (size_t)ld);
    st5* C = (st5*)malloc(sizeof(st5) * (size_t)(lq > 0 ? lq : 1));
    trn7* dt = (trn7*)malloc(sizeof(trn7) * (size_t)ld);
    colm1_states(q, C);
    for (int j = 0; j < ld; j++) { prev[j] = ZERO5; dt[j] = get_trn(d, j); }
    real best = 0;
    int bi = -1, bj = -1, nt = 0;
    for (int i = 0; i < lq; i++) {
        trn7 qt = get_trn(q, i);
        for (int j = 0; j < ld; j++) {
            const trn7 t = dt[j];
            st5 up = (i == 0) ? ZERO5 : prev[j];
            st5 left, diag;
            if (j == 0) {
                left = (i % 32 == 31) ? ZERO5 : C[i];
                diag = (i % 32 == 31 || i % 32 == 0) ? ZERO5 : C[i - 1];
            } else {
                left = cur[j - 1];
                diag = (i == 0) ? ZERO5 : prev[j - 1];
            }
            real sc = in_corner(lq, ld, edge, i, j) ? (real)-9.f : S[(size_t)i * ld + j];
            st5 c;
            real v = MAXR((diag.MI + qt.MM) + t.IM, (diag.IM + qt.IM) + t.MM);
            v = MAXR(v, (diag.DN + qt.DM) + t.MM);
            v = MAXR(v, (diag.ND + qt.MM) + t.DM);
            v = MAXR(v, (diag.MM + qt.MM) + t.MM);
            c.MM = MAXR(v + sc, (real)0);
            c.MI = MAXR((up.MM + qt.MM) + t.MI, (up.MI + qt.MM) + t.II);
            c.IM = MAXR((left.MM + qt.MI) + t.MM, (left.IM + qt.II) + t.MM);
            c.DN = MAXR(up.MM + qt.MD, up.DN + qt.DD);
            c.ND = MAXR(left.MM + t.MD, left.ND + t.DD);
            cur[j] = c;
            if (btck) {
                int b = ORC_STOP;
                real mx = c.MM;
                if (c.MM != 0) b = ORC_DIAG;
                if (mx < c.MI) { mx = c.MI; b = ORC_UP; }
                if (mx < c.IM) { mx = c.IM; b = ORC_LEFT; }
                if (mx < c.DN) { mx = c.DN; b = ORC_UP; }
                if (mx < c.ND) { mx = c.ND; b = ORC_LEFT; }
                btck[(size_t)i * ld + j] = (signed char)b;
            }
            if (best < c.MM) { best = c.MM; bi = i; bj = j; nt = 1; }
            else if (c.MM == best && best > 0) nt++;
        }
        st5* tmp = prev; prev = cur; cur = tmp;
    }
    free(prev); free(cur); free(C); free(dt);
    *best_out = best; *bx = bj; *by = bi; *nties = nt;
}

/* ---------------------------------------------------------------------- */
/* Warp butterfly sum (shfl_xor 16,8,4,2,1) of 32 values as seen by lane 0. */
static real butterfly32(const real* p)
{
    real a[16], b[8], c[4], dd[2];
    for (int t = 0; t < 16; t++) a[t] = p[t] + p[t + 16];
    for (int t = 0; t < 8; t++) b[t] = a[t] + a[t + 8];
    for (int t = 0; t < 4; t++) c[t] = b[t] + b[t + 4];
    for (int t = 0; t < 2; t++) dd[t] = c[t] + c[t + 2];
    return dd[0] + dd[1];
}

/*
 * DP finalisation of one pair (src/libmycu/cudp/CuBatchDP_final.cu:170-290):
 * traceback from the best cell over the btck bytes, collecting the scores of
 * DIAG cells; correlation sum_k s_k*(s_{k-4}+...+s_{k-1}) in chunks of 32 with
 * a warp butterfly per chunk; score = max + sgn(c/2)*sqrt(|c/2|); psts =
 * #positive collected scores; beginning = (x+1, y+1) after the walk.
 */
void orc_finalize(const real* S, const signed char* btck, int lq, int ld, real maxsc, int x, int y,
                  real* score_out, int* psts_out, int* begx, int* begy)
{
    real cache[36];
    for (int k = 0; k < 36; k++) cache[k] = 0;
    real sum = 0;
    int psts = 0;
    int b = ORC_DIAG;
    (void)lq;
    while (b != ORC_STOP) {
        for (int k = 0; k < 4; k++) cache[k] = cache[k + 32];
        int ndx;
        for (ndx = 4; ndx < 36;) {
            if (x < 0 || y < 0) { b = ORC_STOP; break; }
            size_t qp = (size_t)y * ld + x;
            b = btck[qp];
            if (b == ORC_STOP) break;
            if (b == ORC_UP) { y--; continue; }
            if (b == ORC_LEFT) { x--; continue; }
            cache[ndx] = S[qp];
            if (cache[ndx] > 0) psts++;
            x--; y--;
            ndx++;
        }
        real p[32];
        for (int t = 0; t < 32; t++)
            p[t] = (ndx <= t + 4) ? (real)0
                 : cache[t + 4] * (((cache[t] + cache[t + 1]) + cache[t + 2]) + cache[t + 3]);
        sum += butterfly32(p);
    }
    sum *= (real)0.5f;
    sum = sum < 0 ? -SQRT(-sum) : SQRT(sum);
    *score_out = maxsc + sum;
    *psts_out = psts;
    *begx = x + 1;
    *begy = y + 1;
}

/* ---------------------------------------------------------------------- */
/* Score threshold for passing to phase 2 (src/libmycu/cualn/JobDispatcher.cpp:809-860). */
void orc_score_threshold(size_t nqyposs, size_t dbsize, float eval, float gK, float glambda,
                         float* scorethld, float* logevthld)
{
    size_t sspace = nqyposs * dbsize;
    float e = eval;
    if (e <= 0.0f) { *scorethld = 999.0f; *logevthld = -99.0f; return; }
    *logevthld = logf(e);
    if (e < 1.0f) e *= 10.0f; else e *= 3.0f;
    e /= gK * sspace;
    if (e <= 0.0f) { *scorethld = 999.0f; return; }
    e = logf(e);
    float s = -e / glambda;
    if (s < 0.0f) s = 0.0f;
    *scorethld = s;
}

/* Gertz (2005) length adjustment -> effective search space
 * (src/libpro/srcsco/AbstractScoreMatrix.cpp:303-380), float arithmetic. */
void orc_length_adjustment(float lambda, float K, float alpha, float beta,
                           size_t m, unsigned long long n, size_t N,
                           unsigned long long* searchspace, unsigned long long* deltalen)
{
    *searchspace = (unsigned long long)m * n;
    *deltalen = 0;
    if (lambda <= 0.0f || K <= 0.0f || N < 1) return;
    const int maxit = 20;
    const float logK = logf(K);
    const float alratio = alpha / lambda;
    const float max_mn = (float)((m > n) ? m : n);
    float length = 0.0f, min_length = 0.0f, max_length = 0.0f, nxt_length = 0.0f;
    float sspace = 0.0f, space2 = 0.0f;
    int converged = 0;
    float a = (float)N;
    float b = (float)(n + m * N);
    float c = (float)(m * n) - max_mn / K;
    if (c < 0.0f) return;
    max_length = 2.0f * c / (b + sqrtf(b * b - 4.0f * a * c));
    for (int j = 0; j < maxit; j++) {
        length = nxt_length;
        sspace = (m - length) * (n - N * length);
        nxt_length = alratio * (logK + logf(sspace)) + beta;
        if (length <= nxt_length) {
            min_length = length;
            if (nxt_length - length <= 1.0f) { converged = 1; break; }
            if (min_length == max_length) break;
        } else
            max_length = length;
        if (nxt_length < min_length || max_length < nxt_length)
            nxt_length = (!j) ? max_length : (min_length + max_length) * 0.5f;
    }
    if (converged) {
        length = ceilf(min_length);
        if (length <= max_length) {
            space2 = (m - length) * (n - N * length);
            nxt_length = alratio * (logK + logf(space2)) + beta;
            if (length <= nxt_length) { min_length = length; sspace = space2; }
        }
    }
    *searchspace = (unsigned long long)sspace;
    *deltalen = (unsigned long long)min_length;
}
