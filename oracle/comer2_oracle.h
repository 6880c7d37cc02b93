/*
 * comer2_oracle.h -- CPU oracle of the COMER2 search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * algorithm (minmarg/comer2, src/libmycu/...), used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product (comer2_b200) never links or calls it.
 *
 * The same source builds twice: REAL=float (liborc32.so) follows the
 * reference's float operation order, REAL=double (liborc64.so) is the FP64
 * error reference.  CUDA fast intrinsics (__logf, __fdividef) are replaced by
 * the C library's IEEE functions, so the float build differs from the
 * reference's device results by rounding only.
 *
 * PARITY PINNED to the reference's own results on a B200 where that build's
 * results are valid: its comer program, built for sm_100a from its sources
 * and run on three seeded workloads with the SS and context-vector score
 * terms off (with them on, that build's score matrix holds invalid cells).
 * For every hit it reported (tests/golden/ref_*_w00_plain.json,
 * tests/test_ref_golden.py) this oracle gives the same DP score, expected
 * score and score range, and -- given the lambda and K the reference computed
 * for the pair, which on that build are not valid values -- the same E-value
 * and the same MAP alignment.  The SS and CV terms are pinned through the
 * reference's own table readers and constants (oracle/ref_tables.cpp), and
 * the length adjustment through its own code (oracle/ref_lenadj.cpp).
 */
#ifndef COMER2_ORACLE_H
#define COMER2_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    float ssswgt, cvswgt;
    int mapaln;                 /* MAPALN option: 1 -> init shift 0.002, no prior rounding */
    const float* ssss;          /* card x card symmetric SS score table */
    int ssss_card;
    const float* cvkeys;        /* smoothed CV map keys [cvcard] */
    const float* cvvals;        /* smoothed CV map values [cvcard] */
    int cvcard, cvshift;
    /* context-vector constants (orc_cv_constants) */
    float cv_lokappa0, cv_pownu0, cv_cterm;
} orc_params;

typedef struct {
    int len;
    float eno;
    const float* bkg;           /* [20] */
    const float* trn;           /* [(len+1)*7]: row i = transitions into position i */
    const float* trg;           /* [len*20] */
    const float* cv;            /* [len*19] */
    const float* cvprior;       /* [len] */
    const float* cvnorm2;       /* [len] */
    const float* ss;            /* [len*3] C,E,H */
    const unsigned char* aa;    /* [len] */
} orc_profile;

/* btck codes of the reference (src/libmycu/cudp/CuBatchDP_com.h:99-104) */
enum { ORC_STOP = 0, ORC_LEFT = 1, ORC_UP = 2, ORC_DIAG = 3 };

#ifdef __cplusplus
}
#endif
#endif
