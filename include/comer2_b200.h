/*
 * comer2_b200.h -- C ABI of the B200 implementation of the COMER2 search hot
 * path (profile-profile scores, Viterbi ranking DP, E-value statistics and
 * MAP alignment).
 *
 * The reference has no plugin API for this path; its boundary is the C++
 * class CuBatchProcessing (src/libmycu/cupro/CuBatchProcessing.cuh:47-244),
 * driven by DevCommThread (src/libmycu/cualn/DevCommThread.cpp:155-165,296-356).
 * Each entry point below names the reference call it replaces.
 *
 * Conventions: plain C types, pointers and sizes only; every call returns a
 * c2_status; a handle is used by one host thread at a time; the last error
 * text of a handle is available through c2_last_error().  No call traps or
 * aborts: device-side problems come back as status codes.
 */
#ifndef COMER2_B200_H
#define COMER2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    C2_OK = 0,
    C2_ERR_ARG = 1,        /* invalid argument or inconsistent sizes */
    C2_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    C2_ERR_NOMEM = 3,      /* device or host allocation failed */
    C2_ERR_STATE = 4,      /* call out of order (e.g. search before upload) */
    C2_ERR_CAPACITY = 5,   /* a size exceeds a compiled limit */
    C2_ERR_DEVICE = 6      /* a kernel reported an error status */
} c2_status;

/* Search parameters: comer.par constants, option values and score tables.
 * Replaces the Configuration[] / MOptions / SSSScores / CVS2Scores state the
 * reference passes to CuBatchProcessing's constructor and CuDeviceMemory
 * (CuBatchProcessing.cuh:51-60, CuDeviceMemory.cuh:640-760). */
typedef struct {
    float ungapped_lambda, ungapped_K, ungapped_H;        /* [UNGAPPED]  */
    float gapped_lambda, gapped_K, gapped_H;             /* [GAPPED_A_1] */
    float gapped_alpha, gapped_beta;
    float eval;            /* EVAL */
    float ssswgt;          /* SSSWGT (>= 0; 0 leaves the SS term out) */
    float cvswgt;          /* CVSWGT (>= 0; 0 leaves the context-vector term out) */
    float minpp;           /* MINPP */
    int32_t mapaln;        /* MAPALN: 1 MAP alignments; 0 the Viterbi DP's own alignments */
    int32_t x_uninf;       /* X_UNINF */
    int32_t ssemodel;      /* SSEMODEL: 0 observed statistics, 1 and 2 the SS18 variants */
    const float* ssss;     /* SS score table, ssss_card x ssss_card, symmetric */
    int32_t ssss_card;
    const float* cvs2s_keys;    /* smoothed CV score map: keys, step 0.5 */
    const float* cvs2s_values;  /* values */
    int32_t cvs2s_card;
    int32_t cvs2s_shift;        /* number of negative keys */
    const float* sse_nn_weights;  /* SS18 model weights + adjustment constants */
    int32_t n_sse_nn_weights;
} c2_params;

/* A set of profiles in structure-of-arrays form over concatenated positions
 * (the field set of PM2DVectorFields, src/libmycu/cupro/PM2DVectorFields.h:48-81).
 * trn holds nprofiles + npositions rows of 7 log-space transition values
 * (MM MI MD IM II DM DD; IM..DD scaled by 0.4, log 0 = -32768): row
 * offsets[k] + k + i holds the transitions into position i of profile k. */
typedef struct {
    int32_t nprofiles;
    int64_t npositions;
    const int32_t* lengths;   /* [nprofiles] */
    const int64_t* offsets;   /* [nprofiles] first position of each profile */
    const float* bkg;         /* [nprofiles][20] background probabilities */
    const float* eno;         /* [nprofiles] effective number of observations */
    const float* trn;         /* [npositions + nprofiles][7] */
    const float* trg;         /* [npositions][20] target probabilities */
    const float* cv;          /* [npositions][19] context vectors */
    const float* cvprior;     /* [npositions] */
    const float* cvnorm2;     /* [npositions] */
    const float* ss;          /* [npositions][3] SS probabilities C,E,H */
    const uint8_t* ssstate;   /* [npositions] 'C','E','H' */
    const uint8_t* aa;        /* [npositions] residue letters */
} c2_profiles;

/* Per-pair result of phase 1 (Viterbi ranking DP). */
typedef struct {
    float best;          /* maximum MM score over the pair's DP matrix */
    uint32_t coords;     /* (x << 16) | y of the maximum, x = db, y = query */
} c2_p1_result;

/* Per-pair result of the DP finalisation (one record per pair whose phase-1
 * maximum exceeds the score threshold).  Layout of the reference's phase-1
 * output section (TDP2OutputAlnData dp2oadScore..dp2oadEndCoords,
 * src/libmycu/cuss/CuBatchSS_com.h:45-53). */
typedef struct {
    float score;         /* max + sgn(c/2) sqrt(|c/2|) with the correlation c */
    int32_t profile;     /* db profile index */
    int32_t psts;        /* number of positive substitution scores on the path */
    uint32_t beg;        /* (x << 16) | y, 1-based beginning of the path */
    uint32_t end;        /* (x << 16) | y of the maximum */
    int32_t passed;      /* score > threshold */
} c2_dp_result;

/* One reported hit: a db profile whose log E-value is within the threshold,
 * with its statistics and MAP alignment.  The fields are those of the
 * reference's TDP2OutputAlnData record (src/libmycu/cuss/CuBatchSS_com.h:45-78)
 * after FinalizeMAPDP_MAP, which replaces psts, beg and end with the MAP
 * alignment's values (src/libmycu/cumapdp/CuBatchMAPDP_map_final.cu:318-330). */
typedef struct {
    int32_t profile;     /* db profile index */
    float score;         /* DP score */
    float logE;          /* log E-value (SS18 model) */
    float logEpA;        /* log E-value of the pair alone */
    float lambda, K;     /* computed ungapped lambda and K of the pair's scores */
    float lambda_est, K_est;  /* derived gapped lambda and K */
    float E, H;          /* expected score and relative entropy */
    int32_t smin, smax;  /* score range */
    int32_t psts;        /* positive, non-identical aligned pairs of the MAP alignment */
    int32_t idts;        /* identities */
    int32_t gaps;        /* gap positions */
    int32_t alnlen;      /* alignment length */
    uint32_t beg;        /* (x << 16) | y, 1-based beginning */
    uint32_t end;        /* (x << 16) | y, 0-based end */
    int64_t aln_offset;  /* offset of the 5 NUL-terminated strings (query, middle,
                            target, query SS, target SS) in the alignment buffer */
} c2_hit;

typedef struct c2_handle c2_handle;

/* Create a handle on a device; replaces CuBatchProcessing's constructor and
 * CuDeviceMemory's table caching (CuDeviceMemory.cu:640-760). */
c2_status c2_create(int device, const c2_params* params, c2_handle** out);

/* Release all device and host resources of a handle. */
c2_status c2_destroy(c2_handle* h);

/* Copy the handle's last error message into buf (always NUL-terminated). */
c2_status c2_last_error(const c2_handle* h, char* buf, size_t bufsize);

/* Upload (and repack for the device) a database; replaces
 * CuBatchProcessing::TransferCPMData (CuBatchProcessing.cuh:79-82) and
 * SetDbDetails(db_len, nseqs) (:73).  db_total_positions/profiles describe
 * the whole database (for the threshold and search space); 0 means "this
 * upload is the whole database".  The records are packed by up to 16 host
 * threads into two pinned staging buffers (2 x 56 MiB, held for the call)
 * and copied on the handle's stream; the call returns when the copies are
 * done.  Profiles must be contiguous (offsets[k] = sum of earlier lengths),
 * each of 1..65535 positions. */
c2_status c2_upload_db(c2_handle* h, const c2_profiles* db,
                       uint64_t db_total_positions, uint64_t db_total_profiles);

/* Set the query profile (profile 0 of q); replaces SetQueryLen and the query
 * part of ProcessScoreMatrix (CuBatchProcessing.cuh:87-99).  Computes the
 * score threshold and log E threshold as JobDispatcher::CalculateScoreThreshold
 * (src/libmycu/cualn/JobDispatcher.cpp:809-860). */
c2_status c2_set_query(c2_handle* h, const c2_profiles* q);

/* Run phase 1 (fused score matrix + Viterbi DP max) of the current query over
 * the uploaded database on the device, asynchronously on the handle's stream;
 * results stay on the device.  Replaces ComputeScoreMatrixDevice +
 * PerformCompleteDynProgDevice's DP launches (CuBatchProcessing.cu:324-372). */
c2_status c2_run_phase1(c2_handle* h);

/* Wait for the handle's stream and copy phase-1 results, one per db profile. */
c2_status c2_get_phase1(c2_handle* h, c2_p1_result* out, int32_t n);

/* Run the DP finalisation (traceback, correlation score, pass decision) for
 * the pairs whose phase-1 maximum exceeds the threshold; replaces
 * FinalizeDP/FinalizeDPPro (src/libmycu/cudp/CuBatchDP_final.cu:55-396).
 * Returns the number of finalised pairs in *ncand. */
c2_status c2_run_finalize(c2_handle* h, int32_t* ncand);

/* Copy finalisation records (in ascending profile order). */
c2_status c2_get_finalize(c2_handle* h, c2_dp_result* out, int32_t n);

/* The FP32 score and modular-score matrices (row-major [Lq][L], L the db
 * profile's length) of one finalised pair of the current query, as the
 * traceback sweep of c2_run_finalize computed them; either pointer may be
 * NULL.  Valid until the next c2_run_finalize.  C2_ERR_ARG if the profile is
 * not among the finalised pairs.  The reference keeps these matrices in its
 * device heap (sections ddsBegOfOrgScores / ddsEndOfOrgScores,
 * src/libmycu/cupro/CuBatchProcessing.cu:451-452) without an accessor; this
 * one serves inspection and the parity tests. */
c2_status c2_get_pair_scores(c2_handle* h, int32_t profile, float* scores, float* modscores);

/* Compute the statistics and E-values of the finalised pairs whose score
 * exceeds the threshold; replaces CuBatchSS::CalculateAlnStatisticsDevice
 * (src/libmycu/cuss/CuBatchSS.cu:196-265).  *npassed receives their number. */
c2_status c2_run_stats(c2_handle* h, int32_t* npassed);

/* MAP-align the pairs whose log E-value is within the threshold; replaces
 * CuBatchMAPDP::PerformCompleteMAPDynProgDevice (CuBatchMAPDP.cu:150-513).
 * *nhits receives the number of hits. */
c2_status c2_run_map(c2_handle* h, int32_t* nhits);

/* Copy the hits, sorted by log E-value (then profile index), and their
 * alignment strings.  alns may be NULL to query the required size, which is
 * returned in *aln_bytes; n must be at least the number of hits. */
c2_status c2_get_hits(c2_handle* h, c2_hit* hits, int32_t n, char* alns, size_t* aln_bytes);

/* One complete search of a query over the uploaded database: set the query,
 * phase 1, finalisation, statistics and MAP alignment; replaces
 * CuBatchProcessing::ProcessScoreMatrix (CuBatchProcessing.cuh:87-99).
 * *nhits receives the number of hits; copy them with c2_get_hits. */
c2_status c2_search(c2_handle* h, const c2_profiles* query, int32_t* nhits);

/* Search the database uploaded to src from dst as well (same device, no
 * copy); dst keeps its own query, results and scratch.  No reference
 * counterpart (the reference copies each db chunk to every worker's device
 * heap, CuDeviceMemory.cu:1073). */
c2_status c2_share_db(c2_handle* dst, const c2_handle* src);

/* Results of one query of a batch: hits and alignment strings as c2_get_hits
 * returns them (valid during the call); status != C2_OK: the query failed. */
typedef void (*c2_batch_cb)(void* user, int32_t query, c2_status status, const c2_hit* hits, int32_t nhits,
                            const char* alns, size_t aln_bytes);

/* Search every profile of queries (one query each) over the uploaded
 * database with nworkers (1..8) worker handles sharing it, one host thread
 * and CUDA stream each; cb receives each query's results as it completes
 * (serialised, from the worker threads).  Replaces the query loop of the
 * reference's JobDispatcher and DevCommThread
 * (src/libmycu/cualn/JobDispatcher.cpp:967-1213, DevCommThread.cpp:155-356).
 * Phase 1 runs one query at a time; with two or more workers a query's
 * phase 2 runs beside the next query's phase 1, whose grid then leaves some
 * SMs free (c2_set_batch_sm_reserve; default nsm / 18, 8 on a B200).  Two
 * workers are the fastest on the 64-query configuration. */
c2_status c2_search_batch(c2_handle* h, const c2_profiles* queries, int32_t nworkers, c2_batch_cb cb, void* user);

/* SMs the phase-1 kernels of a multi-worker c2_search_batch leave to the
 * phase-2 sweeps running beside them (-1: the default, nsm / 18). */
c2_status c2_set_batch_sm_reserve(c2_handle* h, int32_t nsm);

/* Result files in the reference's formats (-f 0 Plain, -f 1 JSON): the
 * writers' inputs besides the hits, as the comer program has them. */
enum { C2_REPORT_PLAIN = 0, C2_REPORT_JSON = 1 };

typedef struct {
    const char* progname;           /* program name, may be NULL */
    const char* progversion;        /* may be NULL */
    const char* const* references;  /* NULL-terminated citation lines, may be NULL */
    const char* query_desc;         /* query description, may be NULL */
    int32_t query_length;
    float query_eno;
    int32_t query_has_ss;           /* the query carries SS predictions */
    const char* const* db_names;    /* database names */
    int32_t n_db_names;
    uint64_t db_positions;          /* database size (positions) */
    uint64_t db_profiles;           /* number of database profiles */
    float logevthld;                /* log of the E-value threshold */
    double searchspace;             /* effective search space (c2_get_search_space) */
    int32_t deltalen;               /* length adjustment (c2_get_search_space) */
    float ref_lambda, ref_K;        /* ungapped reference lambda and K */
    float gapped_lambda, gapped_K;  /* expected gapped lambda and K */
    int32_t print_ss;               /* SS lines in Plain alignments (SS weight > 0) */
    int32_t dsclen, dscwidth, alnwidth, show, nhits, nalns;  /* options DSCLEN DSCWIDTH ALNWIDTH SHOW NOHITS NOALNS */
    /* per database profile, indexed by c2_hit.profile */
    const char* const* db_desc;     /* descriptions, may be NULL */
    const int32_t* db_lengths;
    const float* db_eno;
    const uint8_t* db_has_ss;       /* SS predictions present; NULL: all have them */
} c2_report_info;

/* Format one query's result file from its hits (as c2_get_hits returns them,
 * sorted by log E-value).  out == NULL: *out_bytes receives the size needed
 * (with the terminating NUL).  Replaces the reference's result writers
 * (src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp, ...JSON.cpp and
 * src/libmycu/cualn/AlnWriterPlain.cpp, AlnWriterJSON.cpp).  No GPU needed. */
c2_status c2_format_report(int32_t format, const c2_report_info* info, const c2_hit* hits, int32_t nhits,
                           const char* alns, char* out, size_t* out_bytes);

/* Effective search space and length adjustment used for the current query
 * (AbstractScoreMatrix::ComputeLengthAdjustment,
 * src/libpro/srcsco/AbstractScoreMatrix.cpp:247-380). */
c2_status c2_get_search_space(const c2_handle* h, uint64_t* searchspace, uint64_t* deltalen);

/* Thresholds computed for the current query. */
c2_status c2_get_thresholds(const c2_handle* h, float* scorethld, float* logevthld);

/* The same values -- effective search space, length adjustment, score and
 * log E-value thresholds -- for a query of this length against the uploaded
 * database (its totals), without setting a query: what a caller of
 * c2_search_batch needs for the result files of each query
 * (AbstractScoreMatrix::ComputeLengthAdjustment,
 * src/libpro/srcsco/AbstractScoreMatrix.cpp:303-380;
 * JobDispatcher::CalculateScoreThreshold, src/libmycu/cualn/JobDispatcher.cpp:809-860). */
c2_status c2_get_query_limits(const c2_handle* h, int32_t query_length, uint64_t* searchspace, uint64_t* deltalen,
                              float* score_threshold, float* logE_threshold);

/* Make the handle issue its work on a caller-owned CUDA stream (a
 * cudaStream_t passed as void*; NULL restores the handle's own stream). */
c2_status c2_set_stream(c2_handle* h, void* stream);

/* Synchronize the handle's stream. */
c2_status c2_sync(c2_handle* h);

/* Device memory budget of the handle, in bytes (0: none): a buffer that
 * would take the handle's device memory beyond it is refused with
 * C2_ERR_NOMEM before cudaMalloc; c2_search then processes its candidate
 * pairs in groups whose phase-2 scratch fits.  Replaces the reference's
 * --dev-mem limit on its device heap (CuDeviceMemory, src/comer/comer.h
 * usage: "Maximum amount of GPU memory (MB) that can be used").  Worker
 * handles of c2_search_batch draw on the same budget. */
c2_status c2_set_device_memory_limit(c2_handle* h, uint64_t bytes);

/* Device memory the handle's buffers hold now, in bytes. */
c2_status c2_get_device_memory_use(const c2_handle* h, uint64_t* bytes);

/* Number of CUDA devices (0 when none is usable): the reference's --dev-N
 * option uses up to that many (src/comer/comer.h:50-57, comer.cpp:192-194). */
c2_status c2_get_device_count(int32_t* count);

/* Free and total memory of the handle's device (cudaMemGetInfo). */
c2_status c2_get_device_memory_info(const c2_handle* h, uint64_t* free_bytes, uint64_t* total_bytes);

/* Device bytes that c2_upload_db of a database with these sizes (its longest
 * profile max_length positions) holds, with the per-profile phase-1 buffers
 * and, in the tensor-core score mode, the packed score operands: what a
 * caller needs to cut a database too large for the budget into chunks, each
 * uploaded with the whole database's totals and searched in turn (the
 * reference's reader feeds the device in portions sized from --dev-mem:
 * TdDataReader::GetNextData, src/libmycu/cupro/TdDataReader.cpp:543-570). */
c2_status c2_db_device_bytes(const c2_handle* h, int64_t npositions, int32_t nprofiles, int32_t max_length,
                             uint64_t* bytes);

/* Number of candidate groups the last c2_search processed its phase 2 in
 * (1 unless a device memory budget split it).  After a search of several
 * groups, c2_get_pair_scores holds only the last group's pairs. */
c2_status c2_get_search_groups(const c2_handle* h, int32_t* ngroups);

/* Bound of the waits between the strips of one pair in the phase-2 sweeps
 * (traceback DP, MAP forward/backward, MAP DP): a strip polls its
 * predecessor's progress at most `polls` times (0 restores the default,
 * 2^22 polls with 128 ns sleeps, about a second), then gives up, the sweep
 * finishes without faulting and c2_get_finalize / c2_run_stats /
 * c2_get_hits return C2_ERR_DEVICE ("a strip wait ... timed out").  The
 * next c2_set_query clears the error.  No counterpart in the reference,
 * whose kernels neither wait on one another nor time out. */
c2_status c2_set_wait_limit(c2_handle* h, uint32_t polls);

/* Number of kernel launches issued by the handle since creation. */
c2_status c2_launch_count(const c2_handle* h, uint64_t* n);

/* Score arithmetic of phase 1 (no counterpart in the reference, which has
 * only FP32):
 *   C2_SCORE_FP32     the three score contractions in FP32 on the CUDA cores;
 *   C2_SCORE_BF16_TC  the contractions as split-BF16 (hi + lo) tensor-core
 *                     products with FP32 accumulation; the DP stays FP32.
 * In BF16 mode the phase-1 maxima (c2_get_phase1) carry the BF16 rounding;
 * pairs within a 2e-3 relative margin of the score threshold are recomputed
 * in FP32 (traceback sweep), so the finalised scores, hits, E-values and
 * alignments are those of the FP32 mode.  Default: C2_SCORE_FP32. */
#define C2_SCORE_FP32 0
#define C2_SCORE_BF16_TC 1
c2_status c2_set_score_mode(c2_handle* h, int32_t mode);

/* Reader of the reference's binary profile database (`db2bin` output,
 * format v2.2: Db::WriteBinaryHeader, src/libpro/srcpro/Db.cpp:733-741;
 * BinaryWriteProfile_v2_2, src/libpro/srcpro/PMProfileModel.cpp:1468-1930),
 * the input the reference's reader threads stream (TdDataReader,
 * CuDbReader).  c2_db2bin_info gives the sizes; c2_db2bin_read fills
 * caller-owned arrays with the c2_profiles field set (position-major; SS
 * states upper case).  err (may be NULL) receives a message on failure. */
c2_status c2_db2bin_info(const char* path, int32_t* nprofiles, int64_t* npositions, char* err, size_t errlen);
c2_status c2_db2bin_read(const char* path, int32_t* lengths, int64_t* offsets, float* bkg, float* eno, float* trn,
                         float* trg, float* cv, float* cvprior, float* cvnorm2, float* ss, uint8_t* ssstate,
                         uint8_t* aa, char* err, size_t errlen);
/* The same for profiles [k0, k1) only, so that a database larger than host
 * or device memory streams through in chunks, as the reference's reader
 * threads feed it to the device in portions (TdDataReader::GetNextData and
 * ReadDataChunk, src/libmycu/cupro/TdDataReader.cpp:543-686).  The arrays are sized for the range (k1 - k0
 * profiles, their positions, and their positions + profiles transition rows);
 * offsets[] start at 0 for profile k0.  c2_db2bin_lengths gives every
 * profile's length (nprofiles entries) to plan the ranges. */
c2_status c2_db2bin_lengths(const char* path, int32_t* lengths, char* err, size_t errlen);
c2_status c2_db2bin_read_range(const char* path, int32_t k0, int32_t k1, int32_t* lengths, int64_t* offsets,
                               float* bkg, float* eno, float* trn, float* trg, float* cv, float* cvprior,
                               float* cvnorm2, float* ss, uint8_t* ssstate, uint8_t* aa, char* err, size_t errlen);
/* Profile descriptions of the same database (the section after the
 * description end addresses, PMProfileModel.cpp:1529-1533): buf == NULL gives
 * the bytes needed in *bytes; otherwise buf receives the NUL-terminated
 * descriptions back to back and offsets[k] (nprofiles entries) the start of
 * profile k's.  The reference's reader keeps them for its result writers
 * (CuDbReader / TdDataReader, cupro/TdDataReader.cpp:132-975). */
c2_status c2_db2bin_descriptions(const char* path, char* buf, size_t* bytes, int64_t* offsets, char* err,
                                 size_t errlen);

/* Differentiable alignment (no counterpart in the reference, whose
 * forward-backward only feeds its MAP alignment).  Log-partition of the MAP
 * forward model -- the recursion of src/libmycu/cumapdp/CuBatchMAPDP_fwd.cu
 * with true exp/log (hardware forms, ~1e-7 relative) -- for the current
 * query against db profiles
 * `profiles[0..npairs)`, over the score matrix S = s0 + wss*ss + wcv*cv
 * (amino-acid score; SS and context-vector terms before their weights) and
 * with theta[7] (MM MI MD IM II DM DD, may be NULL = 0) added to the query's
 * transition log-probabilities in every cell update.  logz[k] receives
 * log sum over cells exp(F.MM) of pair k.  Keeps what c2_logz_bwd needs
 * (the scores and each 32-row strip's last forward row: the backward sweep
 * recomputes a strip's forward states from the row above it); a new query or
 * c2_logz_fwd call replaces them. */
c2_status c2_logz_fwd(c2_handle* h, const int32_t* profiles, int32_t npairs, const float* theta, float wss,
                      float wcv, float* logz);

/* The same for npairs independent pairs (a training batch): pair k aligns
 * query query_of_pair[k] of the queries given to c2_set_query_batch (their
 * own lengths; the handle's search query is not used or changed) with db
 * profile profiles[k].  c2_logz_bwd and c2_logz_cells then serve these
 * pairs.  c2_set_query_batch packs and uploads the queries once (profiles of
 * up to 65,535 positions, the c2_profiles field set). */
c2_status c2_set_query_batch(c2_handle* h, const c2_profiles* queries);
c2_status c2_logz_fwd_batch(c2_handle* h, const int32_t* query_of_pair, const int32_t* profiles, int32_t npairs,
                            const float* theta, float wss, float wcv, float* logz);

/* Gradients of the last c2_logz_fwd: grad[9 * k + t] = dlogZ_k/dtheta_t
 * (t < 7), grad[9 * k + 7] = dlogZ_k/dwss, grad[9 * k + 8] = dlogZ_k/dwcv. */
c2_status c2_logz_bwd(c2_handle* h, float* grad);

/* Per-cell results of pair k after c2_logz_bwd, row-major [Lq][L] (Lq the
 * pair's query length, L its db profile length):
 * dlogz_ds = dlogZ/dS (expected MM emissions), post = MM state posterior
 * exp(F.MM + B.MM - logZ).  Either pointer may be NULL. */
c2_status c2_logz_cells(c2_handle* h, int32_t pair, float* dlogz_ds, float* post);

/* Phase 1 (as c2_run_phase1 in the default C2_SCORE_FP32 mode) that allocates
 * nothing.  No counterpart in the reference.  It always scores in FP32; a
 * handle set to C2_SCORE_BF16_TC is refused with C2_ERR_STATE.  Its scratch
 * (work counter, strip-boundary rows) lives in one static 16 MiB device array
 * per device, so the grid is limited to the 8-warp blocks whose boundary rows
 * fit; a database whose longest profile exceeds 52,416 positions is rejected
 * with C2_ERR_CAPACITY.  Results go to caller-owned
 * device arrays of nprofiles entries (d_best: DP maxima, d_coords: packed
 * (column << 16 | row) of the maximum), in the layout c2_get_phase1 reports.
 * The array is shared by every call on the device: calls that overlap on the
 * GPU race.  The first call on a device looks up the array's address; make it
 * before any stream capture.  Enqueued on the handle's stream. */
c2_status c2_run_phase1_static(c2_handle* h, float* d_best, uint32_t* d_coords);

#ifdef __cplusplus
}
#endif
#endif
