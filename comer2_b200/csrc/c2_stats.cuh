// c2_stats.cuh -- arguments of the statistics and MAP kernels.
#pragma once
#include <cuda_runtime.h>

namespace c2 {

// per-pair statistics record (the reference's TDP2OutputAlnData phase-2
// fields, src/libmycu/cuss/CuBatchSS_com.h:54-70, plus the SS18 EVD parameters)
enum : int {
    ST_MIN = 0, ST_MAX, ST_E, ST_H, ST_LAMBDA, ST_K, ST_LAMBDA_EST, ST_K_EST,
    ST_LOGE, ST_LOGEPA, ST_MU, ST_SCALE, STATS_NOUT
};

struct StatsArgs {
    int Lq;
    int npass;                  // passed pairs
    const int* p2_cand;         // passed pair -> candidate index
    const int* cand_prof;       // candidate -> profile
    const long long* cand_off;  // candidate -> scratch offset
    const int* plen;
    const long long* poff;
    const float* peno;          // per-profile ENO
    const unsigned char* qaa;   // query residues
    const unsigned char* daa;   // db residues (per position)
    const float* smat;          // [L][Lq] scores per candidate
    const float* fscore;        // DP scores per candidate
    const int* fpsts;           // positive-score counts per candidate
    const float* nnw;           // SS18 weights and adjustment constants
    int ssemodel, xuninf;
    float qeno, searchspace, reflambda, refK, expglambda, expgK;
    float* out;                 // [npass][STATS_NOUT]
};

// MAP stage: one warp per pair whose log E-value is within the threshold
struct MapArgs {
    int Lq;
    int nmap;
    const int* map_cand;        // MAP pair -> candidate index
    const int* map_pass;        // MAP pair -> passed-pair index (stats record)
    const int* cand_prof;
    const long long* cand_off;
    const int* plen;
    const long long* poff;
    const float* qrec;          // query records (transitions at QR_TRN, column -1 states)
    const float* drec;          // db records (transitions at DR_TRN)
    const float* qtrn_bwd;      // [Lq][7] query transitions out of each position
    const float* dtrn_bwd;      // [npos][7] db transitions out of each position
    const float* smat;          // [L][Lq] per candidate
    const float* mmat;          // [L][Lq] per candidate (modular scores)
    const float* stats;         // [npass][STATS_NOUT]
    float* fb;                  // F (MAP.MM forward values), per candidate [nstrips][L + 31][32] in
                                // wavefront order (c2_map.cu, skew_base)
    float* bb;                  // B (backward values), the same layout
    signed char* btck;          // [L][Lq] per candidate: MAP traceback codes
    float* pairf;               // [nmap][4]: maxF, logZ, map max, (unused)
    unsigned* pairc;            // [nmap]: MAP end coordinates
    float* bnd;                 // per candidate at 10 x (cand_off / Lq): two last-row buffers [5][L]
    int* prog;                  // [ncand][nstrips] finished columns per strip
    float* bnd_b;               // backward sweep's strip-boundary rows (same layout as bnd)
    int* prog_b;                // backward sweep's strip progress (same layout as prog)
    const int* items;           // work item -> m * nstrips + strip (ready-time order)
    unsigned long long* pairk;  // [nmap] MAP DP maximum and end cell, packed for atomicMax
    int* status;
    int* counter;
    unsigned spin;              // polls before a strip wait gives up (pipe_wait)
    float minpp;
    int modscores;
    // traceback outputs
    const unsigned char* qaa;
    const unsigned char* qss;
    const unsigned char* daa;
    const unsigned char* dss;
    int* aln_info;              // [nmap][8]: alnlen, idts, psts, gaps, beg, end, 0, 0
    char* aln;                  // [nmap][5][Lq + Lmax + 1]
    int alnstride;
};

}  // namespace c2
