// c2_adj.cuh -- arguments of the log-partition (differentiable alignment)
// kernels in c2_adj.cu.
#pragma once
#include "c2_device.cuh"

namespace c2 {
// Per-cell arrays are in wavefront order: cell (i, j) of a pair is element
//   off[pair] + ((i / 32) * (L + 31) + j + i % 32) * 32 + i % 32
// (strip i / 32, wavefront step j + i % 32, lane i % 32), so that the 32 cells
// a warp updates in one step of a strip are 128 contiguous bytes.
// Every pair has its own query (c2_logz_fwd_batch; one query for all pairs in
// c2_logz_fwd): query length Lq, nstrips = (Lq + 31) / 32 strips, its rows in
// the concatenated query arrays from qpos.  Work items are (pair, strip)
// pairs in the order of their dependencies (items_f: strip s after strip
// s - 1 of the same pair; items_b: strip s after s + 1); a strip's per-strip
// results sit at soff[pair] + s.
struct AdjArgs {
    int npairs;
    int nitems;             // strips of all pairs
    const int* prof;        // [npairs] db profile of each pair
    const int* pLq;         // [npairs] query length
    const long long* qpos;  // [npairs] first row of the pair's query in qrec / qcfx
    const int* qidx;        // [npairs] query index (qbkg, and qtrn rows from qpos + qidx)
    const long long* soff;  // [npairs] first strip of the pair in the per-strip arrays
    const int2* items_f;    // [nitems] (pair, strip) of the forward sweep
    const int2* items_b;    // [nitems] (pair, strip) of the backward sweep
    const long long* off;   // [npairs] first cell of each pair (nstrips (L + 31) 32 cells a pair)
    const long long* roff;  // [npairs] first float of each pair's row buffers (nstrips 5 L floats a pair)
    const int* plen;
    const long long* poff;
    const float* qrec;      // query records (c2_device.cuh layout), queries concatenated
    const float* drec;      // db records
    const float* pbkg;      // db backgrounds
    const float* qbkg;      // query backgrounds [nqueries][20]
    const float* ssss;      // SS score table [card][card]
    const float* cvvals;    // CV map values
    ScoreConsts sc;
    const float* qtrn;      // query transitions (raw rows, Lq + 1 a query)
    const float* dtrn;      // db transitions (raw rows, one extra per profile)
    const float* qcfx;      // [rows][6] exact column -1 states: MI IM DN of row r, of row r - 1
    float theta[7];
    float wss, wcv;
    float* S;               // [cells] score s0 + wss ss + wcv cv
    float* pss;             // [cells] SS term before its weight
    float* pcv;             // [cells] CV term before its weight
    float* gS;              // [cells] dlogZ/dS
    float* post;            // [cells] MM state posterior
    float* frow;            // forward checkpoint rows: per pair [nstrips][5][L], row 32 s + 31 of strip s
    float* brow;            // outside values of row 32 s, per pair [nstrips][5][L]
    int* prog;              // [2][nitems] columns published of frow / brow rows (by soff + strip)
    float* zpart;           // [nitems][2] (max, scaled sum) of a strip's exp(F.MM)
    float* gpart;           // [nitems][9] a strip's gradient sums
    float* Fall;            // forward states of every strip, when they fit (else null): strip s of
                            // pair m at Fall + 5 off[m] + s (L + 31) 160, [step][state][lane]
    float* scratch;         // per backward warp (Fall null): forward states of its strip, [(Lmax + 31) * 5 * 32]
    long long scratch_stride;
    int* counter;           // [2] work counters of the forward and backward sweeps
    int* status;            // device status (PIPE_ERR_TIMEOUT)
    unsigned spin;          // polls before a strip wait gives up
    float* logz;            // [npairs]
    float* grad;            // [npairs][9]: dlogZ/dtheta[7], dlogZ/dwss, dlogZ/dwcv
};

constexpr int ADJ_WARPS = 4;   // warps per CTA of the sweeps

// resident CTAs per SM of the two sweeps (their persistent grids)
cudaError_t adj_occupancy(int* fwd_ctas_per_sm, int* bwd_ctas_per_sm);
cudaError_t launch_adj_fwd(const AdjArgs& a, int grid, cudaStream_t st);
cudaError_t launch_adj_bwd(const AdjArgs& a, int grid, cudaStream_t st);
}  // namespace c2
