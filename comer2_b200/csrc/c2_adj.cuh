// c2_adj.cuh -- arguments of the log-partition (differentiable alignment)
// kernels in c2_adj.cu.
#pragma once
#include "c2_device.cuh"

namespace c2 {
// Per-cell arrays are in wavefront order: cell (i, j) of a pair is element
//   off[pair] + ((i / 32) * (L + 31) + j + i % 32) * 32 + i % 32
// (strip i / 32, wavefront step j + i % 32, lane i % 32), so that the 32 cells
// a warp updates in one step of a strip are 128 contiguous bytes.
struct AdjArgs {
    int Lq;
    int npairs;
    int nstrips;            // (Lq + 31) / 32
    const int* prof;        // [npairs] db profile of each pair
    const long long* off;   // [npairs] first cell of each pair (nstrips (L + 31) 32 cells a pair)
    const long long* roff;  // [npairs] first float of each pair's row buffers (nstrips 5 L floats a pair)
    const int* plen;
    const long long* poff;
    const float* qrec;      // query records (c2_device.cuh layout)
    const float* drec;      // db records
    const float* pbkg;      // db backgrounds
    const float* qbkg;      // query background
    const float* ssss;      // SS score table [card][card]
    const float* cvvals;    // CV map values
    ScoreConsts sc;
    const float* qtrn;      // [Lq + 1][7] query transitions (raw rows)
    const float* dtrn;      // db transitions (raw rows, one extra per profile)
    const float* qcfx;      // [Lq][6] exact column -1 states: MI IM DN of row r, of row r - 1
    float theta[7];
    float wss, wcv;
    float* S;               // [cells] score s0 + wss ss + wcv cv
    float* pss;             // [cells] SS term before its weight
    float* pcv;             // [cells] CV term before its weight
    float* gS;              // [cells] dlogZ/dS
    float* post;            // [cells] MM state posterior
    float* frow;            // forward checkpoint rows: per pair [nstrips][5][L], row 32 s + 31 of strip s
    float* brow;            // outside values of row 32 s, per pair [nstrips][5][L]
    int* prog;              // [2][npairs * nstrips] columns published of frow / brow rows
    float* zpart;           // [npairs * nstrips][2] (max, scaled sum) of a strip's exp(F.MM)
    float* gpart;           // [npairs * nstrips][9] a strip's gradient sums
    float* scratch;         // per backward warp: forward states of its strip, [(Lmax + 31) * 5 * 32]
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
