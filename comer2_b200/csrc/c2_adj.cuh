// c2_adj.cuh -- arguments of the log-partition (differentiable alignment)
// kernels in c2_adj.cu.
#pragma once
#include "c2_device.cuh"

namespace c2 {
struct AdjArgs {
    int Lq;
    int npairs;
    const int* prof;        // [npairs] db profile of each pair
    const long long* off;   // [npairs] first cell of each pair (cells column-major: j * Lq + i)
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
    long long ncells;       // stride of the state planes
    float* p0;              // [cells] amino-acid score
    float* pss;             // [cells] SS term before its weight
    float* pcv;             // [cells] CV term before its weight
    float* F;               // [5][cells] forward states
    float* B;               // [5][cells] outside states
    float* logz;            // [npairs]
    float* gS;              // [cells] dlogZ/dS
    float* post;            // [cells] MM state posterior
    float* grad;            // [npairs][9]: dlogZ/dtheta[7], dlogZ/dwss, dlogZ/dwcv
};

cudaError_t launch_adj_fwd(const AdjArgs& a, cudaStream_t st);
cudaError_t launch_adj_bwd(const AdjArgs& a, cudaStream_t st);
}  // namespace c2
