// c2_adj.cu -- differentiable alignment: log-partition of the MAP forward
// model over (query, db profile) pairs and its adjoint.
//
// No counterpart in the reference, whose forward-backward (cumapdp/) only
// feeds the MAP alignment.  The model is the reference's MAP forward
// recursion (src/libmycu/cumapdp/CuBatchMAPDP_fwd.cu:72-478: five states,
// query and db transition log-probabilities, the column -1 states of its
// 32-row blocks, a local start term log 1 in the MM state) evaluated with
// exact expf/logf and over the score matrix
//     S = s0 + wss * ss + wcv * cv
// (amino-acid score, and the SS and context-vector terms before their
// weights), with seven offsets theta (MM MI MD IM II DM DD) added to the query
// transitions of every cell update.  logZ = log sum over cells exp(F.MM).
// The backward sweep is the transposed recursion (outside values B, with the
// local end term in MM), so exp(F + B - logZ) is a state posterior and every
// edge posterior exp(F(pred) + edge + B(succ) - logZ) is a derivative of
// logZ.  Gradients: dlogZ/dS per cell (the MM emission edges), dlogZ/dtheta
// (edges by the query transition they use), dlogZ/dwss and dlogZ/dwcv.
//
// Sizes are those of batch alignment studies (hundreds of pairs of a few
// hundred positions): one warp per pair, strips of 32 query rows processed
// in turn, all five states of F and B stored per cell.
#include <cuda_runtime.h>

#include "c2_adj.cuh"

namespace c2 {

#define FULL 0xffffffffu
constexpr float XLOG0 = -99.f;   // the MAP model's log 0


struct X5 { float MM, MI, IM, DN, ND; };

__device__ __forceinline__ float xlse2(float a, float b)
{
    const float m = fmaxf(a, b);
    return logf(expf(a - m) + expf(b - m)) + m;
}

// log(e^v1 + ... + e^v5 + 1): the 1 is the local start (forward) or end (backward)
__device__ __forceinline__ float xlse5p1(float v1, float v2, float v3, float v4, float v5)
{
    float m = fmaxf(fmaxf(fmaxf(v1, v2), fmaxf(v3, v4)), fmaxf(v5, 0.f));
    return logf(expf(v1 - m) + expf(v2 - m) + expf(v3 - m) + expf(v4 - m) + expf(v5 - m) + expf(-m)) + m;
}

// transitions of position i of a profile whose raw rows start at t0: the
// forward recursion's (MM MD IM DM DD into i, MI II out of i) and the
// backward's (all out of i); log 0 outside [0, len)
__device__ __forceinline__ void xtrn_fwd(const float* __restrict__ t0, int i, int len, float* t7)
{
    if (i < 0 || i >= len) {
        for (int k = 0; k < 7; k++) t7[k] = XLOG0;
        return;
    }
    const float* a = t0 + (long long)i * 7;
    t7[TMM] = a[0]; t7[TMI] = a[7 + 1]; t7[TMD] = a[2];
    t7[TIM] = a[3]; t7[TII] = a[7 + 4]; t7[TDM] = a[5]; t7[TDD] = a[6];
}

__device__ __forceinline__ void xtrn_bwd(const float* __restrict__ t0, int i, int len, float* t7)
{
    if (i < 0 || i >= len) {
        for (int k = 0; k < 7; k++) t7[k] = XLOG0;
        return;
    }
    const float* b = t0 + (long long)(i + 1) * 7;
    for (int k = 0; k < 7; k++) t7[k] = b[k];
}

// ---------------------------------------------------------------------------
// score parts per cell (the arithmetic of cell_score, weights left out)
__global__ void __launch_bounds__(256) adj_score_kernel(AdjArgs a)
{
    const int pr = blockIdx.x;
    if (pr >= a.npairs) return;
    const int p = a.prof[pr];
    const int L = a.plen[p], Lq = a.Lq;
    const long long base = a.off[pr];
    const float* bd = a.pbkg + (long long)p * NAA;
    const ScoreConsts& sc = a.sc;
    const int card = sc.ssss_card;
    for (long long c = threadIdx.x; c < (long long)Lq * L; c += blockDim.x) {
        const int j = (int)(c / Lq), i = (int)(c - (long long)j * Lq);
        const float* qr = a.qrec + (long long)i * QR_STRIDE;
        const float* dr = a.drec + (a.poff[p] + j) * DR_STRIDE;
        float s = 0.f;
        for (int k = 0; k < NAA; k++) s = fmaf(__fdividef(qr[QR_TRG + k], 0.5f * (a.qbkg[k] + bd[k])), dr[DR_TRG + k], s);
        const float s0 = __logf(s) - sc.shift;
        float dot = 0.f;
        for (int k = 0; k < NCV; k++) dot = fmaf(qr[QR_CV + k], dr[DR_CV + k], dot);
        dot += sc.lokappa0;
        const float det = qr[QR_CN] * dr[DR_CN] - dot * dot;
        const float cvs = sc.cterm + sc.pownu0 * __logf(det) - qr[QR_PRIOR] - dr[DR_PRIOR];
        float cvm;
        if (cvs <= sc.cvkey_first) cvm = sc.cvval_first;
        else if (sc.cvkey_last <= cvs) cvm = sc.cvval_last;
        else cvm = a.cvvals[min(max(sc.cvshift + (int)rintf(2.f * cvs), 0), sc.cvcard - 1)];
        const float q0 = qr[QR_SS], q1 = qr[QR_SS + 1], q2 = qr[QR_SS + 2];
        const int i0 = (int)(q0 * 9.999f), i1 = 10 + (int)(q1 * 9.999f), i2 = 20 + (int)(q2 * 9.999f);
        const int pk = __float_as_int(dr[DR_SSIDX]);
        const int dk[3] = {pk & 0xff, (pk >> 8) & 0xff, (pk >> 16) & 0xff};
        float ss = 0.f;
        for (int t = 0; t < 3; t++) {
            const int cc = dk[t];
            const float u = q0 * a.ssss[i0 * card + cc] + q1 * a.ssss[i1 * card + cc] + q2 * a.ssss[i2 * card + cc];
            ss = fmaf(dr[DR_SS + t], u, ss);
        }
        if (-99.f < ss) {
            ss += qr[QR_HQ] * dr[DR_HD] * 0.1111111f;
            ss -= 0.05f;
        }
        a.p0[base + c] = s0;
        a.pss[base + c] = ss;
        a.pcv[base + c] = cvm;
    }
}

__device__ __forceinline__ float adj_score(const AdjArgs& a, long long k)
{
    return a.p0[k] + a.wss * a.pss[k] + a.wcv * a.pcv[k];
}

// ---------------------------------------------------------------------------
// forward sweep: one warp per pair, strips of 32 rows in turn, lane t at
// column k - t at step k; all five states stored; per-lane online
// log-sum-exp of F.MM for logZ
__global__ void __launch_bounds__(128) adj_fwd_kernel(AdjArgs a)
{
    const int lane = threadIdx.x & 31;
    const int pr = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (pr >= a.npairs) return;
    const int p = a.prof[pr];
    const int L = a.plen[p], Lq = a.Lq;
    const long long base = a.off[pr], NC = a.ncells;
    const float* dt0 = a.dtrn + (a.poff[p] + p) * 7;
    const X5 INIT = {0.f, XLOG0, XLOG0, XLOG0, XLOG0};
    float zm = -INFINITY, zs = 0.f;
    const int nstrips = (Lq + 31) >> 5;
    for (int s = 0; s < nstrips; s++) {
        const int r = s * 32 + lane;
        const bool act = r < Lq;
        float q7[7];
        xtrn_fwd(a.qtrn, r, Lq, q7);
#pragma unroll
        for (int k = 0; k < 7; k++) q7[k] += a.theta[k];
        const float* cf = a.qcfx + (long long)(act ? r : 0) * 6;
        const X5 LB = (lane == 31) ? INIT : X5{0.f, cf[0], cf[1], cf[2], XLOG0};
        const X5 DB = (lane == 31 || lane == 0) ? INIT : X5{0.f, cf[3], cf[4], cf[5], XLOG0};
        X5 mine = INIT, upp = INIT;
        float t7[7];
        for (int k = 0; k < 7; k++) t7[k] = XLOG0;
        __syncwarp();   // the previous strip's last row is visible to lane 0
        for (int k = 0; k < L + 31; k++) {
            float tc[7];
            xtrn_fwd(dt0, k, L, tc);
#pragma unroll
            for (int i = 0; i < 7; i++) {
                const float x = __shfl_up_sync(FULL, t7[i], 1);
                t7[i] = (lane == 0) ? tc[i] : x;
            }
            X5 up;
            up.MM = __shfl_up_sync(FULL, mine.MM, 1);
            up.MI = __shfl_up_sync(FULL, mine.MI, 1);
            up.IM = __shfl_up_sync(FULL, mine.IM, 1);
            up.DN = __shfl_up_sync(FULL, mine.DN, 1);
            up.ND = __shfl_up_sync(FULL, mine.ND, 1);
            const int j = k - lane;
            if (lane == 0) {
                if (s > 0 && k < L) {
                    const long long kk = base + (long long)k * Lq + (r - 1);
                    up = X5{a.F[kk], a.F[NC + kk], a.F[2 * NC + kk], a.F[3 * NC + kk], a.F[4 * NC + kk]};
                } else {
                    up = INIT;
                }
            }
            X5 left = mine, diag = upp;
            if (j == 0) { left = LB; diag = DB; }
            const bool valid = act && j >= 0 && j < L;
            const float sc = valid ? adj_score(a, base + (long long)j * Lq + r) : XLOG0;
            X5 nw;
            nw.MM = xlse5p1(((diag.MI + q7[TMM]) + t7[TIM]) + sc, ((diag.IM + q7[TIM]) + t7[TMM]) + sc,
                            ((diag.DN + q7[TDM]) + t7[TMM]) + sc, ((diag.ND + q7[TMM]) + t7[TDM]) + sc,
                            ((diag.MM + q7[TMM]) + t7[TMM]) + sc);
            nw.MI = xlse2((up.MM + q7[TMM]) + t7[TMI], (up.MI + q7[TMM]) + t7[TII]);
            nw.IM = xlse2((left.MM + q7[TMI]) + t7[TMM], (left.IM + q7[TII]) + t7[TMM]);
            nw.DN = xlse2(up.MM + q7[TMD], up.DN + q7[TDD]);
            nw.ND = xlse2(left.MM + t7[TMD], left.ND + t7[TDD]);
            if (valid) {
                const long long kk = base + (long long)j * Lq + r;
                a.F[kk] = nw.MM;
                a.F[NC + kk] = nw.MI;
                a.F[2 * NC + kk] = nw.IM;
                a.F[3 * NC + kk] = nw.DN;
                a.F[4 * NC + kk] = nw.ND;
                if (nw.MM > zm) { zs = zs * expf(zm - nw.MM) + 1.f; zm = nw.MM; }
                else zs += expf(nw.MM - zm);
            }
            mine = nw;
            upp = up;
        }
    }
    // combine the lanes' (max, sum) pairs
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const float om = __shfl_xor_sync(FULL, zm, o), os = __shfl_xor_sync(FULL, zs, o);
        const float m = fmaxf(zm, om);
        zs = (m == -INFINITY) ? 0.f : zs * expf(zm - m) + os * expf(om - m);
        zm = m;
    }
    if (lane == 0) a.logz[pr] = logf(zs) + zm;
}

// ---------------------------------------------------------------------------
// backward sweep on the mirrored matrix (row Lq-1-r', column L-1-j'):
// outside values of the five states
__global__ void __launch_bounds__(128) adj_bwd_kernel(AdjArgs a)
{
    const int lane = threadIdx.x & 31;
    const int pr = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (pr >= a.npairs) return;
    const int p = a.prof[pr];
    const int L = a.plen[p], Lq = a.Lq;
    const long long base = a.off[pr], NC = a.ncells;
    const float* dt0 = a.dtrn + (a.poff[p] + p) * 7;
    const X5 INIT = {0.f, XLOG0, XLOG0, XLOG0, XLOG0};
    const int nstrips = (Lq + 31) >> 5;
    for (int s = 0; s < nstrips; s++) {
        const int rm = s * 32 + lane;
        const int r = Lq - 1 - rm;
        const bool act = rm < Lq;
        float q7[7];
        xtrn_bwd(a.qtrn, r, Lq, q7);
#pragma unroll
        for (int k = 0; k < 7; k++) q7[k] += a.theta[k];
        X5 mine = INIT, upp = INIT;
        float t7[7];
        for (int k = 0; k < 7; k++) t7[k] = XLOG0;
        __syncwarp();
        for (int k = 0; k < L + 31; k++) {
            float tc[7];
            xtrn_bwd(dt0, L - 1 - k, L, tc);
#pragma unroll
            for (int i = 0; i < 7; i++) {
                const float x = __shfl_up_sync(FULL, t7[i], 1);
                t7[i] = (lane == 0) ? tc[i] : x;
            }
            X5 dn;
            dn.MM = __shfl_up_sync(FULL, mine.MM, 1);
            dn.MI = __shfl_up_sync(FULL, mine.MI, 1);
            dn.IM = __shfl_up_sync(FULL, mine.IM, 1);
            dn.DN = __shfl_up_sync(FULL, mine.DN, 1);
            dn.ND = __shfl_up_sync(FULL, mine.ND, 1);
            const int j = k - lane;   // mirrored column
            const int ca = L - 1 - j; // actual column
            if (lane == 0) {
                if (s > 0 && k < L) {
                    const long long kk = base + (long long)(L - 1 - k) * Lq + (r + 1);
                    dn = X5{a.B[kk], a.B[NC + kk], a.B[2 * NC + kk], a.B[3 * NC + kk], a.B[4 * NC + kk]};
                } else {
                    dn = INIT;
                }
            }
            X5 rt = mine, dg = upp;
            if (j == 0) { rt = INIT; dg = INIT; }
            const bool valid = act && j >= 0 && j < L;
            // score of the diagonal successor (r + 1, ca + 1)
            const float sco = (valid && r + 1 < Lq && ca + 1 < L) ? adj_score(a, base + (long long)(ca + 1) * Lq + r + 1)
                                                                   : XLOG0;
            X5 nw;
            nw.MM = xlse5p1((dn.MI + q7[TMM]) + t7[TMI], (rt.IM + q7[TMI]) + t7[TMM], dn.DN + q7[TMD],
                            rt.ND + t7[TMD], ((dg.MM + q7[TMM]) + t7[TMM]) + sco);
            nw.MI = xlse2(((dg.MM + q7[TMM]) + t7[TIM]) + sco, (dn.MI + q7[TMM]) + t7[TII]);
            nw.IM = xlse2(((dg.MM + q7[TIM]) + t7[TMM]) + sco, (rt.IM + q7[TII]) + t7[TMM]);
            nw.DN = xlse2(((dg.MM + q7[TDM]) + t7[TMM]) + sco, dn.DN + q7[TDD]);
            nw.ND = xlse2(((dg.MM + q7[TMM]) + t7[TDM]) + sco, rt.ND + t7[TDD]);
            if (valid) {
                const long long kk = base + (long long)ca * Lq + r;
                a.B[kk] = nw.MM;
                a.B[NC + kk] = nw.MI;
                a.B[2 * NC + kk] = nw.IM;
                a.B[3 * NC + kk] = nw.DN;
                a.B[4 * NC + kk] = nw.ND;
            }
            mine = nw;
            upp = dn;
        }
    }
}

// ---------------------------------------------------------------------------
// gradients: one CTA per pair; per cell the edge posteriors of every
// incoming edge, exp(F(pred) + edge + B(cell) - logZ)
__device__ __forceinline__ float block_sum(float v, float* red)
{
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    return t;
}

__global__ void __launch_bounds__(256) adj_grad_kernel(AdjArgs a)
{
    __shared__ float red[8];
    const int pr = blockIdx.x;
    if (pr >= a.npairs) return;
    const int p = a.prof[pr];
    const int L = a.plen[p], Lq = a.Lq;
    const long long base = a.off[pr], NC = a.ncells;
    const float* dt0 = a.dtrn + (a.poff[p] + p) * 7;
    const float lz = a.logz[pr];
    const X5 INIT = {0.f, XLOG0, XLOG0, XLOG0, XLOG0};
    float g[9];
    for (int k = 0; k < 9; k++) g[k] = 0.f;
    auto ld5 = [&](const float* P, long long kk) { return X5{P[kk], P[NC + kk], P[2 * NC + kk], P[3 * NC + kk], P[4 * NC + kk]}; };
    for (long long c = threadIdx.x; c < (long long)Lq * L; c += blockDim.x) {
        const int j = (int)(c / Lq), i = (int)(c - (long long)j * Lq);
        const long long kk = base + c;
        float q7[7], t7[7];
        xtrn_fwd(a.qtrn, i, Lq, q7);
        for (int k = 0; k < 7; k++) q7[k] += a.theta[k];
        xtrn_fwd(dt0, j, L, t7);
        const X5 up = (i == 0) ? INIT : ld5(a.F, kk - 1);
        X5 left, diag;
        if (j == 0) {
            const float* cf = a.qcfx + (long long)i * 6;
            left = (i % 32 == 31) ? INIT : X5{0.f, cf[0], cf[1], cf[2], XLOG0};
            diag = (i % 32 == 31 || i % 32 == 0) ? INIT : X5{0.f, cf[3], cf[4], cf[5], XLOG0};
        } else {
            left = ld5(a.F, kk - Lq);
            diag = (i == 0) ? INIT : ld5(a.F, kk - Lq - 1);
        }
        const X5 b = ld5(a.B, kk);
        const float s = adj_score(a, kk);
        // MM: five emission edges
        const float eMM = b.MM - lz;
        const float m1 = expf(((diag.MI + q7[TMM]) + t7[TIM]) + s + eMM);
        const float m2 = expf(((diag.IM + q7[TIM]) + t7[TMM]) + s + eMM);
        const float m3 = expf(((diag.DN + q7[TDM]) + t7[TMM]) + s + eMM);
        const float m4 = expf(((diag.ND + q7[TMM]) + t7[TDM]) + s + eMM);
        const float m5 = expf(((diag.MM + q7[TMM]) + t7[TMM]) + s + eMM);
        const float gs = (m1 + m2 + m3 + m4) + m5;
        // MI, IM, DN (ND uses no query transition)
        const float i1 = expf((up.MM + q7[TMM]) + t7[TMI] + b.MI - lz);
        const float i2 = expf((up.MI + q7[TMM]) + t7[TII] + b.MI - lz);
        const float l1 = expf((left.MM + q7[TMI]) + t7[TMM] + b.IM - lz);
        const float l2 = expf((left.IM + q7[TII]) + t7[TMM] + b.IM - lz);
        const float d1 = expf(up.MM + q7[TMD] + b.DN - lz);
        const float d2 = expf(up.DN + q7[TDD] + b.DN - lz);
        g[TMM] += m1 + m4 + m5 + i1 + i2;
        g[TIM] += m2;
        g[TDM] += m3;
        g[TMI] += l1;
        g[TII] += l2;
        g[TMD] += d1;
        g[TDD] += d2;
        g[7] += gs * a.pss[kk];
        g[8] += gs * a.pcv[kk];
        a.gS[kk] = gs;
        a.post[kk] = expf(ld5(a.F, kk).MM + b.MM - lz);
    }
    for (int k = 0; k < 9; k++) {
        const float t = block_sum(g[k], red);
        if (threadIdx.x == 0) a.grad[(long long)pr * 9 + k] = t;
    }
}

cudaError_t launch_adj_fwd(const AdjArgs& a, cudaStream_t st)
{
    if (a.npairs <= 0) return cudaSuccess;
    adj_score_kernel<<<a.npairs, 256, 0, st>>>(a);
    adj_fwd_kernel<<<(a.npairs + 3) / 4, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_bwd(const AdjArgs& a, cudaStream_t st)
{
    if (a.npairs <= 0) return cudaSuccess;
    adj_bwd_kernel<<<(a.npairs + 3) / 4, 128, 0, st>>>(a);
    adj_grad_kernel<<<a.npairs, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace c2
