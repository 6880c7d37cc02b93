// c2_adj.cu -- differentiable alignment: log-partition of the MAP forward
// model over (query, db profile) pairs and its adjoint.
//
// No counterpart in the reference, whose forward-backward (cumapdp/) only
// feeds the MAP alignment.  The model is the reference's MAP forward
// recursion (src/libmycu/cumapdp/CuBatchMAPDP_fwd.cu:72-478: five states,
// query and db transition log-probabilities, the column -1 states of its
// 32-row blocks, a local start term log 1 in the MM state) evaluated with
// true exponentials and logarithms (the hardware base-2 forms, relative
// error ~1e-7 at these arguments; the reference's MAP stage uses coarse
// approximations instead) over the score matrix
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
// Layout and schedule.  Per-cell arrays (scores, dlogZ/dS, posteriors) are
// in wavefront order (c2_adj.cuh).  Both sweeps run one strip of 32 query
// rows of one pair per warp, strips handed out by a global counter in the
// order of their dependencies (all pairs' strip 0, then strip 1, ...; the
// backward sweep from the last strip up), so a pair is swept by up to
// nstrips warps at once, each trailing the strip it depends on by about 40
// columns (bounded waits on published progress, as the phase-2 sweeps).
// Memory: the forward sweep keeps the last row of every strip (5 states x L
// per strip, the rows the next strip reads) and each strip's partial log-sum,
// and, when they fit (20 bytes a cell), every forward state.  The backward
// sweep takes its strip's forward states from there, or -- checkpointing,
// when they did not fit -- recomputes them from the checkpoint row above into
// a per-warp scratch (32 rows x (L + 31) x 5 states); it then runs the
// outside recursion over the same rows (bottom row first) and forms every
// edge posterior of the strip as it goes.  B is never stored for the matrix,
// and with checkpointing neither is F: memory per cell is then the 3 score
// arrays and the 2 outputs.
#include <cuda_runtime.h>

#include <algorithm>

#include "c2_adj.cuh"

namespace c2 {

#define FULL 0xffffffffu
constexpr float XLOG0 = -99.f;   // the MAP model's log 0


struct X5 { float MM, MI, IM, DN, ND; };

// e^x and ln x through the hardware base-2 forms (ex2.approx / lg2.approx,
// denormal results and arguments flushed: the terms they drop are below
// e^-87 of the largest term of a sum)
constexpr float XLOG2E = 1.4426950408889634f, XLN2 = 0.6931471805599453f;
__device__ __forceinline__ float xexp(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x * XLOG2E));
    return y;
}
__device__ __forceinline__ float xlog(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y * XLN2;
}

// the larger term's exponential is ex2(0) = 1 exactly, the smaller one's
// difference exactly -|a - b|
__device__ __forceinline__ float xlse2(float a, float b)
{
    const float m = fmaxf(a, b);
    return xlog(1.f + xexp(-fabsf(a - b))) + m;
}

// log(e^v1 + ... + e^v5 + 1): the 1 is the local start (forward) or end (backward)
__device__ __forceinline__ float xlse5p1(float v1, float v2, float v3, float v4, float v5)
{
    float m = fmaxf(fmaxf(fmaxf(v1, v2), fmaxf(v3, v4)), fmaxf(v5, 0.f));
    return xlog(xexp(v1 - m) + xexp(v2 - m) + xexp(v3 - m) + xexp(v4 - m) + xexp(v5 - m) + xexp(-m)) + m;
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
// cell (i, j) of a pair whose wavefront block starts at base
__device__ __forceinline__ long long fw_cell(long long base, int L, int i, int j)
{
    const int l = i & 31;
    return base + ((long long)(i >> 5) * (L + 31) + j + l) * 32 + l;
}

// ---------------------------------------------------------------------------
// score parts per cell: one warp per (pair, strip), lane = query row, the
// strip's wavefront steps in turn (coalesced stores).  The db records the
// lanes read (the 46 score fields of 32 consecutive columns per step) are
// staged per 32-column chunk in a shared ring of 64 columns, ADJ_REC floats
// apart (odd: the lanes' reads of consecutive columns hit distinct banks).
constexpr int ADJ_REC = 47, ADJ_RECF = 46;

__device__ __forceinline__ void adj_stage_records(float* ring, const float* __restrict__ d0, int c0, int L, int lane)
{
    const int nc = min(32, L - c0);
    for (int e = lane; e < nc * ADJ_RECF; e += 32) {
        const int c = e / ADJ_RECF, f = e - c * ADJ_RECF;
        ring[((c0 + c) & 63) * ADJ_REC + f] = __ldg(d0 + (long long)(c0 + c) * DR_STRIDE + f);
    }
}

__global__ void __launch_bounds__(ADJ_WARPS * 32) adj_score_kernel(AdjArgs a)
{
    __shared__ float rings[ADJ_WARPS][64 * ADJ_REC];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* ring = rings[wid];
    const int nw = gridDim.x * ADJ_WARPS;
    const ScoreConsts& sc = a.sc;
    const int card = sc.ssss_card;
    for (int it = blockIdx.x * ADJ_WARPS + wid; it < a.nitems; it += nw) {
        const int2 ms = a.items_f[it];
        const int m = ms.x, s = ms.y;
        const int p = a.prof[m];
        const int L = a.plen[p], Lq = a.pLq[m];
        const int r = 32 * s + lane;
        const bool act = r < Lq;
        const float* qr = a.qrec + (a.qpos[m] + (act ? r : 0)) * QR_STRIDE;
        const float* bd = a.pbkg + (long long)p * NAA;
        const float* qb = a.qbkg + (long long)a.qidx[m] * NAA;
        // the query row's amino-acid odds for this pair, CV vector and SS values
        float qt[NAA], qc[NCV];
#pragma unroll
        for (int k = 0; k < NAA; k++) qt[k] = __fdividef(qr[QR_TRG + k], 0.5f * (qb[k] + bd[k]));
#pragma unroll
        for (int k = 0; k < NCV; k++) qc[k] = qr[QR_CV + k];
        const float qcn = qr[QR_CN], qpr = qr[QR_PRIOR], qhq = qr[QR_HQ];
        const float q0 = qr[QR_SS], q1 = qr[QR_SS + 1], q2 = qr[QR_SS + 2];
        const int i0 = (int)(q0 * 9.999f), i1 = 10 + (int)(q1 * 9.999f), i2 = 20 + (int)(q2 * 9.999f);
        const long long cb = a.off[m] + (long long)s * (L + 31) * 32;
        const float* d0 = a.drec + a.poff[p] * DR_STRIDE;
        __syncwarp();
        adj_stage_records(ring, d0, 0, L, lane);
        __syncwarp();
        for (int k = 0; k < L + 31; k++) {
            const int j = k - lane;
            if (act && j >= 0 && j < L) {
                const float* dr = ring + (j & 63) * ADJ_REC;
                float sa = 0.f;
#pragma unroll
                for (int t = 0; t < NAA; t++) sa = fmaf(qt[t], dr[DR_TRG + t], sa);
                const float s0 = __logf(sa) - sc.shift;
                float dot = 0.f;
#pragma unroll
                for (int t = 0; t < NCV; t++) dot = fmaf(qc[t], dr[DR_CV + t], dot);
                dot += sc.lokappa0;
                const float det = qcn * dr[DR_CN] - dot * dot;
                const float cvs = sc.cterm + sc.pownu0 * __logf(det) - qpr - dr[DR_PRIOR];
                float cvm;
                if (cvs <= sc.cvkey_first) cvm = sc.cvval_first;
                else if (sc.cvkey_last <= cvs) cvm = sc.cvval_last;
                else cvm = a.cvvals[min(max(sc.cvshift + (int)rintf(2.f * cvs), 0), sc.cvcard - 1)];
                const int pk = __float_as_int(dr[DR_SSIDX]);
                const int dk[3] = {pk & 0xff, (pk >> 8) & 0xff, (pk >> 16) & 0xff};
                float ss = 0.f;
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    const int cc = dk[t];
                    const float u = q0 * a.ssss[i0 * card + cc] + q1 * a.ssss[i1 * card + cc] + q2 * a.ssss[i2 * card + cc];
                    ss = fmaf(dr[DR_SS + t], u, ss);
                }
                if (-99.f < ss) {
                    ss += qhq * dr[DR_HD] * 0.1111111f;
                    ss -= 0.05f;
                }
                const long long c = cb + (long long)k * 32 + lane;
                const float p0 = s0, pss = ss, pcv = cvm;
                a.S[c] = p0 + a.wss * pss + a.wcv * pcv;
                a.pss[c] = pss;
                a.pcv[c] = pcv;
            }
            if ((k & 31) == 31) {
                // columns of the next chunk into the slots of the chunk before this one
                __syncwarp();
                if (k + 1 < L) adj_stage_records(ring, d0, k + 1, L, lane);
                __syncwarp();
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row buffer of a strip's neighbour, ADJ_RG columns at a time, in the warp's
// shared buffer rab[32][8] (slot c & 31: column c).  Forward: row 32 s - 1
// (frow of strip s - 1) at columns c0 + l; backward: row 32 s + 32 (brow of
// strip s + 1) at mirrored columns c0 + l, i.e. L - 1 - c0 - l.  WAIT: the
// neighbour strip is being swept now; wait for those columns first (a strip
// then trails its neighbour by about 32 + ADJ_RG columns).
constexpr int ADJ_RG = 8;
template <bool MIRROR, bool WAIT>
__device__ __forceinline__ void adj_load_row(const AdjArgs& a, float* rab, const float* __restrict__ row, bool have,
                                             const int* flag, int c0, int L, int lane, bool& broken)
{
    if (WAIT && have) pipe_wait(flag, min(c0 + ADJ_RG, L), lane, a.status, broken, a.spin);
    const int c = c0 + lane;
    if (lane < ADJ_RG) {
        const float init[5] = {0.f, XLOG0, XLOG0, XLOG0, XLOG0};
        float v[5];
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const int col = MIRROR ? L - 1 - c : c;
            v[f] = (have && c < L) ? (WAIT ? __ldcg(row + (long long)f * L + col) : row[(long long)f * L + col])
                                   : init[f];
        }
        float* o = rab + (c & 31) * 8;
        *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
        o[4] = v[4];
    }
    __syncwarp();
}

// Raw transition rows of a pair's db profile (rows 0..L; row r holds the
// transitions into position r, MI and II of row r + 1 those out of position
// r) in the warp's shared ring trs[128][7] by sequence index q: q = row in the
// forward sweep, q = L - row in the mirrored backward sweep.  A step's lanes
// read rows q in [k - 31, k + 1]; chunks of 32 are staged two ahead.
template <bool MIRROR>
__device__ __forceinline__ void adj_stage_trn(float* trs, const float* __restrict__ dt0, int q0, int L, int lane)
{
    const int nq = min(32, L + 1 - q0);
    for (int e = lane; e < nq * 7; e += 32) {
        const int q = q0 + e / 7, f = e % 7;
        const int row = MIRROR ? L - q : q;
        trs[(q & 127) * 7 + f] = __ldg(dt0 + (long long)row * 7 + f);
    }
}

// forward transitions of column j (rows j and j + 1) from the forward ring
__device__ __forceinline__ void ring_trn_fwd(const float* trs, int j, int L, float* t7)
{
    if (j < 0 || j >= L) {
#pragma unroll
        for (int k = 0; k < 7; k++) t7[k] = XLOG0;
        return;
    }
    const float* a = trs + (j & 127) * 7;
    const float* b = trs + ((j + 1) & 127) * 7;
    t7[TMM] = a[0]; t7[TMI] = b[1]; t7[TMD] = a[2];
    t7[TIM] = a[3]; t7[TII] = b[4]; t7[TDM] = a[5]; t7[TDD] = a[6];
}

// L1 prefetch of one 128-byte line (the lines a sweep reads a few steps
// ahead; the loads themselves then hit L1 instead of waiting on L2)
constexpr int ADJ_PF = 4;
__device__ __forceinline__ void pf_l1(const void* p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Forward recursion over strip s of pair m (lane = row 32 s + lane).
// RECOMP false (forward sweep): the row above comes from the strip above as
// it is swept; the strip's last row goes to frow (published for the strip
// below) and the lane's cells into the online log-sum (zm, zs).
// RECOMP true (backward sweep): the row above from the complete checkpoint,
// every state into the warp's scratch Fw[(k * 5 + state) * 32 + lane].
template <bool RECOMP>
__device__ __forceinline__ void adj_fwd_strip(const AdjArgs& a, int m, int s, int lane, float* rab, float* trs,
                                              float* __restrict__ Fw, bool& broken, float& zm, float& zs)
{
    const int p = a.prof[m];
    const int L = a.plen[p], Lq = a.pLq[m], ns = (Lq + 31) >> 5;
    const long long cb = a.off[m] + (long long)s * (L + 31) * 32;
    const float* dt0 = a.dtrn + (a.poff[p] + p) * 7;
    const float* above = a.frow + a.roff[m] + (long long)(s > 0 ? s - 1 : 0) * 5 * L;   // read when s > 0
    float* mine_row = a.frow + a.roff[m] + (long long)s * 5 * L;
    const int* pf = a.prog + a.soff[m];
    const int r = 32 * s + lane;
    const bool act = r < Lq;
    const X5 INIT = {0.f, XLOG0, XLOG0, XLOG0, XLOG0};
    float q7[7];
    xtrn_fwd(a.qtrn + (a.qpos[m] + a.qidx[m]) * 7, r, Lq, q7);
#pragma unroll
    for (int k = 0; k < 7; k++) q7[k] += a.theta[k];
    const float* cf = a.qcfx + (a.qpos[m] + (act ? r : 0)) * 6;
    const X5 LB = (lane == 31) ? INIT : X5{0.f, cf[0], cf[1], cf[2], XLOG0};
    const X5 DB = (lane == 31 || lane == 0) ? INIT : X5{0.f, cf[3], cf[4], cf[5], XLOG0};
    const bool wr_row = !RECOMP && lane == 31 && s + 1 < ns;
    X5 mine = INIT, upp = INIT;
    // the lane's score of the next step, loaded a step ahead
    float scn = (act && lane == 0 && L > 0) ? a.S[cb + lane] : XLOG0;
    const int* pwait = pf + (s > 0 ? s - 1 : 0);   // strip s - 1's progress (s > 0)
    __syncwarp();
    adj_stage_trn<false>(trs, dt0, 0, L, lane);
    adj_stage_trn<false>(trs, dt0, 32, L, lane);
    adj_load_row<false, !RECOMP>(a, rab, above, s > 0, pwait, 0, L, lane, broken);
    for (int k = 0; k < L + 31; k++) {
        const int j = k - lane;
        float t7[7];
        ring_trn_fwd(trs, j, L, t7);
        X5 up;
        up.MM = __shfl_up_sync(FULL, mine.MM, 1);
        up.MI = __shfl_up_sync(FULL, mine.MI, 1);
        up.IM = __shfl_up_sync(FULL, mine.IM, 1);
        up.DN = __shfl_up_sync(FULL, mine.DN, 1);
        up.ND = __shfl_up_sync(FULL, mine.ND, 1);
        {
            const int src = k & 31;
            const float4 ba = *reinterpret_cast<const float4*>(rab + src * 8);
            const float b4 = rab[src * 8 + 4];
            if (lane == 0) up = X5{ba.x, ba.y, ba.z, ba.w, b4};
            if ((src & (ADJ_RG - 1)) == ADJ_RG - 1) {
                __syncwarp();
                adj_load_row<false, !RECOMP>(a, rab, above, s > 0, pwait, k + 1, L, lane, broken);
            }
            if (src == 31) {
                if (k + 33 <= L) adj_stage_trn<false>(trs, dt0, k + 33, L, lane);
                __syncwarp();
            }
        }
        X5 left = mine, diag = upp;
        if (j == 0) { left = LB; diag = DB; }
        const bool valid = act && j >= 0 && j < L;
        const float sc = valid ? scn : XLOG0;
        if (act && j + 1 >= 0 && j + 1 < L) scn = a.S[cb + (long long)(k + 1) * 32 + lane];
        X5 nw;
        nw.MM = xlse5p1(((diag.MI + q7[TMM]) + t7[TIM]) + sc, ((diag.IM + q7[TIM]) + t7[TMM]) + sc,
                        ((diag.DN + q7[TDM]) + t7[TMM]) + sc, ((diag.ND + q7[TMM]) + t7[TDM]) + sc,
                        ((diag.MM + q7[TMM]) + t7[TMM]) + sc);
        nw.MI = xlse2((up.MM + q7[TMM]) + t7[TMI], (up.MI + q7[TMM]) + t7[TII]);
        nw.IM = xlse2((left.MM + q7[TMI]) + t7[TMM], (left.IM + q7[TII]) + t7[TMM]);
        nw.DN = xlse2(up.MM + q7[TMD], up.DN + q7[TDD]);
        nw.ND = xlse2(left.MM + t7[TMD], left.ND + t7[TDD]);
        if (valid) {
            if (RECOMP || Fw) {
                float* o = Fw + (long long)k * 160 + lane;
                o[0] = nw.MM; o[32] = nw.MI; o[64] = nw.IM; o[96] = nw.DN; o[128] = nw.ND;
            }
            if (!RECOMP) {
                if (nw.MM > zm) { zs = zs * xexp(zm - nw.MM) + 1.f; zm = nw.MM; }
                else zs += xexp(nw.MM - zm);
            }
            if (wr_row) {
                mine_row[j] = nw.MM; mine_row[L + j] = nw.MI; mine_row[2 * L + j] = nw.IM;
                mine_row[3 * L + j] = nw.DN; mine_row[4 * L + j] = nw.ND;
                pipe_publish(a.prog + a.soff[m] + s, j, L);
            }
        }
        mine = nw;
        upp = up;
    }
}

// forward sweep: logZ partial sums per strip, checkpoint rows
__global__ void __launch_bounds__(ADJ_WARPS * 32) adj_fwd_kernel(AdjArgs a)
{
    __shared__ __align__(16) float rabs[ADJ_WARPS][32 * 8];
    __shared__ float trss[ADJ_WARPS][128 * 7];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    bool broken = false;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.nitems) break;
        const int2 ms = a.items_f[item];
        const int m = ms.x, s = ms.y;
        float zm = -INFINITY, zs = 0.f;
        // the strip's forward states kept for the backward sweep when they fit
        float* Fw = a.Fall ? a.Fall + 5 * a.off[m] + (long long)s * (a.plen[a.prof[m]] + 31) * 160 : nullptr;
        adj_fwd_strip<false>(a, m, s, lane, rabs[wid], trss[wid], Fw, broken, zm, zs);
        // combine the lanes' (max, sum) pairs
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const float om = __shfl_xor_sync(FULL, zm, o), os = __shfl_xor_sync(FULL, zs, o);
            const float mx = fmaxf(zm, om);
            zs = (mx == -INFINITY) ? 0.f : zs * xexp(zm - mx) + os * xexp(om - mx);
            zm = mx;
        }
        if (lane == 0) {
            const long long o = a.soff[m] + s;
            a.zpart[2 * o] = zm;
            a.zpart[2 * o + 1] = zs;
        }
        __syncwarp();
    }
}

// logZ of each pair from its strips' partial sums, in strip order
__global__ void adj_logz_kernel(AdjArgs a)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.npairs) return;
    float zm = -INFINITY, zs = 0.f;
    const int ns = (a.pLq[m] + 31) >> 5;
    for (int s = 0; s < ns; s++) {
        const long long it = a.soff[m] + s;
        const float om = a.zpart[2 * it], os = a.zpart[2 * it + 1];
        const float mx = fmaxf(zm, om);
        zs = (mx == -INFINITY) ? 0.f : zs * xexp(zm - mx) + os * xexp(om - mx);
        zm = mx;
    }
    a.logz[m] = logf(zs) + zm;
}

// ---------------------------------------------------------------------------
// backward sweep with the gradients.  Strip s of pair m: lane t holds row
// i = 32 s + 31 - t (the strip's rows bottom first), mirrored column
// jm = k - t at step k, actual column ca = L - 1 - jm.  The outside values B
// follow the transposed recursion; at every cell the posteriors of its
// incoming edges exp(F(pred) + edge + B(cell) - logZ) come from the
// recomputed forward states of the strip (and the checkpoint row above it).
__device__ __forceinline__ X5 fw_ld5(const float* __restrict__ Fw, int k, int l)
{
    const float* o = Fw + (long long)k * 160 + l;
    return X5{o[0], o[32], o[64], o[96], o[128]};
}

__device__ __forceinline__ void adj_bwd_strip(const AdjArgs& a, int m, int s, int lane, float* rab, float* trs,
                                              const float* __restrict__ Fw, bool& broken)
{
    const int p = a.prof[m];
    const int L = a.plen[p], Lq = a.pLq[m], ns = (Lq + 31) >> 5;
    const long long base = a.off[m];
    const long long cb = base + (long long)s * (L + 31) * 32;
    const float lz = a.logz[m];
    const float* dt0 = a.dtrn + (a.poff[p] + p) * 7;
    const bool has_below = s + 1 < ns;
    const float* below = a.brow + a.roff[m] + (long long)(has_below ? s + 1 : s) * 5 * L;   // read when has_below
    float* mine_row = a.brow + a.roff[m] + (long long)s * 5 * L;
    const float* fab = a.frow + a.roff[m] + (long long)(s > 0 ? s - 1 : 0) * 5 * L;   // row 32 s - 1 (s > 0)
    const int* pb = a.prog + a.nitems + a.soff[m] + (has_below ? s + 1 : s);
    const int t = lane;
    const int lf = 31 - t;            // the lane's row within the strip
    const int i = 32 * s + lf;
    const bool act = i < Lq;
    const X5 INIT = {0.f, XLOG0, XLOG0, XLOG0, XLOG0};
    float qb[7], qf[7];
    const float* qt0 = a.qtrn + (a.qpos[m] + a.qidx[m]) * 7;
    xtrn_bwd(qt0, i, Lq, qb);
    xtrn_fwd(qt0, i, Lq, qf);
#pragma unroll
    for (int k = 0; k < 7; k++) { qb[k] += a.theta[k]; qf[k] += a.theta[k]; }
    // column -1 states of row i (the forward's left and diagonal at column 0)
    const float* cf = a.qcfx + (a.qpos[m] + (act ? i : 0)) * 6;
    const X5 LB = (lf == 31) ? INIT : X5{0.f, cf[0], cf[1], cf[2], XLOG0};
    const X5 DB = (lf == 31 || lf == 0) ? INIT : X5{0.f, cf[3], cf[4], cf[5], XLOG0};
    const bool wr_row = (t == 31) && s > 0;
    float g[9];
#pragma unroll
    for (int k = 0; k < 9; k++) g[k] = 0.f;
    X5 mine = INIT, upp = INIT;
    __syncwarp();
    adj_stage_trn<true>(trs, dt0, 0, L, lane);
    adj_stage_trn<true>(trs, dt0, 32, L, lane);
    adj_load_row<true, true>(a, rab, below, has_below, pb, 0, L, lane, broken);
    for (int k = 0; k < L + 31; k++) {
        const int jm = k - t;
        const int ca = L - 1 - jm;
        {
            // the rows step k + ADJ_PF reads first: forward states of its
            // diagonal row (5 lines), its own score, SS and CV rows, and lane
            // 0's diagonal successor in the strip below
            const int kq = k + ADJ_PF;
            const int kfq = L + 30 - kq;   // forward step of the lanes' own cells then
            if (kq < L + 31) {
                if (lane < 5 && kfq - 2 >= 0) pf_l1(Fw + (long long)(kfq - 2) * 160 + lane * 32);
                else if (kfq >= 0 && kfq < L + 31) {
                    if (lane == 5) pf_l1(a.S + cb + (long long)kfq * 32);
                    else if (lane == 6) pf_l1(a.pss + cb + (long long)kfq * 32);
                    else if (lane == 7) pf_l1(a.pcv + cb + (long long)kfq * 32);
                }
                if (lane == 8 && s + 1 < ns && L - kq >= 0 && L - kq < L)
                    pf_l1(a.S + cb + (long long)(L + 31) * 32 + (long long)(L - kq) * 32);
            }
        }
        // transitions out of column ca (row ca + 1, sequence index jm) and,
        // for the edge posteriors, into it (rows ca and ca + 1)
        const bool colv = jm >= 0 && jm < L;
        float tb[7], tf[7];
        {
            const float* b = trs + (jm & 127) * 7;         // row ca + 1
            const float* c = trs + ((jm + 1) & 127) * 7;   // row ca
#pragma unroll
            for (int f = 0; f < 7; f++) tb[f] = colv ? b[f] : XLOG0;
            tf[TMM] = c[0]; tf[TMI] = b[1]; tf[TMD] = c[2];
            tf[TIM] = c[3]; tf[TII] = b[4]; tf[TDM] = c[5]; tf[TDD] = c[6];
        }
        X5 dn;
        dn.MM = __shfl_up_sync(FULL, mine.MM, 1);
        dn.MI = __shfl_up_sync(FULL, mine.MI, 1);
        dn.IM = __shfl_up_sync(FULL, mine.IM, 1);
        dn.DN = __shfl_up_sync(FULL, mine.DN, 1);
        dn.ND = __shfl_up_sync(FULL, mine.ND, 1);
        {
            const int src = k & 31;
            const float4 ba = *reinterpret_cast<const float4*>(rab + src * 8);
            const float b4 = rab[src * 8 + 4];
            if (lane == 0) dn = X5{ba.x, ba.y, ba.z, ba.w, b4};
            if ((src & (ADJ_RG - 1)) == ADJ_RG - 1) {
                __syncwarp();
                adj_load_row<true, true>(a, rab, below, has_below, pb, k + 1, L, lane, broken);
            }
            if (src == 31) {
                if (k + 33 <= L) adj_stage_trn<true>(trs, dt0, k + 33, L, lane);
                __syncwarp();
            }
        }
        X5 rt = mine, dg = upp;
        if (jm == 0) { rt = INIT; dg = INIT; }
        const bool valid = act && jm >= 0 && jm < L;
        // score of the diagonal successor (i + 1, ca + 1)
        const float sco = (valid && i + 1 < Lq && ca + 1 < L) ? a.S[fw_cell(base, L, i + 1, ca + 1)] : XLOG0;
        X5 nw;
        nw.MM = xlse5p1((dn.MI + qb[TMM]) + tb[TMI], (rt.IM + qb[TMI]) + tb[TMM], dn.DN + qb[TMD],
                        rt.ND + tb[TMD], ((dg.MM + qb[TMM]) + tb[TMM]) + sco);
        nw.MI = xlse2(((dg.MM + qb[TMM]) + tb[TIM]) + sco, (dn.MI + qb[TMM]) + tb[TII]);
        nw.IM = xlse2(((dg.MM + qb[TIM]) + tb[TMM]) + sco, (rt.IM + qb[TII]) + tb[TMM]);
        nw.DN = xlse2(((dg.MM + qb[TDM]) + tb[TMM]) + sco, dn.DN + qb[TDD]);
        nw.ND = xlse2(((dg.MM + qb[TMM]) + tb[TDM]) + sco, rt.ND + tb[TDD]);
        // rows past the query (the last strip's first lanes) are the matrix
        // edge for the rows above them
        if (!act) nw = INIT;
        if (valid) {
            // edge posteriors of cell (i, ca): its forward predecessors
            const int kf = ca + lf;
            const X5 own = fw_ld5(Fw, kf, lf);
            X5 up, left, diag;
            if (i == 0) up = INIT;
            else if (lf == 0) up = X5{fab[ca], fab[L + ca], fab[2 * L + ca], fab[3 * L + ca], fab[4 * L + ca]};
            else up = fw_ld5(Fw, kf - 1, lf - 1);
            if (ca == 0) {
                left = LB;
                diag = DB;
            } else {
                left = fw_ld5(Fw, kf - 1, lf);
                if (i == 0) diag = INIT;
                else if (lf == 0)
                    diag = X5{fab[ca - 1], fab[L + ca - 1], fab[2 * L + ca - 1], fab[3 * L + ca - 1], fab[4 * L + ca - 1]};
                else diag = fw_ld5(Fw, kf - 2, lf - 1);
            }
            const long long kk = cb + (long long)kf * 32 + lf;
            const float sc = a.S[kk];
            const X5& b = nw;
            // MM: five emission edges
            const float eMM = b.MM - lz;
            const float m1 = xexp(((diag.MI + qf[TMM]) + tf[TIM]) + sc + eMM);
            const float m2 = xexp(((diag.IM + qf[TIM]) + tf[TMM]) + sc + eMM);
            const float m3 = xexp(((diag.DN + qf[TDM]) + tf[TMM]) + sc + eMM);
            const float m4 = xexp(((diag.ND + qf[TMM]) + tf[TDM]) + sc + eMM);
            const float m5 = xexp(((diag.MM + qf[TMM]) + tf[TMM]) + sc + eMM);
            const float gs = (m1 + m2 + m3 + m4) + m5;
            // MI, IM, DN (ND uses no query transition)
            const float i1 = xexp((up.MM + qf[TMM]) + tf[TMI] + b.MI - lz);
            const float i2 = xexp((up.MI + qf[TMM]) + tf[TII] + b.MI - lz);
            const float l1 = xexp((left.MM + qf[TMI]) + tf[TMM] + b.IM - lz);
            const float l2 = xexp((left.IM + qf[TII]) + tf[TMM] + b.IM - lz);
            const float d1 = xexp(up.MM + qf[TMD] + b.DN - lz);
            const float d2 = xexp(up.DN + qf[TDD] + b.DN - lz);
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
            a.post[kk] = xexp(own.MM + b.MM - lz);
            if (wr_row) {
                mine_row[ca] = nw.MM; mine_row[L + ca] = nw.MI; mine_row[2 * L + ca] = nw.IM;
                mine_row[3 * L + ca] = nw.DN; mine_row[4 * L + ca] = nw.ND;
                pipe_publish(a.prog + a.nitems + a.soff[m] + s, jm, L);
            }
        }
        mine = nw;
        upp = dn;
    }
    // the strip's gradient sums
#pragma unroll
    for (int f = 0; f < 9; f++) {
        float v = g[f];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        g[f] = v;
    }
    if (lane == 0) {
        float* o = a.gpart + (a.soff[m] + s) * 9;
#pragma unroll
        for (int f = 0; f < 9; f++) o[f] = g[f];
    }
}

__global__ void __launch_bounds__(ADJ_WARPS * 32) adj_bwd_kernel(AdjArgs a)
{
    __shared__ __align__(16) float rabs[ADJ_WARPS][32 * 8];
    __shared__ float trss[ADJ_WARPS][128 * 7];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* const scr = a.Fall ? nullptr : a.scratch + ((long long)blockIdx.x * ADJ_WARPS + wid) * a.scratch_stride;
    bool broken = false;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter + 1, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.nitems) break;
        const int2 ms = a.items_b[item];
        const int m = ms.x, s = ms.y;
        const float* Fw;
        if (a.Fall) {
            // the forward sweep kept the strip's states
            Fw = a.Fall + 5 * a.off[m] + (long long)s * (a.plen[a.prof[m]] + 31) * 160;
        } else {
            // checkpointing: the strip's states again, from the row above
            float zm = 0.f, zs = 0.f;
            adj_fwd_strip<true>(a, m, s, lane, rabs[wid], trss[wid], scr, broken, zm, zs);
            Fw = scr;
        }
        __syncwarp();
        adj_bwd_strip(a, m, s, lane, rabs[wid], trss[wid], Fw, broken);
        __syncwarp();
    }
}

// gradients of each pair: its strips' sums in strip order
__global__ void adj_gsum_kernel(AdjArgs a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= a.npairs * 9) return;
    const int m = x / 9, f = x % 9;
    const int ns = (a.pLq[m] + 31) >> 5;
    float v = 0.f;
    for (int s = 0; s < ns; s++) v += a.gpart[(a.soff[m] + s) * 9 + f];
    a.grad[x] = v;
}

cudaError_t adj_occupancy(int* fwd_ctas_per_sm, int* bwd_ctas_per_sm)
{
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(fwd_ctas_per_sm, adj_fwd_kernel, ADJ_WARPS * 32, 0);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bwd_ctas_per_sm, adj_bwd_kernel, ADJ_WARPS * 32, 0);
}

cudaError_t launch_adj_fwd(const AdjArgs& a, int grid, cudaStream_t st)
{
    if (a.npairs <= 0) return cudaSuccess;
    const int sgrid = std::min((a.nitems + ADJ_WARPS - 1) / ADJ_WARPS, 1184);
    adj_score_kernel<<<sgrid, 128, 0, st>>>(a);
    adj_fwd_kernel<<<grid, ADJ_WARPS * 32, 0, st>>>(a);
    adj_logz_kernel<<<(a.npairs + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_bwd(const AdjArgs& a, int grid, cudaStream_t st)
{
    if (a.npairs <= 0) return cudaSuccess;
    adj_bwd_kernel<<<grid, ADJ_WARPS * 32, 0, st>>>(a);
    adj_gsum_kernel<<<(a.npairs * 9 + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace c2
