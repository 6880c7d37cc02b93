// c2_kernels.cu -- phase-1 (fused score matrix + Viterbi DP) and DP
// finalisation kernels for sm_100a.
//
// Phase 1 replaces the reference's CalcSM_Init_SMEMUnroll2x +
// CalcSM_SSSS_CVS2S_SMEMUnroll2x_2 (src/libmycu/cusco/) and the per-diagonal
// ExecDP_Btck_Unroll32x launches (src/libmycu/cudp/CuBatchDP.cu:149-320,
// CuBatchDP_init_btck.cu:65-494).  Instead of materialising the L_q x N score
// matrix and a traceback byte per cell in HBM, one persistent warp owns one
// (query, db profile) pair at a time:
//  * lanes own query rows (a strip of 32 rows at a time); the query-row
//    operands of the score live in registers for the whole strip;
//  * each step, the warp reads one db column record with warp-uniform
//    (broadcast) loads and every lane scores its row against it; the score
//    goes to a per-lane ring in shared memory;
//  * the DP runs as an anti-diagonal wavefront: lane t processes column k-t at
//    step k, taking its "up" states from lane t-1 by __shfl_up_sync, its
//    "diagonal" states from the previous step's "up", and the column's
//    transitions passed down the lanes the same way;
//  * the strip's last row is handed to the next strip through a per-warp
//    boundary buffer (global memory, L2 resident).
// For the pairs that pass the phase-1 threshold, p2s_kernel stores the FP32
// scores column-major for the finalisation, statistics and MAP stages, and the
// traceback sweep (p1tc_kernel) runs the same DP on them again, storing btck
// codes.
#include <cuda_bf16.h>

#include <algorithm>

#include "c2_device.cuh"

namespace c2 {

#define FULL 0xffffffffu

__device__ __forceinline__ int corner_edge(int lq, int ld)
{
    // GetCornerMaxlen, src/libmycu/cudp/CuBatchDP_init_btck.cuh:118-127
    int m = lq > ld ? lq : ld;
    int e = (int)rintf(0.34f * (float)m);
    return e > 60 ? 60 : e;
}

__device__ __forceinline__ bool in_corner(int lq, int ld, int e, int y, int x)
{
    // CellYXinCorners, src/libmycu/cudp/CuBatchDP_init_btck.cuh:129-145
    return (lq <= y + e && x <= e + y - lq) || (ld - e + y <= x && y < e);
}

// Score of (own query row, db column) -- src/libmycu/cusco/CuBatchScoreMatrix_Init.cu:129-182,
// _ssss.cuh:48-131, _cvs2s.cuh:47-136.  The aa term uses the per-pair row
// factors Qt[a] = q(a) / (0.5 (bq(a) + bd(a))); the SS term uses the per-row
// table U[c] = sum_s p_q(s) T[idx_q(s)][c].
struct RowOps {
    float Qt[NAA];
    float qcv[NCV];
    float cq, pq, hq;
};

// cvtab holds each CV map value CVREP times ([cvcard][CVREP]); a lane reads
// replica lane % CVREP so that lanes reading different entries rarely share a bank.
template <int CVREP>
__device__ __forceinline__ float cell_score(const RowOps& R, const float4* __restrict__ rp,
                                            const float* __restrict__ U, const float* __restrict__ cvtab,
                                            const ScoreConsts& sc, int lane, float& mod_out)
{
    float4 v;
    // aa term (two accumulators shorten the dependent FMA chain)
    float s = 0.f, s2 = 0.f;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        v = rp[i];
        s = fmaf(R.Qt[4 * i + 0], v.x, s);
        s2 = fmaf(R.Qt[4 * i + 1], v.y, s2);
        s = fmaf(R.Qt[4 * i + 2], v.z, s);
        s2 = fmaf(R.Qt[4 * i + 3], v.w, s2);
    }
    s += s2;
    const float s0 = __logf(s) - sc.shift;
    // CV term: dot product over [20,39), then (cq)(cd) - (dot+1/kappa0)^2
    float dot = 0.f, dot2 = 0.f;
#pragma unroll
    for (int i = 5; i < 10; i++) {
        v = rp[i];
        const int b = 4 * i - DR_CV;
        dot = fmaf(R.qcv[b + 0], v.x, dot);
        dot2 = fmaf(R.qcv[b + 1], v.y, dot2);
        dot = fmaf(R.qcv[b + 2], v.z, dot);
        if (b + 3 < NCV) dot2 = fmaf(R.qcv[b + 3], v.w, dot2);
    }
    dot += dot2;
    const float cd = v.w;  // DR_CN = 39
    v = rp[10];            // 40 prior, 41..43 ss
    const float pd = v.x;
    const float ds0 = v.y, ds1 = v.z, ds2 = v.w;
    const float4 v11 = rp[11];  // 44 ss idx, 45 hd
    dot += sc.lokappa0;
    float det = R.cq * cd - dot * dot;
    float cvs = sc.cterm + sc.pownu0 * __logf(det) - R.pq - pd;
    float cvm;
    if (cvs <= sc.cvkey_first) cvm = sc.cvval_first;
    else if (sc.cvkey_last <= cvs) cvm = sc.cvval_last;
    else {
        // clamp keeps the shared-memory read in bounds for any table/argument
        const int ix = min(max(sc.cvshift + (int)rintf(2.f * cvs), 0), sc.cvcard - 1);
        cvm = cvtab[ix * CVREP + (lane & (CVREP - 1))];
    }
    cvm *= sc.cvswgt;
    // SS term
    const int pk = __float_as_int(v11.x);
    float ss = ds0 * U[(pk & 0xff) * 32 + lane];
    ss = fmaf(ds1, U[((pk >> 8) & 0xff) * 32 + lane], ss);
    ss = fmaf(ds2, U[((pk >> 16) & 0xff) * 32 + lane], ss);
    if (-99.f < ss) {
        ss += R.hq * v11.y * 0.1111111f;
        ss -= 0.05f;
        ss *= sc.ssswgt;
    }
    const float add = ss + cvm;
    mod_out = add - 0.5f * sc.cvswgt;   // modular score of the MAP stage
    return s0 + add;
}

struct St5 { float MM, MI, IM, DN, ND; };

// asynchronous global->shared copies (cp.async, 16 B each)
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Stage the records of columns [REC_CHUNK*m, REC_CHUNK*(m+1)) (clipped to L)
// into ring slots; records of consecutive columns are contiguous in HBM, so a
// chunk is one contiguous range copied by all lanes in 16-byte pieces.  Every
// call commits one group (possibly empty) so that wait_group counts stay aligned.
__device__ __forceinline__ void stage_chunk(float* rec, const float* __restrict__ dr, int m, int L, int lane)
{
    const int c0 = m * REC_CHUNK;
    const int nc = min(REC_CHUNK, L - c0);
    if (nc > 0) {
        const int n16 = nc * (DR_STRIDE / 4);
        float* dst = rec + (c0 & (REC_SLOTS - 1)) * DR_STRIDE;
        const float* src = dr + (long long)c0 * DR_STRIDE;
        for (int i = lane; i < n16; i += 32) cp_async16(dst + 4 * i, src + 4 * i);
    }
    cp_async_commit();
}

__global__ void __launch_bounds__(P1_WARPS * 32, 2)
p1_kernel(P1Args a, const float* __restrict__ qbkg)
{
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cvcard = a.sc.cvcard;
    const int card = a.sc.ssss_card;
    float* cvtab = smem;                                      // [cvcard][32]
    float* wb = smem + cvcard * 32 + wid * P1_WARP_FLOATS;
    float* ring = wb;                                         // [32][32]
    float* U = wb + 32 * 32;                                  // [card][32]
    float* rec = U + MAX_SSSS_CARD * 32;                      // [REC_SLOTS][DR_STRIDE] db records
    for (int i = threadIdx.x; i < cvcard * 32; i += blockDim.x) cvtab[i] = a.cvvals[i >> 5];
    __syncthreads();

    const long long slot = (long long)blockIdx.x * P1_WARPS + wid;
    const int Lmax = (int)(a.botstride / 10);
    float* bot0 = a.bot + slot * a.botstride;
    const int Lq = a.Lq;
    const int nstrips = (Lq + 31) >> 5;
    const ScoreConsts sc = a.sc;

    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.nwork) break;
        const int p = a.order[item];
        const int L = a.plen[p];
        const long long off = a.poff[p];
        const float* __restrict__ dr = a.drec + off * DR_STRIDE;
        const float* __restrict__ bd = a.pbkg + (long long)p * NAA;
        const int edge = corner_edge(Lq, L);
        float best = 0.f;
        int brow = 0x7fffffff, bcol = 0x7fffffff;
        float* botr = bot0;
        float* botw = bot0 + 5 * Lmax;

        for (int s = 0; s < nstrips; s++) {
            const int r = s * 32 + lane;
            const bool act = r < Lq;
            const float* __restrict__ qr = a.qrec + (long long)(act ? r : Lq - 1) * QR_STRIDE;
            RowOps R;
#pragma unroll
            for (int i = 0; i < NAA; i++)
                R.Qt[i] = __fdividef(qr[QR_TRG + i], 0.5f * (qbkg[i] + bd[i]));
#pragma unroll
            for (int i = 0; i < NCV; i++) R.qcv[i] = qr[QR_CV + i];
            R.cq = qr[QR_CN];
            R.pq = qr[QR_PRIOR];
            R.hq = qr[QR_HQ];
            {
                // this strip's SS row tables (built once per query, c2_set_query)
                const float* __restrict__ us = a.qU + (long long)s * MAX_SSSS_CARD * 32 + lane;
#pragma unroll 8
                for (int c = 0; c < card; c++) U[c * 32 + lane] = __ldg(us + c * 32);
            }
            float q7[7];
#pragma unroll
            for (int i = 0; i < 7; i++) q7[i] = act ? qr[QR_TRN + i] : LOG0;
            // column -1 boundary states of this row and of the row above
            const bool z_left = (lane == 31);
            const bool z_diag = (lane == 31 || lane == 0);
            const St5 LB = z_left ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                  : St5{0.f, qr[QR_C + 0], qr[QR_C + 1], qr[QR_C + 2], LOG0};
            const St5 DB = z_diag ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                  : St5{0.f, qr[QR_CP + 0], qr[QR_CP + 1], qr[QR_CP + 2], LOG0};
            __syncwarp();

            St5 mine = {0.f, 0.f, 0.f, 0.f, 0.f};
            St5 upp = {0.f, 0.f, 0.f, 0.f, 0.f};
            float t7[7];
#pragma unroll
            for (int i = 0; i < 7; i++) t7[i] = LOG0;
            // strip-boundary prefetch: lane i holds column c0 + i of the row above
            float bcur[5], bnxt[5];
#pragma unroll
            for (int f = 0; f < 5; f++) {
                bcur[f] = 0.f;
                bnxt[f] = 0.f;
                if (s > 0) {
                    if (lane < L) bcur[f] = botr[f * Lmax + lane];
                    if (32 + lane < L) bnxt[f] = botr[f * Lmax + 32 + lane];
                }
            }
            const bool wr_bot = (lane == 31) && (s + 1 < nstrips);
            const int nsteps = L + 31;
            // db column records are staged into shared memory one chunk ahead
            stage_chunk(rec, dr, 0, L, lane);
            stage_chunk(rec, dr, 1, L, lane);
            for (int k = 0; k < nsteps; k++) {
                if ((k & (REC_CHUNK - 1)) == 0 && k < L) {
                    cp_async_wait_1();
                    __syncwarp();
                }
                // ---- score stage: column k for every lane's row
                float tc[7];
                if (k < L) {
                    const float4* rp = reinterpret_cast<const float4*>(rec + (k & (REC_SLOTS - 1)) * DR_STRIDE);
                    float mod;
                    float S = cell_score<32>(R, rp, U, cvtab, sc, lane, mod);
                    if (!act) S = -9.f;
                    ring[(k & 31) * 32 + lane] = S;
                    const float4 ta = rp[12], tb = rp[13];
                    tc[0] = ta.x; tc[1] = ta.y; tc[2] = ta.z; tc[3] = ta.w;
                    tc[4] = tb.x; tc[5] = tb.y; tc[6] = tb.z;
                    if ((k & (REC_CHUNK - 1)) == REC_CHUNK - 1) {
                        // chunk fully read by every lane: refill its slots two chunks ahead
                        __syncwarp();
                        stage_chunk(rec, dr, (k >> REC_CHUNK_LOG) + 2, L, lane);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 7; i++) tc[i] = LOG0;
                }
                // ---- DP stage: column j = k - lane
#pragma unroll
                for (int i = 0; i < 7; i++) {
                    const float x = __shfl_up_sync(FULL, t7[i], 1);
                    t7[i] = (lane == 0) ? tc[i] : x;
                }
                St5 up;
                up.MM = __shfl_up_sync(FULL, mine.MM, 1);
                up.MI = __shfl_up_sync(FULL, mine.MI, 1);
                up.IM = __shfl_up_sync(FULL, mine.IM, 1);
                up.DN = __shfl_up_sync(FULL, mine.DN, 1);
                up.ND = __shfl_up_sync(FULL, mine.ND, 1);
                {
                    const int src = k & 31;
                    const float b0 = __shfl_sync(FULL, bcur[0], src);
                    const float b1 = __shfl_sync(FULL, bcur[1], src);
                    const float b2 = __shfl_sync(FULL, bcur[2], src);
                    const float b3 = __shfl_sync(FULL, bcur[3], src);
                    const float b4 = __shfl_sync(FULL, bcur[4], src);
                    if (lane == 0) up = St5{b0, b1, b2, b3, b4};
                    if (src == 31) {
#pragma unroll
                        for (int f = 0; f < 5; f++) {
                            bcur[f] = bnxt[f];
                            const int c = k + 33 + lane;
                            bnxt[f] = (s > 0 && c < L) ? botr[f * Lmax + c] : 0.f;
                        }
                    }
                }
                const int j = k - lane;
                St5 left = mine, diag = upp;
                if (j == 0) { left = LB; diag = DB; }
                float S = -9.f;
                if (j >= 0 && j < L) {
                    S = ring[(j & 31) * 32 + lane];
                    if (in_corner(Lq, L, edge, r, j)) S = -9.f;
                }
                St5 nw;
                {
                    float v = fmaxf((diag.MI + q7[TMM]) + t7[TIM], (diag.IM + q7[TIM]) + t7[TMM]);
                    v = fmaxf(v, (diag.DN + q7[TDM]) + t7[TMM]);
                    v = fmaxf(v, (diag.ND + q7[TMM]) + t7[TDM]);
                    v = fmaxf(v, (diag.MM + q7[TMM]) + t7[TMM]);
                    nw.MM = fmaxf(v + S, 0.f);
                    nw.MI = fmaxf((up.MM + q7[TMM]) + t7[TMI], (up.MI + q7[TMM]) + t7[TII]);
                    nw.IM = fmaxf((left.MM + q7[TMI]) + t7[TMM], (left.IM + q7[TII]) + t7[TMM]);
                    nw.DN = fmaxf(up.MM + q7[TMD], up.DN + q7[TDD]);
                    nw.ND = fmaxf(left.MM + t7[TMD], left.ND + t7[TDD]);
                }
                const bool valid = act && j >= 0 && j < L;
                if (valid && nw.MM > best) { best = nw.MM; brow = r; bcol = j; }
                if (wr_bot && j >= 0 && j < L) {
                    botw[0 * Lmax + j] = nw.MM;
                    botw[1 * Lmax + j] = nw.MI;
                    botw[2 * Lmax + j] = nw.IM;
                    botw[3 * Lmax + j] = nw.DN;
                    botw[4 * Lmax + j] = nw.ND;
                }
                mine = nw;
                upp = up;
            }
            cp_async_wait_all();
            float* t = botr; botr = botw; botw = t;
            __syncwarp();
        }
        // warp arg-max: largest score, then smallest row, then smallest column
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const float ob = __shfl_xor_sync(FULL, best, o);
            const int orr = __shfl_xor_sync(FULL, brow, o);
            const int oc = __shfl_xor_sync(FULL, bcol, o);
            if (ob > best || (ob == best && (orr < brow || (orr == brow && oc < bcol)))) {
                best = ob; brow = orr; bcol = oc;
            }
        }
        if (lane == 0) {
            const unsigned xy = (best > 0.f) ? (((unsigned)bcol << 16) | ((unsigned)brow & 0xffffu)) : 0u;
            a.best[p] = best;
            a.coords[p] = xy;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Phase 1, chunked: the same arithmetic as p1_kernel, scheduled in chunks of
// 32 db columns.  Per chunk, every lane first scores its query row against
// the 32 columns (independent cells: the FMA chains of consecutive columns
// overlap), writing scores and the columns' DP transitions to shared-memory
// rings; then the warp advances the anti-diagonal wavefront by 32 steps.
// Wavefront steps whose 32 cells all lie inside the matrix (every chunk but
// the first and the last ones of a strip) run without bounds checks.
//
// Score rings are indexed by anti-diagonal: the score of cell (row i of the
// strip, column j) sits in slot (i + j) & 63, so at step k every lane reads
// slot k & 63 and a DP stage reads 32 consecutive slots from one base.

// Pair of FP32 adds.  The packed sm_100 form (add.rn.f32x2) gives the same
// bits with ~1 % fewer instructions here, but measured 2 % slower in the
// tensor-core phase-1 kernel (5.53 vs 5.42 ms on 5,000 profiles), so the pairs
// stay two scalar adds; the pairing keeps the shared sums explicit.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

// Maximum of three (sm_100 three-input max.f32; exact, like two fmaxf)
__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// One lane of the wavefront DP.  Every Viterbi candidate of the reference's
// recurrence is (state + query transition) + db transition, evaluated in that
// order, with the sums that two candidates or two steps share computed once:
//   X = (up.MM, up.DN) + (qMM, qDM)   W = (up.MM, up.DN) + (qMD, qDD)
//   Y = (up.MI, up.IM) + (qMM, qIM)   z = up.ND + qMM
// X, Y and z are the up-sums of this step and the diagonal sums of the next
// (the diagonal predecessor of a cell is the up-neighbour of its left one).
struct WfLane {
    float MM, MI, IM, DN, ND;     // own state at the previous step (left)
    float2 X, Y;                  // up-sums of the previous step
    float z;
    float2 qX, qW, qY;            // (qMM, qDM), (qMD, qDD), (qMM, qIM)
    float qMM, qMI, qII;
    float2 XB, YB;                // diagonal sums of the column -1 boundary state
    float zB, lbMM, lbIM, lbND;   // and the column -1 left state
    float bnxt[5];                // row above the strip: columns [32m+32, 32m+64) (lane i: column 32m+32+i)
    float best;
    int kbest;
};

__device__ __forceinline__ void wf_init(WfLane& D, const float* q7, const St5& LB, const St5& DB)
{
    D.qX = make_float2(q7[TMM], q7[TDM]);
    D.qW = make_float2(q7[TMD], q7[TDD]);
    D.qY = make_float2(q7[TMM], q7[TIM]);
    D.qMM = q7[TMM];
    D.qMI = q7[TMI];
    D.qII = q7[TII];
    D.XB = add2(make_float2(DB.MM, DB.DN), D.qX);
    D.YB = add2(make_float2(DB.MI, DB.IM), D.qY);
    D.zB = DB.ND + q7[TMM];
    D.lbMM = LB.MM;
    D.lbIM = LB.IM;
    D.lbND = LB.ND;
    D.MM = D.MI = D.IM = D.DN = D.ND = 0.f;
    D.X = D.Y = make_float2(0.f, 0.f);
    D.z = 0.f;
    D.best = 0.f;
    D.kbest = 0;
}

// Row above the strip, 32 column slots: states MM, MI, IM, DN as a float4
// per slot ([32][4]), ND after them ([32] at BND_ND)
__device__ __forceinline__ void bnd_put(float* bnd, int slot, float mm, float mi, float im, float dn, float nd)
{
    *reinterpret_cast<float4*>(bnd + slot * 4) = make_float4(mm, mi, im, dn);
    bnd[BND_ND + slot] = nd;
}

// Wavefront steps [k0, k0 + nst) of a strip (k0 a multiple of 32, nst <= 32;
// 32 when !CHECK).  ring: diagonal-indexed scores, RLD floats per slot.
// Column records (DPT_N transitions, P1C_TRS floats apart): with TMIRROR,
// tcol points at this lane's record for step k0 and the next 31 follow
// without wrapping; otherwise tcol is a ring of TMASK + 1 records indexed by
// column & TMASK.  bnd: row above the strip for columns [k0, k0 + 32).
// TB (traceback sweep): each cell's traceback code also goes to the warp's
// column ring btr (column j in slot j & 31, the lane's own row), and column
// k - 31, complete for every row at step k, is stored to the pair's code
// matrix bt (column-major, Lq rows; r = this lane's query row).
template <bool CHECK, int RLD, bool TMIRROR, int TMASK, bool TB = false>
__device__ __forceinline__ void wf_steps(WfLane& D, int k0, int nst, int lane, int L, bool act,
                                         const float* __restrict__ ring, const float* __restrict__ tcol,
                                         float* __restrict__ bnd, bool wr_bot, signed char (*btr)[33] = nullptr,
                                         signed char* __restrict__ bt = nullptr, int Lq = 0, int r = 0)
{
    const float* __restrict__ rb = ring + (k0 & (P1C_RING - 1)) * RLD + lane;
    if (!CHECK) nst = 32;
    int ub = -1;
    // the instruction cache holds both variants of both kernels at these depths
    constexpr int UNR = CHECK ? 2 : 4;
#pragma unroll UNR
    for (int u = 0; u < nst; u++) {
        const float S = rb[u * RLD];
        const float* __restrict__ tp =
            TMIRROR ? tcol + u * P1C_TRS : tcol + ((k0 + u - lane) & TMASK) * P1C_TRS;
        const float4 ta = *reinterpret_cast<const float4*>(tp);       // MM MM IM MM
        const float4 tb = *reinterpret_cast<const float4*>(tp + 4);   // MD DD MI II
        const float tDM = tp[8];
        float uMM = __shfl_up_sync(FULL, D.MM, 1);
        float uMI = __shfl_up_sync(FULL, D.MI, 1);
        float uIM = __shfl_up_sync(FULL, D.IM, 1);
        float uDN = __shfl_up_sync(FULL, D.DN, 1);
        float uND = __shfl_up_sync(FULL, D.ND, 1);
        {
            // row above the strip at column k (lane 0's column), broadcast reads
            const float4 ba = *reinterpret_cast<const float4*>(bnd + u * 4);
            const float b4 = bnd[BND_ND + u];
            if (lane == 0) { uMM = ba.x; uMI = ba.y; uIM = ba.z; uDN = ba.w; uND = b4; }
        }
        const int j = k0 + u - lane;
        float2 Xd = D.X, Yd = D.Y;
        float zd = D.z, lMM = D.MM, lIM = D.IM, lND = D.ND;
        if (CHECK && j == 0) {
            Xd = D.XB; Yd = D.YB; zd = D.zB;
            lMM = D.lbMM; lIM = D.lbIM; lND = D.lbND;
        }
        const float2 T0 = make_float2(ta.x, ta.y), T1 = make_float2(ta.z, ta.w), T2 = make_float2(tb.x, tb.y);
        const float2 X = add2(make_float2(uMM, uDN), D.qX);
        const float2 W = add2(make_float2(uMM, uDN), D.qW);
        const float2 Y = add2(make_float2(uMI, uIM), D.qY);
        const float z = uND + D.qMM;
        const float2 c53 = add2(Xd, T0);   // diag MM + MM + MM, diag DN + DM + MM
        const float2 c12 = add2(Yd, T1);   // diag MI + MM + IM, diag IM + IM + MM
        const float v = max3f(max3f(c12.x, c12.y, c53.y), zd + tDM, c53.x);
        const float nMM = fmaxf(v + S, 0.f);
        const float nMI = fmaxf(X.x + tb.z, Y.x + tb.w);
        const float2 c89 = add2(make_float2(lMM + D.qMI, lIM + D.qII), T0);
        const float2 cND = add2(make_float2(lMM, lND), T2);
        const float nIM = fmaxf(c89.x, c89.y);
        const float nDN = fmaxf(W.x, W.y);
        const float nND = fmaxf(cND.x, cND.y);
        // inactive lanes (rows past the query) carry LOG0 query transitions:
        // their MM stays 0 and never beats a maximum
        const bool inm = !CHECK || (j >= 0 && j < L);
        if ((!CHECK || act) && inm && nMM > D.best) { D.best = nMM; ub = u; }
        if (TB) {
            // ExecDP_Btck's code: DIAG if MM > 0, then the first strictly larger
            // of MI (UP), IM (LEFT), DN (UP), ND (LEFT)
            if (act && inm) {
                int b = BT_STOP;
                float mx = nMM;
                if (nMM != 0.f) b = BT_DIAG;
                if (mx < nMI) { mx = nMI; b = BT_UP; }
                if (mx < nIM) { mx = nIM; b = BT_LEFT; }
                if (mx < nDN) { mx = nDN; b = BT_UP; }
                if (mx < nND) b = BT_LEFT;
                btr[j & 31][lane] = (signed char)b;
            }
            const int cfl = k0 + u - 31;
            if (act && (!CHECK || (cfl >= 0 && cfl < L))) bt[(long long)cfl * Lq + r] = btr[cfl & 31][lane];
        }
        if (wr_bot) {
            // lane 31's cell (column k0 + u - 31) into the slot lane 0 read at
            // the top of this step; bot_flush stores the 32 columns per chunk
            bnd_put(bnd, u, nMM, nMI, nIM, nDN, nND);
        }
        D.MM = nMM; D.MI = nMI; D.IM = nIM; D.DN = nDN; D.ND = nND;
        D.X = X; D.Y = Y; D.z = z;
    }
    if (ub >= 0) D.kbest = k0 + ub;
}

// The strip's last row after a DP stage over [k0, k0 + 32): slot l of bnd
// holds lane 31's states at column k0 - 31 + l; the warp stores the columns
// inside the matrix to the boundary buffer, one coalesced segment per state
__device__ __forceinline__ void bot_flush(const float* __restrict__ bnd, float* __restrict__ botw, int k0, int L,
                                          int Lmax, int lane)
{
    const int c = k0 - 31 + lane;
    if (c >= 0 && c < L) {
        const float4 a = *reinterpret_cast<const float4*>(bnd + lane * 4);
        botw[0 * Lmax + c] = a.x;
        botw[1 * Lmax + c] = a.y;
        botw[2 * Lmax + c] = a.z;
        botw[3 * Lmax + c] = a.w;
        botw[4 * Lmax + c] = bnd[BND_ND + lane];
    }
}

// Corner cells (CellYXinCorners): row r keeps S = -9 at columns j <= cA(r)
// and j >= cB(r).
__device__ __forceinline__ int corner_a(int r, int Lq, int edge) { return (Lq <= r + edge) ? edge + r - Lq : -1; }
__device__ __forceinline__ int corner_b(int r, int L, int edge) { return (r < edge) ? L - edge + r : 0x7fffffff; }

__global__ void __launch_bounds__(P1C_WARPS * 32, 1)
p1c_kernel(P1Args a, const float* __restrict__ qbkg)
{
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cvcard = a.sc.cvcard;
    const int card = a.sc.ssss_card;
    float* cvtab = smem;                                      // [cvcard][P1C_CVREP]
    float* wb = smem + cvcard * P1C_CVREP + wid * P1C_WARP_FLOATS;
    float* ring = wb;                                         // [P1C_RING][32] scores
    float* trn = ring + P1C_RING * 32;                        // [P1C_RING][P1C_TRS] transitions
    float* U = trn + P1C_RING * P1C_TRS;                      // [card][32]
    float* rec = U + MAX_SSSS_CARD * 32;                      // [REC_SLOTS][DR_STRIDE] db records
    float* bnd = rec + REC_SLOTS * DR_STRIDE;                 // [BND_FLOATS] row above the strip
    for (int i = threadIdx.x; i < cvcard * P1C_CVREP; i += blockDim.x) cvtab[i] = a.cvvals[i / P1C_CVREP];
    __syncthreads();

    const long long slotw = (long long)blockIdx.x * P1C_WARPS + wid;
    const int Lmax = (int)(a.botstride / 10);
    float* bot0 = a.bot + slotw * a.botstride;
    const int Lq = a.Lq;
    const int nstrips = (Lq + 31) >> 5;
    const ScoreConsts sc = a.sc;

    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.nwork) break;
        const int p = a.order[item];
        const int L = a.plen[p];
        const long long off = a.poff[p];
        const float* __restrict__ dr = a.drec + off * DR_STRIDE;
        const float* __restrict__ bd = a.pbkg + (long long)p * NAA;
        const int edge = corner_edge(Lq, L);
        float* botr = bot0;
        float* botw = bot0 + 5 * Lmax;
        float pbest = 0.f;
        int prow = 0x7fffffff, pcol = 0x7fffffff;

        for (int s = 0; s < nstrips; s++) {
            const int r = s * 32 + lane;
            const bool act = r < Lq;
            const float* __restrict__ qr = a.qrec + (long long)(act ? r : Lq - 1) * QR_STRIDE;
            RowOps R;
#pragma unroll
            for (int i = 0; i < NAA; i++)
                R.Qt[i] = __fdividef(qr[QR_TRG + i], 0.5f * (qbkg[i] + bd[i]));
#pragma unroll
            for (int i = 0; i < NCV; i++) R.qcv[i] = qr[QR_CV + i];
            R.cq = qr[QR_CN];
            R.pq = qr[QR_PRIOR];
            R.hq = qr[QR_HQ];
            {
                // this strip's SS row tables (built once per query, c2_set_query)
                const float* __restrict__ us = a.qU + (long long)s * MAX_SSSS_CARD * 32 + lane;
#pragma unroll 8
                for (int c = 0; c < card; c++) U[c * 32 + lane] = __ldg(us + c * 32);
            }
            WfLane D;
            float q7[7];
#pragma unroll
            for (int i = 0; i < 7; i++) q7[i] = act ? qr[QR_TRN + i] : LOG0;
            // column -1 boundary states of this row and of the row above
            const bool z_left = (lane == 31);
            const bool z_diag = (lane == 31 || lane == 0);
            const St5 LB = z_left ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                  : St5{0.f, qr[QR_C + 0], qr[QR_C + 1], qr[QR_C + 2], LOG0};
            const St5 DB = z_diag ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                  : St5{0.f, qr[QR_CP + 0], qr[QR_CP + 1], qr[QR_CP + 2], LOG0};
            // corner cells of this row: j <= cA or j >= cB
            const int cA = corner_a(r, Lq, edge);
            const int cB = corner_b(r, L, edge);
            wf_init(D, q7, LB, DB);
            float bc[5];
#pragma unroll
            for (int f = 0; f < 5; f++) {
                bc[f] = 0.f;
                D.bnxt[f] = 0.f;
                if (s > 0) {
                    if (lane < L) bc[f] = botr[f * Lmax + lane];
                    if (32 + lane < L) D.bnxt[f] = botr[f * Lmax + 32 + lane];
                }
            }
            const bool wr_bot = (lane == 31) && (s + 1 < nstrips);
            __syncwarp();
            // columns [0, 32) of the row above, lane i holding column i
            bnd_put(bnd, lane, bc[0], bc[1], bc[2], bc[3], bc[4]);
            stage_chunk(rec, dr, 0, L, lane);
            stage_chunk(rec, dr, 1, L, lane);
            const int nch = (L + 31) >> 5;        // chunks holding columns
            const int kend = L + 31;              // wavefront steps of the strip
            for (int m = 0; 32 * m < kend; m++) {
                // ---- score stage: columns [32m, min(32m + 32, L))
                if (m < nch) {
                    const int c0 = 32 * m, c1 = min(c0 + 32, L);
                    // does any row of the strip have corner cells in this chunk?
                    const bool hasc = __any_sync(FULL, cA >= c0 || cB < c1);
                    for (int c = c0; c < c1; c++) {
                        if ((c & (REC_CHUNK - 1)) == 0) {
                            cp_async_wait_1();
                            __syncwarp();
                        }
                        const float* rc = rec + (c & (REC_SLOTS - 1)) * DR_STRIDE;
                        float mod;
                        float Sc = cell_score<P1C_CVREP>(R, reinterpret_cast<const float4*>(rc), U, cvtab, sc, lane, mod);
                        (void)mod;
                        if (hasc && (c <= cA || c >= cB)) Sc = -9.f;
                        ring[((c + lane) & (P1C_RING - 1)) * 32 + lane] = Sc;
                        if (lane < DPT_N) trn[(c & (P1C_RING - 1)) * P1C_TRS + lane] = rc[DR_TRN + dpt_src(lane)];
                        if ((c & (REC_CHUNK - 1)) == REC_CHUNK - 1) {
                            // group fully read by every lane: refill its slots two groups ahead
                            __syncwarp();
                            stage_chunk(rec, dr, (c >> REC_CHUNK_LOG) + 2, L, lane);
                        }
                    }
                }
                __syncwarp();
                // ---- DP stage: wavefront steps [32m, 32m + 32)
                const int k0 = 32 * m, k1 = min(k0 + 32, kend);
                if (m >= 1 && k0 + 31 < L && k1 == k0 + 32)
                    wf_steps<false, 32, false, P1C_RING - 1>(D, k0, 32, lane, L, act, ring, trn, bnd, wr_bot);
                else
                    wf_steps<true, 32, false, P1C_RING - 1>(D, k0, k1 - k0, lane, L, act, ring, trn, bnd, wr_bot);
                __syncwarp();
                if (s + 1 < nstrips) bot_flush(bnd, botw, k0, L, Lmax, lane);
                __syncwarp();
                // next 32 columns of the row above the strip
                bnd_put(bnd, lane, D.bnxt[0], D.bnxt[1], D.bnxt[2], D.bnxt[3], D.bnxt[4]);
#pragma unroll
                for (int f = 0; f < 5; f++) {
                    const int cc = k0 + 64 + lane;
                    D.bnxt[f] = (s > 0 && cc < L) ? botr[f * Lmax + cc] : 0.f;
                }
                __syncwarp();
            }
            cp_async_wait_all();
            // this strip's maximum: largest score, then smallest row, then smallest column
            {
                float b = D.best;
                int rr = (D.best > 0.f) ? r : 0x7fffffff;
                int cc = (D.best > 0.f) ? D.kbest - lane : 0x7fffffff;
                if (b > pbest || (b == pbest && (rr < prow || (rr == prow && cc < pcol)))) {
                    pbest = b; prow = rr; pcol = cc;
                }
            }
            float* t = botr; botr = botw; botw = t;
            __syncwarp();
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const float ob = __shfl_xor_sync(FULL, pbest, o);
            const int orr = __shfl_xor_sync(FULL, prow, o);
            const int oc = __shfl_xor_sync(FULL, pcol, o);
            if (ob > pbest || (ob == pbest && (orr < prow || (orr == prow && oc < pcol)))) {
                pbest = ob; prow = orr; pcol = oc;
            }
        }
        if (lane == 0) {
            const unsigned xy = (pbest > 0.f) ? (((unsigned)pcol << 16) | ((unsigned)prow & 0xffffu)) : 0u;
            a.best[p] = pbest;
            a.coords[p] = xy;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Traceback sweep, chunked: the DP finalisation's FP32 recomputation of the
// candidates (ExecDP_Btck_Unroll32x, src/libmycu/cudp/CuBatchDP_init_btck.cu:
// 303-360) with p1c_kernel's schedule -- per 32-column chunk the scores of the
// strip (also stored to the pair's score and modular-score matrices, column-
// major, coalesced) and then 32 wavefront steps that also store the traceback
// codes.  Work items are (candidate, strip) in the strip pipeline of
// c2_device.cuh: strip s waits, before DP stage m, for the strip above to have
// published the columns of chunk m + 1 of its last row (loaded into registers
// during the stage) and publishes its own last row once per chunk.  The
// arithmetic is p1c_kernel's, so the maxima equal phase 1's in the FP32 form.
// Phase-2 score matrices: the FP32 scores and modular scores of every cell of
// the candidate pairs, column-major per pair (the layout of the finalisation,
// statistics and MAP stages), by cell_score -- the arithmetic of phase 1's
// FP32 form.  One warp per (candidate, strip) at a time, lanes own query rows,
// db records staged in shared memory as in phase 1; no dependencies between
// work items, so every resident warp works.
__global__ void __launch_bounds__(P2S_WARPS * 32)
p2s_kernel(P1Args a, const float* __restrict__ qbkg)
{
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cvcard = a.sc.cvcard;
    const int card = a.sc.ssss_card;
    float* cvtab = smem;                                      // [cvcard][P1TC_CVREP]
    float* U = smem + cvcard * P1TC_CVREP + wid * P2S_WARP_FLOATS;   // [card][32]
    float* rec = U + MAX_SSSS_CARD * 32;                      // [REC_SLOTS][DR_STRIDE] db records
    for (int i = threadIdx.x; i < cvcard * P1TC_CVREP; i += blockDim.x) cvtab[i] = a.cvvals[i / P1TC_CVREP];
    __syncthreads();
    const int Lq = a.Lq;
    const int nstrips = (Lq + 31) >> 5;
    const int nitems = a.nwork * nstrips;
    const ScoreConsts sc = a.sc;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter + 1, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= nitems) break;
        const int cand = a.worder[item / nstrips];
        const int s = item % nstrips;
        const int p = a.order[cand];
        const int L = a.plen[p];
        const float* __restrict__ dr = a.drec + a.poff[p] * DR_STRIDE;
        const float* __restrict__ bd = a.pbkg + (long long)p * NAA;
        const long long coff = a.cand_off[cand];
        float* smt = a.smat + coff;
        float* mmt = a.mmat + coff;
        const int r = s * 32 + lane;
        const bool act = r < Lq;
        const float* __restrict__ qr = a.qrec + (long long)(act ? r : Lq - 1) * QR_STRIDE;
        RowOps R;
#pragma unroll
        for (int i = 0; i < NAA; i++)
            R.Qt[i] = __fdividef(qr[QR_TRG + i], 0.5f * (qbkg[i] + bd[i]));
#pragma unroll
        for (int i = 0; i < NCV; i++) R.qcv[i] = qr[QR_CV + i];
        R.cq = qr[QR_CN];
        R.pq = qr[QR_PRIOR];
        R.hq = qr[QR_HQ];
        __syncwarp();
        {
            // this strip's SS row tables (built once per query, c2_set_query)
            const float* __restrict__ us = a.qU + (long long)s * MAX_SSSS_CARD * 32 + lane;
#pragma unroll 8
            for (int c = 0; c < card; c++) U[c * 32 + lane] = __ldg(us + c * 32);
        }
        stage_chunk(rec, dr, 0, L, lane);
        stage_chunk(rec, dr, 1, L, lane);
        // a staged chunk of REC_CHUNK columns at a time: its cells are
        // independent, so their chains overlap
        for (int c0 = 0; c0 < L; c0 += REC_CHUNK) {
            cp_async_wait_1();
            __syncwarp();
#pragma unroll
            for (int u = 0; u < REC_CHUNK; u++) {
                const int c = c0 + u;
                if (c < L) {
                    const float* rc = rec + (c & (REC_SLOTS - 1)) * DR_STRIDE;
                    float mod;
                    const float Sc =
                        cell_score<P1TC_CVREP>(R, reinterpret_cast<const float4*>(rc), U, cvtab, sc, lane, mod);
                    if (act) {
                        smt[(long long)c * Lq + r] = Sc;
                        mmt[(long long)c * Lq + r] = mod;
                    }
                }
            }
            __syncwarp();
            stage_chunk(rec, dr, (c0 >> REC_CHUNK_LOG) + 2, L, lane);
        }
        cp_async_wait_all();
        __syncwarp();
    }
}

// Traceback sweep over the candidate pairs: the FP32 Viterbi DP again, on the
// score matrices p2s_kernel wrote (read a 32-column chunk at a time into the
// anti-diagonal ring), with the btck code of every cell stored column-major
// and the strips of a pair pipelined over warps.
__global__ void __launch_bounds__(P1TC_WARPS * 32, 1)
p1tc_kernel(P1Args a, const float* __restrict__ qbkg)
{
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __shared__ signed char btr_all[P1TC_WARPS][32][33];
    signed char(*btr)[33] = btr_all[wid];
    float* wb = smem + wid * P1TC_WARP_FLOATS;
    float* ring = wb;                                         // [P1C_RING][32] scores
    float* trn = ring + P1C_RING * 32;                        // [P1C_RING][P1C_TRS] transitions
    float* bnd = trn + P1C_RING * P1C_TRS;                    // [BND_FLOATS] row above the strip
    (void)qbkg;

    const int Lq = a.Lq;
    const int nstrips = (Lq + 31) >> 5;
    const int nitems = a.nwork * nstrips;
    bool broken = false;

    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= nitems) break;
        const int iv = a.items[item];
        const int rank = iv / nstrips, s = iv - rank * nstrips;
        const int cand = a.worder[rank];
        const int p = a.order[cand];
        const int L = a.plen[p];
        const long long off = a.poff[p];
        const float* __restrict__ dr = a.drec + off * DR_STRIDE;
        const int edge = corner_edge(Lq, L);
        const long long coff = a.cand_off[cand];
        signed char* bt = a.btck + coff;
        const float* smt = a.smat + coff;
        float* pb = a.bnd + (coff / Lq) * 10;
        const float* botr = pb + ((s + 1) & 1) * 5 * L;   // last row of strip s-1
        float* botw = pb + (s & 1) * 5 * L;
        int* pf = a.prog + (long long)cand * nstrips;
        const int r = s * 32 + lane;
        const bool act = r < Lq;
        const float* __restrict__ qr = a.qrec + (long long)(act ? r : Lq - 1) * QR_STRIDE;
        WfLane D;
        {
            float q7[7];
#pragma unroll
            for (int i = 0; i < 7; i++) q7[i] = act ? qr[QR_TRN + i] : LOG0;
            const bool z_left = (lane == 31);
            const bool z_diag = (lane == 31 || lane == 0);
            const St5 LB = z_left ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                  : St5{0.f, qr[QR_C + 0], qr[QR_C + 1], qr[QR_C + 2], LOG0};
            const St5 DB = z_diag ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                  : St5{0.f, qr[QR_CP + 0], qr[QR_CP + 1], qr[QR_CP + 2], LOG0};
            wf_init(D, q7, LB, DB);
        }
        const int cA = corner_a(r, Lq, edge);
        const int cB = corner_b(r, L, edge);
        // columns [0, 32) of the row above, lane i holding column i
        float bc[5];
        if (s > 0) pipe_wait(pf + s - 1, min(32, L), lane, a.status, broken, a.spin);
#pragma unroll
        for (int f = 0; f < 5; f++) {
            bc[f] = (s > 0 && lane < L) ? __ldcg(botr + f * L + lane) : 0.f;
            D.bnxt[f] = 0.f;
        }
        const bool wr_bot = (lane == 31) && (s + 1 < nstrips);
        __syncwarp();
        bnd_put(bnd, lane, bc[0], bc[1], bc[2], bc[3], bc[4]);
        const int nch = (L + 31) >> 5;
        const int kend = L + 31;
        for (int m = 0; 32 * m < kend; m++) {
            // ---- score stage: columns [32m, min(32m + 32, L)) from the score
            // matrix (the lanes' rows of one column: one 128-byte line), and
            // the columns' transitions
            if (m < nch) {
                const int c0 = 32 * m, c1 = min(c0 + 32, L);
                const bool hasc = __any_sync(FULL, cA >= c0 || cB < c1);
#pragma unroll 8
                for (int c = c0; c < c1; c++) {
                    float Sc = act ? __ldcg(smt + (long long)c * Lq + r) : 0.f;
                    if (hasc && (c <= cA || c >= cB)) Sc = -9.f;
                    ring[((c + lane) & (P1C_RING - 1)) * 32 + lane] = Sc;
                    if (lane < DPT_N)
                        trn[(c & (P1C_RING - 1)) * P1C_TRS + lane] = __ldg(dr + (long long)c * DR_STRIDE + DR_TRN + dpt_src(lane));
                }
            }
            // the row above for chunk m + 1, loaded while this stage runs
            const int k0 = 32 * m, k1 = min(k0 + 32, kend);
            if (s > 0 && k0 + 32 < L) {
                pipe_wait(pf + s - 1, min(k0 + 64, L), lane, a.status, broken, a.spin);
#pragma unroll
                for (int f = 0; f < 5; f++) {
                    const int cc = k0 + 32 + lane;
                    D.bnxt[f] = (cc < L) ? __ldcg(botr + f * L + cc) : 0.f;
                }
            } else {
#pragma unroll
                for (int f = 0; f < 5; f++) D.bnxt[f] = 0.f;
            }
            __syncwarp();
            // ---- DP stage: wavefront steps [32m, 32m + 32), traceback codes stored
            if (m >= 1 && k0 + 31 < L && k1 == k0 + 32)
                wf_steps<false, 32, false, P1C_RING - 1, true>(D, k0, 32, lane, L, act, ring, trn, bnd, wr_bot, btr,
                                                               bt, Lq, r);
            else
                wf_steps<true, 32, false, P1C_RING - 1, true>(D, k0, k1 - k0, lane, L, act, ring, trn, bnd, wr_bot,
                                                              btr, bt, Lq, r);
            __syncwarp();
            if (s + 1 < nstrips) {
                // last row of columns [k0 - 31, k0] to the pair's buffer, then published
                bot_flush(bnd, botw, k0, L, L, lane);
                __syncwarp();
                if (lane == 0) {
                    __threadfence();
                    pipe_st_release(pf + s, min(k1 - 31, L));
                }
            }
            __syncwarp();
            bnd_put(bnd, lane, D.bnxt[0], D.bnxt[1], D.bnxt[2], D.bnxt[3], D.bnxt[4]);
            __syncwarp();
        }
        // the strip's maximum: largest score, then smallest row, then smallest column
        float best = D.best;
        int brow = (best > 0.f) ? r : 0x7fffffff;
        int bcol = (best > 0.f) ? D.kbest - lane : 0x7fffffff;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const float ob = __shfl_xor_sync(FULL, best, o);
            const int orr = __shfl_xor_sync(FULL, brow, o);
            const int oc = __shfl_xor_sync(FULL, bcol, o);
            if (ob > best || (ob == best && (orr < brow || (orr == brow && oc < bcol)))) {
                best = ob; brow = orr; bcol = oc;
            }
        }
        // pair maximum over strips as one 64-bit key (best >= 0 orders by its bits)
        if (lane == 0 && best > 0.f) {
            const unsigned cell = ((unsigned)brow << 16) | ((unsigned)bcol & 0xffffu);
            atomicMax(a.tbkey + cand,
                      ((unsigned long long)__float_as_uint(best) << 32) | (unsigned long long)(0xffffffffu - cell));
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Tensor-core score path (layouts in c2_device.cuh).

__device__ __forceinline__ unsigned bf16_bits(float x)
{
    return (unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// hi and lo BF16 parts of x: hi = bf16(x), lo = bf16(x - hi)
__device__ __forceinline__ void bf16_split(float x, unsigned& hi, unsigned& lo)
{
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi = (unsigned)__bfloat16_as_ushort(h);
    lo = bf16_bits(x - __bfloat162float(h));
}

// D += A * B, m16n8k16, BF16 inputs, FP32 accumulation
// first product of a chain: C = 0 (no accumulator zeroing)
__device__ __forceinline__ void mma_bf16_z(float* d, const unsigned* a, unsigned b0, unsigned b1)
{
    const float z = 0.f;
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%10,%10,%10,%10};\n"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(z));
}

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// mbarrier and bulk (non-tensor, non-multicast) async copy helpers
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Tensor memory (TMEM) as a per-lane store of loop-invariant fragments: the
// allocating warp takes ncols columns for the CTA; warp w reads and writes
// lanes [32 (w % 4), 32 (w % 4) + 32) only (32x32b shape: thread i <-> lane
// 32 (w % 4) + i, consecutive 32-bit columns).
__device__ __forceinline__ void tmem_alloc(unsigned* dst_smem, unsigned ncols)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_st16(unsigned taddr, const unsigned* v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// 32 columns into v; the wait takes v as operands so no use of v can be
// scheduled before the load has completed
__device__ __forceinline__ void tmem_ld32(unsigned taddr, unsigned* v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
          "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                   "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                   "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]),
                   "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]),
                   "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// one thread: expect `bytes` on the barrier and start the copy global -> shared
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Wait for phase `parity` of the barrier to complete; gives up after a bounded
// number of polls (returns false; the caller records a device status).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
    const unsigned a = smem_u32(bar);
    for (int it = 0; it < (1 << 22); it++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Pack the db operands of one profile per CTA (4 warps over its 8-column
// tiles) and its column records.  lok: 1/kappa0 (CV column k = 19); wss: SS
// weight (SS operand and its folded columns k = 30, 31).
__global__ void __launch_bounds__(128) tc_pack_kernel(const float* __restrict__ drec, const long long* __restrict__ poff,
                                                      const int* __restrict__ plen, const long long* __restrict__ ttile,
                                                      unsigned* __restrict__ tcdb, float* __restrict__ cold, float lok,
                                                      float wss)
{
    const int p = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int L = plen[p];
    const long long off = poff[p];
    const int ntiles = ((L + 31) >> 5) * 4;
    const int g = lane >> 2, q = lane & 3;
    for (int t = wid; t < ntiles; t += 4) {
        const int col = 8 * t + g;
        const bool valid = col < L;
        const float* rc = drec + (off + (valid ? col : 0)) * DR_STRIDE;
        const int pk = __float_as_int(rc[DR_SSIDX]);
        const int i0 = pk & 0xff, i1 = (pk >> 8) & 0xff, i2 = (pk >> 16) & 0xff;
        unsigned* out = tcdb + (ttile[p] + t) * (long long)TC_TILE_WORDS;
#pragma unroll
        for (int d = 0; d < 3; d++) {
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                float v[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int k = 16 * kt + 2 * q + (e & 1) + (e >> 1) * 8;
                    float x = 0.f;
                    if (valid) {
                        if (d == 0) x = (k < NAA) ? rc[DR_TRG + k] : 0.f;
                        else if (d == 1) x = (k < NCV) ? rc[DR_CV + k] : (k == NCV) ? lok : 0.f;
                        else if (k == i0) x = wss * rc[DR_SS];
                        else if (k == i1) x = wss * rc[DR_SS + 1];
                        else if (k == i2) x = wss * rc[DR_SS + 2];
                        else if (k == TC_SS_KMAX) x = wss * (rc[DR_HD] * 0.1111111f);
                        else if (k == TC_SS_KMAX + 1) x = -0.05f * wss;
                    }
                    v[e] = x;
                }
                unsigned h[4], l[4];
#pragma unroll
                for (int e = 0; e < 4; e++) bf16_split(v[e], h[e], l[e]);
                unsigned* o = out + ((d * 2 + kt) * 2) * 64 + lane * 2;
                o[0] = h[0] | (h[1] << 16);
                o[1] = h[2] | (h[3] << 16);
                o[64] = l[0] | (l[1] << 16);
                o[65] = l[2] | (l[3] << 16);
            }
        }
    }
    for (int c = threadIdx.x; c < L; c += blockDim.x) {
        const float* rc = drec + (off + c) * DR_STRIDE;
        float* o = cold + (off + c) * P1C_TRS;
#pragma unroll
        for (int i = 0; i < DPT_N; i++) o[i] = rc[DR_TRN + dpt_src(i)];
        o[CO_CD] = rc[DR_CN];
        o[CO_PD2] = 2.f * rc[DR_PRIOR];
        o[11] = 0.f;
    }
}

// Score epilogue of one cell of the tensor-core form from its three
// contractions (the CV one with 1/kappa0 folded in, the SS one the complete
// weighted SS term):
//   x   = 2 (cterm + pownu0 ln(cq cd - dot^2) - prior_q - prior_d)
//   cvm = w_cv T[shift + rint(x)] (T clamped; the key range tests when the
//         table is not uniform)
//   S   = (ln(aa) - shift) + (ss + cvm), evaluated as ln(aa) + (ss +
//         (cvm - shift)) with the table pre-shifted: a reassociation within
//         the rounding of the split-BF16 products (this form only ranks the
//         pairs; the candidates are rescored in FP32)
// (cell_score is the FP32 form; src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cu)
constexpr float C2_LN2 = 0.693147180559945309f;
// hardware base-2 logarithm, denormal inputs flushed (the arguments here, an
// amino-acid odds sum and a CV determinant, are far above the denormal range)
__device__ __forceinline__ float lg2_ftz(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
template <bool CVUNIF>
__device__ __forceinline__ float tc_cell(float daa, float dot, float ss, float cq, float rq2, float cd, float pd2,
                                         const float* __restrict__ cvl, const TcConsts& tc)
{
    // rq2 = c2 - 2 prior_q (per row); the table values and vfw, vlw carry the
    // -shift of the amino-acid term, so the cell is ln(daa) + (ss + cv)
    const float det = fmaf(-dot, dot, cq * cd);
    const float x = fmaf(tc.p2l, lg2_ftz(det), rq2) - pd2;
    const int ix = min(max(__float2int_rn(x), tc.ilo), tc.ihi);
    float cvm = cvl[ix * P1T_CVREP];
    if (!CVUNIF) {
        cvm = (tc.kl2 <= x) ? tc.vlw - tc.shift : cvm;
        cvm = (x <= tc.kf2) ? tc.vfw - tc.shift : cvm;
    }
    return fmaf(lg2_ftz(daa), C2_LN2, ss + cvm);
}

// Stage the column records of chunk m (32 columns) into the column ring
// (3 chunks; chunks at slot 0 also into the mirror slots 96..127)
__device__ __forceinline__ void stage_cols(float* cring, const float* __restrict__ cold, int m, int L, int lane)
{
    const int c0 = 32 * m;
    const int nc = min(32, L - c0);
    if (nc > 0) {
        const int base = c0 % P1T_CMOD;
        float* dst = cring + base * P1C_TRS;
        const float* src = cold + (long long)c0 * P1C_TRS;
        for (int i = lane; i < nc * (P1C_TRS / 4); i += 32) cp_async16(dst + 4 * i, src + 4 * i);
        if (base == 0) {
            float* mir = cring + P1T_CMOD * P1C_TRS;
            for (int i = lane; i < nc * (P1C_TRS / 4); i += 32) cp_async16(mir + 4 * i, src + 4 * i);
        }
    }
    cp_async_commit();
}

// Phase 1 with the score contractions on the tensor cores: per 32-column
// chunk the warp computes the 32 x 32 score tile with mma.sync (fragment
// layout: lane (g, q) holds rows g, g + 8 of each 16-row tile and columns
// 2q, 2q + 1 of each 8-column tile), applies the epilogue per cell, writes the
// scores into the ring, then advances the same wavefront DP as p1c_kernel.
// CVUNIF: the CV table's key range coincides with its index clamp (TcConsts)
template <bool CVUNIF>
__global__ void __launch_bounds__(P1T_WARPS * 32, 1)
p1t_kernel(P1Args a, const float* __restrict__ qbkg)
{
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cvcard = a.sc.cvcard;
    float* cvtab = smem;                                      // [cvcard][P1T_CVREP], x CV weight
    float* wb = smem + cvcard * P1T_CVREP + wid * P1T_WARP_FLOATS;
    float* ring = wb;                                         // [64 anti-diagonals][P1T_RLD] scores
    float* cring = ring + P1C_RING * P1T_RLD;                 // [P1T_CRING][P1C_TRS] column records
    float* bnd = cring + P1T_CRING * P1C_TRS;                 // [BND_FLOATS] row above the strip
    unsigned* btile = reinterpret_cast<unsigned*>(bnd + BND_FLOATS);   // [TC_TILE_WORDS] db operand tile
    unsigned long long* tbar = reinterpret_cast<unsigned long long*>(btile + TC_TILE_WORDS);
    for (int i = threadIdx.x; i < cvcard * P1T_CVREP; i += blockDim.x)
        cvtab[i] = a.cvvals[i / P1T_CVREP] * a.sc.cvswgt - a.tc.shift;
    __shared__ unsigned tmem_base;
    if (lane == 0) {
        mbar_init(tbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // query CV / SS A fragments of the current strip live in TMEM (64 columns
    // per warp; warps w, w + 4, w + 8 share lanes and take 128-column blocks)
    if (wid == 0) tmem_alloc(&tmem_base, P1T_TMEM_COLS);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const unsigned tq = tmem_base + ((unsigned)(32 * (wid & 3)) << 16) + (unsigned)((wid >> 2) * 128);
    unsigned tph = 0;   // phase parity of the tile slot's barrier
    // a tile wait that gave up: the warp issues no further tile copies and
    // waits for none, and before it exits waits (bounded) once more for the
    // copy it gave up on, so that no copy into this CTA's shared memory is in
    // flight when the CTA ends
    bool tbroken = false;
    unsigned tpend = 0;

    const long long slotw = (long long)blockIdx.x * P1T_WARPS + wid;
    const int Lmax = (int)(a.botstride / 10);
    float* bot0 = a.bot + slotw * a.botstride;
    const int Lq = a.Lq;
    const int nstrips = (Lq + 31) >> 5;
    const TcConsts tc = a.tc;
    const int g = lane >> 2, q = lane & 3;
    // this lane's CV table replica, offset so that index 0 is the table's key 0
    const float* __restrict__ cvl = cvtab + a.sc.cvshift * P1T_CVREP + (lane & (P1T_CVREP - 1));

    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.nwork) break;
        const int p = a.order[item];
        const int L = a.plen[p];
        const long long off = a.poff[p];
        const float* __restrict__ cold = a.cold + off * P1C_TRS;
        const unsigned* __restrict__ tb0 = a.tcdb + a.ttile[p] * (long long)TC_TILE_WORDS;
        const float* __restrict__ bd = a.pbkg + (long long)p * NAA;
        const int edge = corner_edge(Lq, L);
        float* botr = bot0;
        float* botw = bot0 + 5 * Lmax;
        float pbest = 0.f;
        int prow = 0x7fffffff, pcol = 0x7fffffff;

        for (int s = 0; s < nstrips; s++) {
            const int r = s * 32 + lane;
            const bool act = r < Lq;
            const float* __restrict__ qr = a.qrec + (long long)(act ? r : Lq - 1) * QR_STRIDE;
            // amino-acid A fragments of this strip, scaled for the pair and split
            // (q(a) / (0.5 (bq(a) + bd(a))), as cell_score's Qt), kept in registers
            unsigned Aaa[2][2][2][4];   // [mtile][ktile][split][reg]
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                float wk[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int k = 16 * kt + 2 * q + (e & 1) + (e >> 1) * 8;
                    wk[e] = (k < NAA) ? 0.5f * (qbkg[k] + bd[k]) : 1.f;
                }
#pragma unroll
                for (int mt = 0; mt < 2; mt++) {
                    const float4* src = reinterpret_cast<const float4*>(
                        a.qaa + ((((long long)s * 2 + mt) * 2 + kt) * 32 + lane) * 8);
                    const float4 u0 = __ldg(src), u1 = __ldg(src + 1);
                    const float v[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
                    unsigned h[8], l[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        // element e: register e / 2, k index 2q + (e & 1) + 8 (e >= 4)
                        const float x = __fdividef(v[e], wk[(e & 1) + ((e >> 2) << 1)]);
                        bf16_split(x, h[e], l[e]);
                    }
#pragma unroll
                    for (int w = 0; w < 4; w++) {
                        Aaa[mt][kt][0][w] = h[2 * w] | (h[2 * w + 1] << 16);
                        Aaa[mt][kt][1][w] = l[2 * w] | (l[2 * w + 1] << 16);
                    }
                }
            }
            // this strip's query CV / SS fragments into TMEM: column 4 idx + w holds
            // word w of fragment idx = ((mt * 2 + dot) * 2 + ktile) * 2 + split
            {
                const uint4* src = reinterpret_cast<const uint4*>(a.qa + (long long)s * TC_QA_WORDS) + lane;
#pragma unroll
                for (int blk = 0; blk < 4; blk++) {
                    unsigned v[16];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const uint4 x = __ldg(src + (4 * blk + i) * 32);
                        v[4 * i + 0] = x.x; v[4 * i + 1] = x.y; v[4 * i + 2] = x.z; v[4 * i + 3] = x.w;
                    }
                    tmem_st16(tq + 16 * blk, v);
                }
                tmem_wait_st();
            }
            // query row terms of this lane's fragment rows 32 s + 16 mt + g + 8 hh:
            // cvnorm and twice the CV log prior
            float rq[2][2][2];
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int hh = 0; hh < 2; hh++) {
                    const int rr = s * 32 + 16 * mt + g + 8 * hh;
                    const float* qx = a.qrec + (long long)min(rr, Lq - 1) * QR_STRIDE;
                    rq[mt][hh][0] = qx[QR_CN];
                    rq[mt][hh][1] = tc.c2 - 2.f * qx[QR_PRIOR];
                }
            WfLane D;
            {
                float q7[7];
#pragma unroll
                for (int i = 0; i < 7; i++) q7[i] = act ? qr[QR_TRN + i] : LOG0;
                const bool z_left = (lane == 31);
                const bool z_diag = (lane == 31 || lane == 0);
                const St5 LB = z_left ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                      : St5{0.f, qr[QR_C + 0], qr[QR_C + 1], qr[QR_C + 2], LOG0};
                const St5 DB = z_diag ? St5{0.f, 0.f, 0.f, 0.f, 0.f}
                                      : St5{0.f, qr[QR_CP + 0], qr[QR_CP + 1], qr[QR_CP + 2], LOG0};
                wf_init(D, q7, LB, DB);
            }
            const int cA = corner_a(r, Lq, edge);
            const int cB = corner_b(r, L, edge);
            float bc[5];
#pragma unroll
            for (int f = 0; f < 5; f++) {
                bc[f] = 0.f;
                D.bnxt[f] = 0.f;
                if (s > 0) {
                    if (lane < L) bc[f] = botr[f * Lmax + lane];
                    if (32 + lane < L) D.bnxt[f] = botr[f * Lmax + 32 + lane];
                }
            }
            const bool wr_bot = (lane == 31) && (s + 1 < nstrips);
            __syncwarp();
            bnd_put(bnd, lane, bc[0], bc[1], bc[2], bc[3], bc[4]);
            stage_cols(cring, cold, 0, L, lane);
            stage_cols(cring, cold, 1, L, lane);
            const int nch = (L + 31) >> 5;
            const int kend = L + 31;
            // db operand tiles T = 4m + nt stream through the slot, one tile ahead:
            // tile T + 1 loads while tile T's products and epilogue run (and
            // the first tile of a chunk during the DP stage before it)
            const int ntile = 4 * nch;
            if (lane == 0 && !tbroken) bulk_load(btile, tb0, TC_TILE_WORDS * 4, tbar);
            for (int m = 0; 32 * m < kend; m++) {
                if (m < nch) {
                    cp_async_wait_1();   // column records of chunk m have landed
                    __syncwarp();
                    // the next chunk's db operands (12 KB) towards L2 while this one is used
                    if (m + 1 < nch) {
                        const char* nx = reinterpret_cast<const char*>(tb0 + (long long)(4 * m + 4) * TC_TILE_WORDS);
#pragma unroll
                        for (int i = 0; i < 3; i++)
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(nx + (i * 32 + lane) * 128));
                    }
                    // does any row of the strip have corner cells in this chunk?
                    const bool hasc = __any_sync(FULL, cA >= 32 * m || cB < 32 * m + 32);
                    const float* cbase = cring + ((32 * m) % P1T_CMOD) * P1C_TRS;
                    // ---- score stage: 32 x 32 tile of chunk m on the tensor cores
#pragma unroll 2
                    for (int nt = 0; nt < 4; nt++) {
                        const int T = 4 * m + nt;
                        if (!tbroken && !__all_sync(FULL, mbar_wait(tbar, tph))) {
                            tbroken = true;
                            tpend = tph;
                            if (lane == 0 && a.status) atomicCAS(a.status, 0, PIPE_ERR_TIMEOUT);
                        }
                        tph ^= 1u;
                        const unsigned* bt = btile + lane * 2;
                        uint2 B[3][2][2];
#pragma unroll
                        for (int d = 0; d < 3; d++)
#pragma unroll
                            for (int kt = 0; kt < 2; kt++)
#pragma unroll
                                for (int sp = 0; sp < 2; sp++)
                                    B[d][kt][sp] = *reinterpret_cast<const uint2*>(bt + ((d * 2 + kt) * 2 + sp) * 64);
                        // slot free once every lane holds its fragments: tile T + 1 into it
                        __syncwarp();
                        if (lane == 0 && T + 1 < ntile && !tbroken) {
                            // the warp's reads of the slot before the async-proxy write
                            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                            bulk_load(btile, tb0 + (long long)(T + 1) * TC_TILE_WORDS, TC_TILE_WORDS * 4, tbar);
                        }
                        const int cl = 8 * nt + 2 * q;   // column within the chunk
                        const float* cr0 = cbase + cl * P1C_TRS;
                        const float cd[2] = {cr0[CO_CD], cr0[P1C_TRS + CO_CD]};
                        const float pd[2] = {cr0[CO_PD2], cr0[P1C_TRS + CO_PD2]};
#pragma unroll
                        for (int mt = 0; mt < 2; mt++) {
                            float acc[3][4];
#pragma unroll
                            for (int kt = 0; kt < 2; kt++) {
                                if (kt == 0) mma_bf16_z(acc[0], Aaa[mt][kt][1], B[0][kt][0].x, B[0][kt][0].y);
                                else mma_bf16(acc[0], Aaa[mt][kt][1], B[0][kt][0].x, B[0][kt][0].y);
                                mma_bf16(acc[0], Aaa[mt][kt][0], B[0][kt][1].x, B[0][kt][1].y);
                                mma_bf16(acc[0], Aaa[mt][kt][0], B[0][kt][0].x, B[0][kt][0].y);
                            }
                            unsigned Q[32];   // (dot, ktile, split) fragments of this m-tile
                            tmem_ld32(tq + 32 * mt, Q);
#pragma unroll
                            for (int d = 1; d < 3; d++)
#pragma unroll
                                for (int kt = 0; kt < 2; kt++) {
                                    const unsigned* Ah = Q + (((d - 1) * 2 + kt) * 2 + 0) * 4;
                                    const unsigned* Al = Q + (((d - 1) * 2 + kt) * 2 + 1) * 4;
                                    if (kt == 0) mma_bf16_z(acc[d], Al, B[d][kt][0].x, B[d][kt][0].y);
                                    else mma_bf16(acc[d], Al, B[d][kt][0].x, B[d][kt][0].y);
                                    mma_bf16(acc[d], Ah, B[d][kt][1].x, B[d][kt][1].y);
                                    mma_bf16(acc[d], Ah, B[d][kt][0].x, B[d][kt][0].y);
                                }
                            // epilogue: cell (row 16 mt + g + 8 hh, column 32 m + cl + e) is
                            // register 2 hh + e; its score goes to anti-diagonal row + column
                            float S[4];
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                S[i] = tc_cell<CVUNIF>(acc[0][i], acc[1][i], acc[2][i], rq[mt][i >> 1][0],
                                                       rq[mt][i >> 1][1], cd[i & 1], pd[i & 1], cvl, tc);
                            if (hasc) {
#pragma unroll
                                for (int i = 0; i < 4; i++) {
                                    const int rr = 32 * s + 16 * mt + g + 8 * (i >> 1), cc = 32 * m + cl + (i & 1);
                                    // (padding columns past L keep -inf)
                                    if (cc < L && (cc <= corner_a(rr, Lq, edge) || cc >= corner_b(rr, L, edge)))
                                        S[i] = -9.f;
                                }
                            }
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                const int row = 16 * mt + g + 8 * (i >> 1);
                                // anti-diagonal (32 m + cl + e + row) & 63
                                ring[((cl + (i & 1) + row) ^ ((m & 1) << 5)) * P1T_RLD + row] = S[i];
                            }
                        }
                    }
                }
                __syncwarp();
                // ---- DP stage: wavefront steps [32m, 32m + 32).  A full stage
                // after the first runs without bounds checks also where it passes
                // the matrix edge: the last chunk's padding columns (zero operands)
                // score -inf, so MM stays 0 there, and their other states reach
                // only cells past the edge
                const int k0 = 32 * m, k1 = min(k0 + 32, kend);
                const float* tcol = cring + ((k0 - lane + P1T_CMOD) % P1T_CMOD) * P1C_TRS;
                if (m >= 1 && k1 == k0 + 32)
                    wf_steps<false, P1T_RLD, true, 0>(D, k0, 32, lane, L, act, ring, tcol, bnd, wr_bot);
                else
                    wf_steps<true, P1T_RLD, true, 0>(D, k0, k1 - k0, lane, L, act, ring, tcol, bnd, wr_bot);
                __syncwarp();
                if (s + 1 < nstrips) bot_flush(bnd, botw, k0, L, Lmax, lane);
                __syncwarp();
                bnd_put(bnd, lane, D.bnxt[0], D.bnxt[1], D.bnxt[2], D.bnxt[3], D.bnxt[4]);
#pragma unroll
                for (int f = 0; f < 5; f++) {
                    const int cc = k0 + 64 + lane;
                    D.bnxt[f] = (s > 0 && cc < L) ? botr[f * Lmax + cc] : 0.f;
                }
                // chunk m - 1's records are no longer read: chunk m + 2 into its slots
                stage_cols(cring, cold, m + 2, L, lane);
                __syncwarp();
            }
            cp_async_wait_all();
            {
                float b = D.best;
                int rr = (D.best > 0.f) ? r : 0x7fffffff;
                int cc = (D.best > 0.f) ? D.kbest - lane : 0x7fffffff;
                if (b > pbest || (b == pbest && (rr < prow || (rr == prow && cc < pcol)))) {
                    pbest = b; prow = rr; pcol = cc;
                }
            }
            float* t = botr; botr = botw; botw = t;
            __syncwarp();
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const float ob = __shfl_xor_sync(FULL, pbest, o);
            const int orr = __shfl_xor_sync(FULL, prow, o);
            const int oc = __shfl_xor_sync(FULL, pcol, o);
            if (ob > pbest || (ob == pbest && (orr < prow || (orr == prow && oc < pcol)))) {
                pbest = ob; prow = orr; pcol = oc;
            }
        }
        if (lane == 0) {
            const unsigned xy = (pbest > 0.f) ? (((unsigned)pcol << 16) | ((unsigned)prow & 0xffffu)) : 0u;
            a.best[p] = pbest;
            a.coords[p] = xy;
        }
        __syncwarp();
    }
    if (tbroken) (void)mbar_wait(tbar, tpend);
    // every warp is past its last TMEM access: the allocating warp frees it
    tmem_fence_before();
    __syncthreads();
    if (wid == 0) {
        tmem_fence_after();
        tmem_dealloc(tmem_base, P1T_TMEM_COLS);
    }
}

// Warp butterfly sum as the reference's FinalizeDPPro reduction
// (src/libmycu/cudp/CuBatchDP_final.cu:254-260).
__device__ __forceinline__ float warp_butterfly(float v)
{
    v += __shfl_xor_sync(FULL, v, 16);
    v += __shfl_xor_sync(FULL, v, 8);
    v += __shfl_xor_sync(FULL, v, 4);
    v += __shfl_xor_sync(FULL, v, 2);
    v += __shfl_xor_sync(FULL, v, 1);
    return v;
}

// DP finalisation, one warp per candidate pair
// (src/libmycu/cudp/CuBatchDP_final.cu:170-290).
__global__ void __launch_bounds__(256) fin_kernel(FinArgs a)
{
    __shared__ float cache[8][36];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int c = blockIdx.x * 8 + wid;
    if (c >= a.ncand) return;
    const int p = a.cand_prof[c];
    const int Lq = a.Lq;
    const int L = a.plen[p];
    const signed char* bt = a.btck + a.cand_off[c];
    const float* sm = a.smat + a.cand_off[c];
    float* ch = cache[wid];
    // maximum and end cell from the traceback sweep (FP32 scores)
    const unsigned long long key = a.tbkey[c];
    const float maxsc = __uint_as_float((unsigned)(key >> 32));
    const unsigned cell = 0xffffffffu - (unsigned)(key & 0xffffffffu);
    const unsigned xx = (key != 0ull) ? (((cell & 0xffffu) << 16) | (cell >> 16)) : 0u;
    // ... which must reproduce the phase-1 maximum of this pair (exactly when
    // phase 1 used the same FP32 scores, within tol after BF16 scores)
    if (lane == 0 && a.status) {
        const float pb = a.best[p];
        const bool ok = (a.tol == 0.f) ? (maxsc == pb && xx == a.coords[p]) : (fabsf(maxsc - pb) <= a.tol * fmaxf(1.f, pb));
        if (!ok) atomicCAS(a.status, 0, 2);
    }
    int x = (int)(xx >> 16), y = (int)(xx & 0xffff);
    int psts = 0;
    int b = BT_DIAG;
    int ndx = 0;
    float sum = 0.f;
    if (lane < 4) ch[32 + lane] = 0.f;
    __syncwarp();
    // the walk is bounded by the number of cells on any monotone path
    int guard = Lq + L + 2;
    while (b != BT_STOP) {
        if (lane < 4) ch[lane] = ch[32 + lane];
        __syncwarp();
        if (lane == 0) {
            for (ndx = 4; ndx < 36;) {
                if (x < 0 || y < 0 || --guard < 0) { b = BT_STOP; break; }
                const long long qp = (long long)x * Lq + y;
                b = bt[qp];
                if (b == BT_STOP) break;
                if (b == BT_UP) { y--; continue; }
                if (b == BT_LEFT) { x--; continue; }
                ch[ndx] = sm[qp];
                if (ch[ndx] > 0.f) psts++;
                x--; y--;
                ndx++;
            }
        }
        __syncwarp();
        b = __shfl_sync(FULL, b, 0);
        ndx = __shfl_sync(FULL, ndx, 0);
        float cs = 0.f;
        if (!(ndx <= lane + 4))
            cs = ch[lane + 4] * (((ch[lane] + ch[lane + 1]) + ch[lane + 2]) + ch[lane + 3]);
        sum += warp_butterfly(cs);
        __syncwarp();
    }
    if (lane == 0) {
        sum *= 0.5f;
        sum = sum < 0.f ? -sqrtf(-sum) : sqrtf(sum);
        const float sc = maxsc + sum;
        a.score[c] = sc;
        a.psts[c] = psts;
        a.beg[c] = ((unsigned)(x + 1) << 16) | ((unsigned)(y + 1) & 0xffffu);
        a.endc[c] = xx;
        a.passed[c] = (a.scorethld < maxsc && a.scorethld < sc) ? 1 : 0;
        (void)L;
    }
}

// ---------------------------------------------------------------------------
// launchers (host)
size_t p1t_smem_bytes(int cvcard)
{
    return (size_t)(cvcard * P1T_CVREP + P1T_WARPS * P1T_WARP_FLOATS) * sizeof(float);
}

int p1t_blocks_per_sm(int cvcard, cudaError_t* err)
{
    int n = 0;
    const size_t sm = p1t_smem_bytes(cvcard);
    cudaError_t e = cudaFuncSetAttribute(p1t_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(p1t_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, p1t_kernel<true>, P1T_WARPS * 32, sm);
    if (err) *err = e;
    return n;
}

cudaError_t launch_tc_pack(const float* drec, const long long* poff, const int* plen, const long long* ttile,
                           int nprof, unsigned* tcdb, float* cold, float lok, float wss, cudaStream_t st)
{
    if (nprof <= 0) return cudaSuccess;
    tc_pack_kernel<<<nprof, 128, 0, st>>>(drec, poff, plen, ttile, tcdb, cold, lok, wss);
    return cudaGetLastError();
}

size_t p1c_smem_bytes(int cvcard)
{
    return (size_t)(cvcard * P1C_CVREP + P1C_WARPS * P1C_WARP_FLOATS) * sizeof(float);
}

int p1c_blocks_per_sm(int cvcard)
{
    int n = 0;
    const size_t sm = p1c_smem_bytes(cvcard);
    cudaFuncSetAttribute(p1c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, p1c_kernel, P1C_WARPS * 32, sm);
    return n;
}

size_t p1_smem_bytes(int cvcard)
{
    return (size_t)(cvcard * 32 + P1_WARPS * P1_WARP_FLOATS) * sizeof(float);
}

cudaError_t launch_p1(const P1Args& a, const float* qbkg, int which, int grid, cudaStream_t st)
{
    if (which == P1K_TENSOR) {
        const size_t sm = p1t_smem_bytes(a.sc.cvcard);
        if (a.tc.uniform) {
            cudaFuncSetAttribute(p1t_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            p1t_kernel<true><<<grid, P1T_WARPS * 32, sm, st>>>(a, qbkg);
        } else {
            cudaFuncSetAttribute(p1t_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            p1t_kernel<false><<<grid, P1T_WARPS * 32, sm, st>>>(a, qbkg);
        }
        return cudaGetLastError();
    }
    if (which == P1K_CHUNKED) {
        const size_t sm = p1c_smem_bytes(a.sc.cvcard);
        cudaFuncSetAttribute(p1c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        p1c_kernel<<<grid, P1C_WARPS * 32, sm, st>>>(a, qbkg);
        return cudaGetLastError();
    }
    const size_t sm = p1_smem_bytes(a.sc.cvcard);
    if (which == P1K_TRACEBACK) {
        // the score matrices first (their own work counter, a.counter[1]),
        // then the sweep over them
        const size_t sms = (size_t)(a.sc.cvcard * P1TC_CVREP + P2S_WARPS * P2S_WARP_FLOATS) * sizeof(float);
        cudaError_t e = cudaFuncSetAttribute(p2s_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms);
        if (e != cudaSuccess) return e;
        int occ = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p2s_kernel, P2S_WARPS * 32, sms)) != cudaSuccess)
            return e;
        int dev = 0, nsm = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        const long long nit = (long long)a.nwork * ((a.Lq + 31) / 32);
        const int gs = (int)std::min<long long>((long long)std::max(occ, 1) * nsm, (nit + P2S_WARPS - 1) / P2S_WARPS);
        p2s_kernel<<<gs, P2S_WARPS * 32, sms, st>>>(a, qbkg);
        const size_t smt = (size_t)P1TC_WARPS * P1TC_WARP_FLOATS * sizeof(float);
        if ((e = cudaFuncSetAttribute(p1tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smt)) != cudaSuccess)
            return e;
        p1tc_kernel<<<grid, P1TC_WARPS * 32, smt, st>>>(a, qbkg);
    } else {
        cudaFuncSetAttribute(p1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        p1_kernel<<<grid, P1_WARPS * 32, sm, st>>>(a, qbkg);
    }
    return cudaGetLastError();
}

int p1_blocks_per_sm(int cvcard)
{
    int n = 0;
    const size_t sm = p1_smem_bytes(cvcard);
    cudaFuncSetAttribute(p1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, p1_kernel, P1_WARPS * 32, sm);
    return n > 0 ? n : 1;
}

cudaError_t launch_fin(const FinArgs& a, cudaStream_t st)
{
    if (a.ncand <= 0) return cudaSuccess;
    const int grid = (a.ncand + 7) / 8;
    fin_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace c2
