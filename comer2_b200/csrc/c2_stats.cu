// c2_stats.cu -- alignment statistics of the pairs that pass the DP stage,
// one CTA of 32 x 21 threads per pair (threadIdx.y = unscaled score
// -10..10, threadIdx.x = one of the 32 scaled scores of that unit), the
// layout of the reference's CalcStatParamsDynPlmProfile
// (src/libmycu/cuss/CuBatchSS_dynplm.cu:193-430).  The reference spreads
// this over five dynamic-parallelism launches per pair; here one kernel
// computes, per pair:
//  * the histogram of rint(32 s) over the pair's score matrix (cells whose
//    query or db residue is 'X' skipped when X_UNINF) in shared memory
//    (_dynplm.cu:80-183);
//  * probabilities, expected score, score range, lambda by Newton-Raphson
//    with bisection, relative entropy and K (_expected.cuh, _minmax.cuh,
//    _lambda.cuh, _entropy.cuh, _K.cuh);
//  * the SS18 E-value: NN-predicted EVD location and scale, the p-value of
//    the score combined with the NBD p-value of the positive-score count by
//    the empirical Brown's method (_SS18.cuh, _NN.cuh, cusf/).
#include "c2_device.cuh"
#include "c2_stats.cuh"

namespace c2 {

#define FULL 0xffffffffu
constexpr int NDS = 21, SCF = 32, SMIN = -320, NSCALED = 641;
constexpr float LOG_SP_MIN = -8.7336545e+01f, LOG_SP_MAX = 8.8722839e+01f;
constexpr float LN1K = 6.90775527898213681510242167860f;
constexpr float MACHEPF = 5.9604644775390625e-8f, BIGSPNUM = 16777216.0f;

__device__ __forceinline__ float wsum(float v)
{
    v += __shfl_down_sync(FULL, v, 16);
    v += __shfl_down_sync(FULL, v, 8);
    v += __shfl_down_sync(FULL, v, 4);
    v += __shfl_down_sync(FULL, v, 2);
    v += __shfl_down_sync(FULL, v, 1);
    return v;
}

// Two-level sums over the 21 x 32 block (each warp's butterfly, then the 21
// warp totals by warp 0); results valid in every thread.  Calls alternate
// between two halves of the scratch, so no trailing barrier is needed: a
// half is rewritten two calls later, after every thread has passed the first
// barrier of the call in between (and so has read this call's result).
struct BlockSums {
    float2 t[2][32];
    float2 r[2];
};

__device__ __forceinline__ float block_sum(float v, BlockSums& S, int& ph)
{
    v = wsum(v);
    if (threadIdx.x == 0) S.t[ph][threadIdx.y].x = v;
    __syncthreads();
    if (threadIdx.y == 0) {
        float u = threadIdx.x < NDS ? S.t[ph][threadIdx.x].x : 0.f;
        u = wsum(u);
        if (threadIdx.x == 0) S.r[ph].x = u;
    }
    __syncthreads();
    const float r = S.r[ph].x;
    ph ^= 1;
    return r;
}

// two sums in one pass, each in block_sum's order
__device__ __forceinline__ float2 block_sum2(float a, float b, BlockSums& S, int& ph)
{
    a = wsum(a);
    b = wsum(b);
    if (threadIdx.x == 0) S.t[ph][threadIdx.y] = make_float2(a, b);
    __syncthreads();
    if (threadIdx.y == 0) {
        float2 u = threadIdx.x < NDS ? S.t[ph][threadIdx.x] : make_float2(0.f, 0.f);
        u.x = wsum(u.x);
        u.y = wsum(u.y);
        if (threadIdx.x == 0) S.r[ph] = u;
    }
    __syncthreads();
    const float2 r = S.r[ph];
    ph ^= 1;
    return r;
}

// ---- special functions (Cephes incbet / igam / igamc of S. L. Moshier,
// in logarithmic form as the reference's cusf functions evaluate them)
__device__ float betacf1(float a, float b, float x)
{
    float k1 = a, k2 = a + b, k3 = a, k4 = a + 1.f, k5 = 1.f, k6 = b - 1.f, k7 = a + 1.f, k8 = a + 2.f;
    float pkm2 = 0.f, qkm2 = 1.f, pkm1 = 1.f, qkm1 = 1.f, ans = 1.f, r = 0.f, t, xk, pk, qk;
    for (int n = 0; n < 100; n++) {
        xk = -__fdividef(x * k1 * k2, k3 * k4);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        xk = __fdividef(x * k5 * k6, k7 * k8);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (qk != 0.f) r = __fdividef(pk, qk);
        if (r != 0.f) { t = fabsf(__fdividef(ans - r, r)); ans = r; } else t = 1.f;
        if (t < MACHEPF) break;
        k1 += 1.f; k2 += 1.f; k3 += 2.f; k4 += 2.f; k5 += 1.f; k6 -= 1.f; k7 += 2.f; k8 += 2.f;
        if ((fabsf(qk) + fabsf(pk)) > BIGSPNUM) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
        if ((fabsf(qk) < MACHEPF) || (fabsf(pk) < MACHEPF)) { pkm2 *= BIGSPNUM; pkm1 *= BIGSPNUM; qkm2 *= BIGSPNUM; qkm1 *= BIGSPNUM; }
    }
    return ans;
}

__device__ float betacf2(float a, float b, float x)
{
    float k1 = a, k2 = b - 1.f, k3 = a, k4 = a + 1.f, k5 = 1.f, k6 = a + b, k7 = a + 1.f, k8 = a + 2.f;
    float pkm2 = 0.f, qkm2 = 1.f, pkm1 = 1.f, qkm1 = 1.f, ans = 1.f, r = 0.f, t, xk, pk, qk;
    const float z = __fdividef(x, 1.f - x);
    for (int n = 0; n < 100; n++) {
        xk = -__fdividef(z * k1 * k2, k3 * k4);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        xk = __fdividef(z * k5 * k6, k7 * k8);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (qk != 0.f) r = __fdividef(pk, qk);
        if (r != 0.f) { t = fabsf(__fdividef(ans - r, r)); ans = r; } else t = 1.f;
        if (t < MACHEPF) break;
        k1 += 1.f; k2 -= 1.f; k3 += 2.f; k4 += 2.f; k5 += 1.f; k6 += 1.f; k7 += 2.f; k8 += 2.f;
        if ((fabsf(qk) + fabsf(pk)) > BIGSPNUM) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
        if ((fabsf(qk) < MACHEPF) || (fabsf(pk) < MACHEPF)) { pkm2 *= BIGSPNUM; pkm1 *= BIGSPNUM; qkm2 *= BIGSPNUM; qkm1 *= BIGSPNUM; }
    }
    return ans;
}

__device__ float betaps(float a, float b, float x)
{
    float y = a * __logf(x) + (b - 1.f) * __logf(1.f - x) - __logf(a);
    y -= lgammaf(a) + lgammaf(b);
    y += lgammaf(a + b);
    const float t = __fdividef(x, 1.f - x);
    float s = 0.f, u = 1.f;
    for (int it = 0; it < 1000; it++) {
        b -= 1.f;
        if (b == 0.f) break;
        a += 1.f;
        u *= __fdividef(t * b, a);
        s += u;
        if (!(fabsf(u) > MACHEPF)) break;
    }
    return y + __logf(1.f + s);
}

__device__ float lbetainc_helper(float a, float b, float x)
{
    float t = 1.f - x, ans;
    if (b > 10.f && fabsf(__fdividef(b * x, a)) < 0.3f) return betaps(a, b, x);
    ans = x * __fdividef(a + b - 2.f, a - 1.f);
    if (ans < 1.f) { ans = betacf1(a, b, x); t = b * __logf(t); }
    else { ans = betacf2(a, b, x); t = (b - 1.f) * __logf(t); }
    t += a * __logf(x) + lgammaf(a + b) - lgammaf(a) - lgammaf(b);
    t += __logf(__fdividef(ans, a));
    return t;
}

__device__ float lbetainc(float aa, float bb, float xx)
{
    if (xx <= 0.f || xx >= 1.f) {
        if (xx == 0.f) return -999.f;
        if (xx == 1.f) return 0.f;
        return 999.f;
    }
    if (aa <= 0.f) return 999.f;
    if (aa <= 1.f) {
        float ans = lbetainc_helper(aa + 1.f, bb, xx);
        ans = ans > LOG_SP_MIN ? __expf(ans) : 0.f;
        const float t = aa * __logf(xx) + bb * __logf(1.f - xx) + lgammaf(aa + bb) - lgammaf(aa + 1.f) - lgammaf(bb);
        if (t > LOG_SP_MIN) ans += __expf(t);
        return ans != 0.f ? __logf(ans) : -999.f;
    }
    return lbetainc_helper(aa, bb, xx);
}

__device__ float lgammainc_P(float a, float x);

__device__ float lgammainc_Q(float a, float x)
{
    if (x <= 0.f || a <= 0.f) return 0.f;
    if (x < 1.f || x < a) {
        float ans = lgammainc_P(a, x);
        ans = ans > LOG_SP_MIN ? __expf(ans) : 0.f;
        return ans < 1.f ? __logf(1.f - ans) : -999.f;
    }
    const float ax = a * __logf(x) - x - lgammaf(a);
    float y = 1.f - a, z = x + y + 1.f, c = 0.f;
    float pkm2 = 1.f, qkm2 = x, pkm1 = x + 1.f, qkm1 = z * x;
    float ans = __fdividef(pkm1, qkm1), t, yc, pk, qk, r;
    for (int it = 0; it < 1000; it++) {
        c += 1.f; y += 1.f; z += 2.f;
        yc = y * c;
        pk = pkm1 * z - pkm2 * yc;
        qk = qkm1 * z - qkm2 * yc;
        if (qk != 0.f) { r = __fdividef(pk, qk); t = fabsf(__fdividef(ans - r, r)); ans = r; } else t = 1.f;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (fabsf(pk) > BIGSPNUM) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
        if (!(t > MACHEPF)) break;
    }
    return __logf(ans) + ax;
}

__device__ float lgammainc_P(float a, float x)
{
    if (x <= 0.f || a <= 0.f) return -999.f;
    if (x > 1.f && x > a) {
        // the complement, evaluated directly (no recursion on the device)
        const float ax = a * __logf(x) - x - lgammaf(a);
        float y = 1.f - a, z = x + y + 1.f, c = 0.f;
        float pkm2 = 1.f, qkm2 = x, pkm1 = x + 1.f, qkm1 = z * x;
        float ans = __fdividef(pkm1, qkm1), t, yc, pk, qk, r;
        for (int it = 0; it < 1000; it++) {
            c += 1.f; y += 1.f; z += 2.f;
            yc = y * c;
            pk = pkm1 * z - pkm2 * yc;
            qk = qkm1 * z - qkm2 * yc;
            if (qk != 0.f) { r = __fdividef(pk, qk); t = fabsf(__fdividef(ans - r, r)); ans = r; } else t = 1.f;
            pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
            if (fabsf(pk) > BIGSPNUM) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
            if (!(t > MACHEPF)) break;
        }
        float q = __logf(ans) + ax;
        q = q > LOG_SP_MIN ? __expf(q) : 0.f;
        return q < 1.f ? __logf(1.f - q) : -999.f;
    }
    const float ax = a * __logf(x) - x - lgammaf(a);
    float r = a, c = 1.f, ans = 1.f;
    for (int it = 0; it < 1000; it++) {
        r += 1.f;
        c *= __fdividef(x, r);
        ans += c;
        if (!(__fdividef(c, ans) > MACHEPF)) break;
    }
    return __logf(ans) + ax - __logf(a);
}

// ---- SS18 model (src/libmycu/cuss/CuBatchSS_SS18.cuh:104-459, _NN.cuh)
__device__ __forceinline__ float nn_act(float x) { return __fdividef(2.f, 1.f + __expf(-x)) - 1.f; }

__device__ float nn4(const float* w, const float in[4], float factor)
{
    float h[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
        float s = w[t * 5] + in[0] * w[t * 5 + 1] + in[1] * w[t * 5 + 2] + in[2] * w[t * 5 + 3] + in[3] * w[t * 5 + 4];
        h[t] = nn_act(s) * w[20 + t + 1];
    }
    const float o = w[20] + h[0] + h[1] + h[2] + h[3];
    return nn_act(o) * factor;
}

__device__ void predict_evd(const StatsArgs& a, int nq, int nd, float qeno, float deno, float lambda,
                            float* mu, float* scale)
{
    const float* w = a.nnw;
    float q1 = (float)nq, d1 = (float)nd, qe = qeno, de = deno;
    if (qe < de) { float t = qe; qe = de; de = t; t = q1; q1 = d1; d1 = t; }
    else if (qe == de && q1 < d1) { float t = q1; q1 = d1; d1 = t; }
    const float ie[4] = {0.05f * qe, __fdividef(__logf(q1), LN1K), 0.05f * de, __fdividef(__logf(d1), LN1K)};
    float emu = nn4(w, ie, 30.f);
    float lr = __fdividef(rintf(lambda * 10.f), 10.f);
    if (lr <= 0.f) lr = 0.1f;
    if (10.f < lr) lr = 10.f;
    float l1 = (float)nq, l2 = (float)nd;
    if (l1 < l2) { float t = l1; l1 = l2; l2 = t; }
    const float il[4] = {0.2f * lr, __fdividef(__logf(l1), LN1K), __fdividef(__logf(l2), LN1K), 0.f};
    float lmu = nn4(w + 25, il, 30.f);
    float lsc = nn4(w + 50, il, 5.f);
    const float* adj = w + 75;
    if (a.ssemodel == 2) adj = w + 84;
    if (emu < 3.f) emu = 3.f;
    if (lmu < 3.f) lmu = 3.f;
    if (lsc < 0.1f) lsc = 0.1f;
    lsc = adj[6] * (__expf(lsc) - 1.f);
    if (lsc < 0.1f) lsc = 0.1f;
    if (5.f < lsc) lsc = 5.f;
    float scaleE = adj[4] * emu + adj[5];
    if (scaleE < 0.1f) scaleE = 0.1f;
    if (5.f < scaleE) scaleE = 5.f;
    emu = adj[0] * emu + adj[1];
    lmu = adj[2] * lmu + adj[3];
    float alpha = adj[7], ibeta = adj[8];
    if (0.f < lambda) {
        const float m = fminf(10.f, __fdividef(1.f, lambda));
        alpha -= alpha * 0.1f * m;
        ibeta += (1.f - ibeta) * 0.1f * m;
    }
    *mu = alpha * emu + (1.f - alpha) * lmu;
    *scale = (1.f - ibeta) * scaleE + ibeta * lsc;
}

__device__ float evalue_ss18(const StatsArgs& a, int nq, int nd, float score, float psts, float K,
                             float mu, float scale)
{
    if (mu <= 0.f || scale <= 0.f) return __logf(a.expgK * a.searchspace) - a.expglambda * score;
    const float l1l2 = (float)((unsigned)nq * (unsigned)nd);
    const float Kref = a.refK;
    float lkmn = __fdividef(mu, scale);
    if (K > Kref && 0.f < K && K < 1.f && 0.f < Kref && Kref < 1.f) lkmn += __logf(__fdividef(K, Kref));
    float lexp = lkmn - __fdividef(score, scale);
    if (a.ssemodel == 2) lexp += -9.210340372f;
    float lp = lexp;
    if (-4.605170186f <= lexp) {
        if (LOG_SP_MAX - 3.f < lexp) lp = 0.f;
        else {
            lp = __expf(lexp);
            if (LOG_SP_MAX - 3.f < lp) lp = 0.f;
            else lp = __logf(1.f - __expf(-lp));
        }
    }
    const float pn = rintf(__fdividef(100000.f * psts, __powf(fmaxf(l1l2, 625.f), 1.5f)));
    const float lpp = lbetainc(pn + 1.f, 0.1f, 0.757213f);
    lp = lgammainc_Q(1.346206f, __fdividef(-lp - lpp, 1.485656f));
    lexp = lp;
    if (-4.605170186f <= lp) {
        const float p = __expf(lp);
        lexp = 77.f;
        if (p < 1.f) lexp = __logf(-__logf(1.f - p));
    }
    lexp += __logf(__fdividef(a.searchspace, l1l2));
    return lexp;
}

// ---- the per-pair statistics kernel
__global__ void __launch_bounds__(SCF * NDS, 2) stats_kernel(StatsArgs a)
{
    __shared__ float counts[NSCALED + 31];
    __shared__ float P[NDS][SCF + 1];
    __shared__ float pu[NDS];
    __shared__ BlockSums bsm;
    int ph = 0;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * SCF + tx;
    const int pi = blockIdx.x;              // passed-pair index
    const int c = a.p2_cand[pi];            // candidate index
    const int p = a.cand_prof[c];
    const int Lq = a.Lq, L = a.plen[p];
    const long long off = a.poff[p];
    const float* __restrict__ sm = a.smat + a.cand_off[c];
    __shared__ unsigned hist[NSCALED];
    for (int k = tid; k < NSCALED + 31; k += SCF * NDS) counts[k] = 0.f;
    for (int k = tid; k < NSCALED; k += SCF * NDS) hist[k] = 0u;
    __syncthreads();
    // histogram of rint(32 s), s clamped to [-10, 10]: warp ty takes db
    // columns, its lanes the query rows of a column (coalesced reads), eight
    // rows per lane loaded before their counts are added (loads in flight)
    for (int x = ty; x < L; x += NDS) {
        if (a.xuninf && a.daa[off + x] == 'X') continue;
        const float* __restrict__ col = sm + (long long)x * Lq;
        for (int y0 = tx; y0 < Lq; y0 += 8 * SCF) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int y = y0 + u * SCF;
                v[u] = y < Lq ? col[y] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int y = y0 + u * SCF;
                if (y >= Lq || (a.xuninf && a.qaa[y] == 'X')) continue;
                const float s = v[u] < -10.f ? -10.f : (v[u] > 10.f ? 10.f : v[u]);
                atomicAdd(&hist[(int)rintf(s * SCF) - SMIN], 1u);
            }
        }
    }
    __syncthreads();
    for (int k = tid; k < NSCALED; k += SCF * NDS) counts[k] = (float)hist[k];
    __syncthreads();
    // probability layout: row ty holds the scaled scores of unscaled score ty-10
    const int u = ty - 10;
    int left = u * SCF - (SCF >> 1) - SMIN, right = u * SCF + (SCF >> 1) - SMIN;
    if (u <= 0) { left++; if (left < 0) left = 0; }
    if (0 <= u) { right--; if (NSCALED - 1 < right) right = NSCALED - 1; }
    float cnt = (tx + left <= right) ? counts[left + tx] : 0.f;
    P[ty][tx] = cnt;
    {
        const float rs = wsum(cnt);
        if (tx == 0) pu[ty] = rs;
    }
    __syncthreads();
    const float total = block_sum(cnt, bsm, ph);
    if (ty == 0 && tx < NDS) pu[tx] = __fdividef(pu[tx], total);
    P[ty][tx] = __fdividef(P[ty][tx], total);
    __syncthreads();
    const float sc = (float)(left + tx + SMIN);
    float E = block_sum(sc * P[ty][tx], bsm, ph);
    // score range over nonzero probabilities (including 0)
    float vmin = P[ty][tx] != 0.f ? sc : 0.f, vmax = vmin;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        vmin = fminf(vmin, __shfl_down_sync(FULL, vmin, o));
        vmax = fmaxf(vmax, __shfl_down_sync(FULL, vmax, o));
    }
    __shared__ float mm2[2][NDS];
    if (tx == 0) { mm2[0][ty] = vmin; mm2[1][ty] = vmax; }
    __syncthreads();
    __shared__ float smin, smax;
    if (ty == 0 && tx == 0) {
        float a0 = 0.f, a1 = 0.f;
        for (int y = 0; y < NDS; y++) { a0 = fminf(a0, mm2[0][y]); a1 = fmaxf(a1, mm2[1][y]); }
        smin = a0; smax = a1;
    }
    __syncthreads();
    const float mn = smin, mx = smax;
    // lambda: Newton-Raphson with bisection (CuBatchSS_lambda.cuh:136-262)
    float lambda = -1.f;
    if (!(0.f <= E || mx <= 0.f)) {
        auto feq = [&](float x, float* dfo) {
            float lf = 0.f, ldf = 0.f;
            if (mn <= sc && sc <= mx) {
                const float s2 = sc - mx;
                const float yy = x * s2;
                if (LOG_SP_MIN < yy) { lf = __expf(yy) * P[ty][tx]; ldf = lf * s2; }
            }
            float f, df = 0.f;
            if (dfo) {
                const float2 fd = block_sum2(lf, ldf, bsm, ph);
                f = fd.x;
                df = fd.y;
            } else {
                f = block_sum(lf, bsm, ph);
            }
            float xx = x * -mx;
            if (LOG_SP_MIN < xx) { xx = __expf(xx); f -= xx; df += xx * mx; }
            if (dfo) *dfo = df;
            return f;
        };
        const float x1 = 1.0e-5f, x2 = 10.0f;
        float fl = feq(x1, nullptr);
        float f = feq(x2, nullptr);
        if (!((fl > 0.f && f > 0.f) || (fl < 0.f && f < 0.f))) {
            float xl, xh;
            if (fl < 0.f) { xl = x1; xh = x2; } else { xh = x1; xl = x2; }
            float rts = 0.5f * (x1 + x2), dxold = fabsf(x2 - x1), dx = dxold, df;
            f = feq(rts, &df);
            int n, flag = 0;
            for (n = 0; n < 32; n++) {
                if (((((rts - xh) * df - f) * ((rts - xl) * df - f)) > 0.f) || (fabsf(2.f * f) > fabsf(dxold * df))) {
                    dxold = dx; dx = 0.5f * (xh - xl); rts = xl + dx;
                    if (xl == rts) flag = 1;
                } else {
                    dxold = dx; dx = __fdividef(f, df);
                    const float t0 = rts; rts -= dx;
                    if (t0 == rts) flag = 1;
                }
                if (fabsf(dx) < 1.0e-4f) flag = 1;
                if (flag) break;
                f = feq(rts, &df);
                if (f < 0.f) xl = rts; else xh = rts;
            }
            lambda = (n == 32) ? -1.f : rts;
        }
    }
    // relative entropy
    float H = -1.f;
    if (lambda > 0.f) {
        float v = 0.f;
        if (mn <= sc && sc <= mx) {
            const float yy = lambda * sc;
            if (LOG_SP_MIN < yy && yy < LOG_SP_MAX - 3.f) v = __expf(yy) * yy * P[ty][tx];
        }
        H = block_sum(v, bsm, ph);
    }
    lambda *= SCF;  // rescaled even when the root search failed (-1 -> -32)
    E = __fdividef(E, SCF);
    __syncthreads();
    if (ty == 10) P[10][tx] = 1.f;
    __syncthreads();
    int minu = 0, maxu = 0;
    for (int y = 0; y < NDS; y++)
        if (pu[y] != 0.f) { const int s = y - 10; minu = min(minu, s); maxu = max(maxu, s); }
    // K (CuBatchSS_K.cuh:60-318); each length's convolution reads the previous length's values
    float K = -1.f;
    if (!(0.f <= E || lambda <= 0.f || H <= 0.f)) {
        if (minu == -1 && maxu == 1) {
            const float mnp = pu[-1 + 10], mxp = pu[1 + 10];
            K = __fdividef((mnp - mxp) * (mnp - mxp), mnp);
        } else if (minu == -1 || maxu == 1) {
            if (maxu != 1) K = __fdividef(lambda, H) * (1.f - __expf(-lambda)) * (E * E);
            else K = __fdividef(H, lambda) * (1.f - __expf(-lambda));
        } else {
            float sigma = 0.f, Pj = 1.f;
            int minscore = minu, maxscore = maxu;
            const int range = maxu - minu + 1;
            const int isc = left + tx + SMIN;
            for (int j = 1; j <= 32 && 1.0e-4f < Pj; j++) {
                float pji = 0.f, pj = 0.f;
                if (minscore <= isc && isc <= maxscore && -32 <= isc && isc <= 32) {
                    const float etols = (isc < 0) ? lambda * (float)isc : 0.f;
                    if (LOG_SP_MIN < etols) {
                        const int lo = (maxscore - isc < range) ? maxu - (maxscore - isc) : minu;
                        const int hi = (isc - minscore < range) ? minu + (isc - minscore) : maxu;
                        for (int i = lo; i <= hi; i++) {
                            int yy = ty, xx = tx - i;
                            if (32 <= xx) { xx -= 32; if (yy + 1 < NDS) yy++; else continue; }
                            else if (xx < 0) { xx += 32; if (0 < yy) yy--; else continue; }
                            pji += P[yy][xx] * pu[i + 10];
                        }
                        pj = pji * __expf(etols);
                    }
                }
                __syncthreads();
                P[ty][tx] = pji;
                Pj = block_sum(pj, bsm, ph);
                sigma += __fdividef(Pj, (float)j);
                minscore += minu;
                maxscore += maxu;
            }
            K = __fdividef(lambda * __expf(-2.f * sigma), H * (1.f - __expf(-lambda)));
        }
    }
    if (tx == 0 && ty == 0) {
        const float score = a.fscore[c];
        const float psts = (float)a.fpsts[c];
        float* o = a.out + (size_t)pi * STATS_NOUT;
        o[ST_MIN] = (float)minu; o[ST_MAX] = (float)maxu; o[ST_E] = E; o[ST_H] = H;
        o[ST_LAMBDA] = lambda; o[ST_K] = K;
        o[ST_LAMBDA_EST] = 0.f < lambda ? lambda * __fdividef(a.expglambda, a.reflambda) : -1.f;
        o[ST_K_EST] = 0.f < K ? K * __fdividef(a.expgK, a.refK) : -1.f;
        const float l1l2 = (float)((unsigned)Lq * (unsigned)L);
        o[ST_LOGEPA] = (lambda <= 0.f || K <= 0.f) ? __logf(a.refK * l1l2) - a.reflambda * score
                                                   : __logf(K * l1l2) - lambda * score;
        if (a.ssemodel == 0) {
            // observed-statistics model: the expected gapped lambda and K over
            // the search space (CalcSignificanceObsDynPlmProfile,
            // src/libmycu/cuss/CuBatchSS_dynplm.cu:594-676; CalculateEvalueObs,
            // CuBatchSS_SS18.cuh:372-384)
            o[ST_MU] = 0.f; o[ST_SCALE] = 0.f;
            o[ST_LOGE] = __logf(a.expgK * a.searchspace) - a.expglambda * score;
        } else {
            float mu, scale;
            predict_evd(a, Lq, L, a.qeno, a.peno[p], lambda, &mu, &scale);
            o[ST_MU] = mu; o[ST_SCALE] = scale;
            o[ST_LOGE] = evalue_ss18(a, Lq, L, score, psts, K, mu, scale);
        }
    }
}

cudaError_t launch_stats(const StatsArgs& a, cudaStream_t st)
{
    if (a.npass <= 0) return cudaSuccess;
    stats_kernel<<<a.npass, dim3(SCF, NDS), 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace c2
