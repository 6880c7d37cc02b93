// c2_host.cu -- C ABI of the B200 COMER2 search hot path (host side).
//
// Replaces the reference's CuBatchProcessing / CuDeviceMemory host logic
// (src/libmycu/cupro/CuBatchProcessing.cu:229-694, CuDeviceMemory.cu) for the
// stages built here.  All state is per handle; nothing lives in __constant__
// memory, so handles on the same device are independent.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/comer2_b200.h"
#include "c2_device.cuh"

namespace c2 {
size_t p1_smem_bytes(int cvcard);
cudaError_t launch_p1(const P1Args& a, const float* qbkg, bool tb, int grid, cudaStream_t st);
int p1_blocks_per_sm(int cvcard);
cudaError_t launch_fin(const FinArgs& a, cudaStream_t st);
}  // namespace c2

using namespace c2;

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t cnt) {
        if (cnt <= n && p) return cudaSuccess;
        release();
        if (cnt == 0) cnt = 1;
        cudaError_t e = cudaMalloc((void**)&p, cnt * sizeof(T));
        if (e == cudaSuccess) n = cnt;
        return e;
    }
};

struct c2_handle {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream in use
    cudaStream_t own_stream = nullptr;  // the handle's own stream
    std::string err;
    uint64_t launches = 0;
    int nsm = 0;
    int grid = 0;
    // parameters
    c2_params prm{};
    std::vector<float> ssss, cvkeys, cvvals, nnw;
    ScoreConsts sc{};
    DevBuf<float> d_ssss, d_cvvals, d_nnw;
    DevBuf<int> d_status;
    // database
    int nprof = 0;
    int64_t npos = 0;
    uint64_t total_pos = 0, total_prof = 0;
    int Lmax = 0;
    std::vector<int32_t> h_plen;
    std::vector<int64_t> h_poff;
    DevBuf<float> d_drec, d_pbkg;
    DevBuf<int> d_plen, d_order;
    DevBuf<long long> d_poff;
    // query
    int Lq = 0;
    float qeno = 0.f;
    std::vector<float> h_qrec;
    DevBuf<float> d_qrec, d_qbkg;
    float scorethld = 0.f, logevthld = 0.f;
    unsigned long long searchspace = 0, deltalen = 0;
    // phase 1
    DevBuf<float> d_best;
    DevBuf<unsigned> d_coords;
    DevBuf<int> d_counter;
    DevBuf<float> d_bot;
    long long botstride = 0;
    // finalisation
    int ncand = 0;
    std::vector<int> h_cand;
    std::vector<long long> h_cand_off;
    DevBuf<int> d_cand_prof;
    DevBuf<long long> d_cand_off;
    DevBuf<signed char> d_btck;
    DevBuf<float> d_smat;
    DevBuf<float> d_fscore;
    DevBuf<int> d_fpsts, d_fpassed;
    DevBuf<unsigned> d_fbeg, d_fend;
};

static c2_status fail(c2_handle* h, c2_status st, const char* fmt, ...)
{
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return st;
}

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(h, C2_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                            \
    } while (0)

// Context-vector constants exactly as _TCTXVECT computes them in float
// (src/libpro/srcpro/TCTXVECT.cpp:26-54).
static void cv_constants(float* lokappa0, float* pownu0, float* cterm)
{
    const int dim = NCV;
    const float kappa0 = 0.1f;
    const float nu0 = (float)dim;
    float lo = 1.f / kappa0;
    float pw = -0.5f * (nu0 + 2.f);
    float ct = (0.5f * dim + pw) * (logf(kappa0) - logf(kappa0 + 2.f));
    float sum = 0.0f;
    for (int ii = 1; ii <= dim; ii++) sum += logf(nu0 + 1.0f - ii) - 0.69314718055994530941723212146f;
    ct += sum;
    *lokappa0 = lo;
    *pownu0 = pw;
    *cterm = ct;
}

static inline float hmax(float a, float b) { return a < b ? b : a; }

// ---------------------------------------------------------------------------
extern "C" c2_status c2_create(int device, const c2_params* p, c2_handle** out)
{
    if (!out || !p) return C2_ERR_ARG;
    *out = nullptr;
    if (!p->ssss || p->ssss_card <= 0 || p->ssss_card > MAX_SSSS_CARD || !p->cvs2s_keys ||
        !p->cvs2s_values || p->cvs2s_card <= 1 || p->cvs2s_card > MAX_CVCARD || p->cvs2s_shift < 0)
        return C2_ERR_ARG;
    if (p->ssswgt <= 0.f || p->cvswgt <= 0.f) return C2_ERR_ARG;  // SS and CV terms both in use
    c2_handle* h = new c2_handle();
    h->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete h;
        return C2_ERR_CUDA;
    }
    h->prm = *p;
    h->ssss.assign(p->ssss, p->ssss + (size_t)p->ssss_card * p->ssss_card);
    h->cvkeys.assign(p->cvs2s_keys, p->cvs2s_keys + p->cvs2s_card);
    h->cvvals.assign(p->cvs2s_values, p->cvs2s_values + p->cvs2s_card);
    if (p->sse_nn_weights && p->n_sse_nn_weights > 0)
        h->nnw.assign(p->sse_nn_weights, p->sse_nn_weights + p->n_sse_nn_weights);
    h->prm.ssss = nullptr;
    h->prm.cvs2s_keys = h->prm.cvs2s_values = h->prm.sse_nn_weights = nullptr;
    ScoreConsts& sc = h->sc;
    sc.ssswgt = p->ssswgt;
    sc.cvswgt = p->cvswgt;
    sc.shift = p->mapaln ? 0.002f : 0.0003f;  // CuBatchScoreMatrix_Init.cuh:14-15
    cv_constants(&sc.lokappa0, &sc.pownu0, &sc.cterm);
    sc.cvkey_first = h->cvkeys.front();
    sc.cvkey_last = h->cvkeys.back();
    sc.cvval_first = h->cvvals.front();
    sc.cvval_last = h->cvvals.back();
    sc.cvcard = p->cvs2s_card;
    sc.cvshift = p->cvs2s_shift;
    sc.ssss_card = p->ssss_card;
    c2_status st = C2_OK;
    do {
        if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) { st = C2_ERR_CUDA; break; }
        h->stream = h->own_stream;
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { st = C2_ERR_CUDA; break; }
        h->nsm = prop.multiProcessorCount;
        h->grid = h->nsm * p1_blocks_per_sm(sc.cvcard);
        if (h->d_ssss.ensure(h->ssss.size()) || h->d_cvvals.ensure(h->cvvals.size()) ||
            h->d_status.ensure(1) || h->d_counter.ensure(4)) { st = C2_ERR_NOMEM; break; }
        if (cudaMemcpy(h->d_ssss.p, h->ssss.data(), h->ssss.size() * 4, cudaMemcpyHostToDevice) ||
            cudaMemcpy(h->d_cvvals.p, h->cvvals.data(), h->cvvals.size() * 4, cudaMemcpyHostToDevice) ||
            cudaMemset(h->d_status.p, 0, sizeof(int))) { st = C2_ERR_CUDA; break; }
        if (!h->nnw.empty()) {
            if (h->d_nnw.ensure(h->nnw.size()) ||
                cudaMemcpy(h->d_nnw.p, h->nnw.data(), h->nnw.size() * 4, cudaMemcpyHostToDevice)) { st = C2_ERR_CUDA; break; }
        }
    } while (0);
    if (st != C2_OK) {
        if (h->own_stream) cudaStreamDestroy(h->own_stream);
        delete h;
        return st;
    }
    *out = h;
    return C2_OK;
}

extern "C" c2_status c2_destroy(c2_handle* h)
{
    if (!h) return C2_ERR_ARG;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return C2_OK;
}

extern "C" c2_status c2_last_error(const c2_handle* h, char* buf, size_t n)
{
    if (!h || !buf || n == 0) return C2_ERR_ARG;
    snprintf(buf, n, "%s", h->err.c_str());
    return C2_OK;
}

static c2_status check_profiles(c2_handle* h, const c2_profiles* d)
{
    if (!d || d->nprofiles <= 0 || d->npositions <= 0 || !d->lengths || !d->offsets || !d->bkg ||
        !d->trn || !d->trg || !d->cv || !d->cvprior || !d->cvnorm2 || !d->ss || !d->aa)
        return fail(h, C2_ERR_ARG, "profiles: null field or empty set");
    int64_t acc = 0;
    for (int k = 0; k < d->nprofiles; k++) {
        if (d->lengths[k] <= 0 || d->lengths[k] > 65535)
            return fail(h, C2_ERR_ARG, "profile %d: length %d outside [1,65535]", k, d->lengths[k]);
        if (d->offsets[k] != acc) return fail(h, C2_ERR_ARG, "profile %d: offsets not contiguous", k);
        acc += d->lengths[k];
    }
    if (acc != d->npositions) return fail(h, C2_ERR_ARG, "profiles: lengths sum %lld != npositions %lld",
                                          (long long)acc, (long long)d->npositions);
    return C2_OK;
}

// DP transitions of position i of profile k (MMp, MIc, MDp, IMp, IIc, DMp, DDp)
static inline void trn_of(const c2_profiles* d, int k, int i, float* t7)
{
    const float* a = d->trn + ((size_t)d->offsets[k] + k + i) * 7;
    const float* b = a + 7;
    t7[TMM] = a[0]; t7[TMI] = b[1]; t7[TMD] = a[2];
    t7[TIM] = a[3]; t7[TII] = b[4]; t7[TDM] = a[5]; t7[TDD] = a[6];
}

static inline int ss_index(int state, float prb) { return state * 10 + (int)(prb * 9.999f); }

extern "C" c2_status c2_upload_db(c2_handle* h, const c2_profiles* d, uint64_t tot_pos, uint64_t tot_prof)
{
    if (!h) return C2_ERR_ARG;
    c2_status st = check_profiles(h, d);
    if (st != C2_OK) return st;
    CK(cudaSetDevice(h->device));
    const int P = d->nprofiles;
    const int64_t N = d->npositions;
    h->nprof = P;
    h->npos = N;
    h->total_pos = tot_pos ? tot_pos : (uint64_t)N;
    h->total_prof = tot_prof ? tot_prof : (uint64_t)P;
    h->h_plen.assign(d->lengths, d->lengths + P);
    h->h_poff.assign(d->offsets, d->offsets + P);
    h->Lmax = *std::max_element(h->h_plen.begin(), h->h_plen.end());
    // position records
    std::vector<float> rec((size_t)N * DR_STRIDE, 0.f);
    const float lok = h->sc.lokappa0;
    for (int k = 0; k < P; k++) {
        const int L = d->lengths[k];
        const int64_t o = d->offsets[k];
        for (int i = 0; i < L; i++) {
            const int64_t pos = o + i;
            float* r = rec.data() + (size_t)pos * DR_STRIDE;
            memcpy(r + DR_TRG, d->trg + pos * NAA, NAA * 4);
            memcpy(r + DR_CV, d->cv + pos * NCV, NCV * 4);
            r[DR_CN] = (d->cvnorm2[pos] + 1.0f) + lok;
            const float pr = d->cvprior[pos];
            r[DR_PRIOR] = h->prm.mapaln ? pr : (float)(int)pr;
            const float* s3 = d->ss + pos * NSS;
            r[DR_SS + 0] = s3[0]; r[DR_SS + 1] = s3[1]; r[DR_SS + 2] = s3[2];
            const int pk = ss_index(0, s3[0]) | (ss_index(1, s3[1]) << 8) | (ss_index(2, s3[2]) << 16);
            memcpy(r + DR_SSIDX, &pk, 4);
            r[DR_HD] = s3[2] + 0.1f;
            trn_of(d, k, i, r + DR_TRN);
            r[DR_AA] = (float)d->aa[pos];
        }
    }
    std::vector<float> bkg(d->bkg, d->bkg + (size_t)P * NAA);
    std::vector<int> order(P);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d->lengths[a] > d->lengths[b]; });
    std::vector<long long> poff(d->offsets, d->offsets + P);
    if (h->d_drec.ensure(rec.size()) || h->d_pbkg.ensure(bkg.size()) || h->d_plen.ensure(P) ||
        h->d_order.ensure(P) || h->d_poff.ensure(P) || h->d_best.ensure(P) || h->d_coords.ensure(P))
        return fail(h, C2_ERR_NOMEM, "device allocation for %d profiles / %lld positions failed", P, (long long)N);
    CK(cudaMemcpy(h->d_drec.p, rec.data(), rec.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_pbkg.p, bkg.data(), bkg.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_plen.p, d->lengths, (size_t)P * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_order.p, order.data(), (size_t)P * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_poff.p, poff.data(), (size_t)P * 8, cudaMemcpyHostToDevice));
    // strip-boundary scratch: per warp slot, two rows of 5 states
    const int lm = (h->Lmax + 31) & ~31;
    h->botstride = 10LL * lm;
    if (h->d_bot.ensure((size_t)h->grid * P1_WARPS * h->botstride))
        return fail(h, C2_ERR_NOMEM, "strip-boundary scratch allocation failed");
    h->Lq = 0;
    return C2_OK;
}

extern "C" c2_status c2_set_query(c2_handle* h, const c2_profiles* q)
{
    if (!h) return C2_ERR_ARG;
    c2_status st = check_profiles(h, q);
    if (st != C2_OK) return st;
    if (h->nprof <= 0) return fail(h, C2_ERR_STATE, "set_query before upload_db");
    CK(cudaSetDevice(h->device));
    const int Lq = q->lengths[0];
    h->Lq = Lq;
    h->qeno = q->eno ? q->eno[0] : 0.f;
    h->h_qrec.assign((size_t)Lq * QR_STRIDE, 0.f);
    // column -1 boundary states (see oracle colm1_states; CuBatchDP_init_btck.cu:117-262)
    std::vector<float> cMI(Lq), cIM(Lq), cDN(Lq);
    for (int r = 0; r < Lq; r++) {
        float t[7];
        trn_of(q, 0, r, t);
        float uMM = 0.f, uMI = 0.f, uDN = 0.f;
        if (r % 32 != 0) { uMI = cMI[r - 1]; uDN = cDN[r - 1]; }
        cMI[r] = hmax((uMM + t[TMM]) + LOG0, (uMI + t[TMM]) + LOG0);
        if (r % 32 == 0) cIM[r] = hmax((0.f + t[TMI]) + LOG0, (0.f + t[TII]) + LOG0);
        else cIM[r] = (0.f + t[TMI]) + LOG0;
        cDN[r] = hmax(uMM + t[TMD], uDN + t[TDD]);
    }
    const float lok = h->sc.lokappa0;
    for (int r = 0; r < Lq; r++) {
        float* rr = h->h_qrec.data() + (size_t)r * QR_STRIDE;
        memcpy(rr + QR_TRG, q->trg + (size_t)r * NAA, NAA * 4);
        memcpy(rr + QR_CV, q->cv + (size_t)r * NCV, NCV * 4);
        rr[QR_CN] = (q->cvnorm2[r] + 1.0f) + lok;
        const float pr = q->cvprior[r];
        rr[QR_PRIOR] = h->prm.mapaln ? pr : (float)(int)pr;
        const float* s3 = q->ss + (size_t)r * NSS;
        rr[QR_SS + 0] = s3[0]; rr[QR_SS + 1] = s3[1]; rr[QR_SS + 2] = s3[2];
        rr[QR_HQ] = s3[2] + 0.1f;
        trn_of(q, 0, r, rr + QR_TRN);
        rr[QR_C + 0] = cMI[r]; rr[QR_C + 1] = cIM[r]; rr[QR_C + 2] = cDN[r];
        if (r > 0) { rr[QR_CP + 0] = cMI[r - 1]; rr[QR_CP + 1] = cIM[r - 1]; rr[QR_CP + 2] = cDN[r - 1]; }
    }
    if (h->d_qrec.ensure(h->h_qrec.size()) || h->d_qbkg.ensure(NAA))
        return fail(h, C2_ERR_NOMEM, "query allocation failed");
    CK(cudaMemcpyAsync(h->d_qrec.p, h->h_qrec.data(), h->h_qrec.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_qbkg.p, q->bkg, NAA * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // thresholds: JobDispatcher::CalculateScoreThreshold (JobDispatcher.cpp:809-860)
    {
        size_t sspace = (size_t)Lq * (size_t)h->total_pos;
        float e = h->prm.eval;
        if (e <= 0.0f) { h->scorethld = 999.0f; h->logevthld = -99.0f; }
        else {
            h->logevthld = logf(e);
            e = (e < 1.0f) ? e * 10.0f : e * 3.0f;
            e /= h->prm.gapped_K * sspace;
            if (e <= 0.0f) h->scorethld = 999.0f;
            else {
                float s = -logf(e) / h->prm.gapped_lambda;
                h->scorethld = s < 0.0f ? 0.0f : s;
            }
        }
    }
    return C2_OK;
}

extern "C" c2_status c2_get_thresholds(const c2_handle* h, float* s, float* le)
{
    if (!h || !s || !le) return C2_ERR_ARG;
    *s = h->scorethld;
    *le = h->logevthld;
    return C2_OK;
}

static void fill_p1(c2_handle* h, P1Args& a)
{
    memset(&a, 0, sizeof a);
    a.qrec = h->d_qrec.p;
    a.Lq = h->Lq;
    a.drec = h->d_drec.p;
    a.plen = h->d_plen.p;
    a.poff = h->d_poff.p;
    a.pbkg = h->d_pbkg.p;
    a.counter = h->d_counter.p;
    a.ssss = h->d_ssss.p;
    a.cvvals = h->d_cvvals.p;
    a.sc = h->sc;
    a.bot = h->d_bot.p;
    a.botstride = h->botstride;
    a.best = h->d_best.p;
    a.coords = h->d_coords.p;
    a.status = h->d_status.p;
}

extern "C" c2_status c2_run_phase1(c2_handle* h)
{
    if (!h) return C2_ERR_ARG;
    if (h->nprof <= 0 || h->Lq <= 0) return fail(h, C2_ERR_STATE, "run_phase1 needs a database and a query");
    CK(cudaSetDevice(h->device));
    P1Args a;
    fill_p1(h, a);
    a.nwork = h->nprof;
    a.order = h->d_order.p;
    CK(cudaMemsetAsync(h->d_counter.p, 0, sizeof(int), h->stream));
    CK(launch_p1(a, h->d_qbkg.p, false, h->grid, h->stream));
    h->launches++;
    return C2_OK;
}

extern "C" c2_status c2_set_stream(c2_handle* h, void* stream)
{
    if (!h) return C2_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return C2_OK;
}

extern "C" c2_status c2_sync(c2_handle* h)
{
    if (!h) return C2_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    return C2_OK;
}

extern "C" c2_status c2_get_phase1(c2_handle* h, c2_p1_result* out, int32_t n)
{
    if (!h || !out || n < h->nprof) return C2_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float> b(h->nprof);
    std::vector<unsigned> c(h->nprof);
    CK(cudaMemcpy(b.data(), h->d_best.p, (size_t)h->nprof * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(c.data(), h->d_coords.p, (size_t)h->nprof * 4, cudaMemcpyDeviceToHost));
    for (int k = 0; k < h->nprof; k++) { out[k].best = b[k]; out[k].coords = c[k]; }
    return C2_OK;
}

extern "C" c2_status c2_run_finalize(c2_handle* h, int32_t* ncand)
{
    if (!h || !ncand) return C2_ERR_ARG;
    if (h->nprof <= 0 || h->Lq <= 0) return fail(h, C2_ERR_STATE, "run_finalize needs a database and a query");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float> b(h->nprof);
    CK(cudaMemcpy(b.data(), h->d_best.p, (size_t)h->nprof * 4, cudaMemcpyDeviceToHost));
    h->h_cand.clear();
    h->h_cand_off.clear();
    long long acc = 0;
    for (int k = 0; k < h->nprof; k++) {
        if (b[k] > h->scorethld) {  // FinalizeDPPro: maxsc <= scorethld -> not passed
            h->h_cand.push_back(k);
            h->h_cand_off.push_back(acc);
            acc += (long long)h->Lq * h->h_plen[k];
        }
    }
    h->ncand = (int)h->h_cand.size();
    *ncand = h->ncand;
    if (h->ncand == 0) return C2_OK;
    const int nc = h->ncand;
    if (h->d_cand_prof.ensure(nc) || h->d_cand_off.ensure(nc) || h->d_btck.ensure((size_t)acc) ||
        h->d_smat.ensure((size_t)acc) || h->d_fscore.ensure(nc) || h->d_fpsts.ensure(nc) ||
        h->d_fpassed.ensure(nc) || h->d_fbeg.ensure(nc) || h->d_fend.ensure(nc))
        return fail(h, C2_ERR_NOMEM, "finalisation scratch for %d pairs (%lld cells) failed", nc, acc);
    CK(cudaMemcpyAsync(h->d_cand_prof.p, h->h_cand.data(), (size_t)nc * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_cand_off.p, h->h_cand_off.data(), (size_t)nc * 8, cudaMemcpyHostToDevice, h->stream));
    P1Args a;
    fill_p1(h, a);
    a.nwork = nc;
    a.order = h->d_cand_prof.p;
    a.cand_off = h->d_cand_off.p;
    a.btck = h->d_btck.p;
    a.smat = h->d_smat.p;
    CK(cudaMemsetAsync(h->d_counter.p, 0, sizeof(int), h->stream));
    const int grid = std::min(h->grid, (nc + P1_WARPS - 1) / P1_WARPS);
    CK(launch_p1(a, h->d_qbkg.p, true, grid, h->stream));
    h->launches++;
    FinArgs f;
    f.Lq = h->Lq;
    f.ncand = nc;
    f.cand_prof = h->d_cand_prof.p;
    f.cand_off = h->d_cand_off.p;
    f.plen = h->d_plen.p;
    f.btck = h->d_btck.p;
    f.smat = h->d_smat.p;
    f.best = h->d_best.p;
    f.coords = h->d_coords.p;
    f.scorethld = h->scorethld;
    f.score = h->d_fscore.p;
    f.psts = h->d_fpsts.p;
    f.beg = h->d_fbeg.p;
    f.endc = h->d_fend.p;
    f.passed = h->d_fpassed.p;
    CK(launch_fin(f, h->stream));
    h->launches++;
    return C2_OK;
}

extern "C" c2_status c2_get_finalize(c2_handle* h, c2_dp_result* out, int32_t n)
{
    if (!h || (!out && n > 0) || n < h->ncand) return C2_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    int stw = 0;
    CK(cudaMemcpy(&stw, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (stw != 0) return fail(h, C2_ERR_DEVICE, "device status %d (traceback DP disagrees with phase 1)", stw);
    const int nc = h->ncand;
    if (nc == 0) return C2_OK;
    std::vector<float> sc(nc);
    std::vector<int> ps(nc), pa(nc);
    std::vector<unsigned> bg(nc), en(nc);
    CK(cudaMemcpy(sc.data(), h->d_fscore.p, nc * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ps.data(), h->d_fpsts.p, nc * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(pa.data(), h->d_fpassed.p, nc * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(bg.data(), h->d_fbeg.p, nc * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(en.data(), h->d_fend.p, nc * 4, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nc; i++) {
        out[i].score = sc[i];
        out[i].profile = h->h_cand[i];
        out[i].psts = ps[i];
        out[i].beg = bg[i];
        out[i].end = en[i];
        out[i].passed = pa[i];
    }
    return C2_OK;
}

extern "C" c2_status c2_launch_count(const c2_handle* h, uint64_t* n)
{
    if (!h || !n) return C2_ERR_ARG;
    *n = h->launches;
    return C2_OK;
}
