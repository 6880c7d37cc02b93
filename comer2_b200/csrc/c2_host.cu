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
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <atomic>
#include <thread>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/comer2_b200.h"
#include "c2_device.cuh"
#include "c2_stats.cuh"
#include "c2_adj.cuh"

namespace c2 {
cudaError_t launch_stats(const StatsArgs& a, cudaStream_t st);
cudaError_t launch_map(const MapArgs& a, const float* qtrn, const float* dtrn, const float* qcf, int nsm,
                       int* counter, cudaStream_t st, int* nlaunch);
cudaError_t launch_viterbi_aln(const MapArgs& a, cudaStream_t st);
size_t p1_smem_bytes(int cvcard);
cudaError_t launch_p1(const P1Args& a, const float* qbkg, int which, int grid, cudaStream_t st);
int p1_blocks_per_sm(int cvcard);
int p1c_blocks_per_sm(int cvcard);
int p1t_blocks_per_sm(int cvcard, cudaError_t* err);
cudaError_t launch_aln_pack(const char* aln, int alnstride, const int* info, const long long* off, int nm, char* dst,
                            cudaStream_t st);
cudaError_t launch_tc_pack(const float* drec, const long long* poff, const int* plen, const long long* ttile,
                           int nprof, unsigned* tcdb, float* cold, float lok, float wss, cudaStream_t st);
cudaError_t launch_fin(const FinArgs& a, cudaStream_t st);
}  // namespace c2

using namespace c2;

// Device memory budget of a handle (c2_set_device_memory_limit; the
// reference's --dev-mem): bytes held by the handle's buffers, and the limit
// (0: none).  Shared by the buffers that draw on it, which may outlive the
// handle (a database store kept by another handle).
struct Budget {
    size_t limit = 0;
    size_t used = 0;
    std::mutex mu;
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    std::shared_ptr<Budget> bud;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            cudaFree(p);
            if (bud) {
                std::lock_guard<std::mutex> lk(bud->mu);
                bud->used -= n * sizeof(T);
            }
        }
        p = nullptr;
        n = 0;
        bud.reset();
    }
    // at least cnt elements; a request beyond the budget fails as an
    // allocation failure would, before cudaMalloc
    cudaError_t ensure(size_t cnt, const std::shared_ptr<Budget>& b = nullptr) {
        if (cnt <= n && p) return cudaSuccess;
        release();
        if (cnt == 0) cnt = 1;
        const size_t bytes = cnt * sizeof(T);
        if (b) {
            std::lock_guard<std::mutex> lk(b->mu);
            if (b->limit && b->used + bytes > b->limit) return cudaErrorMemoryAllocation;
            b->used += bytes;
        }
        cudaError_t e = cudaMalloc((void**)&p, bytes);
        if (e == cudaSuccess) {
            n = cnt;
            bud = b;
        } else {
            p = nullptr;
            if (b) {
                std::lock_guard<std::mutex> lk(b->mu);
                b->used -= bytes;
            }
        }
        return e;
    }
};

// Device copy of an uploaded database: shared by the handles that search it
// (c2_share_db), freed with the last of them.
struct DbStore {
    DevBuf<float> d_drec, d_pbkg, d_dtrn, d_peno;
    DevBuf<int> d_plen, d_order;
    DevBuf<long long> d_poff;
    DevBuf<unsigned char> d_daa, d_dss;
    // tensor-core score operands, packed on first use (under tc_mu)
    DevBuf<unsigned> d_tcdb;
    DevBuf<long long> d_ttile;
    DevBuf<float> d_cold;
    bool tc_ready = false;
    std::mutex tc_mu;
};

struct c2_handle {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream in use
    cudaStream_t own_stream = nullptr;  // the handle's own stream
    std::string err;
    uint64_t launches = 0;
    int nsm = 0;
    int grid = 0;
    int score_mode = C2_SCORE_FP32;   // phase-1 score arithmetic (c2_set_score_mode)
    int p1_reserve = 0;               // SMs the phase-1 kernels leave free (multi-query batches)
    int batch_reserve = -1;           // c2_set_batch_sm_reserve (-1: nsm / BATCH_RESERVE_DIV)
    std::shared_ptr<Budget> budget = std::make_shared<Budget>();   // c2_set_device_memory_limit
    unsigned spin = PIPE_SPIN;        // polls before a phase-2 strip wait gives up (c2_set_wait_limit)
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
    std::shared_ptr<DbStore> db;
    // query
    int Lq = 0;
    float qeno = 0.f;
    std::vector<float> h_qrec;
    DevBuf<float> d_qrec, d_qbkg, d_qtrn, d_qcf, d_qcfx, d_qU;
    // differentiable alignment (c2_logz_fwd / c2_logz_bwd)
    std::vector<int> adj_prof, adj_Lq;
    std::vector<long long> adj_off, adj_roff;   // per pair: first cell (wavefront order), first row-buffer float
    long long adj_cells = 0, adj_rows = 0;
    int adj_Lmax = 0, adj_bgrid = 0, adj_nitems = 0;   // longest profile of the pairs; backward CTAs; strips
    bool adj_fwd_done = false, adj_batch = false;      // adj_batch: the pairs' queries are in d_adjq*
    float adj_theta[7] = {0, 0, 0, 0, 0, 0, 0};
    float adj_wss = 0.f, adj_wcv = 0.f;
    DevBuf<int> d_adjprof, d_adjprog, d_adjctr, d_adjLq, d_adjqidx;
    DevBuf<long long> d_adjoff, d_adjroff, d_adjqpos, d_adjsoff;
    DevBuf<int2> d_adjitems;
    DevBuf<float> d_adjbuf, d_adjlogz, d_adjgrad, d_adjpart, d_adjscr;
    DevBuf<float> d_adjF;            // all forward states, when they fit (no recompute in the backward sweep)
    bool adj_keepF = false;
    DevBuf<float> d_adjqrec, d_adjqtrn, d_adjqcfx, d_adjqbkg;   // queries of c2_set_query_batch
    std::vector<int> adj_qlen;                                   // their lengths
    std::vector<long long> adj_qstart;                           // and first rows
    DevBuf<unsigned char> d_qaa, d_qss;
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
    DevBuf<int> d_cand_prof, d_worder, d_tbitems, d_mapitems;
    DevBuf<long long> d_cand_off;
    DevBuf<signed char> d_btck;
    DevBuf<float> d_smat, d_mmat;
    // strip pipeline of the phase-2 sweeps: last-row buffers, progress words
    DevBuf<float> d_bnd;
    DevBuf<unsigned long long> d_tbkey;
    // tensor-core query operands
    DevBuf<unsigned> d_qa;
    DevBuf<float> d_qaaf;
    DevBuf<int> d_prog;
    size_t bnd_half = 0, prog_half = 0;   // floats / words of one sweep's strip-pipeline scratch
    DevBuf<float> d_fscore;
    DevBuf<int> d_fpsts, d_fpassed;
    DevBuf<unsigned> d_fbeg, d_fend;
    std::vector<float> h_fscore;
    std::vector<int> h_fpassed;
    // statistics
    int npass = 0;
    std::vector<int> h_p2;          // passed pair -> candidate index
    DevBuf<int> d_p2;
    DevBuf<float> d_stats;
    std::vector<float> h_stats;
    // MAP
    int nmap = 0;
    std::vector<int> h_mapcand, h_mappass;
    DevBuf<int> d_mapcand, d_mappass, d_alninfo;
    DevBuf<float> d_fb, d_bb, d_pairf;
    DevBuf<unsigned> d_pairc;
    DevBuf<unsigned long long> d_pairk;
    DevBuf<char> d_aln, d_alnpack;
    DevBuf<long long> d_alnoff;
    int alnstride = 0;
    // hits of a search run in candidate groups (c2_search under a device
    // memory budget), merged and sorted; c2_get_hits serves them when valid
    bool acc_valid = false;
    int ngroups = 1;
    std::vector<c2_hit> acc_hits;
    std::vector<char> acc_alns;
    // worker handles of c2_search_batch (sharing this handle's database)
    std::vector<c2_handle*> workers;
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

// device status words: 2 = the traceback DP's maximum differs from phase 1,
// 3 = a phase-2 sweep gave up waiting for the strip above it
static const char* status_text(int st)
{
    switch (st) {
    case 2: return "traceback DP disagrees with phase 1";
    case PIPE_ERR_TIMEOUT: return "a strip wait in a phase-2 sweep timed out";
    default: return "unknown device error";
    }
}

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

// Schraudolph (1999) exponential and its inverse as the MAP kernels evaluate
// them (fused multiply-add), for the host-side boundary states
static inline float host_fexp(float x)
{
    if (!(-16.f < x)) return 0.f;
    const int i = (int)fmaf(12102203.16f, x, 1064631197.0f);
    float f;
    memcpy(&f, &i, 4);
    return f;
}
static inline float host_flog(float x)
{
    if (!(3.8e-11f < x)) return -99.f;
    int i;
    memcpy(&i, &x, 4);
    return (float)(i - 1064631197) * 8.2629582959339e-08f;
}
static inline float host_lse2(float a, float b)
{
    const float mx = hmax(a, b);
    return host_flog(host_fexp(a - mx) + host_fexp(b - mx)) + mx;
}

// Gertz (2005) length adjustment for the effective search space, float
// arithmetic as AbstractScoreMatrix::ComputeLengthAdjustment
// (src/libpro/srcsco/AbstractScoreMatrix.cpp:303-380)
static void length_adjustment(float lambda, float K, float alpha, float beta, size_t m, uint64_t n, size_t N,
                              unsigned long long* searchspace, unsigned long long* deltalen)
{
    *searchspace = (unsigned long long)m * n;
    *deltalen = 0;
    if (lambda <= 0.0f || K <= 0.0f || N < 1) return;
    const int maxit = 20;
    const float logK = logf(K);
    const float alratio = alpha / lambda;
    const float max_mn = (float)((m > n) ? m : n);
    float length = 0.0f, min_length = 0.0f, max_length = 0.0f, nxt_length = 0.0f;
    float sspace = 0.0f, space2 = 0.0f;
    bool converged = false;
    const float a = (float)N;
    const float b = (float)(n + m * N);
    const float c = (float)(m * n) - max_mn / K;
    if (c < 0.0f) return;
    max_length = 2.0f * c / (b + sqrtf(b * b - 4.0f * a * c));
    for (int j = 0; j < maxit; j++) {
        length = nxt_length;
        sspace = (m - length) * (n - N * length);
        nxt_length = alratio * (logK + logf(sspace)) + beta;
        if (length <= nxt_length) {
            min_length = length;
            if (nxt_length - length <= 1.0f) { converged = true; break; }
            if (min_length == max_length) break;
        } else
            max_length = length;
        if (nxt_length < min_length || max_length < nxt_length)
            nxt_length = (!j) ? max_length : (min_length + max_length) * 0.5f;
    }
    if (converged) {
        length = ceilf(min_length);
        if (length <= max_length) {
            space2 = (m - length) * (n - N * length);
            nxt_length = alratio * (logK + logf(space2)) + beta;
            if (length <= nxt_length) { min_length = length; sspace = space2; }
        }
    }
    *searchspace = (unsigned long long)sspace;
    *deltalen = (unsigned long long)min_length;
}

// ---------------------------------------------------------------------------
extern "C" c2_status c2_create(int device, const c2_params* p, c2_handle** out)
{
    if (!out || !p) return C2_ERR_ARG;
    *out = nullptr;
    if (!p->ssss || p->ssss_card <= 0 || p->ssss_card > MAX_SSSS_CARD || !p->cvs2s_keys ||
        !p->cvs2s_values || p->cvs2s_card <= 1 || p->cvs2s_card > std::min(MAX_CVCARD, P1TC_MAX_CVCARD) ||
        p->cvs2s_shift < 0)
        return C2_ERR_ARG;
    // SS and CV term weights: 0 leaves a term out, as the reference's score
    // kernels are then not launched (cusco/CuBatchScoreMatrix.cu:273-352)
    if (!(p->ssswgt >= 0.f) || !(p->cvswgt >= 0.f)) return C2_ERR_ARG;
    // SSEMODEL 0 (observed statistics), 1 and 2 (SS18 variants); MAPALN 1
    // (MAP alignments) or 0 (the Viterbi DP's alignments, as FinalizeDP_ALN
    // draws them; cupro/CuBatchProcessing.cu:477-510)
    if (p->ssemodel < 0 || p->ssemodel > 2 || (p->mapaln != 0 && p->mapaln != 1)) return C2_ERR_ARG;
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
        if (h->d_ssss.ensure(h->ssss.size(), h->budget) || h->d_cvvals.ensure(h->cvvals.size(), h->budget) ||
            h->d_status.ensure(1, h->budget) || h->d_counter.ensure(4, h->budget)) { st = C2_ERR_NOMEM; break; }
        if (cudaMemcpy(h->d_ssss.p, h->ssss.data(), h->ssss.size() * 4, cudaMemcpyHostToDevice) ||
            cudaMemcpy(h->d_cvvals.p, h->cvvals.data(), h->cvvals.size() * 4, cudaMemcpyHostToDevice) ||
            cudaMemset(h->d_status.p, 0, sizeof(int))) { st = C2_ERR_CUDA; break; }
        if (!h->nnw.empty()) {
            if (h->d_nnw.ensure(h->nnw.size(), h->budget) ||
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
    for (c2_handle* w : h->workers) c2_destroy(w);
    h->workers.clear();
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

// Dispatch lag of the sweeps' work-item order, in wavefront steps: strip s of
// a pair is handed out about `lag` steps' worth of work after strip s - 1.
// The physical lag is about 96 steps for the traceback sweep (the row above
// is loaded a 32-column chunk ahead and published once per chunk) and about
// 48 for the MAP sweeps (8 columns at a time); handing strips out later than
// that leaves fewer warps polling for their predecessor, and the values below
// were chosen by measurement (kernel times on configs 1 and 4 with lags of
// 64 / 96 / 128 / 160-192 / 256-320: traceback sweep 21.4 -> 16.3 ms, MAP DP
// 22.4 -> 17.5-18.0 ms and MAP forward-backward 74.4 -> 72.3 ms on config 4).
constexpr int STRIP_LAG_TB = 320, STRIP_LAG_MAP = 192;

// Work-item table of a strip-pipelined sweep over np pairs (in processing
// order, lengths lens): item (p, s) at key p + K s, K = pairs started per
// strip lag (lag steps) when nwarps warps are busy, so that strip s of a pair is handed
// out about when strip s - 1 is far enough ahead.  Ties keep s order, so
// (p, s - 1) always precedes (p, s).

static void strip_items(const std::vector<int>& lens, int nstrips, int nwarps, int lag, std::vector<int>& items)
{
    const int np = (int)lens.size();
    double lm = 31.0;
    for (int L : lens) lm += (double)L / std::max(1, np);
    const double K = (double)lag * nwarps / (nstrips * lm);
    // key(p, s) = p + K s = b + f_s with bucket b = p + floor(K s) and
    // f_s = frac(K s): each bucket holds one item per strip, ordered by f_s
    // and, for equal f_s, larger s first (its p is smaller); the same order
    // in every bucket, so the table is emitted bucket by bucket in linear time
    std::vector<long long> fl(nstrips);
    std::vector<double> fr(nstrips);
    for (int s = 0; s < nstrips; s++) {
        const double ks = K * s;
        fl[s] = (long long)std::floor(ks);
        fr[s] = ks - (double)fl[s];
    }
    std::vector<int> perm(nstrips);
    std::iota(perm.begin(), perm.end(), 0);
    std::sort(perm.begin(), perm.end(), [&](int x, int y) { return fr[x] < fr[y] || (fr[x] == fr[y] && x > y); });
    items.clear();
    items.reserve((size_t)np * nstrips);
    const long long bmax = (long long)np - 1 + fl[nstrips - 1];
    for (long long b = 0; b <= bmax; b++)
        for (int s : perm) {
            const long long p = b - fl[s];
            if (p >= 0 && p < np) items.push_back((int)p * nstrips + s);
        }
}

// candidate margin and traceback tolerance of the BF16 score mode (relative)
constexpr float C2_TC_MARGIN = 2e-3f;
constexpr float C2_TC_TOL = 2e-3f;

// BF16 round to nearest even, as the device conversion does
static inline uint32_t bf16_rn_bits(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0u;   // NaN
    return (u + 0x7fffu + ((u >> 16) & 1u)) >> 16;
}

static inline float bf16_to_f(uint32_t b)
{
    const uint32_t u = b << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static inline int ss_index(int state, float prb) { return state * 10 + (int)(prb * 9.999f); }

// Position record of every db position (DR_* layout) for profiles [k0, k1),
// written from out on (out holds the record of position offsets[k0] first)
static void pack_records(const c2_profiles* d, float lok, bool mapaln, int k0, int k1, float* out)
{
    const int64_t base = d->offsets[k0];
    for (int k = k0; k < k1; k++) {
        const int L = d->lengths[k];
        const int64_t o = d->offsets[k];
        for (int i = 0; i < L; i++) {
            const int64_t pos = o + i;
            float* r = out + (size_t)(pos - base) * DR_STRIDE;
            memcpy(r + DR_TRG, d->trg + pos * NAA, NAA * 4);
            memcpy(r + DR_CV, d->cv + pos * NCV, NCV * 4);
            r[DR_CN] = (d->cvnorm2[pos] + 1.0f) + lok;
            const float pr = d->cvprior[pos];
            r[DR_PRIOR] = mapaln ? pr : (float)(int)pr;
            const float* s3 = d->ss + pos * NSS;
            r[DR_SS + 0] = s3[0]; r[DR_SS + 1] = s3[1]; r[DR_SS + 2] = s3[2];
            const int pk = ss_index(0, s3[0]) | (ss_index(1, s3[1]) << 8) | (ss_index(2, s3[2]) << 16);
            memcpy(r + DR_SSIDX, &pk, 4);
            r[DR_HD] = s3[2] + 0.1f;
            r[DR_HD + 1] = 0.f;   // pad
            r[DR_HD + 2] = 0.f;
            trn_of(d, k, i, r + DR_TRN);
            r[DR_AA] = (float)d->aa[pos];
        }
    }
}

// Pinned staging of the record upload: two buffers and their copy events.
// The destructor waits for copies in flight before freeing the buffers.
namespace {
struct RecStage {
    float* buf[2] = {nullptr, nullptr};
    bool pinned[2] = {false, false};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    bool sync = false;
    ~RecStage()
    {
        if (sync) cudaStreamSynchronize(st);
        for (int b = 0; b < 2; b++) {
            if (ev[b]) cudaEventDestroy(ev[b]);
            if (buf[b] && pinned[b]) cudaFreeHost(buf[b]);
            else free(buf[b]);
        }
    }
};
}  // namespace

// The db position records to d_drec: chunks of whole profiles (up to 2^18
// positions, 56 MiB of records) are packed by host threads into two pinned
// buffers in turn, each copied asynchronously while the next chunk is packed
// (the reference's reader overlaps its double-buffered pinned transfers the
// same way: cupro/TdDataReader.cpp, CuDeviceMemory.cu:1073).
static c2_status upload_records(c2_handle* h, const c2_profiles* d)
{
    const int P = d->nprofiles;
    const int64_t N = d->npositions;
    const int64_t cap = std::max<int64_t>(int64_t(1) << 18, h->Lmax);
    const float lok = h->sc.lokappa0;
    const bool mapaln = h->prm.mapaln != 0;
    RecStage S;
    for (int b = 0; b < 2; b++) {
        const size_t bytes = (size_t)cap * DR_STRIDE * 4;
        if (cudaHostAlloc(reinterpret_cast<void**>(&S.buf[b]), bytes, cudaHostAllocDefault) == cudaSuccess) {
            S.pinned[b] = true;
        } else {
            // no pinned memory to be had: pageable staging (cudaMemcpyAsync
            // then returns once it has taken the source over)
            (void)cudaGetLastError();
            S.buf[b] = static_cast<float*>(malloc(bytes));
            if (!S.buf[b]) return fail(h, C2_ERR_NOMEM, "record staging buffer of %zu bytes", bytes);
        }
        CK(cudaEventCreateWithFlags(&S.ev[b], cudaEventDisableTiming));
    }
    S.st = h->stream;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::max(1u, std::min(16u, hw));
    const int64_t* off = d->offsets;
    auto end_of = [&](int k) -> int64_t { return k < P ? off[k] : N; };
    bool used[2] = {false, false};
    int b = 0;
    for (int k0 = 0; k0 < P;) {
        const int64_t p0 = off[k0];
        // profiles [k0, k1): the most whose positions fit in a buffer (at least
        // one; cap >= Lmax).  Profiles before the first one starting past the
        // window start inside it; only the last of them can end past it.
        int k1 = (int)(std::upper_bound(off + k0 + 1, off + P, p0 + cap) - off);
        while (k1 > k0 + 1 && end_of(k1) - p0 > cap) k1--;
        const int64_t p1 = end_of(k1);
        if (used[b]) CK(cudaEventSynchronize(S.ev[b]));
        float* out = S.buf[b];
        // host threads over position ranges of whole profiles
        const int nth = (int)std::max<int64_t>(1, std::min<int64_t>(nt, (p1 - p0) / 16384));
        std::vector<std::thread> pool;
        int ka = k0;
        for (int t = 0; t < nth; t++) {
            int kb = k1;
            if (t + 1 < nth) {
                const int64_t tgt = p0 + (p1 - p0) * (t + 1) / nth;
                kb = (int)(std::upper_bound(off + ka, off + k1, tgt) - off);
                kb = std::max(kb, ka);
            }
            if (kb > ka) {
                float* o = out + (size_t)(off[ka] - p0) * DR_STRIDE;
                try {
                    pool.emplace_back(pack_records, d, lok, mapaln, ka, kb, o);
                } catch (...) {
                    pack_records(d, lok, mapaln, ka, kb, o);   // no thread to be had: pack here
                }
            }
            ka = kb;
        }
        for (auto& th : pool) th.join();
        S.sync = true;
        CK(cudaMemcpyAsync(h->db->d_drec.p + (size_t)p0 * DR_STRIDE, out, (size_t)(p1 - p0) * DR_STRIDE * 4,
                           cudaMemcpyHostToDevice, h->stream));
        CK(cudaEventRecord(S.ev[b], h->stream));
        used[b] = true;
        b ^= 1;
        k0 = k1;
    }
    // the raw transitions ([N + P][7] floats, the MAP and statistics stages'
    // copy) through the same buffers: copied into a pinned buffer by the host
    // threads while the previous piece goes over the bus, instead of one
    // synchronous copy from pageable memory
    {
        const size_t total = (size_t)(N + P) * 7 * sizeof(float);
        const size_t piece = (size_t)cap * DR_STRIDE * 4;
        const char* src = reinterpret_cast<const char*>(d->trn);
        char* dst = reinterpret_cast<char*>(h->db->d_dtrn.p);
        for (size_t o = 0; o < total; o += piece) {
            const size_t n = std::min(piece, total - o);
            if (used[b]) CK(cudaEventSynchronize(S.ev[b]));
            char* out = reinterpret_cast<char*>(S.buf[b]);
            const int nth = (int)std::max<size_t>(1, std::min<size_t>((size_t)nt, n >> 22));
            std::vector<std::thread> pool;
            for (int t = 0; t < nth; t++) {
                const size_t a0 = n * t / nth, a1 = n * (t + 1) / nth;
                try {
                    pool.emplace_back([=]() { memcpy(out + a0, src + o + a0, a1 - a0); });
                } catch (...) {
                    memcpy(out + a0, src + o + a0, a1 - a0);   // no thread to be had: copy here
                }
            }
            for (auto& th : pool) th.join();
            S.sync = true;
            CK(cudaMemcpyAsync(dst + o, out, n, cudaMemcpyHostToDevice, h->stream));
            CK(cudaEventRecord(S.ev[b], h->stream));
            used[b] = true;
            b ^= 1;
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    return C2_OK;
}

extern "C" c2_status c2_upload_db(c2_handle* h, const c2_profiles* d, uint64_t tot_pos, uint64_t tot_prof)
{
    if (!h) return C2_ERR_ARG;
    c2_status st = check_profiles(h, d);
    if (st != C2_OK) return st;
    CK(cudaSetDevice(h->device));
    const int P = d->nprofiles;
    const int64_t N = d->npositions;
    h->db = std::make_shared<DbStore>();   // handles sharing the previous database keep it
    h->nprof = P;
    h->npos = N;
    h->total_pos = tot_pos ? tot_pos : (uint64_t)N;
    h->total_prof = tot_prof ? tot_prof : (uint64_t)P;
    h->h_plen.assign(d->lengths, d->lengths + P);
    h->h_poff.assign(d->offsets, d->offsets + P);
    h->Lmax = *std::max_element(h->h_plen.begin(), h->h_plen.end());
    std::vector<float> bkg(d->bkg, d->bkg + (size_t)P * NAA);
    std::vector<int> order(P);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d->lengths[a] > d->lengths[b]; });
    std::vector<long long> poff(d->offsets, d->offsets + P);
    if (h->db->d_drec.ensure((size_t)N * DR_STRIDE, h->budget) || h->db->d_pbkg.ensure(bkg.size(), h->budget) || h->db->d_plen.ensure(P, h->budget) ||
        h->db->d_order.ensure(P, h->budget) || h->db->d_poff.ensure(P, h->budget) || h->d_best.ensure(P, h->budget) || h->d_coords.ensure(P, h->budget))
        return fail(h, C2_ERR_NOMEM, "device allocation for %d profiles / %lld positions failed", P, (long long)N);
    if (h->db->d_dtrn.ensure((size_t)(N + P) * 7, h->budget))
        return fail(h, C2_ERR_NOMEM, "device allocation of db transitions failed");
    if ((st = upload_records(h, d)) != C2_OK) return st;   // the records and the raw transitions
    CK(cudaMemcpy(h->db->d_pbkg.p, bkg.data(), bkg.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->db->d_plen.p, d->lengths, (size_t)P * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->db->d_order.p, order.data(), (size_t)P * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->db->d_poff.p, poff.data(), (size_t)P * 8, cudaMemcpyHostToDevice));
    // raw transitions, residues, SS states and ENOs for the statistics and MAP stages
    if (h->db->d_daa.ensure((size_t)N, h->budget) || h->db->d_dss.ensure((size_t)N, h->budget) ||
        h->db->d_peno.ensure((size_t)P, h->budget))
        return fail(h, C2_ERR_NOMEM, "device allocation of db side arrays failed");
    CK(cudaMemcpy(h->db->d_daa.p, d->aa, (size_t)N, cudaMemcpyHostToDevice));
    if (d->ssstate) CK(cudaMemcpy(h->db->d_dss.p, d->ssstate, (size_t)N, cudaMemcpyHostToDevice));
    else CK(cudaMemset(h->db->d_dss.p, ' ', (size_t)N));
    if (d->eno) CK(cudaMemcpy(h->db->d_peno.p, d->eno, (size_t)P * 4, cudaMemcpyHostToDevice));
    else CK(cudaMemset(h->db->d_peno.p, 0, (size_t)P * 4));
    // strip-boundary scratch: per warp slot, two rows of 5 states
    const int lm = (h->Lmax + 31) & ~31;
    h->botstride = 10LL * lm;
    if (h->d_bot.ensure((size_t)h->grid * P1_WARPS * h->botstride, h->budget))
        return fail(h, C2_ERR_NOMEM, "strip-boundary scratch allocation failed");
    h->Lq = 0;
    h->db->tc_ready = false;
    return C2_OK;
}

// Search the database uploaded to src from dst as well (same device; no
// copy): dst gets its own query, result and scratch buffers.
extern "C" c2_status c2_share_db(c2_handle* dst, const c2_handle* src)
{
    if (!dst || !src || dst == src) return C2_ERR_ARG;
    c2_handle* h = dst;   // error reports go to dst
    if (!src->db || src->nprof <= 0) return fail(dst, C2_ERR_STATE, "share_db: the source handle has no database");
    if (dst->device != src->device) return fail(dst, C2_ERR_ARG, "share_db: handles on different devices");
    CK(cudaSetDevice(dst->device));
    dst->db = src->db;
    dst->nprof = src->nprof;
    dst->npos = src->npos;
    dst->total_pos = src->total_pos;
    dst->total_prof = src->total_prof;
    dst->h_plen = src->h_plen;
    dst->h_poff = src->h_poff;
    dst->Lmax = src->Lmax;
    const int P = dst->nprof;
    const int lm = (dst->Lmax + 31) & ~31;
    dst->botstride = 10LL * lm;
    if (dst->d_best.ensure(P, dst->budget) || dst->d_coords.ensure(P, dst->budget) ||
        dst->d_bot.ensure((size_t)dst->grid * P1_WARPS * dst->botstride, dst->budget))
        return fail(dst, C2_ERR_NOMEM, "share_db: per-handle buffers for %d profiles failed", P);
    dst->Lq = 0;
    return C2_OK;
}

// Score fields of the query records (profile 0 of q): target probabilities,
// context vector, CV norm and prior, SS probabilities, P(H) + 0.1
static void qrec_score_fields(const c2_handle* h, const c2_profiles* q, float* qrec)
{
    const int Lq = q->lengths[0];
    const float lok = h->sc.lokappa0;
    for (int r = 0; r < Lq; r++) {
        float* rr = qrec + (size_t)r * QR_STRIDE;
        memcpy(rr + QR_TRG, q->trg + (size_t)r * NAA, NAA * 4);
        memcpy(rr + QR_CV, q->cv + (size_t)r * NCV, NCV * 4);
        rr[QR_CN] = (q->cvnorm2[r] + 1.0f) + lok;
        const float pr = q->cvprior[r];
        rr[QR_PRIOR] = h->prm.mapaln ? pr : (float)(int)pr;
        const float* s3 = q->ss + (size_t)r * NSS;
        rr[QR_SS + 0] = s3[0]; rr[QR_SS + 1] = s3[1]; rr[QR_SS + 2] = s3[2];
        rr[QR_HQ] = s3[2] + 0.1f;
    }
}

// Column -1 states of the query rows in the log-partition model (the MAP
// forward's boundary with exact exp/log): per row MI IM DN of the row and of
// the row before
static void colm1_exact(const c2_profiles* q, float* qx)
{
    const int Lq = q->lengths[0];
    auto xl2 = [](double a, double b) { const double m = std::max(a, b); return std::log(std::exp(a - m) + std::exp(b - m)) + m; };
    double pMI = 0, pIM = 0, pDN = 0;
    for (int r = 0; r < Lq; r++) {
        float t[7];
        trn_of(q, 0, r, t);
        const double L0 = -99.0;
        double uMI = L0, uDN = L0;
        if (r % 32 != 0) { uMI = pMI; uDN = pDN; }
        const double mi = xl2((0.0 + t[TMM]) + L0, (uMI + t[TMM]) + L0);
        const double im = (r % 32 == 0) ? xl2((0.0 + t[TMI]) + L0, (L0 + t[TII]) + L0)
                                        : xl2((0.0 + t[TMI]) + L0, ((((0.0 + t[TMI]) + L0) + t[TII]) + L0));
        const double dn = xl2(0.0 + t[TMD], uDN + t[TDD]);
        float* c = qx + (size_t)r * 6;
        c[0] = (float)mi; c[1] = (float)im; c[2] = (float)dn;
        c[3] = (float)pMI; c[4] = (float)pIM; c[5] = (float)pDN;
        pMI = mi; pIM = im; pDN = dn;
    }
}

// Effective search space and thresholds of a query of length Lq against the
// database totals: AbstractScoreMatrix::ComputeLengthAdjustment
// (libpro/srcsco/AbstractScoreMatrix.cpp:303-380) and
// JobDispatcher::CalculateScoreThreshold (cualn/JobDispatcher.cpp:809-860)
static void query_limits(const c2_handle* h, int Lq, unsigned long long* searchspace, unsigned long long* deltalen,
                         float* scorethld, float* logevthld)
{
    length_adjustment(h->prm.gapped_lambda, h->prm.gapped_K, h->prm.gapped_alpha, h->prm.gapped_beta,
                      (size_t)Lq, h->total_pos, (size_t)h->total_prof, searchspace, deltalen);
    size_t sspace = (size_t)Lq * (size_t)h->total_pos;
    float e = h->prm.eval;
    if (e <= 0.0f) {
        *scorethld = 999.0f;
        *logevthld = -99.0f;
    } else {
        *logevthld = logf(e);
        e = (e < 1.0f) ? e * 10.0f : e * 3.0f;
        e /= h->prm.gapped_K * sspace;
        if (e <= 0.0f) *scorethld = 999.0f;
        else {
            const float sc = -logf(e) / h->prm.gapped_lambda;
            *scorethld = sc < 0.0f ? 0.0f : sc;
        }
    }
}

extern "C" c2_status c2_set_query(c2_handle* h, const c2_profiles* q)
{
    if (!h) return C2_ERR_ARG;
    c2_status st = check_profiles(h, q);
    if (st != C2_OK) return st;
    if (h->nprof <= 0) return fail(h, C2_ERR_STATE, "set_query before upload_db");
    CK(cudaSetDevice(h->device));
    // a new search starts with a clear device status word and no results
    CK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
    h->h_cand.clear();
    h->h_cand_off.clear();
    h->ncand = h->npass = h->nmap = 0;
    h->acc_valid = false;
    h->ngroups = 1;
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
    qrec_score_fields(h, q, h->h_qrec.data());
    for (int r = 0; r < Lq; r++) {
        float* rr = h->h_qrec.data() + (size_t)r * QR_STRIDE;
        trn_of(q, 0, r, rr + QR_TRN);
        rr[QR_C + 0] = cMI[r]; rr[QR_C + 1] = cIM[r]; rr[QR_C + 2] = cDN[r];
        if (r > 0) { rr[QR_CP + 0] = cMI[r - 1]; rr[QR_CP + 1] = cIM[r - 1]; rr[QR_CP + 2] = cDN[r - 1]; }
    }
    if (h->d_qrec.ensure(h->h_qrec.size(), h->budget) || h->d_qbkg.ensure(NAA, h->budget))
        return fail(h, C2_ERR_NOMEM, "query allocation failed");
    // tensor-core query operands (layouts in c2_device.cuh): context vectors
    // (k = 19: 1, the 1/kappa0 column) and SS row tables
    // U[r][c] = sum_s p_q(s) T[idx_q(s)][c] (k = 30: P(H) + 0.1, k = 31: 1) as
    // split BF16 A fragments, amino-acid rows unscaled in fragment order
    {
        const int ns = (Lq + 31) / 32;
        const int card = h->sc.ssss_card;
        std::vector<float> U((size_t)Lq * 32, 0.f);
        for (int r = 0; r < Lq; r++) {
            const float* s3 = q->ss + (size_t)r * NSS;
            const int i0 = (int)(s3[0] * 9.999f), i1 = 10 + (int)(s3[1] * 9.999f), i2 = 20 + (int)(s3[2] * 9.999f);
            for (int c = 0; c < card; c++)
                U[(size_t)r * 32 + c] = s3[0] * h->ssss[(size_t)i0 * card + c] + s3[1] * h->ssss[(size_t)i1 * card + c] +
                                        s3[2] * h->ssss[(size_t)i2 * card + c];
        }
        // the same tables per strip, [strip][MAX_SSSS_CARD][32] (lane = row), for
        // the FP32 kernels
        {
            std::vector<float> qU((size_t)ns * MAX_SSSS_CARD * 32, 0.f);
            for (int r = 0; r < Lq; r++)
                for (int c = 0; c < card; c++)
                    qU[((size_t)(r / 32) * MAX_SSSS_CARD + c) * 32 + (r % 32)] = U[(size_t)r * 32 + c];
            if (h->d_qU.ensure(qU.size(), h->budget)) return fail(h, C2_ERR_NOMEM, "query SS table allocation failed");
            CK(cudaMemcpyAsync(h->d_qU.p, qU.data(), qU.size() * 4, cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        auto aval = [&](int d, int r, int k) -> float {
            if (r >= Lq) return 0.f;
            if (d == 0) return k < NCV ? q->cv[(size_t)r * NCV + k] : (k == NCV ? 1.f : 0.f);
            if (k == TC_SS_KMAX) return h->h_qrec[(size_t)r * QR_STRIDE + QR_HQ];
            if (k == TC_SS_KMAX + 1) return 1.f;
            return k < card ? U[(size_t)r * 32 + k] : 0.f;
        };
        std::vector<uint32_t> qa((size_t)ns * TC_QA_WORDS, 0u);
        std::vector<float> qaa((size_t)ns * TC_QAA_FLOATS, 0.f);
        for (int s = 0; s < ns; s++)
            for (int mt = 0; mt < 2; mt++)
                for (int kt = 0; kt < 2; kt++)
                    for (int lane = 0; lane < 32; lane++) {
                        const int g = lane >> 2, qq = lane & 3;
                        for (int d = 0; d < 2; d++)
                            for (int w = 0; w < 4; w++) {
                                const int r = 32 * s + 16 * mt + g + ((w & 1) ? 8 : 0);
                                const int k = 16 * kt + 2 * qq + ((w >> 1) ? 8 : 0);
                                const float x0 = aval(d, r, k), x1 = aval(d, r, k + 1);
                                const uint32_t h0 = bf16_rn_bits(x0), h1 = bf16_rn_bits(x1);
                                const uint32_t l0 = bf16_rn_bits(x0 - bf16_to_f(h0));
                                const uint32_t l1 = bf16_rn_bits(x1 - bf16_to_f(h1));
                                const size_t base = (size_t)(((s * 2 + mt) * 2 + d) * 2 + kt) * 2;
                                qa[((base + 0) * 32 + lane) * 4 + w] = h0 | (h1 << 16);
                                qa[((base + 1) * 32 + lane) * 4 + w] = l0 | (l1 << 16);
                            }
                        for (int e = 0; e < 8; e++) {
                            const int r = 32 * s + 16 * mt + g + (((e >> 1) & 1) << 3);
                            const int k = 16 * kt + 2 * qq + (e & 1) + ((e >> 2) << 3);
                            qaa[((size_t)((s * 2 + mt) * 2 + kt) * 32 + lane) * 8 + e] =
                                (r < Lq && k < NAA) ? q->trg[(size_t)r * NAA + k] : 0.f;
                        }
                    }
        if (h->d_qa.ensure(qa.size(), h->budget) || h->d_qaaf.ensure(qaa.size(), h->budget))
            return fail(h, C2_ERR_NOMEM, "query operand allocation failed");
        CK(cudaMemcpyAsync(h->d_qa.p, qa.data(), qa.size() * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_qaaf.p, qaa.data(), qaa.size() * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaMemcpyAsync(h->d_qrec.p, h->h_qrec.data(), h->h_qrec.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_qbkg.p, q->bkg, NAA * 4, cudaMemcpyHostToDevice, h->stream));
    // MAP forward: column -1 states of the query rows (log-sum-exp form of the
    // Viterbi boundary; src/libmycu/cumapdp/CuBatchMAPDP_fwd.cu:72-478)
    {
        std::vector<float> qcf((size_t)Lq * 6, 0.f);
        float pMI = 0.f, pIM = 0.f, pDN = 0.f;
        for (int r = 0; r < Lq; r++) {
            float t[7];
            trn_of(q, 0, r, t);
            const float L0 = -99.f;
            float uMM = 0.f, uMI = L0, uDN = L0;
            if (r % 32 != 0) { uMI = pMI; uDN = pDN; }
            const float mi = host_lse2((uMM + t[TMM]) + L0, (uMI + t[TMM]) + L0);
            float im;
            if (r % 32 == 0) im = host_lse2((0.f + t[TMI]) + L0, (L0 + t[TII]) + L0);
            else im = host_lse2((0.f + t[TMI]) + L0, ((((0.f + t[TMI]) + L0) + t[TII]) + L0));
            const float dn = host_lse2(uMM + t[TMD], uDN + t[TDD]);
            float* c = qcf.data() + (size_t)r * 6;
            c[0] = mi; c[1] = im; c[2] = dn;
            c[3] = pMI; c[4] = pIM; c[5] = pDN;
            pMI = mi; pIM = im; pDN = dn;
        }
        if (h->d_qcf.ensure(qcf.size(), h->budget) || h->d_qtrn.ensure((size_t)(Lq + 1) * 7, h->budget) || h->d_qaa.ensure(Lq, h->budget) ||
            h->d_qss.ensure(Lq, h->budget))
            return fail(h, C2_ERR_NOMEM, "query side arrays allocation failed");
        CK(cudaMemcpyAsync(h->d_qcf.p, qcf.data(), qcf.size() * 4, cudaMemcpyHostToDevice, h->stream));
        // the same column -1 states with exact exp/log, for the log-partition model
        std::vector<float> qx((size_t)Lq * 6, 0.f);
        colm1_exact(q, qx.data());
        if (h->d_qcfx.ensure(qx.size(), h->budget)) return fail(h, C2_ERR_NOMEM, "query side arrays allocation failed");
        CK(cudaMemcpyAsync(h->d_qcfx.p, qx.data(), qx.size() * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->adj_fwd_done = false;
        CK(cudaMemcpyAsync(h->d_qtrn.p, q->trn, (size_t)(Lq + 1) * 7 * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_qaa.p, q->aa, (size_t)Lq, cudaMemcpyHostToDevice, h->stream));
        if (q->ssstate) CK(cudaMemcpyAsync(h->d_qss.p, q->ssstate, (size_t)Lq, cudaMemcpyHostToDevice, h->stream));
        else CK(cudaMemsetAsync(h->d_qss.p, ' ', (size_t)Lq, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    query_limits(h, Lq, &h->searchspace, &h->deltalen, &h->scorethld, &h->logevthld);
    return C2_OK;
}

extern "C" c2_status c2_get_query_limits(const c2_handle* h, int32_t query_length, uint64_t* searchspace,
                                         uint64_t* deltalen, float* score_threshold, float* logE_threshold)
{
    if (!h || query_length <= 0 || !searchspace || !deltalen || !score_threshold || !logE_threshold)
        return C2_ERR_ARG;
    if (h->nprof <= 0) return C2_ERR_STATE;
    unsigned long long ss = 0, dl = 0;
    query_limits(h, query_length, &ss, &dl, score_threshold, logE_threshold);
    *searchspace = ss;
    *deltalen = dl;
    return C2_OK;
}

extern "C" c2_status c2_get_thresholds(const c2_handle* h, float* s, float* le)
{
    if (!h || !s || !le) return C2_ERR_ARG;
    *s = h->scorethld;
    *le = h->logevthld;
    return C2_OK;
}

// Epilogue constants of the tensor-core form (TcConsts in c2_device.cuh)
static TcConsts tc_consts(const ScoreConsts& sc)
{
    TcConsts t;
    t.shift = sc.shift;
    t.p2l = 2.f * sc.pownu0 * 0.693147180559945309f;
    t.c2 = 2.f * sc.cterm;
    t.kf2 = 2.f * sc.cvkey_first;
    t.kl2 = 2.f * sc.cvkey_last;
    t.vfw = sc.cvval_first * sc.cvswgt;
    t.vlw = sc.cvval_last * sc.cvswgt;
    t.ilo = -sc.cvshift;
    t.ihi = sc.cvcard - 1 - sc.cvshift;
    // x <= 2 key_first gives index <= 0 and x >= 2 key_last index >= card - 1
    // when the keys sit at the table's ends: the clamp alone is exact then
    t.uniform = (sc.cvshift + (int)rintf(t.kf2) <= 0 && sc.cvshift + (int)rintf(t.kl2) >= sc.cvcard - 1) ? 1 : 0;
    return t;
}

// Pack the db operands of the tensor-core path (once per database).
static c2_status tc_prepare_db(c2_handle* h)
{
    std::lock_guard<std::mutex> lk(h->db->tc_mu);
    if (h->db->tc_ready) return C2_OK;
    std::vector<long long> tt(h->nprof);
    long long ntiles = 0;
    for (int k = 0; k < h->nprof; k++) {
        tt[k] = ntiles;
        ntiles += (long long)((h->h_plen[k] + 31) / 32) * 4;
    }
    if (h->db->d_ttile.ensure(h->nprof, h->budget) || h->db->d_tcdb.ensure((size_t)ntiles * TC_TILE_WORDS, h->budget) ||
        h->db->d_cold.ensure((size_t)h->npos * P1C_TRS, h->budget))
        return fail(h, C2_ERR_NOMEM, "tensor-core db operands (%lld tiles) allocation failed", ntiles);
    CK(cudaMemcpyAsync(h->db->d_ttile.p, tt.data(), (size_t)h->nprof * 8, cudaMemcpyHostToDevice, h->stream));
    CK(launch_tc_pack(h->db->d_drec.p, h->db->d_poff.p, h->db->d_plen.p, h->db->d_ttile.p, h->nprof, h->db->d_tcdb.p, h->db->d_cold.p,
                      h->sc.lokappa0, h->sc.ssswgt, h->stream));
    h->launches++;
    CK(cudaStreamSynchronize(h->stream));
    h->db->tc_ready = true;
    return C2_OK;
}

extern "C" c2_status c2_set_score_mode(c2_handle* h, int32_t mode)
{
    if (!h) return C2_ERR_ARG;
    if (mode != C2_SCORE_FP32 && mode != C2_SCORE_BF16_TC) return fail(h, C2_ERR_ARG, "unknown score mode %d", mode);
    if (mode == C2_SCORE_BF16_TC) {
        // the SS constants ride in K columns 30 and 31, and dropping the
        // reference's "-99 < ss" guard needs table entries well above -99
        if (h->sc.ssss_card > TC_SS_KMAX)
            return fail(h, C2_ERR_ARG, "tensor-core score form needs an SS table of at most %d states", TC_SS_KMAX);
        for (float v : h->ssss)
            if (!(v >= SS_FOLD_MIN))
                return fail(h, C2_ERR_ARG, "tensor-core score form needs SS table entries >= %g", (double)SS_FOLD_MIN);
        if (h->sc.cvcard > P1T_MAX_CVCARD)
            return fail(h, C2_ERR_ARG, "tensor-core score form holds CV maps of at most %d entries (this one: %d)",
                        P1T_MAX_CVCARD, h->sc.cvcard);
    }
    h->score_mode = mode;
    return C2_OK;
}

static void fill_p1(c2_handle* h, P1Args& a)
{
    memset(&a, 0, sizeof a);
    a.qrec = h->d_qrec.p;
    a.Lq = h->Lq;
    a.drec = h->db->d_drec.p;
    a.plen = h->db->d_plen.p;
    a.poff = h->db->d_poff.p;
    a.pbkg = h->db->d_pbkg.p;
    a.counter = h->d_counter.p;
    a.ssss = h->d_ssss.p;
    a.cvvals = h->d_cvvals.p;
    a.qU = h->d_qU.p;
    a.sc = h->sc;
    a.bot = h->d_bot.p;
    a.botstride = h->botstride;
    a.best = h->d_best.p;
    a.coords = h->d_coords.p;
    a.status = h->d_status.p;
    a.spin = h->spin;
}

extern "C" c2_status c2_run_phase1(c2_handle* h)
{
    if (!h) return C2_ERR_ARG;
    if (h->nprof <= 0 || h->Lq <= 0) return fail(h, C2_ERR_STATE, "run_phase1 needs a database and a query");
    CK(cudaSetDevice(h->device));
    P1Args a;
    fill_p1(h, a);
    a.nwork = h->nprof;
    a.order = h->db->d_order.p;
    CK(cudaMemsetAsync(h->d_counter.p, 0, sizeof(int), h->stream));
    if (h->score_mode == C2_SCORE_BF16_TC) {
        c2_status st = tc_prepare_db(h);
        if (st != C2_OK) return st;
        a.tcdb = h->db->d_tcdb.p;
        a.ttile = h->db->d_ttile.p;
        a.cold = h->db->d_cold.p;
        a.qa = h->d_qa.p;
        a.qaa = h->d_qaaf.p;
        a.tc = tc_consts(h->sc);
        cudaError_t oe = cudaSuccess;
        int gt = (h->nsm - h->p1_reserve) * p1t_blocks_per_sm(h->sc.cvcard, &oe);
        if (gt < 1)
            return fail(h, C2_ERR_CUDA, "tensor-core phase-1 kernel does not fit on an SM (%s)",
                        cudaGetErrorString(oe));
        gt = std::min(gt, h->grid * P1_WARPS / P1T_WARPS);
        CK(launch_p1(a, h->d_qbkg.p, P1K_TENSOR, gt, h->stream));
        h->launches++;
        return C2_OK;
    }
    // chunked kernel: one CTA of P1C_WARPS warps per SM, within the boundary-row slots
    // allocated for the strip kernel's grid (h->grid x P1_WARPS)
    int gc = (h->nsm - h->p1_reserve) * p1c_blocks_per_sm(h->sc.cvcard);
    if (gc < 1) return fail(h, C2_ERR_CUDA, "phase-1 kernel does not fit on an SM");
    gc = std::min(gc, h->grid * P1_WARPS / P1C_WARPS);
    CK(launch_p1(a, h->d_qbkg.p, P1K_CHUNKED, gc, h->stream));
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

extern "C" c2_status c2_set_device_memory_limit(c2_handle* h, uint64_t bytes)
{
    if (!h) return C2_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->budget->mu);
    h->budget->limit = (size_t)bytes;
    return C2_OK;
}

extern "C" c2_status c2_get_device_memory_use(const c2_handle* h, uint64_t* bytes)
{
    if (!h || !bytes) return C2_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->budget->mu);
    *bytes = h->budget->used;
    return C2_OK;
}

extern "C" c2_status c2_get_device_count(int32_t* count)
{
    if (!count) return C2_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        (void)cudaGetLastError();
        n = 0;
    }
    *count = n;
    return C2_OK;
}

extern "C" c2_status c2_get_device_memory_info(const c2_handle* h, uint64_t* free_bytes, uint64_t* total_bytes)
{
    if (!h || !free_bytes || !total_bytes) return C2_ERR_ARG;
    if (cudaSetDevice(h->device) != cudaSuccess) return C2_ERR_CUDA;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return C2_ERR_CUDA;
    *free_bytes = fr;
    *total_bytes = tot;
    return C2_OK;
}

// Device bytes of a database upload of this size and of the per-profile
// phase-1 buffers that come with it: the c2_upload_db allocations, and in the
// tensor-core score mode the operands tc_prepare_db packs (at most
// ceil(L / 32) * 4 tiles a profile, i.e. npositions / 8 + 4 nprofiles).
extern "C" c2_status c2_db_device_bytes(const c2_handle* h, int64_t npositions, int32_t nprofiles, int32_t max_length,
                                        uint64_t* bytes)
{
    if (!h || !bytes || npositions < 0 || nprofiles < 0 || max_length < 0) return C2_ERR_ARG;
    const uint64_t N = (uint64_t)npositions, P = (uint64_t)nprofiles;
    uint64_t b = N * DR_STRIDE * sizeof(float)                 // d_drec
                 + P * NAA * sizeof(float)                     // d_pbkg
                 + P * (sizeof(int) * 2 + sizeof(long long))   // d_plen, d_order, d_poff
                 + P * (sizeof(float) + sizeof(unsigned))      // d_best, d_coords
                 + (N + P) * 7 * sizeof(float)                 // d_dtrn
                 + N * 2                                        // d_daa, d_dss
                 + P * sizeof(float);                           // d_peno
    const uint64_t lm = ((uint64_t)max_length + 31) & ~31ull;
    b += (uint64_t)h->grid * P1_WARPS * 10 * lm * sizeof(float);   // d_bot
    if (h->score_mode == C2_SCORE_BF16_TC) {
        const uint64_t ntiles = N / 8 + 4 * P;
        b += P * sizeof(long long) + ntiles * TC_TILE_WORDS * sizeof(unsigned) + N * P1C_TRS * sizeof(float);
    }
    *bytes = b;
    return C2_OK;
}

extern "C" c2_status c2_set_wait_limit(c2_handle* h, uint32_t polls)
{
    if (!h) return C2_ERR_ARG;
    h->spin = polls ? polls : PIPE_SPIN;
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

// Pairs whose phase-1 maximum passes the candidate cut, ascending profile
// order.  FinalizeDPPro: maxsc <= scorethld -> not passed.  With BF16 phase-1
// scores the cut is lowered by a margin far above their error; the FP32
// traceback sweep then applies the exact cut (fin_kernel).
static c2_status select_candidates(c2_handle* h, std::vector<int>& cand)
{
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float> b(h->nprof);
    CK(cudaMemcpy(b.data(), h->d_best.p, (size_t)h->nprof * 4, cudaMemcpyDeviceToHost));
    const float cut = (h->score_mode == C2_SCORE_FP32)
                          ? h->scorethld
                          : h->scorethld - C2_TC_MARGIN * std::max(1.0f, std::fabs(h->scorethld));
    cand.clear();
    for (int k = 0; k < h->nprof; k++)
        if (b[k] > cut) cand.push_back(k);
    return C2_OK;
}

// Traceback sweep and finalisation of the candidate pairs `cand` (ascending
// profile order).
static c2_status finalize_set(c2_handle* h, const std::vector<int>& cand, int32_t* ncand)
{
    h->h_cand = cand;
    h->h_cand_off.clear();
    long long acc = 0;
    for (int k : cand) {
        h->h_cand_off.push_back(acc);
        acc += (long long)h->Lq * h->h_plen[k];
    }
    h->ncand = (int)h->h_cand.size();
    *ncand = h->ncand;
    if (h->ncand == 0) return C2_OK;
    const int nc = h->ncand;
    // strip-pipeline scratch: two halves, the second for the MAP backward sweep
    h->bnd_half = (size_t)(acc / h->Lq) * 10;
    h->prog_half = (size_t)nc * ((h->Lq + 31) / 32);
    if (h->d_cand_prof.ensure(nc, h->budget) || h->d_cand_off.ensure(nc, h->budget) || h->d_btck.ensure((size_t)acc, h->budget) ||
        h->d_smat.ensure((size_t)acc, h->budget) || h->d_mmat.ensure((size_t)acc, h->budget) || h->d_fscore.ensure(nc, h->budget) || h->d_fpsts.ensure(nc, h->budget) ||
        h->d_fpassed.ensure(nc, h->budget) || h->d_fbeg.ensure(nc, h->budget) || h->d_fend.ensure(nc, h->budget) ||
        h->d_bnd.ensure(2 * h->bnd_half, h->budget) || h->d_tbkey.ensure(nc, h->budget) || h->d_prog.ensure(2 * h->prog_half, h->budget))
        return fail(h, C2_ERR_NOMEM, "finalisation scratch for %d pairs (%lld cells) failed", nc, acc);
    CK(cudaMemcpyAsync(h->d_cand_prof.p, h->h_cand.data(), (size_t)nc * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_cand_off.p, h->h_cand_off.data(), (size_t)nc * 8, cudaMemcpyHostToDevice, h->stream));
    // traceback sweep order: longest candidates first
    {
        std::vector<int> wo(nc);
        std::iota(wo.begin(), wo.end(), 0);
        std::stable_sort(wo.begin(), wo.end(),
                         [&](int x, int y) { return h->h_plen[h->h_cand[x]] > h->h_plen[h->h_cand[y]]; });
        std::vector<int> lens(nc), items;
        for (int i = 0; i < nc; i++) lens[i] = h->h_plen[h->h_cand[wo[i]]];
        strip_items(lens, (h->Lq + 31) / 32, h->nsm * P1TC_WARPS, STRIP_LAG_TB, items);
        if (h->d_worder.ensure(nc, h->budget) || h->d_tbitems.ensure(items.size(), h->budget))
            return fail(h, C2_ERR_NOMEM, "candidate order allocation failed");
        CK(cudaMemcpyAsync(h->d_worder.p, wo.data(), (size_t)nc * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_tbitems.p, items.data(), items.size() * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    P1Args a;
    fill_p1(h, a);
    a.nwork = nc;
    a.order = h->d_cand_prof.p;
    a.cand_off = h->d_cand_off.p;
    a.btck = h->d_btck.p;
    a.smat = h->d_smat.p;
    a.mmat = h->d_mmat.p;
    a.bnd = h->d_bnd.p;
    a.prog = h->d_prog.p;
    a.tbkey = h->d_tbkey.p;
    a.worder = h->d_worder.p;
    a.items = h->d_tbitems.p;
    const long long nitems = (long long)nc * ((h->Lq + 31) / 32);
    CK(cudaMemsetAsync(h->d_counter.p, 0, 2 * sizeof(int), h->stream));   // the sweep's and the score kernel's
    CK(cudaMemsetAsync(h->d_prog.p, 0, (size_t)nitems * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_tbkey.p, 0, (size_t)nc * sizeof(unsigned long long), h->stream));
    // one CTA of P1TC_WARPS warps per SM, one warp per (candidate, strip) work item at most
    const int grid = (int)std::min<long long>(h->nsm, (nitems + P1TC_WARPS - 1) / P1TC_WARPS);
    CK(launch_p1(a, h->d_qbkg.p, P1K_TRACEBACK, grid, h->stream));   // p2s_kernel, then p1tc_kernel
    h->launches += 2;
    FinArgs f;
    f.Lq = h->Lq;
    f.ncand = nc;
    f.cand_prof = h->d_cand_prof.p;
    f.cand_off = h->d_cand_off.p;
    f.plen = h->db->d_plen.p;
    f.btck = h->d_btck.p;
    f.smat = h->d_smat.p;
    f.best = h->d_best.p;
    f.coords = h->d_coords.p;
    f.scorethld = h->scorethld;
    f.tbkey = h->d_tbkey.p;
    // BF16 phase-1 maxima differ from the FP32 traceback sweep by rounding only
    f.tol = (h->score_mode == C2_SCORE_FP32) ? 0.f : C2_TC_TOL;
    f.status = h->d_status.p;
    f.score = h->d_fscore.p;
    f.psts = h->d_fpsts.p;
    f.beg = h->d_fbeg.p;
    f.endc = h->d_fend.p;
    f.passed = h->d_fpassed.p;
    CK(launch_fin(f, h->stream));
    h->launches++;
    return C2_OK;
}

extern "C" c2_status c2_run_finalize(c2_handle* h, int32_t* ncand)
{
    if (!h || !ncand) return C2_ERR_ARG;
    if (h->nprof <= 0 || h->Lq <= 0) return fail(h, C2_ERR_STATE, "run_finalize needs a database and a query");
    h->acc_valid = false;
    std::vector<int> cand;
    c2_status st = select_candidates(h, cand);
    if (st != C2_OK) return st;
    return finalize_set(h, cand, ncand);
}

extern "C" c2_status c2_get_finalize(c2_handle* h, c2_dp_result* out, int32_t n)
{
    if (!h || (!out && n > 0) || n < h->ncand) return C2_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    int stw = 0;
    CK(cudaMemcpy(&stw, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (stw != 0) return fail(h, C2_ERR_DEVICE, "device status %d (%s)", stw, status_text(stw));
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

// The FP32 score and modular-score matrices of one candidate pair, as the
// traceback sweep of c2_run_finalize stored them (column-major [L][Lq] on the
// device), copied out row-major [Lq][L].
extern "C" c2_status c2_get_pair_scores(c2_handle* h, int32_t profile, float* scores, float* modscores)
{
    if (!h || (!scores && !modscores)) return C2_ERR_ARG;
    const auto it = std::lower_bound(h->h_cand.begin(), h->h_cand.end(), profile);
    if (it == h->h_cand.end() || *it != profile)
        return fail(h, C2_ERR_ARG, "get_pair_scores: profile %d is not a candidate of the current query", profile);
    const size_t c = (size_t)(it - h->h_cand.begin());
    const int Lq = h->Lq, L = h->h_plen[profile];
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float> col((size_t)Lq * L);
    for (int w = 0; w < 2; w++) {
        float* out = w ? modscores : scores;
        if (!out) continue;
        const float* src = (w ? h->d_mmat.p : h->d_smat.p) + h->h_cand_off[c];
        CK(cudaMemcpy(col.data(), src, col.size() * 4, cudaMemcpyDeviceToHost));
        for (int x = 0; x < L; x++)
            for (int y = 0; y < Lq; y++) out[(size_t)y * L + x] = col[(size_t)x * Lq + y];
    }
    return C2_OK;
}

extern "C" c2_status c2_launch_count(const c2_handle* h, uint64_t* n)
{
    if (!h || !n) return C2_ERR_ARG;
    *n = h->launches;
    return C2_OK;
}

extern "C" c2_status c2_get_search_space(const c2_handle* h, uint64_t* ss, uint64_t* dl)
{
    if (!h || !ss || !dl) return C2_ERR_ARG;
    *ss = h->searchspace;
    *dl = h->deltalen;
    return C2_OK;
}

extern "C" c2_status c2_run_stats(c2_handle* h, int32_t* npassed)
{
    if (!h || !npassed) return C2_ERR_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    int stw = 0;
    CK(cudaMemcpy(&stw, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (stw != 0) return fail(h, C2_ERR_DEVICE, "device status %d (%s)", stw, status_text(stw));
    const int nc = h->ncand;
    h->h_p2.clear();
    h->h_fscore.assign(nc, 0.f);
    h->h_fpassed.assign(nc, 0);
    if (nc > 0) {
        CK(cudaMemcpy(h->h_fpassed.data(), h->d_fpassed.p, (size_t)nc * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(h->h_fscore.data(), h->d_fscore.p, (size_t)nc * 4, cudaMemcpyDeviceToHost));
    }
    for (int c = 0; c < nc; c++)
        if (h->h_fpassed[c]) h->h_p2.push_back(c);
    h->npass = (int)h->h_p2.size();
    *npassed = h->npass;
    if (h->npass == 0) return C2_OK;
    if (h->d_p2.ensure(h->npass, h->budget) || h->d_stats.ensure((size_t)h->npass * STATS_NOUT, h->budget))
        return fail(h, C2_ERR_NOMEM, "statistics buffers for %d pairs failed", h->npass);
    CK(cudaMemcpyAsync(h->d_p2.p, h->h_p2.data(), (size_t)h->npass * 4, cudaMemcpyHostToDevice, h->stream));
    StatsArgs a;
    memset(&a, 0, sizeof a);
    a.Lq = h->Lq;
    a.npass = h->npass;
    a.p2_cand = h->d_p2.p;
    a.cand_prof = h->d_cand_prof.p;
    a.cand_off = h->d_cand_off.p;
    a.plen = h->db->d_plen.p;
    a.poff = h->db->d_poff.p;
    a.peno = h->db->d_peno.p;
    a.qaa = h->d_qaa.p;
    a.daa = h->db->d_daa.p;
    a.smat = h->d_smat.p;
    a.fscore = h->d_fscore.p;
    a.fpsts = h->d_fpsts.p;
    a.nnw = h->d_nnw.p;
    a.ssemodel = h->prm.ssemodel;
    a.xuninf = h->prm.x_uninf;
    a.qeno = h->qeno;
    a.searchspace = (float)h->searchspace;
    a.reflambda = h->prm.ungapped_lambda;
    a.refK = h->prm.ungapped_K;
    a.expglambda = h->prm.gapped_lambda;
    a.expgK = h->prm.gapped_K;
    a.out = h->d_stats.p;
    if (!a.nnw || h->nnw.size() < 93) return fail(h, C2_ERR_ARG, "SS18 model weights missing (93 values needed)");
    CK(launch_stats(a, h->stream));
    h->launches++;
    return C2_OK;
}

// MAPALN 0: the hits' alignments are the Viterbi DP's own (FinalizeDP_ALN,
// src/libmycu/cudp/CuBatchDP_aln_final.cu:61-360): the walk from each pair's
// DP maximum through the traceback codes of the finalisation sweep, which no
// MAP sweep has overwritten.
static c2_status viterbi_alignments(c2_handle* h)
{
    const int nm = h->nmap;
    if (h->d_mapcand.ensure(nm, h->budget) || h->d_mappass.ensure(nm, h->budget) ||
        h->d_pairf.ensure((size_t)nm * 4, h->budget) || h->d_pairc.ensure(nm, h->budget) ||
        h->d_alninfo.ensure((size_t)nm * 8, h->budget) || h->d_aln.ensure((size_t)nm * 5 * h->alnstride, h->budget) ||
        h->d_pairk.ensure(nm, h->budget))
        return fail(h, C2_ERR_NOMEM, "alignment buffers for %d pairs failed", nm);
    // each pair's DP maximum and end cell in the MAP DP's key form
    std::vector<unsigned> fend(h->ncand);
    std::vector<unsigned long long> key(nm);
    CK(cudaMemcpy(fend.data(), h->d_fend.p, (size_t)h->ncand * 4, cudaMemcpyDeviceToHost));
    for (int m = 0; m < nm; m++) {
        const int c = h->h_mapcand[m];
        const unsigned xx = fend[c];   // (x << 16) | y
        const unsigned cell = ((xx & 0xffffu) << 16) | (xx >> 16);
        float sc = h->h_fscore[c];
        unsigned bits;
        memcpy(&bits, &sc, 4);
        key[m] = ((unsigned long long)bits << 32) | (unsigned long long)(0xffffffffu - cell);
    }
    CK(cudaMemcpyAsync(h->d_pairk.p, key.data(), (size_t)nm * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_mapcand.p, h->h_mapcand.data(), (size_t)nm * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_mappass.p, h->h_mappass.data(), (size_t)nm * 4, cudaMemcpyHostToDevice, h->stream));
    MapArgs a;
    memset(&a, 0, sizeof a);
    a.Lq = h->Lq;
    a.nmap = nm;
    a.map_cand = h->d_mapcand.p;
    a.map_pass = h->d_mappass.p;
    a.cand_prof = h->d_cand_prof.p;
    a.cand_off = h->d_cand_off.p;
    a.plen = h->db->d_plen.p;
    a.poff = h->db->d_poff.p;
    a.smat = h->d_smat.p;
    a.btck = h->d_btck.p;
    a.pairf = h->d_pairf.p;
    a.pairc = h->d_pairc.p;
    a.pairk = h->d_pairk.p;
    a.status = h->d_status.p;
    a.qaa = h->d_qaa.p;
    a.qss = h->d_qss.p;
    a.daa = h->db->d_daa.p;
    a.dss = h->db->d_dss.p;
    a.aln_info = h->d_alninfo.p;
    a.aln = h->d_aln.p;
    a.alnstride = h->alnstride;
    CK(launch_viterbi_aln(a, h->stream));
    h->launches++;
    return C2_OK;
}

extern "C" c2_status c2_run_map(c2_handle* h, int32_t* nhits)
{
    if (!h || !nhits) return C2_ERR_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    h->h_stats.assign((size_t)h->npass * STATS_NOUT, 0.f);
    if (h->npass > 0)
        CK(cudaMemcpy(h->h_stats.data(), h->d_stats.p, h->h_stats.size() * 4, cudaMemcpyDeviceToHost));
    h->h_mapcand.clear();
    h->h_mappass.clear();
    for (int i = 0; i < h->npass; i++)
        if (!(h->logevthld < h->h_stats[(size_t)i * STATS_NOUT + ST_LOGE])) {  // MAP stage skips logE > threshold
            h->h_mapcand.push_back(h->h_p2[i]);
            h->h_mappass.push_back(i);
        }
    {
        // longest pairs first: their strip chains are the longest
        std::vector<int> ix(h->h_mapcand.size());
        std::iota(ix.begin(), ix.end(), 0);
        std::stable_sort(ix.begin(), ix.end(), [&](int x, int y) {
            return h->h_plen[h->h_cand[h->h_mapcand[x]]] > h->h_plen[h->h_cand[h->h_mapcand[y]]];
        });
        std::vector<int> mc(ix.size()), mp(ix.size());
        for (size_t i = 0; i < ix.size(); i++) { mc[i] = h->h_mapcand[ix[i]]; mp[i] = h->h_mappass[ix[i]]; }
        h->h_mapcand.swap(mc);
        h->h_mappass.swap(mp);
    }
    h->nmap = (int)h->h_mapcand.size();
    *nhits = h->nmap;
    if (h->nmap == 0) return C2_OK;
    const int nm = h->nmap;
    long long cells = 0;
    for (int c : h->h_mapcand) cells += (long long)h->Lq * h->h_plen[h->h_cand[c]];
    (void)cells;
    h->alnstride = h->Lq + h->Lmax + 1;
    if (h->prm.mapaln == 0) return viterbi_alignments(h);
    // F and B in wavefront order: [nstrips][L + 31][32] per candidate, at
    // 32 nstrips (sum of (L + 31) over the candidates before it)
    long long skl = 0;
    for (int c = 0; c < h->ncand; c++) skl += (long long)h->h_plen[h->h_cand[c]] + 31;
    const size_t fbn = (size_t)32 * ((h->Lq + 31) / 32) * (size_t)skl;
    if (h->d_mapcand.ensure(nm, h->budget) || h->d_mappass.ensure(nm, h->budget) || h->d_fb.ensure(fbn, h->budget) || h->d_bb.ensure(fbn, h->budget) ||
        h->d_pairf.ensure((size_t)nm * 4, h->budget) ||
        h->d_pairc.ensure(nm, h->budget) || h->d_alninfo.ensure((size_t)nm * 8, h->budget) || h->d_aln.ensure((size_t)nm * 5 * h->alnstride, h->budget) ||
        h->d_pairk.ensure(nm, h->budget))
        return fail(h, C2_ERR_NOMEM, "MAP buffers for %d pairs failed", nm);
    {
        std::vector<int> lens(nm), items;
        for (int i = 0; i < nm; i++) lens[i] = h->h_plen[h->h_cand[h->h_mapcand[i]]];
        strip_items(lens, (h->Lq + 31) / 32, h->grid * P1_WARPS, STRIP_LAG_MAP, items);
        if (h->d_mapitems.ensure(items.size(), h->budget)) return fail(h, C2_ERR_NOMEM, "MAP work table allocation failed");
        CK(cudaMemcpyAsync(h->d_mapitems.p, items.data(), items.size() * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaMemcpyAsync(h->d_mapcand.p, h->h_mapcand.data(), (size_t)nm * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_mappass.p, h->h_mappass.data(), (size_t)nm * 4, cudaMemcpyHostToDevice, h->stream));
    MapArgs a;
    memset(&a, 0, sizeof a);
    a.Lq = h->Lq;
    a.nmap = nm;
    a.map_cand = h->d_mapcand.p;
    a.map_pass = h->d_mappass.p;
    a.cand_prof = h->d_cand_prof.p;
    a.cand_off = h->d_cand_off.p;
    a.plen = h->db->d_plen.p;
    a.poff = h->db->d_poff.p;
    a.smat = h->d_smat.p;
    a.mmat = h->d_mmat.p;
    a.stats = h->d_stats.p;
    a.fb = h->d_fb.p;
    a.bb = h->d_bb.p;
    a.btck = h->d_btck.p;
    a.pairf = h->d_pairf.p;
    a.pairc = h->d_pairc.p;
    a.bnd = h->d_bnd.p;
    a.prog = h->d_prog.p;
    a.bnd_b = h->d_bnd.p + h->bnd_half;   // the backward sweep's halves of the scratch
    a.prog_b = h->d_prog.p + h->prog_half;
    a.pairk = h->d_pairk.p;
    a.items = h->d_mapitems.p;
    a.status = h->d_status.p;
    a.counter = h->d_counter.p;
    a.spin = h->spin;
    a.minpp = h->prm.minpp;
    a.modscores = (h->prm.ssswgt > 0.f || h->prm.cvswgt > 0.f) ? 1 : 0;
    a.qaa = h->d_qaa.p;
    a.qss = h->d_qss.p;
    a.daa = h->db->d_daa.p;
    a.dss = h->db->d_dss.p;
    a.aln_info = h->d_alninfo.p;
    a.aln = h->d_aln.p;
    a.alnstride = h->alnstride;
    int nl = 0;
    CK(launch_map(a, h->d_qtrn.p, h->db->d_dtrn.p, h->d_qcf.p, h->nsm, h->d_counter.p, h->stream, &nl));
    h->launches += nl;
    return C2_OK;
}

static c2_status hits_direct(c2_handle* h, c2_hit* hits, int32_t n, char* alns, size_t* aln_bytes)
{
    CK(cudaStreamSynchronize(h->stream));
    int stw = 0;
    CK(cudaMemcpy(&stw, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (stw != 0) return fail(h, C2_ERR_DEVICE, "device status %d (%s)", stw, status_text(stw));
    const int nm = h->nmap;
    const size_t per = (size_t)5 * h->alnstride;
    std::vector<int> info((size_t)nm * 8);
    if (nm > 0) CK(cudaMemcpy(info.data(), h->d_alninfo.p, info.size() * 4, cudaMemcpyDeviceToHost));
    size_t need = 0;
    for (int m = 0; m < nm; m++) need += (size_t)5 * (info[(size_t)m * 8] + 1);
    if (!alns || !hits) {
        *aln_bytes = need;
        return (hits || alns) ? C2_ERR_ARG : C2_OK;
    }
    if (n < nm || *aln_bytes < need) return fail(h, C2_ERR_ARG, "output buffers too small (%d hits, %zu bytes)", nm, need);
    (void)per;
    std::vector<int> order(nm);
    std::iota(order.begin(), order.end(), 0);
    auto logE = [&](int m) { return h->h_stats[(size_t)h->h_mappass[m] * STATS_NOUT + ST_LOGE]; };
    auto prof = [&](int m) { return h->h_cand[h->h_mapcand[m]]; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const float ex = logE(x), ey = logE(y);
        if (ex != ey) return ex < ey;
        return prof(x) < prof(y);
    });
    // the strings, packed on the device in hit order (only their bytes cross PCIe)
    std::vector<long long> off((size_t)std::max(nm, 1));
    {
        size_t p = 0;
        for (int i = 0; i < nm; i++) {
            off[order[i]] = (long long)p;
            p += (size_t)5 * (info[(size_t)order[i] * 8] + 1);
        }
    }
    if (nm > 0) {
        if (h->d_alnoff.ensure((size_t)nm, h->budget) || h->d_alnpack.ensure(need, h->budget))
            return fail(h, C2_ERR_NOMEM, "alignment packing buffers failed");
        CK(cudaMemcpyAsync(h->d_alnoff.p, off.data(), (size_t)nm * 8, cudaMemcpyHostToDevice, h->stream));
        CK(launch_aln_pack(h->d_aln.p, h->alnstride, h->d_alninfo.p, h->d_alnoff.p, nm, h->d_alnpack.p, h->stream));
        h->launches++;
        CK(cudaMemcpyAsync(alns, h->d_alnpack.p, need, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    size_t pos = 0;
    for (int i = 0; i < nm; i++) {
        const int m = order[i];
        const float* st = &h->h_stats[(size_t)h->h_mappass[m] * STATS_NOUT];
        const int* in = &info[(size_t)m * 8];
        c2_hit& o = hits[i];
        o.profile = prof(m);
        o.score = h->h_fscore[h->h_mapcand[m]];
        o.logE = st[ST_LOGE];
        o.logEpA = st[ST_LOGEPA];
        o.lambda = st[ST_LAMBDA];
        o.K = st[ST_K];
        o.lambda_est = st[ST_LAMBDA_EST];
        o.K_est = st[ST_K_EST];
        o.E = st[ST_E];
        o.H = st[ST_H];
        o.smin = (int32_t)st[ST_MIN];
        o.smax = (int32_t)st[ST_MAX];
        o.alnlen = in[0];
        o.idts = in[1];
        o.psts = in[2];
        o.gaps = in[3];
        o.beg = (uint32_t)in[4];
        o.end = (uint32_t)in[5];
        o.aln_offset = (int64_t)pos;
        pos += (size_t)5 * (in[0] + 1);
    }
    return C2_OK;
}

extern "C" c2_status c2_get_hits(c2_handle* h, c2_hit* hits, int32_t n, char* alns, size_t* aln_bytes)
{
    if (!h || !aln_bytes) return C2_ERR_ARG;
    if (!h->acc_valid) return hits_direct(h, hits, n, alns, aln_bytes);
    const int nm = (int)h->acc_hits.size();
    if (!alns || !hits) {
        *aln_bytes = h->acc_alns.size();
        return (hits || alns) ? C2_ERR_ARG : C2_OK;
    }
    if (n < nm || *aln_bytes < h->acc_alns.size())
        return fail(h, C2_ERR_ARG, "output buffers too small (%d hits, %zu bytes)", nm, h->acc_alns.size());
    std::copy(h->acc_hits.begin(), h->acc_hits.end(), hits);
    std::copy(h->acc_alns.begin(), h->acc_alns.end(), alns);
    return C2_OK;
}

// Phase-2 buffers sized by the candidate pairs (released between groups)
static void release_phase2(c2_handle* h)
{
    h->d_cand_prof.release(); h->d_cand_off.release(); h->d_btck.release(); h->d_smat.release();
    h->d_mmat.release(); h->d_fscore.release(); h->d_fpsts.release(); h->d_fpassed.release();
    h->d_fbeg.release(); h->d_fend.release(); h->d_bnd.release(); h->d_tbkey.release(); h->d_prog.release();
    h->d_worder.release(); h->d_tbitems.release(); h->d_mapitems.release(); h->d_p2.release(); h->d_stats.release();
    h->d_mapcand.release(); h->d_mappass.release(); h->d_alninfo.release(); h->d_fb.release(); h->d_bb.release();
    h->d_pairf.release(); h->d_pairc.release(); h->d_pairk.release(); h->d_aln.release(); h->d_alnpack.release();
    h->d_alnoff.release();
}

// Device bytes phase 2 takes for one candidate pair of db length L: score,
// modular-score and traceback matrices, strip-boundary rows and progress
// words, the MAP sweeps' F and B in wavefront order, the alignment rows, and
// the per-pair records (an upper estimate of the buffers finalize_set,
// c2_run_stats, c2_run_map and c2_get_hits size by the pairs).
static size_t pair_scratch_bytes(const c2_handle* h, int L)
{
    const size_t Lq = (size_t)h->Lq, ns = (Lq + 31) / 32;
    return 9 * Lq * (size_t)L + 2 * 10 * 4 * (size_t)L + 2 * 4 * ns + 4 * ns * 2 + 2 * 4 * 32 * ns * ((size_t)L + 31) +
           2 * 5 * (Lq + (size_t)h->Lmax + 1) + 512;
}

// Candidate groups whose phase-2 scratch fits the handle's device memory
// budget (one group without a budget).  The phase-2 buffers of an earlier
// search are released first, so the budget's use is the fixed part.
static c2_status plan_groups(c2_handle* h, const std::vector<int>& cand, std::vector<std::vector<int>>& groups)
{
    groups.clear();
    size_t limit, used;
    {
        std::lock_guard<std::mutex> lk(h->budget->mu);
        limit = h->budget->limit;
    }
    if (limit == 0 || cand.empty()) {
        groups.push_back(cand);
        return C2_OK;
    }
    release_phase2(h);
    {
        std::lock_guard<std::mutex> lk(h->budget->mu);
        used = h->budget->used;
    }
    const size_t margin = size_t(1) << 20;
    if (used + margin >= limit)
        return fail(h, C2_ERR_NOMEM, "device memory budget of %zu bytes leaves nothing for phase 2 (%zu in use)", limit,
                    used);
    const size_t avail = (limit - used - margin) / 10 * 9;
    std::vector<int> g;
    size_t gb = 0;
    for (int k : cand) {
        const size_t b = pair_scratch_bytes(h, h->h_plen[k]);
        if (b > avail)
            return fail(h, C2_ERR_NOMEM,
                        "device memory budget: the phase-2 scratch of one pair (profile %d, %d x %d cells, %zu bytes) "
                        "exceeds the %zu bytes left",
                        k, h->Lq, h->h_plen[k], b, avail);
        if (gb + b > avail && !g.empty()) {
            groups.push_back(g);
            g.clear();
            gb = 0;
        }
        g.push_back(k);
        gb += b;
    }
    if (!g.empty()) groups.push_back(g);
    return C2_OK;
}

extern "C" c2_status c2_search(c2_handle* h, const c2_profiles* q, int32_t* nhits)
{
    if (!h || !q || !nhits) return C2_ERR_ARG;
    c2_status st;
    int32_t n = 0;
    if ((st = c2_set_query(h, q)) != C2_OK) return st;
    if ((st = c2_run_phase1(h)) != C2_OK) return st;
    std::vector<int> cand;
    if ((st = select_candidates(h, cand)) != C2_OK) return st;
    std::vector<std::vector<int>> groups;
    if ((st = plan_groups(h, cand, groups)) != C2_OK) return st;
    h->ngroups = (int)groups.size();
    if (groups.size() <= 1) {
        if ((st = finalize_set(h, cand, &n)) != C2_OK) return st;
        if ((st = c2_run_stats(h, &n)) != C2_OK) return st;
        return c2_run_map(h, nhits);
    }
    // candidate groups in turn: finalisation, statistics, MAP and the hits
    // of each group to the host, then one list sorted by log E (then profile)
    std::vector<c2_hit> all;
    std::vector<char> aln;
    for (const auto& g : groups) {
        release_phase2(h);
        if ((st = finalize_set(h, g, &n)) != C2_OK) return st;
        if ((st = c2_run_stats(h, &n)) != C2_OK) return st;
        int32_t nm = 0;
        if ((st = c2_run_map(h, &nm)) != C2_OK) return st;
        size_t bytes = 0;
        if ((st = hits_direct(h, nullptr, 0, nullptr, &bytes)) != C2_OK) return st;
        std::vector<c2_hit> hs((size_t)std::max(nm, 1));
        std::vector<char> as(bytes + 1);
        if ((st = hits_direct(h, hs.data(), nm, as.data(), &bytes)) != C2_OK) return st;
        const int64_t base = (int64_t)aln.size();
        for (int i = 0; i < nm; i++) {
            hs[i].aln_offset += base;
            all.push_back(hs[i]);
        }
        aln.insert(aln.end(), as.begin(), as.begin() + (long)bytes);
    }
    release_phase2(h);
    std::vector<int> order(all.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (all[x].logE != all[y].logE) return all[x].logE < all[y].logE;
        return all[x].profile < all[y].profile;
    });
    h->acc_hits.clear();
    h->acc_alns.clear();
    for (int i : order) {
        c2_hit r = all[i];
        const size_t len = (size_t)5 * (r.alnlen + 1);
        r.aln_offset = (int64_t)h->acc_alns.size();
        h->acc_alns.insert(h->acc_alns.end(), aln.begin() + all[i].aln_offset, aln.begin() + all[i].aln_offset + (long)len);
        h->acc_hits.push_back(r);
    }
    h->acc_valid = true;
    *nhits = (int32_t)h->acc_hits.size();
    return C2_OK;
}

extern "C" c2_status c2_get_search_groups(const c2_handle* h, int32_t* ngroups)
{
    if (!h || !ngroups) return C2_ERR_ARG;
    *ngroups = h->ngroups;
    return C2_OK;
}

// ---------------------------------------------------------------------------
// Phase 1 with no allocation (no counterpart in the reference).  The same
// p1_kernel, launched with its per-call scratch -- the work-queue counter and
// the per-warp strip-boundary rows -- taken from a fixed file-scope device
// array instead of handle buffers, and its results written to caller-owned
// device memory.  For hosts that must not allocate at call time (cudaMalloc
// and cudaFree synchronise the device and can fail under memory pressure).
//
// Scratch: C2_STATIC_SCRATCH_BYTES = 16 MiB; bytes [0, 256) hold the work
// counter (zeroed by every call), the rest holds 10 x Lm floats per warp
// slot, Lm being the longest db profile rounded up to a multiple of 32.  The
// grid shrinks to the number of 8-warp blocks whose slots fit; a database
// whose longest profile needs more than the whole array for one block
// (Lm > 52,428, i.e. a longest profile above 52,416 positions) is rejected.
// The kernel scores in FP32 only: a handle in the tensor-core score mode is
// refused rather than given maxima of the other arithmetic.
// Every call on a device shares the one array: calls whose kernels overlap on
// the GPU (different streams, or different handles on one device) race on it.
// The first call on a device resolves the array's address with
// cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture.
namespace {
constexpr size_t C2_STATIC_SCRATCH_BYTES = size_t(16) << 20;
constexpr size_t C2_STATIC_HDR = 256;
constexpr int C2_STATIC_MAXDEV = 64;
__device__ __align__(256) unsigned char c2_static_scratch[C2_STATIC_SCRATCH_BYTES];
void* g_static_scratch[C2_STATIC_MAXDEV] = {};
std::mutex g_static_mu;
}  // namespace

extern "C" c2_status c2_run_phase1_static(c2_handle* h, float* d_best, uint32_t* d_coords)
{
    if (!h || !d_best || !d_coords) return C2_ERR_ARG;
    if (h->nprof <= 0 || h->Lq <= 0) return fail(h, C2_ERR_STATE, "run_phase1_static needs a database and a query");
    if (h->score_mode != C2_SCORE_FP32)
        return fail(h, C2_ERR_STATE, "run_phase1_static scores in FP32 only; the handle is in score mode %d",
                    h->score_mode);
    if (h->device < 0 || h->device >= C2_STATIC_MAXDEV)
        return fail(h, C2_ERR_ARG, "run_phase1_static: device %d out of range", h->device);
    CK(cudaSetDevice(h->device));
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_scratch[h->device]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, c2_static_scratch);
            if (e != cudaSuccess || !p)
                return fail(h, C2_ERR_CUDA, "run_phase1_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_static_scratch[h->device] = p;
        }
        base = g_static_scratch[h->device];
    }
    const size_t per_block = (size_t)h->botstride * sizeof(float) * P1_WARPS;
    const size_t nblocks = (C2_STATIC_SCRATCH_BYTES - C2_STATIC_HDR) / per_block;
    if (nblocks < 1)
        return fail(h, C2_ERR_CAPACITY,
                    "run_phase1_static: longest db profile (%d positions) exceeds the static scratch limit "
                    "(%zu positions)",
                    h->Lmax, ((C2_STATIC_SCRATCH_BYTES - C2_STATIC_HDR) / (10 * sizeof(float) * P1_WARPS)) & ~size_t(31));
    const int grid = (int)std::min<size_t>((size_t)h->grid, nblocks);
    P1Args a;
    fill_p1(h, a);
    a.nwork = h->nprof;
    a.order = h->db->d_order.p;
    a.counter = (int*)base;
    a.bot = (float*)((char*)base + C2_STATIC_HDR);
    a.best = d_best;
    a.coords = d_coords;
    CK(cudaMemsetAsync(base, 0, sizeof(int), h->stream));
    CK(launch_p1(a, h->d_qbkg.p, P1K_STRIP, grid, h->stream));
    h->launches++;
    return C2_OK;
}

// ---------------------------------------------------------------------------
// Differentiable alignment (no counterpart in the reference): log-partition
// of the MAP forward model and its gradients (model in c2_adj.cu).

static c2_profiles query_view(const c2_profiles* qs, int k, const int64_t* zero);

static void fill_adj(c2_handle* h, AdjArgs& a)
{
    memset(&a, 0, sizeof a);
    const long long NC = h->adj_cells, NR = h->adj_rows;
    a.npairs = (int)h->adj_prof.size();
    a.nitems = h->adj_nitems;
    a.prof = h->d_adjprof.p;
    a.pLq = h->d_adjLq.p;
    a.qpos = h->d_adjqpos.p;
    a.qidx = h->d_adjqidx.p;
    a.soff = h->d_adjsoff.p;
    a.items_f = h->d_adjitems.p;
    a.items_b = h->d_adjitems.p + h->adj_nitems;
    a.off = h->d_adjoff.p;
    a.roff = h->d_adjroff.p;
    a.plen = h->db->d_plen.p;
    a.poff = h->db->d_poff.p;
    a.drec = h->db->d_drec.p;
    a.pbkg = h->db->d_pbkg.p;
    if (h->adj_batch) {
        a.qrec = h->d_adjqrec.p;
        a.qbkg = h->d_adjqbkg.p;
        a.qtrn = h->d_adjqtrn.p;
        a.qcfx = h->d_adjqcfx.p;
    } else {
        a.qrec = h->d_qrec.p;
        a.qbkg = h->d_qbkg.p;
        a.qtrn = h->d_qtrn.p;
        a.qcfx = h->d_qcfx.p;
    }
    a.ssss = h->d_ssss.p;
    a.cvvals = h->d_cvvals.p;
    a.sc = h->sc;
    a.dtrn = h->db->d_dtrn.p;
    for (int k = 0; k < 7; k++) a.theta[k] = h->adj_theta[k];
    a.wss = h->adj_wss;
    a.wcv = h->adj_wcv;
    float* b = h->d_adjbuf.p;
    a.S = b;
    a.pss = b + NC;
    a.pcv = b + 2 * NC;
    a.gS = b + 3 * NC;
    a.post = b + 4 * NC;
    a.frow = b + 5 * NC;
    a.brow = b + 5 * NC + NR;
    a.prog = h->d_adjprog.p;
    a.zpart = h->d_adjpart.p;
    a.gpart = h->d_adjpart.p + 2LL * h->adj_nitems;
    a.Fall = h->adj_keepF ? h->d_adjF.p : nullptr;
    a.scratch = h->d_adjscr.p;
    a.scratch_stride = (long long)(h->adj_Lmax + 31) * 160;
    a.counter = h->d_adjctr.p;
    a.status = h->d_status.p;
    a.spin = h->spin;
    a.logz = h->d_adjlogz.p;
    a.grad = h->d_adjgrad.p;
}

// device status after a sweep (a strip wait that timed out)
static c2_status adj_status(c2_handle* h)
{
    int stw = 0;
    CK(cudaMemcpyAsync(&stw, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (stw != 0) return fail(h, C2_ERR_DEVICE, "device status %d: %s", stw, status_text(stw));
    return C2_OK;
}

// The forward sweep over pairs (query qidx[k] of length Lq[k] from row
// qpos[k] of the query arrays, db profile profiles[k]): per-pair layout,
// work item tables, scratch, launch.
static c2_status logz_fwd_pairs(c2_handle* h, const int32_t* profiles, const int* Lq, const long long* qpos,
                                const int* qidx, int32_t npairs, const float* theta, float wss, float wcv,
                                float* logz)
{
    h->adj_fwd_done = false;
    h->adj_prof.assign(profiles, profiles + npairs);
    h->adj_Lq.assign(Lq, Lq + npairs);
    h->adj_off.resize(npairs);
    h->adj_roff.resize(npairs);
    std::vector<long long> soff(npairs);
    long long acc = 0, racc = 0, sacc = 0;
    int lmax = 0, nsmax = 0;
    for (int k = 0; k < npairs; k++) {
        if (profiles[k] < 0 || profiles[k] >= h->nprof)
            return fail(h, C2_ERR_ARG, "logz_fwd: profile %d out of range", profiles[k]);
        const int L = h->h_plen[profiles[k]];
        const int ns = (Lq[k] + 31) / 32;
        h->adj_off[k] = acc;
        h->adj_roff[k] = racc;
        soff[k] = sacc;
        acc += (long long)ns * (L + 31) * 32;
        racc += (long long)ns * 5 * L;
        sacc += ns;
        lmax = std::max(lmax, L);
        nsmax = std::max(nsmax, ns);
    }
    if (sacc > 0x7fffffff) return fail(h, C2_ERR_CAPACITY, "logz_fwd: %lld strips", sacc);
    const int items = (int)sacc;
    // work items: the forward sweep by strip, the backward sweep by strip
    // from each pair's last one
    std::vector<int2> it((size_t)2 * items);
    {
        size_t f = 0, b = items;
        for (int s = 0; s < nsmax; s++)
            for (int k = 0; k < npairs; k++) {
                const int ns = (Lq[k] + 31) / 32;
                if (s < ns) {
                    it[f++] = make_int2(k, s);
                    it[b++] = make_int2(k, ns - 1 - s);
                }
            }
    }
    h->adj_cells = acc;
    h->adj_rows = racc;
    h->adj_Lmax = lmax;
    h->adj_nitems = items;
    for (int k = 0; k < 7; k++) h->adj_theta[k] = theta ? theta[k] : 0.f;
    h->adj_wss = wss;
    h->adj_wcv = wcv;
    if (h->d_adjprof.ensure(npairs, h->budget) || h->d_adjoff.ensure(npairs, h->budget) ||
        h->d_adjroff.ensure(npairs, h->budget) || h->d_adjLq.ensure(npairs, h->budget) ||
        h->d_adjqpos.ensure(npairs, h->budget) || h->d_adjqidx.ensure(npairs, h->budget) ||
        h->d_adjsoff.ensure(npairs, h->budget) || h->d_adjitems.ensure((size_t)2 * items, h->budget) ||
        h->d_adjbuf.ensure((size_t)(5 * acc + 2 * racc), h->budget) ||
        h->d_adjlogz.ensure(npairs, h->budget) || h->d_adjgrad.ensure((size_t)npairs * 9, h->budget) ||
        h->d_adjprog.ensure((size_t)2 * items, h->budget) || h->d_adjpart.ensure((size_t)11 * items, h->budget) ||
        h->d_adjctr.ensure(2, h->budget))
        return fail(h, C2_ERR_NOMEM, "logz_fwd: scratch for %d pairs (%lld cells) failed", npairs, acc);
    // persistent grids of the sweeps: as many CTAs as are resident (or as
    // there are strips); backward sweep warps each hold a strip's forward
    // states (32 rows x (Lmax + 31) columns x 5 floats), its grid halved while
    // that scratch does not fit (the memory budget or the device)
    int fwd_occ = 4, bwd_occ = 4;
    CK(adj_occupancy(&fwd_occ, &bwd_occ));
    const long long want = std::min<long long>((long long)h->nsm * std::max(bwd_occ, 1), (items + ADJ_WARPS - 1) / ADJ_WARPS);
    h->adj_bgrid = (int)want;
    // The forward sweep keeps every forward state (20 bytes a cell) when that
    // takes at most a quarter of the free device memory and fits the budget;
    // otherwise the backward sweep recomputes each strip's states from the
    // checkpoint row above into per-warp scratch (32 rows x (Lmax + 31)
    // columns x 5 floats), its grid halved while that scratch does not fit.
    h->adj_keepF = false;
    {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && (size_t)acc * 5 * sizeof(float) <= fr / 4 &&
            h->d_adjF.ensure((size_t)acc * 5, h->budget) == cudaSuccess)
            h->adj_keepF = true;
        (void)cudaGetLastError();   // a refused allocation is not an error of what follows
    }
    if (!h->adj_keepF) {
        h->d_adjF.release();
        const size_t per_cta = (size_t)ADJ_WARPS * (lmax + 31) * 160 * sizeof(float);
        h->adj_bgrid = 0;
        for (long long g = want; g >= 1 && h->adj_bgrid == 0; g /= 2)
            if (h->d_adjscr.ensure((size_t)g * per_cta / sizeof(float), h->budget) == cudaSuccess) h->adj_bgrid = (int)g;
        (void)cudaGetLastError();
        if (h->adj_bgrid == 0)
            return fail(h, C2_ERR_NOMEM, "logz_fwd: backward sweep scratch (%zu bytes per CTA) failed", per_cta);
    }
    CK(cudaMemcpyAsync(h->d_adjprof.p, profiles, (size_t)npairs * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjLq.p, Lq, (size_t)npairs * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjqpos.p, qpos, (size_t)npairs * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjqidx.p, qidx, (size_t)npairs * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjsoff.p, soff.data(), (size_t)npairs * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjitems.p, it.data(), it.size() * sizeof(int2), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjoff.p, h->adj_off.data(), (size_t)npairs * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjroff.p, h->adj_roff.data(), (size_t)npairs * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->d_adjprog.p, 0, (size_t)items * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_adjctr.p, 0, 2 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
    AdjArgs a;
    fill_adj(h, a);
    const int grid = (int)std::min<long long>((long long)h->nsm * std::max(fwd_occ, 1), (items + ADJ_WARPS - 1) / ADJ_WARPS);
    CK(launch_adj_fwd(a, grid, h->stream));
    h->launches += 3;
    c2_status st = adj_status(h);
    if (st != C2_OK) return st;
    CK(cudaMemcpyAsync(logz, h->d_adjlogz.p, (size_t)npairs * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->adj_fwd_done = true;
    return C2_OK;
}

extern "C" c2_status c2_logz_fwd(c2_handle* h, const int32_t* profiles, int32_t npairs, const float* theta, float wss,
                                 float wcv, float* logz)
{
    if (!h || !profiles || npairs <= 0 || !logz) return C2_ERR_ARG;
    if (h->nprof <= 0 || h->Lq <= 0) return fail(h, C2_ERR_STATE, "logz_fwd needs a database and a query");
    CK(cudaSetDevice(h->device));
    h->adj_batch = false;
    const std::vector<int> Lq(npairs, h->Lq), qidx(npairs, 0);
    const std::vector<long long> qpos(npairs, 0);
    return logz_fwd_pairs(h, profiles, Lq.data(), qpos.data(), qidx.data(), npairs, theta, wss, wcv, logz);
}

extern "C" c2_status c2_set_query_batch(c2_handle* h, const c2_profiles* queries)
{
    if (!h || !queries) return C2_ERR_ARG;
    c2_status st = check_profiles(h, queries);
    if (st != C2_OK) return st;
    CK(cudaSetDevice(h->device));
    const int nq = queries->nprofiles;
    // the queries' rows as c2_set_query packs them (score fields, exact
    // column -1 states), raw transitions and backgrounds, concatenated; the
    // queries packed by up to 16 host threads
    const long long N = queries->npositions;
    std::vector<float> qrec((size_t)N * QR_STRIDE, 0.f), qcf((size_t)N * 6, 0.f);
    {
        std::atomic<int> next(0);
        auto work = [&]() {
            const int64_t zero = 0;
            for (int q; (q = next.fetch_add(1)) < nq;) {
                const c2_profiles v = query_view(queries, q, &zero);
                const size_t o = (size_t)queries->offsets[q];
                qrec_score_fields(h, &v, qrec.data() + o * QR_STRIDE);
                colm1_exact(&v, qcf.data() + o * 6);
            }
        };
        const int nt = std::max(1, std::min(16, nq / 8));
        std::vector<std::thread> th;
        for (int t = 1; t < nt; t++) th.emplace_back(work);
        work();
        for (auto& t : th) t.join();
    }
    if (h->d_adjqrec.ensure(qrec.size(), h->budget) || h->d_adjqcfx.ensure(qcf.size(), h->budget) ||
        h->d_adjqtrn.ensure((size_t)(N + nq) * 7, h->budget) || h->d_adjqbkg.ensure((size_t)nq * NAA, h->budget))
        return fail(h, C2_ERR_NOMEM, "set_query_batch: query arrays for %d queries failed", nq);
    CK(cudaMemcpyAsync(h->d_adjqrec.p, qrec.data(), qrec.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjqcfx.p, qcf.data(), qcf.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjqtrn.p, queries->trn, (size_t)(N + nq) * 7 * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_adjqbkg.p, queries->bkg, (size_t)nq * NAA * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));   // the host arrays above are freed on return
    h->adj_qlen.assign(queries->lengths, queries->lengths + nq);
    h->adj_qstart.assign(queries->offsets, queries->offsets + nq);
    h->adj_fwd_done = false;
    return C2_OK;
}

extern "C" c2_status c2_logz_fwd_batch(c2_handle* h, const int32_t* query_of_pair, const int32_t* profiles,
                                       int32_t npairs, const float* theta, float wss, float wcv, float* logz)
{
    if (!h || !query_of_pair || !profiles || npairs <= 0 || !logz) return C2_ERR_ARG;
    if (h->nprof <= 0) return fail(h, C2_ERR_STATE, "logz_fwd_batch needs a database");
    if (h->adj_qlen.empty()) return fail(h, C2_ERR_STATE, "logz_fwd_batch needs c2_set_query_batch");
    CK(cudaSetDevice(h->device));
    const int nq = (int)h->adj_qlen.size();
    std::vector<int> Lq(npairs), qidx(npairs);
    std::vector<long long> qpos(npairs);
    for (int k = 0; k < npairs; k++) {
        const int q = query_of_pair[k];
        if (q < 0 || q >= nq) return fail(h, C2_ERR_ARG, "logz_fwd_batch: query %d of pair %d out of range", q, k);
        Lq[k] = h->adj_qlen[q];
        qpos[k] = h->adj_qstart[q];
        qidx[k] = q;
    }
    h->adj_batch = true;
    return logz_fwd_pairs(h, profiles, Lq.data(), qpos.data(), qidx.data(), npairs, theta, wss, wcv, logz);
}

extern "C" c2_status c2_logz_bwd(c2_handle* h, float* grad)
{
    if (!h || !grad) return C2_ERR_ARG;
    if (!h->adj_fwd_done) return fail(h, C2_ERR_STATE, "logz_bwd needs a preceding logz_fwd for the current query");
    CK(cudaSetDevice(h->device));
    AdjArgs a;
    fill_adj(h, a);
    const long long items = h->adj_nitems;
    CK(cudaMemsetAsync(h->d_adjprog.p + items, 0, (size_t)items * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_adjctr.p + 1, 0, sizeof(int), h->stream));
    CK(launch_adj_bwd(a, h->adj_bgrid, h->stream));
    h->launches += 2;
    c2_status st = adj_status(h);
    if (st != C2_OK) return st;
    CK(cudaMemcpyAsync(grad, h->d_adjgrad.p, (size_t)a.npairs * 9 * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return C2_OK;
}

extern "C" c2_status c2_logz_cells(c2_handle* h, int32_t pair, float* dlogz_ds, float* post)
{
    if (!h || (!dlogz_ds && !post)) return C2_ERR_ARG;
    if (!h->adj_fwd_done || pair < 0 || pair >= (int)h->adj_prof.size())
        return fail(h, C2_ERR_STATE, "logz_cells: no such pair after logz_fwd/logz_bwd");
    CK(cudaSetDevice(h->device));
    const int Lq = h->adj_Lq[pair], L = h->h_plen[h->adj_prof[pair]];
    const int ns = (Lq + 31) / 32;
    const size_t n = (size_t)ns * (L + 31) * 32;
    std::vector<float> t(n);
    const long long NC = h->adj_cells;
    for (int w = 0; w < 2; w++) {
        float* dst = w ? post : dlogz_ds;
        if (!dst) continue;
        CK(cudaMemcpy(t.data(), h->d_adjbuf.p + (3 + w) * NC + h->adj_off[pair], n * 4, cudaMemcpyDeviceToHost));
        // wavefront order -> row-major [Lq][L]
        for (int i = 0; i < Lq; i++) {
            const size_t rb = ((size_t)(i >> 5) * (L + 31) + (i & 31)) * 32 + (i & 31);
            for (int j = 0; j < L; j++) dst[(size_t)i * L + j] = t[rb + (size_t)j * 32];
        }
    }
    return C2_OK;
}

// ---------------------------------------------------------------------------
// Multi-query search (replaces the reference's JobDispatcher / DevCommThread
// query loop, src/libmycu/cualn/JobDispatcher.cpp:967-1213 and
// DevCommThread.cpp:155-356): the batch's queries go to worker handles that
// share the database, one host thread and one CUDA stream each, taking the
// next query as they finish one; a query's host-side steps and its
// latency-bound phase-2 kernels overlap other queries' work.

// Query k of a profile set as a one-profile set
static c2_profiles query_view(const c2_profiles* qs, int k, const int64_t* zero)
{
    c2_profiles v;
    memset(&v, 0, sizeof v);
    const int64_t o = qs->offsets[k];
    v.nprofiles = 1;
    v.npositions = qs->lengths[k];
    v.lengths = qs->lengths + k;
    v.offsets = zero;
    v.bkg = qs->bkg + (size_t)k * NAA;
    v.eno = qs->eno ? qs->eno + k : nullptr;
    v.trn = qs->trn + (size_t)(o + k) * 7;
    v.trg = qs->trg + (size_t)o * NAA;
    v.cv = qs->cv + (size_t)o * NCV;
    v.cvprior = qs->cvprior + o;
    v.cvnorm2 = qs->cvnorm2 + o;
    v.ss = qs->ss + (size_t)o * NSS;
    v.ssstate = qs->ssstate ? qs->ssstate + o : nullptr;
    v.aa = qs->aa + o;
    return v;
}

constexpr int BATCH_RESERVE_DIV = 18;   // SMs left free by phase 1 in a multi-worker batch: nsm / 18

static c2_status batch_workers(c2_handle* h, int nw)
{
    // workers made for an earlier database are remade
    for (size_t i = 0; i < h->workers.size(); i++)
        if (h->workers[i]->db != h->db) {
            for (c2_handle* w : h->workers) c2_destroy(w);
            h->workers.clear();
            break;
        }
    while ((int)h->workers.size() < nw - 1) {
        c2_params p = h->prm;
        p.ssss = h->ssss.data();
        p.cvs2s_keys = h->cvkeys.data();
        p.cvs2s_values = h->cvvals.data();
        p.sse_nn_weights = h->nnw.empty() ? nullptr : h->nnw.data();
        c2_handle* w = nullptr;
        c2_status st = c2_create(h->device, &p, &w);
        if (st != C2_OK) return fail(h, st, "batch: creating a worker handle failed");
        w->budget = h->budget;   // the workers draw on the handle's device memory budget
        if ((st = c2_share_db(w, h)) != C2_OK) {
            std::string e = w->err;
            c2_destroy(w);
            return fail(h, st, "batch: %s", e.c_str());
        }
        h->workers.push_back(w);
    }
    // with more than one worker, a query's phase 2 (latency-bound strip
    // sweeps, host round trips) runs beside the next query's phase 1, whose
    // persistent grid leaves a few SMs free for it
    const int reserve = nw <= 1 ? 0
                        : h->batch_reserve >= 0 ? std::min(h->batch_reserve, h->nsm - 1)
                                                : std::max(1, h->nsm / BATCH_RESERVE_DIV);
    h->p1_reserve = reserve;
    for (c2_handle* w : h->workers) {
        w->score_mode = h->score_mode;
        w->spin = h->spin;
        w->p1_reserve = reserve;
    }
    return C2_OK;
}

extern "C" c2_status c2_set_batch_sm_reserve(c2_handle* h, int32_t nsm)
{
    if (!h) return C2_ERR_ARG;
    h->batch_reserve = nsm < 0 ? -1 : nsm;
    return C2_OK;
}

extern "C" c2_status c2_search_batch(c2_handle* h, const c2_profiles* queries, int32_t nworkers, c2_batch_cb cb,
                                     void* user)
{
    if (!h || !cb || nworkers < 1 || nworkers > 8) return C2_ERR_ARG;
    if (h->nprof <= 0 || !h->db) return fail(h, C2_ERR_STATE, "search_batch needs a database");
    c2_status st = check_profiles(h, queries);
    if (st != C2_OK) return st;
    const int nq = queries->nprofiles;
    const int nw = std::min(nworkers, nq);
    if ((st = batch_workers(h, nw)) != C2_OK) return st;
    std::vector<c2_handle*> ws(1, h);
    for (int i = 0; i < nw - 1; i++) ws.push_back(h->workers[i]);
    std::atomic<int> next(0);
    std::mutex mu;       // serialises the callbacks and the first error
    std::mutex p1_mu;    // one query's phase 1 at a time (see below)
    c2_status first = C2_OK;
    std::string first_err;
    auto run = [&](c2_handle* w) {
        const int64_t zero = 0;
        std::vector<c2_hit> hits;
        std::vector<char> alns;
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= nq) break;
            const c2_profiles v = query_view(queries, q, &zero);
            int32_t nh = 0;
            size_t nb = 0;
            // The query's host-side preparation, its phase 2 and its hit copy
            // and callback overlap other workers; phase 1 runs one query at a
            // time (its persistent grid holds every SM but the few reserved
            // for the phase-2 sweeps of the query before).
            c2_status s = c2_set_query(w, &v);
            if (s == C2_OK) {
                std::lock_guard<std::mutex> g(p1_mu);
                s = c2_run_phase1(w);
                if (s == C2_OK && cudaStreamSynchronize(w->stream) != cudaSuccess) s = C2_ERR_CUDA;
            }
            if (s == C2_OK) {
                int32_t n = 0;
                if (s == C2_OK) s = c2_run_finalize(w, &n);
                if (s == C2_OK) s = c2_run_stats(w, &n);
                if (s == C2_OK) s = c2_run_map(w, &nh);
                if (s == C2_OK && cudaStreamSynchronize(w->stream) != cudaSuccess) s = C2_ERR_CUDA;
            }
            if (s == C2_OK) s = c2_get_hits(w, nullptr, 0, nullptr, &nb);
            if (s == C2_OK) {
                hits.resize(std::max(1, nh));
                alns.resize(std::max<size_t>(1, nb));
                s = c2_get_hits(w, hits.data(), nh, alns.data(), &nb);
            }
            std::lock_guard<std::mutex> lk(mu);
            if (s != C2_OK) {
                if (first == C2_OK) {
                    first = s;
                    first_err = "query " + std::to_string(q) + ": " + w->err;
                }
                cb(user, q, s, nullptr, 0, nullptr, 0);
            } else {
                cb(user, q, s, hits.data(), nh, alns.data(), nb);
            }
        }
    };
    std::vector<std::thread> th;
    for (int i = 1; i < nw; i++) th.emplace_back(run, ws[i]);
    run(ws[0]);
    for (auto& t : th) t.join();
    h->p1_reserve = 0;   // the handle's own searches use every SM again
    if (first != C2_OK) return fail(h, first, "search_batch: %s", first_err.c_str());
    return C2_OK;
}
