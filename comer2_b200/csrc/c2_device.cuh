// c2_device.cuh -- device-side layouts and kernel arguments of the B200
// implementation of the COMER2 search hot path.
//
// HBM layout (built by c2_upload_db / c2_set_query):
//  * db position records, DR_STRIDE floats (224 B) per position, everything a
//    score column and a DP column need, so one warp-uniform (broadcast) read
//    stream per column feeds all 32 lanes (lanes own query rows):
//      [0,20)  target probabilities          [20,39) context vector
//      39      cvnorm2 + 1 + 1/kappa0         40      CV log prior
//      [41,44) SS probabilities C,E,H         44      SS table indices, packed
//      45      P(H) + 0.1                     [48,55) DP transitions of the column
//      55      residue letter
//  * query position records, QR_STRIDE floats (256 B), the same fields for the
//    query rows plus the column -1 boundary states of the reference's DP
//    (see c2_host.cu: colm1 states).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace c2 {

constexpr int NAA = 20, NCV = 19, NSS = 3;
constexpr float LOG0 = -32768.0f;

enum : int {
    QR_TRG = 0, QR_CV = 20, QR_CN = 39, QR_PRIOR = 40, QR_SS = 41, QR_SSIDX = 44,
    QR_HQ = 47, QR_TRN = 48, QR_C = 55, QR_CP = 58, QR_STRIDE = 64
};
enum : int {
    DR_TRG = 0, DR_CV = 20, DR_CN = 39, DR_PRIOR = 40, DR_SS = 41, DR_SSIDX = 44,
    DR_HD = 45, DR_TRN = 48, DR_AA = 55, DR_STRIDE = 56
};
// DP transitions of a row/column: MM and MD, IM, DM, DD into the position,
// MI and II out of it (the reference's MMp, MIc, MDp, IMp, IIc, DMp, DDp;
// src/libmycu/cudp/CuBatchDP_init.cuh:132-155)
enum : int { TMM = 0, TMI, TMD, TIM, TII, TDM, TDD };

// btck codes (src/libmycu/cudp/CuBatchDP_com.h:99-104)
enum : int { BT_STOP = 0, BT_LEFT = 1, BT_UP = 2, BT_DIAG = 3 };

struct ScoreConsts {
    float ssswgt, cvswgt, shift;          // term weights, aa-term shift
    float lokappa0, pownu0, cterm;        // context-vector constants
    float cvkey_first, cvkey_last, cvval_first, cvval_last;
    int cvcard, cvshift, ssss_card;
};

constexpr int P1_WARPS = 8;               // warps per CTA of the DP kernels
constexpr int MAX_SSSS_CARD = 32;
// db record staging ring of the phase-1 kernel: 2 chunks of 8 columns
constexpr int REC_CHUNK = 8, REC_CHUNK_LOG = 3, REC_SLOTS = 16;
// shared memory per warp: score ring [32][32], SS row table [32][32], record ring
constexpr int P1_WARP_FLOATS = 32 * 32 + MAX_SSSS_CARD * 32 + REC_SLOTS * DR_STRIDE;
constexpr int MAX_CVCARD = 256;
// Tensor-core (BF16 split) phase-1 kernel.  The three contractions of a cell
// score -- amino acids (K = 20), context vectors (K = 19) and the SS table
// (K = card <= 32, the db side a 3-hot vector of SS probabilities) -- run as
// mma.sync m16n8k16 BF16 products with FP32 accumulation, each operand split
// into hi + lo BF16 parts (x = hi + lo + O(2^-17 x)) and hi*hi + hi*lo +
// lo*hi accumulated.  db operands (B, k16 x n8 fragments) are packed once per
// database in the fragment order of the 32 lanes, 8 db columns per tile:
//   tcdb[tile][dot 3][ktile 2][split 2][lane 32][2 words]
// with every profile padded to a multiple of 32 columns; query operands (A,
// m16 x k16) per query: qa[strip][mtile 2][dot 2: cv, ss][ktile 2][split 2]
// [lane 32][4 words] and the unscaled amino-acid rows qaa[strip][mtile 2]
// [ktile 2][lane 32][8 floats] (scaled per pair by 1 / (0.5 (bq + bd))).
// The constant parts of the CV and SS terms ride in the spare K columns:
// CV k = 19 carries 1 (query) x 1/kappa0 (db), so the CV accumulator is the
// shifted dot product; the SS operand is weighted by the SS weight on the db
// side and k = 30, 31 carry P(H)q + 0.1 x w (P(H)d + 0.1) / 9 and 1 x -0.05 w,
// so the SS accumulator is the complete weighted SS term (the reference's
// "-99 < ss" guard always holds for tables above SS_FOLD_MIN, which the
// tensor-core form requires, with card <= 30).
// Per db position the DP and the score epilogue also read a column record
// cold[pos][P1C_TRS]: the DP transitions in the pair order below (slots
// 0..8), cvnorm, 2 x CV log prior, pad.
constexpr int TC_TILE_WORDS = 3 * 2 * 2 * 32 * 2;
constexpr int TC_QA_WORDS = 2 * 2 * 2 * 2 * 32 * 4;   // per strip
constexpr int TC_QAA_FLOATS = 2 * 2 * 32 * 8;         // per strip
constexpr float SS_FOLD_MIN = -49.f;
constexpr int TC_SS_KMAX = 30;
enum : int { CO_CD = 9, CO_PD2 = 10 };
// DP transition record of a db column, ordered for the packed-pair Viterbi
// step: (MM, MM), (IM, MM), (MD, DD), MI, II, DM.  DPT_SRC packs, per record
// slot i, the transition index (TMM..TDD) in bits [4i, 4i + 4).
constexpr int DPT_N = 9;
constexpr unsigned long long DPT_SRC = 0x541620300ull;
__host__ __device__ constexpr int dpt_src(int i) { return (int)((DPT_SRC >> (4 * i)) & 0xf); }
// chunked phase-1 kernel: 11 warps per CTA, one CTA per SM; per warp a score
// ring of 64 columns x 32 rows, a transition ring of 64 columns (stride 12
// floats: the two 16-byte reads of 8 lanes at consecutive columns cover 32
// distinct banks), the SS row table, the record staging ring and the row
// above the strip for the current chunk
constexpr int P1C_WARPS = 11;
// phase-1 kernel variants of launch_p1
enum : int { P1K_STRIP = 0, P1K_CHUNKED = 1, P1K_TRACEBACK = 2, P1K_TENSOR = 3 };
constexpr int P1C_RING = 64, P1C_TRS = 12, P1C_CVREP = 16;
// row above the strip in the shared-memory DP kernels: [32][4] + [32] floats
constexpr int BND_ND = 32 * 4, BND_FLOATS = 32 * 5;
constexpr int P1C_WARP_FLOATS =
    P1C_RING * 32 + P1C_RING * P1C_TRS + MAX_SSSS_CARD * 32 + REC_SLOTS * DR_STRIDE + BND_FLOATS;
// traceback sweep over the stored score matrices: per warp the score ring, the
// transition ring, the row above and a [32][33]-byte traceback column ring;
// 17 warps per SM.  P1TC_CVREP: CV table replicas of the phase-2 score kernel
constexpr int P1TC_WARPS = 17, P1TC_CVREP = 8;
constexpr int P1TC_WARP_FLOATS = P1C_RING * 32 + P1C_RING * P1C_TRS + BND_FLOATS;
// phase-2 score kernel: 8 warps per CTA, per warp the SS row table and the
// record staging ring; the CV table (P1TC_CVREP replicas) per CTA
constexpr int P2S_WARPS = 8;
constexpr int P2S_WARP_FLOATS = MAX_SSSS_CARD * 32 + REC_SLOTS * DR_STRIDE;

// Largest CV maps the shared-memory layouts hold (opt-in shared memory per CTA
// on sm_100: 227 KB): the phase-2 score kernel, which every search runs, and the
// tensor-core phase-1 kernel (whose 16 bytes of static shared memory hold the
// TMEM address).  The reference's cvs2s map has 93 entries.
constexpr int SMEM_CTA_MAX = 227 * 1024;
constexpr int P1TC_MAX_CVCARD =
    (SMEM_CTA_MAX - P2S_WARPS * P2S_WARP_FLOATS * 4) / (P1TC_CVREP * 4);
// tensor-core kernel: score ring of 64 anti-diagonals with 36 floats each (the
// fragment-layout writes and the per-lane wavefront reads are both free of
// bank conflicts), a column-record ring of 3 chunks plus a mirror of its first
// chunk (slots 96..127), so that the 32 records a lane reads in one DP stage
// never wrap, the row above the strip and one slot for the db operand tile
// (a bulk async copy, one mbarrier); 12 warps fit with a CV table of up to
// 106 entries
constexpr int P1T_WARPS = 12;
constexpr int P1T_RLD = 36, P1T_CRING = 128, P1T_CMOD = 96, P1T_CVREP = 8;
constexpr unsigned P1T_TMEM_COLS = 512;   // TMEM columns of a CTA (3 warps x 128 per lane quarter)
constexpr int P1T_WARP_FLOATS = P1C_RING * P1T_RLD + P1T_CRING * P1C_TRS + BND_FLOATS + TC_TILE_WORDS + 4;
constexpr int P1T_MAX_CVCARD = (SMEM_CTA_MAX - 16 - P1T_WARPS * P1T_WARP_FLOATS * 4) / (P1T_CVREP * 4);

// Epilogue constants of the tensor-core form: x = 2 x (CV score argument)
// = (2 pownu0 ln2) log2(det) + 2 cterm - 2 prior_q - 2 prior_d, compared
// with twice the table keys; table values pre-multiplied by the CV weight.
// uniform: the table index clamp alone reproduces the key range tests.
struct TcConsts {
    float shift, p2l, c2, kf2, kl2, vfw, vlw;
    int ilo, ihi, uniform;
};

struct P1Args {
    const float* qrec;      // [Lq][QR_STRIDE]
    int Lq;
    const float* drec;      // [npos][DR_STRIDE]
    const int* plen;        // [nprof]
    const long long* poff;  // [nprof]
    const float* pbkg;      // [nprof][20]
    int nwork;              // number of work items (profiles or candidates)
    const int* order;       // work item -> profile
    int* counter;           // work-queue head
    const float* ssss;      // [card][card]
    const float* cvvals;    // [cvcard]
    const float* qU;        // [strip][MAX_SSSS_CARD][32] SS row tables of the query rows
    ScoreConsts sc;
    float* bot;             // strip-boundary rows: per warp slot 2 x 5 x Lmax
    long long botstride;    // floats per warp slot
    // phase-1 outputs (indexed by profile)
    float* best;
    unsigned* coords;
    // traceback variant: per work item k, scratch at cand_off[k]
    const long long* cand_off;  // byte offsets into btck / float offsets into smat
    signed char* btck;          // [L][Lq] per candidate (column-major)
    float* smat;                // [L][Lq] per candidate
    float* mmat;                // [L][Lq] per candidate: modular scores
    int* status;                // device error word (0 = ok)
    // strip pipeline of the traceback variant
    float* bnd;                 // per candidate at 10 x (cand_off / Lq): two last-row buffers [5][L]
    int* prog;                  // [ncand][nstrips] finished columns per strip
    unsigned long long* tbkey;  // [ncand] maximum of the traceback sweep and its cell, packed
    const int* worder;          // traceback sweep: rank -> candidate (longest first)
    const int* items;           // traceback sweep: work item -> rank * nstrips + strip
    unsigned spin;              // polls before a strip wait gives up (pipe_wait)
    // tensor-core operands (P1K_TENSOR)
    const unsigned* tcdb;       // db B fragments
    const long long* ttile;     // [nprof] first tile of each profile
    const float* cold;          // [npos][P1C_TRS] column records
    const unsigned* qa;         // query A fragments (cv, ss)
    const float* qaa;           // query amino-acid rows in fragment order
    TcConsts tc;
};

struct FinArgs {
    int Lq;
    int ncand;
    const int* cand_prof;
    const long long* cand_off;
    const int* plen;
    const signed char* btck;
    const float* smat;
    const float* best;
    const unsigned* coords;
    float scorethld;
    const unsigned long long* tbkey;  // [ncand] maxima of the traceback sweep and their cells
    float tol;                  // allowed |phase-1 maximum - traceback maximum| (0: identical)
    int* status;
    // outputs [ncand]
    float* score;
    int* psts;
    unsigned* beg;
    unsigned* endc;
    int* passed;
};

}  // namespace c2

// ---------------------------------------------------------------------------
// Phase-2 sweeps (traceback DP, MAP forward/backward/MAP DP) run one strip of
// one pair per warp: a work item is (pair m, strip s), items are handed out
// in the order of a host-built table from a global counter.  The table puts
// (m, s) after (m, s - 1) (ordered by m + K s, K = pairs started per strip
// lag), so the item a warp waits on was taken earlier by a warp that is
// running, and strips are handed out about when their predecessor is ready.  Strip s writes its last row (5 states
// per column) to bnd[m][s & 1][5][L] and publishes the number of finished
// columns in prog[m * nstrips + s]; strip s+1 waits for the columns it
// prefetches.  A long pair is thus swept by up to nstrips warps at once
// instead of one.
namespace c2 {
constexpr int PIPE_G = 8;                 // columns per progress update
constexpr unsigned PIPE_SPIN = 1u << 22;  // default polls before a wait gives up (c2_set_wait_limit)
constexpr int PIPE_ERR_TIMEOUT = 3;       // device status of an abandoned wait

__device__ __forceinline__ int pipe_ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void pipe_st_release(int* p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Warp-uniform wait until *flag >= need (lane 0 polls).  After `spin` polls
// (at least one) it records PIPE_ERR_TIMEOUT in *status, marks the warp
// broken (no further waits) and returns; the sweep then finishes with invalid
// values -- every cell index stays inside its pair, so nothing is read or
// written out of bounds -- and the host reports the status.
__device__ __forceinline__ void pipe_wait(const int* flag, int need, int lane, int* status, bool& broken,
                                          unsigned spin)
{
    if (broken) return;
    unsigned it = 0;
    for (;;) {
        int ok = 0;
        if (lane == 0) ok = pipe_ld_acquire(flag) >= need;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) break;
        if (++it >= spin) {
            if (lane == 0 && status) atomicCAS(status, 0, PIPE_ERR_TIMEOUT);
            broken = true;
            break;
        }
        __nanosleep(128);
    }
    __syncwarp();
}

// producer side: lane 31 has stored column c of its strip's last row
__device__ __forceinline__ void pipe_publish(int* flag, int c, int L)
{
    if (((c + 1) % PIPE_G) == 0 || c + 1 == L) pipe_st_release(flag, c + 1);
}
}  // namespace c2
