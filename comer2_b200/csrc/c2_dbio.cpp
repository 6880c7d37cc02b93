// c2_dbio.cpp -- reader of the reference's binary profile database (the
// `db2bin` output, format v2.2) into the c2_profiles field set.
//
// File layout (written by Db::WriteBinaryHeader, src/libpro/srcpro/Db.cpp:733-741,
// CalculateAndWriteAddressTable_v2_2 and BinaryWriteProfile_v2_2,
// src/libpro/srcpro/PMProfileModel.cpp:1468-1930):
//   "COMER profile bin database v" "2.2"        (no terminator)
//   size_t nprofiles, uint64 npositions
//   size_t address[79]                          (file offset of every section)
//   int lengths[P]; float eno[P]; float bkg[20][P]
//   float trn[7][P + N]   (MM MI MD IM II DM DD; per profile the beginning
//                          state, then one value per position; natural logs,
//                          x 0.4 for IM II DM DD, -32768 for probability 0)
//   float trg[20][N]; float cv[19][N]; float cvprior[N]; float cvnorm2[N]
//   float ss[3][N]; float hdp1prob[N]; int hdp1index[N]
//   char aa[N]; char ssstate[N] (lower case, ' ' without SS; read as upper case)
//   size_t desc_end[P]; descriptions (NUL terminated)
// The sections are field-major; c2_profiles is position-major.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/comer2_b200.h"

namespace {

constexpr const char* kSig = "COMER profile bin database v";
constexpr const char* kVer = "2.2";
constexpr int kNAA = 20, kNCV = 19, kNSS = 3, kNTRN = 7;
constexpr int kNSECTIONS = 1 + 1 + kNAA + kNTRN + kNAA + kNCV + 1 + 1 + kNSS + 1 + 1 + 1 + 1 + 1 + 1;

struct File {
    FILE* f = nullptr;
    ~File() { if (f) fclose(f); }
};

void set_err(char* err, size_t n, const std::string& m)
{
    if (err && n) {
        std::strncpy(err, m.c_str(), n - 1);
        err[n - 1] = 0;
    }
}

bool read_at(FILE* f, uint64_t off, void* dst, size_t bytes)
{
    if (fseeko(f, (off_t)off, SEEK_SET) != 0) return false;
    return fread(dst, 1, bytes, f) == bytes;
}

struct Header {
    uint64_t nprof = 0, npos = 0, fsize = 0;
    uint64_t addr[kNSECTIONS] = {};
};

c2_status read_header(FILE* f, Header& h, char* err, size_t errlen)
{
    const size_t ls = std::strlen(kSig), lv = std::strlen(kVer);
    std::vector<char> sig(ls + lv);
    if (fread(sig.data(), 1, sig.size(), f) != sig.size() || std::memcmp(sig.data(), kSig, ls) != 0) {
        set_err(err, errlen, "not a COMER binary profile database");
        return C2_ERR_ARG;
    }
    if (std::memcmp(sig.data() + ls, kVer, lv) != 0) {
        set_err(err, errlen, "unsupported binary database version (2.2 expected)");
        return C2_ERR_ARG;
    }
    uint64_t np = 0, nn = 0;
    if (fread(&np, sizeof np, 1, f) != 1 || fread(&nn, sizeof nn, 1, f) != 1 ||
        fread(h.addr, sizeof(uint64_t), kNSECTIONS, f) != (size_t)kNSECTIONS) {
        set_err(err, errlen, "truncated binary database header");
        return C2_ERR_ARG;
    }
    if (np == 0 || np > 0x7fffffffULL) {
        set_err(err, errlen, "invalid number of profiles in the binary database");
        return C2_ERR_ARG;
    }
    // every position takes more than 4 bytes of the file and every section
    // lies inside it: a corrupt count or address is refused here, before any
    // array is sized by it
    if (fseeko(f, 0, SEEK_END) != 0) {
        set_err(err, errlen, "cannot size the binary database");
        return C2_ERR_ARG;
    }
    const uint64_t fsize = (uint64_t)ftello(f);
    if (nn < np || nn > fsize / 4) {
        set_err(err, errlen, "truncated or inconsistent binary database: number of positions");
        return C2_ERR_ARG;
    }
    for (int s = 0; s < kNSECTIONS; s++)
        if (h.addr[s] > fsize) {
            set_err(err, errlen, "truncated or inconsistent binary database: section address");
            return C2_ERR_ARG;
        }
    h.nprof = np;
    h.npos = nn;
    h.fsize = fsize;
    return C2_OK;
}

}  // namespace

extern "C" c2_status c2_db2bin_info(const char* path, int32_t* nprofiles, int64_t* npositions, char* err,
                                    size_t errlen)
{
    if (!path || !nprofiles || !npositions) return C2_ERR_ARG;
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) {
        set_err(err, errlen, std::string("cannot open ") + path);
        return C2_ERR_ARG;
    }
    Header h;
    c2_status st = read_header(F.f, h, err, errlen);
    if (st != C2_OK) return st;
    *nprofiles = (int32_t)h.nprof;
    *npositions = (int64_t)h.npos;
    return C2_OK;
}

namespace {
c2_status read_sections(FILE* f, const Header& h, uint64_t k0, uint64_t k1, int32_t* lengths, int64_t* offsets,
                        float* bkg, float* eno, float* trn, float* trg, float* cv, float* cvprior, float* cvnorm2,
                        float* ss, uint8_t* ssstate, uint8_t* aa, char* err, size_t errlen);
}  // namespace

extern "C" c2_status c2_db2bin_read(const char* path, int32_t* lengths, int64_t* offsets, float* bkg, float* eno,
                                    float* trn, float* trg, float* cv, float* cvprior, float* cvnorm2, float* ss,
                                    uint8_t* ssstate, uint8_t* aa, char* err, size_t errlen)
{
    if (!path || !lengths || !offsets || !bkg || !eno || !trn || !trg || !cv || !cvprior || !cvnorm2 || !ss ||
        !ssstate || !aa)
        return C2_ERR_ARG;
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) {
        set_err(err, errlen, std::string("cannot open ") + path);
        return C2_ERR_ARG;
    }
    Header h;
    c2_status st = read_header(F.f, h, err, errlen);
    if (st != C2_OK) return st;
    try {
        return read_sections(F.f, h, 0, h.nprof, lengths, offsets, bkg, eno, trn, trg, cv, cvprior, cvnorm2, ss,
                             ssstate, aa, err, errlen);
    } catch (...) {
        set_err(err, errlen, "out of host memory reading the binary database");
        return C2_ERR_NOMEM;
    }
}

extern "C" c2_status c2_db2bin_lengths(const char* path, int32_t* lengths, char* err, size_t errlen)
{
    if (!path || !lengths) return C2_ERR_ARG;
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) {
        set_err(err, errlen, std::string("cannot open ") + path);
        return C2_ERR_ARG;
    }
    Header h;
    c2_status st = read_header(F.f, h, err, errlen);
    if (st != C2_OK) return st;
    if (!read_at(F.f, h.addr[0], lengths, h.nprof * sizeof(int32_t))) {
        set_err(err, errlen, "truncated or inconsistent binary database: lengths");
        return C2_ERR_ARG;
    }
    uint64_t acc = 0;
    for (uint64_t k = 0; k < h.nprof; k++) {
        if (lengths[k] < 1) {
            set_err(err, errlen, "truncated or inconsistent binary database: profile length");
            return C2_ERR_ARG;
        }
        acc += (uint64_t)lengths[k];
    }
    if (acc != h.npos) {
        set_err(err, errlen, "truncated or inconsistent binary database: sum of profile lengths");
        return C2_ERR_ARG;
    }
    return C2_OK;
}

extern "C" c2_status c2_db2bin_read_range(const char* path, int32_t k0, int32_t k1, int32_t* lengths,
                                          int64_t* offsets, float* bkg, float* eno, float* trn, float* trg, float* cv,
                                          float* cvprior, float* cvnorm2, float* ss, uint8_t* ssstate, uint8_t* aa,
                                          char* err, size_t errlen)
{
    if (!path || !lengths || !offsets || !bkg || !eno || !trn || !trg || !cv || !cvprior || !cvnorm2 || !ss ||
        !ssstate || !aa || k0 < 0 || k1 <= k0)
        return C2_ERR_ARG;
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) {
        set_err(err, errlen, std::string("cannot open ") + path);
        return C2_ERR_ARG;
    }
    Header h;
    c2_status st = read_header(F.f, h, err, errlen);
    if (st != C2_OK) return st;
    if ((uint64_t)k1 > h.nprof) {
        set_err(err, errlen, "profile range beyond the end of the database");
        return C2_ERR_ARG;
    }
    try {
        return read_sections(F.f, h, (uint64_t)k0, (uint64_t)k1, lengths, offsets, bkg, eno, trn, trg, cv, cvprior,
                             cvnorm2, ss, ssstate, aa, err, errlen);
    } catch (...) {
        set_err(err, errlen, "out of host memory reading the binary database");
        return C2_ERR_NOMEM;
    }
}

namespace {
c2_status read_sections(FILE* f, const Header& h, uint64_t k0, uint64_t k1, int32_t* lengths, int64_t* offsets,
                        float* bkg, float* eno, float* trn, float* trg, float* cv, float* cvprior, float* cvnorm2,
                        float* ss, uint8_t* ssstate, uint8_t* aa, char* err, size_t errlen)
{
    const uint64_t P = h.nprof, N = h.npos;
    int a = 0;
    auto fail = [&](const char* what) {
        set_err(err, errlen, std::string("truncated or inconsistent binary database: ") + what);
        return C2_ERR_ARG;
    };
    // every profile's length (the positions before k0 and the total are
    // needed); profiles [k0, k1) hold Pr profiles and Nr positions from p0 on
    std::vector<int32_t> all(P);
    if (!read_at(f, h.addr[a++], all.data(), P * sizeof(int32_t))) return fail("lengths");
    uint64_t acc = 0, p0 = 0, Nr = 0;
    for (uint64_t k = 0; k < P; k++) {
        if (all[k] < 1) return fail("profile length");
        if (k == k0) p0 = acc;
        if (k0 <= k && k < k1) {
            lengths[k - k0] = all[k];
            offsets[k - k0] = (int64_t)Nr;
            Nr += (uint64_t)all[k];
        }
        acc += (uint64_t)all[k];
    }
    if (acc != N) return fail("sum of profile lengths");
    const uint64_t Pr = k1 - k0;
    if (!read_at(f, h.addr[a++] + k0 * sizeof(float), eno, Pr * sizeof(float))) return fail("ENOs");
    std::vector<float> col(Nr + Pr);
    for (int r = 0; r < kNAA; r++) {
        if (!read_at(f, h.addr[a++] + k0 * sizeof(float), col.data(), Pr * sizeof(float))) return fail("backgrounds");
        for (uint64_t k = 0; k < Pr; k++) bkg[k * kNAA + r] = col[k];
    }
    // transitions: one row per position plus one per profile (its beginning
    // state), so profile k0's rows start at row p0 + k0
    for (int t = 0; t < kNTRN; t++) {
        if (!read_at(f, h.addr[a++] + (p0 + k0) * sizeof(float), col.data(), (Nr + Pr) * sizeof(float)))
            return fail("transitions");
        for (uint64_t i = 0; i < Nr + Pr; i++) trn[i * kNTRN + t] = col[i];
    }
    for (int r = 0; r < kNAA; r++) {
        if (!read_at(f, h.addr[a++] + p0 * sizeof(float), col.data(), Nr * sizeof(float)))
            return fail("target probabilities");
        for (uint64_t i = 0; i < Nr; i++) trg[i * kNAA + r] = col[i];
    }
    for (int r = 0; r < kNCV; r++) {
        if (!read_at(f, h.addr[a++] + p0 * sizeof(float), col.data(), Nr * sizeof(float))) return fail("context vectors");
        for (uint64_t i = 0; i < Nr; i++) cv[i * kNCV + r] = col[i];
    }
    if (!read_at(f, h.addr[a++] + p0 * sizeof(float), cvprior, Nr * sizeof(float))) return fail("context vector priors");
    if (!read_at(f, h.addr[a++] + p0 * sizeof(float), cvnorm2, Nr * sizeof(float))) return fail("context vector norms");
    for (int r = 0; r < kNSS; r++) {
        if (!read_at(f, h.addr[a++] + p0 * sizeof(float), col.data(), Nr * sizeof(float))) return fail("SS probabilities");
        for (uint64_t i = 0; i < Nr; i++) ss[i * kNSS + r] = col[i];
    }
    a += 2;   // HDP1 cluster probabilities and indices: not used by this search path
    if (!read_at(f, h.addr[a++] + p0, aa, Nr)) return fail("residues");
    if (!read_at(f, h.addr[a++] + p0, ssstate, Nr)) return fail("SS states");
    // the description section ends the file: its last end address must be there
    uint64_t dend = 0;
    if (!read_at(f, h.addr[a] + (P - 1) * sizeof(uint64_t), &dend, sizeof dend) || dend < h.addr[a + 1] ||
        dend > h.fsize)
        return fail("descriptions");
    for (uint64_t i = 0; i < Nr; i++) {
        const uint8_t c = ssstate[i];
        ssstate[i] = (c >= 'a' && c <= 'z') ? (uint8_t)(c - 'a' + 'A') : c;   // ' ': no SS prediction
    }
    return C2_OK;
}
}  // namespace

extern "C" c2_status c2_db2bin_descriptions(const char* path, char* buf, size_t* bytes, int64_t* offsets, char* err,
                                            size_t errlen)
{
    if (!path || !bytes || (buf && !offsets)) return C2_ERR_ARG;
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) {
        set_err(err, errlen, std::string("cannot open ") + path);
        return C2_ERR_ARG;
    }
    Header h;
    c2_status st = read_header(F.f, h, err, errlen);
    if (st != C2_OK) return st;
    const uint64_t P = h.nprof;
    const uint64_t ends_at = h.addr[kNSECTIONS - 2], text_at = h.addr[kNSECTIONS - 1];
    try {
        std::vector<uint64_t> ends(P);
        if (!read_at(F.f, ends_at, ends.data(), P * sizeof(uint64_t))) {
            set_err(err, errlen, "truncated or inconsistent binary database: description addresses");
            return C2_ERR_ARG;
        }
        uint64_t prev = text_at;
        for (uint64_t k = 0; k < P; k++) {
            if (ends[k] < prev + 1 || ends[k] > h.fsize) {
                set_err(err, errlen, "truncated or inconsistent binary database: description addresses");
                return C2_ERR_ARG;
            }
            prev = ends[k];
        }
        const uint64_t total = prev - text_at;   // NUL-terminated descriptions back to back
        if (!buf) {
            *bytes = (size_t)total;
            return C2_OK;
        }
        if (*bytes < total) {
            set_err(err, errlen, "description buffer too small");
            return C2_ERR_ARG;
        }
        if (!read_at(F.f, text_at, buf, total)) {
            set_err(err, errlen, "truncated or inconsistent binary database: descriptions");
            return C2_ERR_ARG;
        }
        prev = text_at;
        for (uint64_t k = 0; k < P; k++) {
            offsets[k] = (int64_t)(prev - text_at);
            buf[ends[k] - text_at - 1] = 0;   // each description ends with its NUL
            prev = ends[k];
        }
        *bytes = (size_t)total;
        return C2_OK;
    } catch (...) {
        set_err(err, errlen, "out of host memory reading the binary database");
        return C2_ERR_NOMEM;
    }
}
