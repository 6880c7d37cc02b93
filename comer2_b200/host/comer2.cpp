// comer2.cpp -- the search program over the comer2_b200 C ABI: the reference
// `comer` program's command line, options file, query and database formats
// and result files (src/comer/comer.cpp:34-532, comer.h usage text), with the
// search itself on the B200 through include/comer2_b200.h.
//
//   comer2 -i <query> -d <db>[,<db>...] -o <outdir> [-p <options>] [-f 0|1]
//          [--dev-N=<n>|,<id>[,<id>...]] [--dev-mem=<MB>] [-v] [-h]
//
// Query: a text profile file, possibly several profiles stacked (the COMER
// v2.0 layout read by src/libmycu/cupro/IOProfileModelTxt.cu:47-1030), or a
// database made by makedb + db2bin given as <name>.prd (its <name>.bin is
// read; every profile is a query).  Databases: <name>.bin written by the
// reference's db2bin (format v2.2), several comma-separated names searched as
// one database.  Output: one file per query, <outdir>/<query base name>__<n>.
// json|out (AlnWriter::GetOutputFilename, src/libmycu/cualn/AlnWriter.cpp:
// 358-376), in the reference's JSON (-f 1) or Plain (-f 0) format.
//
// Parameters: the ungapped/gapped statistical constants, the SS score table,
// the context-vector score map and the SS18 model weights of the reference's
// install come from comer2_params.json beside the library (or the file named
// by COMER2_PARAMS); the options file (-p, the format of src/env/options.txt)
// overrides the option values.  --dev-N selects the GPUs (a count or a list),
// --dev-mem bounds the device memory the search may use on each
// (c2_set_device_memory_limit).  A database that does not fit in half
// of that memory (or of the device's free memory), or that is spread over
// several GPUs, is searched in chunks of consecutive profiles, as the
// reference's reader feeds its devices in portions: the chunks go round-robin
// to the GPUs, and a GPU with more than one chunk holds two handles, the next
// chunk read from file and uploaded on one while the other is searched.  The
// results are those of a single search.  The reference's other --dev-* and
// --io-* options are accepted and have no effect here.
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <future>
#include <map>
#include <exception>
#include <thread>
#include <mutex>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/comer2_b200.h"

namespace {

const char* kVersion = "2.03.03";
// citation lines of the reference's result files (liblib/msg.cpp:26-36)
const char* kReferences[] = {
    "Margelevicius, M. (2020). COMER2: GPU-accelerated sensitive and specific homology searches. "
    "Bioinformatics 36, 3570-3572.",
    "Margelevicius, M. (2016). Bayesian nonparametrics in protein remote homology search. "
    "Bioinformatics 32, 2744-2752.",
    nullptr};

int g_verbose = 0;

[[noreturn]] void die(const std::string& m)
{
    throw std::runtime_error(m);
}

void note(int level, const std::string& m)
{
    if (g_verbose >= level) fprintf(stderr, "[comer2] %s\n", m.c_str());
}

// ---------------------------------------------------------------------------
// A small JSON reader for the parameter file: objects, arrays, numbers and
// strings (no escapes beyond \" and \\ are needed there).
struct JVal {
    enum Kind { NUL, NUM, STR, ARR, OBJ } kind = NUL;
    double num = 0;
    std::string str;
    std::vector<JVal> arr;
    std::map<std::string, JVal> obj;
    const JVal& at(const std::string& k) const
    {
        auto it = obj.find(k);
        if (it == obj.end()) die("parameter file: missing key " + k);
        return it->second;
    }
    bool has(const std::string& k) const { return obj.count(k) != 0; }
};

struct JParser {
    const std::string s;
    size_t i = 0;
    explicit JParser(const std::string& t) : s(t) {}
    void ws()
    {
        while (i < s.size() && isspace((unsigned char)s[i])) i++;
    }
    JVal parse()
    {
        ws();
        if (i >= s.size()) die("parameter file: unexpected end");
        JVal v;
        const char c = s[i];
        if (c == '{') {
            v.kind = JVal::OBJ;
            i++;
            ws();
            if (s[i] == '}') { i++; return v; }
            for (;;) {
                ws();
                JVal k = parse();
                if (k.kind != JVal::STR) die("parameter file: object key");
                ws();
                if (s[i++] != ':') die("parameter file: ':' expected");
                v.obj[k.str] = parse();
                ws();
                if (s[i] == ',') { i++; continue; }
                if (s[i] == '}') { i++; break; }
                die("parameter file: ',' or '}' expected");
            }
        } else if (c == '[') {
            v.kind = JVal::ARR;
            i++;
            ws();
            if (s[i] == ']') { i++; return v; }
            for (;;) {
                v.arr.push_back(parse());
                ws();
                if (s[i] == ',') { i++; continue; }
                if (s[i] == ']') { i++; break; }
                die("parameter file: ',' or ']' expected");
            }
        } else if (c == '"') {
            v.kind = JVal::STR;
            i++;
            while (i < s.size() && s[i] != '"') {
                if (s[i] == '\\' && i + 1 < s.size()) i++;
                v.str += s[i++];
            }
            i++;
        } else if (s.compare(i, 4, "null") == 0) {
            i += 4;
        } else {
            v.kind = JVal::NUM;
            char* e = nullptr;
            v.num = strtod(s.c_str() + i, &e);
            if (e == s.c_str() + i) die("parameter file: bad value");
            i = (size_t)(e - s.c_str());
        }
        return v;
    }
};

std::string read_file(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) die("cannot open " + path);
    std::stringstream b;
    b << f.rdbuf();
    return b.str();
}

// option values as key -> value string (options.txt: KEY = value lines, '#'
// comments, [section] lines skipped), as MOptions reads them
std::map<std::string, std::string> parse_options(const std::string& text)
{
    std::map<std::string, std::string> o;
    std::istringstream in(text);
    std::string ln;
    while (std::getline(in, ln)) {
        const size_t a = ln.find_first_not_of(" \t\r");
        if (a == std::string::npos || ln[a] == '#' || ln[a] == '[') continue;
        const size_t eq = ln.find('=');
        if (eq == std::string::npos) continue;
        std::string k = ln.substr(a, eq - a);
        while (!k.empty() && isspace((unsigned char)k.back())) k.pop_back();
        std::istringstream vs(ln.substr(eq + 1));
        std::string v;
        vs >> v;
        o[k] = v;
    }
    return o;
}

// The context-vector score map as CVS2Scores::SmoothScores leaves it
// (src/libpro/srcpro/CVS2Scores.cpp): a 5-wide running mean in float over the
// scores that are not '+', assigned to every entry, then keys missing at step
// 1/2 inserted with the smoothed value, '+' entries taking it too; shift =
// number of negative keys.
const float kCvPlus = 9999.0f, kCvNA = -9999.0f;

void smooth_cvs2s(std::vector<float> keys, const std::vector<float>& vals, std::vector<float>& okeys,
                  std::vector<float>& ovals, int& shift)
{
    std::vector<float> scos(vals);
    const int n_el = (int)scos.size();
    const float incr = 1.0f / 2.0f;
    const int nswin = 5, nswinh = 2;
    std::vector<float> smth(n_el, 0.f);
    float rwin[5] = {0, 0, 0, 0, 0};
    float rsum = 0.f, avg = 0.f;
    int nv = 0, rn = 0, nn = 0;
    auto plus = [](float v) { return v >= kCvPlus; };
    for (int n = 0; n < n_el; n++) {
        const float sc = scos[n];
        if (sc <= kCvNA) die("cvs2s: NA score");
        if (nv < nswinh) nn++;
        if (!plus(sc)) {
            if (nswin <= rn) rn = 0;
            rsum = rsum - rwin[rn];
            rwin[rn++] = sc;
            rsum = rsum + sc;
            avg = rsum / (float)nswin;
            nv++;
        }
        if (nswin <= nv) {
            if (!plus(sc)) {
                if (nswin == nv)
                    for (int p = 0; p < nn; p++) smth[p] = avg;
                smth[nn++] = avg;
                while (nn < n && plus(scos[nn])) smth[nn++] = avg;
            }
            if (n_el == n + 1)
                for (int p = nn; p < n_el; p++) smth[p] = avg;
        }
    }
    float sm = 0.f;
    for (int n = n_el - 1; n >= 0; n--) {
        sm = smth[n];
        scos[n] = sm;
    }
    std::vector<float> kl(keys), vl(scos), sl(smth);
    float pkk = 0.f;
    for (size_t n = 0; n < kl.size();) {
        const float kk = kl[n], sc = vl[n];
        if (n && kk <= pkk) die("cvs2s: keys not sorted");
        if (n && incr < kk - pkk) {
            pkk = pkk + incr;
            kl.insert(kl.begin() + n, pkk);
            vl.insert(vl.begin() + n, sm);
            sl.insert(sl.begin() + n, sm);
            n++;
            continue;
        }
        pkk = kk;
        sm = sl[n];
        if (plus(sc)) vl[n] = sm;
        n++;
    }
    shift = 0;
    for (float k : kl) {
        if (0.0f <= k) break;
        shift++;
    }
    okeys = kl;
    ovals = vl;
}

struct Params {
    c2_params p{};
    std::vector<float> ssss, cvkeys, cvvals, nnw;
    std::map<std::string, std::string> opt;
    int opt_int(const char* k, int d) const
    {
        auto it = opt.find(k);
        return it == opt.end() ? d : atoi(it->second.c_str());
    }
    float opt_float(const char* k, float d) const
    {
        auto it = opt.find(k);
        return it == opt.end() ? d : (float)atof(it->second.c_str());
    }
};

void load_params(const std::string& json_path, const std::string& options_path, Params& P)
{
    JParser jp(read_file(json_path));
    const JVal d = jp.parse();
    const JVal& un = d.at("comer_par").at("UNGAPPED");
    const JVal& ga = d.at("comer_par").at("GAPPED_A_1");
    c2_params& p = P.p;
    p.ungapped_lambda = (float)un.at("Lambda").num;
    p.ungapped_K = (float)un.at("K").num;
    p.ungapped_H = (float)un.at("H").num;
    p.gapped_lambda = (float)ga.at("Lambda").num;
    p.gapped_K = (float)ga.at("K").num;
    p.gapped_H = (float)ga.at("H").num;
    p.gapped_alpha = (float)ga.at("Alpha").num;
    p.gapped_beta = (float)ga.at("Beta").num;
    for (const auto& kv : d.at("options").obj)
        P.opt[kv.first] = kv.second.kind == JVal::STR ? kv.second.str : std::to_string(kv.second.num);
    if (!options_path.empty())
        for (const auto& kv : parse_options(read_file(options_path))) P.opt[kv.first] = kv.second;
    p.eval = P.opt_float("EVAL", 10.f);
    p.ssswgt = P.opt_float("SSSWGT", 0.12f);
    p.cvswgt = P.opt_float("CVSWGT", 0.15f);
    p.minpp = P.opt_float("MINPP", 0.28f);
    p.mapaln = P.opt_int("MAPALN", 1);
    p.x_uninf = P.opt_int("X_UNINF", 1);
    p.ssemodel = P.opt_int("SSEMODEL", 2);
    // SS table: lower triangle, rows r of r + 1 values -> full symmetric matrix
    const int card = (int)d.at("ssss").at("card").num;
    const auto& tri = d.at("ssss").at("tri").arr;
    P.ssss.assign((size_t)card * card, 0.f);
    for (int r = 0; r < card; r++)
        for (int c = 0; c <= r; c++) {
            const float v = (float)tri.at((size_t)r * (r + 1) / 2 + c).num;
            P.ssss[(size_t)r * card + c] = P.ssss[(size_t)c * card + r] = v;
        }
    std::vector<float> rk, rv;
    for (const auto& x : d.at("cvs2s").at("keys").arr) rk.push_back((float)x.num);
    for (const auto& x : d.at("cvs2s").at("values").arr) rv.push_back((float)x.num);
    int shift = 0;
    smooth_cvs2s(rk, rv, P.cvkeys, P.cvvals, shift);
    for (const auto& x : d.at("sse_nn_weights").arr) P.nnw.push_back((float)x.num);
    p.ssss = P.ssss.data();
    p.ssss_card = card;
    p.cvs2s_keys = P.cvkeys.data();
    p.cvs2s_values = P.cvvals.data();
    p.cvs2s_card = (int32_t)P.cvkeys.size();
    p.cvs2s_shift = shift;
    p.sse_nn_weights = P.nnw.data();
    p.n_sse_nn_weights = (int32_t)P.nnw.size();
}

// ---------------------------------------------------------------------------
// Profiles in the c2_profiles field set, owned
struct Profiles {
    std::vector<int32_t> lengths;
    std::vector<int64_t> offsets;
    std::vector<float> bkg, eno, trn, trg, cv, cvprior, cvnorm2, ss;
    std::vector<uint8_t> ssstate, aa;
    std::vector<std::string> desc, name;
    std::vector<uint8_t> has_ss;
    int64_t npos() const { return offsets.empty() ? 0 : offsets.back() + lengths.back(); }
    int nprof() const { return (int)lengths.size(); }
    c2_profiles view() const
    {
        c2_profiles v{};
        v.nprofiles = nprof();
        v.npositions = npos();
        v.lengths = lengths.data();
        v.offsets = offsets.data();
        v.bkg = bkg.data();
        v.eno = eno.data();
        v.trn = trn.data();
        v.trg = trg.data();
        v.cv = cv.data();
        v.cvprior = cvprior.data();
        v.cvnorm2 = cvnorm2.data();
        v.ss = ss.data();
        v.ssstate = ssstate.data();
        v.aa = aa.data();
        return v;
    }
    // profile k alone
    Profiles one(int k) const
    {
        Profiles o;
        const int L = lengths[k];
        const int64_t b = offsets[k];
        o.lengths = {L};
        o.offsets = {0};
        o.bkg.assign(bkg.begin() + (size_t)k * 20, bkg.begin() + (size_t)(k + 1) * 20);
        o.eno = {eno[k]};
        o.trn.assign(trn.begin() + (size_t)(b + k) * 7, trn.begin() + (size_t)(b + k + L + 1) * 7);
        o.trg.assign(trg.begin() + (size_t)b * 20, trg.begin() + (size_t)(b + L) * 20);
        o.cv.assign(cv.begin() + (size_t)b * 19, cv.begin() + (size_t)(b + L) * 19);
        o.cvprior.assign(cvprior.begin() + b, cvprior.begin() + b + L);
        o.cvnorm2.assign(cvnorm2.begin() + b, cvnorm2.begin() + b + L);
        o.ss.assign(ss.begin() + (size_t)b * 3, ss.begin() + (size_t)(b + L) * 3);
        o.ssstate.assign(ssstate.begin() + b, ssstate.begin() + b + L);
        o.aa.assign(aa.begin() + b, aa.begin() + b + L);
        o.desc = {desc[k]};
        o.name = {name[k]};
        o.has_ss = {has_ss[k]};
        return o;
    }
    void append(const Profiles& o)
    {
        const int64_t base = npos();
        for (int k = 0; k < o.nprof(); k++) {
            lengths.push_back(o.lengths[k]);
            offsets.push_back(base + o.offsets[k]);
        }
        auto cat = [](auto& a, const auto& b) { a.insert(a.end(), b.begin(), b.end()); };
        cat(bkg, o.bkg); cat(eno, o.eno); cat(trn, o.trn); cat(trg, o.trg); cat(cv, o.cv);
        cat(cvprior, o.cvprior); cat(cvnorm2, o.cvnorm2); cat(ss, o.ss); cat(ssstate, o.ssstate);
        cat(aa, o.aa); cat(desc, o.desc); cat(name, o.name); cat(has_ss, o.has_ss);
    }
};

// transition working value of a probability: natural log (x 0.4 for the
// IM, II, DM, DD transitions), -32768 for probability 0
// (IOProfileModelTxt.cu:366, 512)
float trn_value(int t7, float p)
{
    if (!(p != 0.f)) return -32768.f;
    const float lg = (float)std::log((double)p);
    return t7 >= 3 ? lg * 0.4f : lg;
}

std::vector<long> ints_of(const std::string& s, size_t from = 0)
{
    std::vector<long> v;
    const char* c = s.c_str() + std::min(from, s.size());
    char* e = nullptr;
    for (;;) {
        while (*c == ' ' || *c == '\t' || *c == '\r') c++;
        if (!*c) break;
        const long x = strtol(c, &e, 10);
        if (e == c) break;
        v.push_back(x);
        c = e;
    }
    return v;
}

std::string after(const std::string& ln, const char* key)
{
    std::string v = ln.substr(strlen(key));
    const size_t a = v.find_first_not_of(" \t");
    v = (a == std::string::npos) ? std::string() : v.substr(a);
    while (!v.empty() && (v.back() == '\r' || v.back() == ' ')) v.pop_back();
    return v;
}

bool starts(const std::string& s, const char* p)
{
    const size_t a = s.find_first_not_of(" \t");
    return a != std::string::npos && s.compare(a, strlen(p), p) == 0;
}

// One or more stacked COMER v2.0 text profiles (full or condensed layout):
// header keys, NULL background, beginning transitions, then per position the
// residue and target probabilities, transitions (9 values, ID and DI
// dropped), MID observations, HDP cluster lines, optional CT:, CV: and SS:
// lines; '*' ends a profile.  Probabilities are integer / SCALE in float.
Profiles read_text_profiles(const std::string& path)
{
    std::istringstream in(read_file(path));
    std::vector<std::string> L;
    for (std::string ln; std::getline(in, ln);) {
        if (!ln.empty() && ln.back() == '\r') ln.pop_back();
        L.push_back(ln);
    }
    Profiles all;
    size_t i = 0;
    const size_t n = L.size();
    auto need = [&](size_t j, const char* what) {
        if (j >= n) die(path + ": truncated profile (" + what + ")");
    };
    while (i < n) {
        if (!starts(L[i], "COMER profile v")) { i++; continue; }
        i++;
        std::string desc, file;
        int len = -1, scale = 10000;
        float eno = 0.f;
        while (i < n && !starts(L[i], "NULL")) {
            const std::string& s = L[i];
            if (starts(s, "DESC:")) desc = after(s.substr(s.find("DESC:")), "DESC:");
            else if (starts(s, "FILE:")) file = after(s.substr(s.find("FILE:")), "FILE:");
            else if (starts(s, "LEN:")) len = atoi(after(s.substr(s.find("LEN:")), "LEN:").c_str());
            else if (starts(s, "EFFNOS:")) eno = (float)atof(after(s.substr(s.find("EFFNOS:")), "EFFNOS:").c_str());
            else if (starts(s, "SCALE:")) scale = atoi(after(s.substr(s.find("SCALE:")), "SCALE:").c_str());
            i++;
        }
        need(i, "NULL");
        if (len < 1 || len > 65535) die(path + ": profile length missing or out of range");
        if (scale < 1) die(path + ": bad SCALE");
        const float fs = (float)scale;
        Profiles P;
        P.lengths = {len};
        P.offsets = {0};
        const std::vector<long> bk = ints_of(L[i], L[i].find("NULL") + 4);
        if (bk.size() < 20) die(path + ": short NULL line");
        for (int a = 0; a < 20; a++) P.bkg.push_back((float)bk[a] / fs);
        P.eno = {eno};
        i += 2;   // POST
        need(i, "beginning transitions");
        std::vector<long> t9 = ints_of(L[i++]);
        if (t9.size() < 9) die(path + ": short beginning transitions");
        auto push_trn = [&](const std::vector<long>& t) {
            const long v[7] = {t[0], t[1], t[2], t[3], t[4], t[6], t[8]};
            for (int k = 0; k < 7; k++) P.trn.push_back(trn_value(k, (float)v[k] / fs));
        };
        push_trn(t9);
        i++;   // beginning MID observations
        bool ss_any = false;
        for (int m = 0; m < len; m++) {
            while (i < n && L[i].find_first_not_of(" \t") == std::string::npos) i++;
            need(i, "position");
            std::istringstream ps(L[i]);
            int num = 0;
            std::string res;
            ps >> num >> res;
            if (num != m + 1 || res.empty()) die(path + ": bad numbering at position " + std::to_string(m + 1));
            P.aa.push_back((uint8_t)res[0]);
            for (int a = 0; a < 20; a++) {
                long x = 0;
                if (!(ps >> x)) die(path + ": short target probabilities at position " + std::to_string(m + 1));
                P.trg.push_back((float)x / fs);
            }
            i++;
            need(i, "transitions");
            t9 = ints_of(L[i++]);
            if (t9.size() < 9) die(path + ": short transitions at position " + std::to_string(m + 1));
            push_trn(t9);
            i++;   // MID observations
            need(i, "HDP entries");
            const std::vector<long> hd = ints_of(L[i++]);
            if (hd.size() >= 2 && hd[1] > 0) i += 2;
            float prior = 0.f, norm2 = 0.f, s3[3] = {0.f, 0.f, 0.f};
            std::vector<float> cvv(19, 0.f);
            uint8_t sst = 'C';
            bool have_cv = false, have_ss = false;
            while (i < n && (starts(L[i], "CT:") || starts(L[i], "CV:") || starts(L[i], "SS:"))) {
                const std::string& s = L[i];
                const size_t a = s.find_first_not_of(" \t");
                if (starts(s, "CV:")) {
                    const std::vector<long> v = ints_of(s, a + 3);
                    if (v.size() < 3 || (long)v.size() < 3 + v[2] || v[2] != 19)
                        die(path + ": bad CV line at position " + std::to_string(m + 1));
                    prior = (float)v[0] / fs;
                    norm2 = (float)v[1] / fs;
                    for (int t = 0; t < 19; t++) cvv[t] = (float)v[3 + t] / fs;
                    have_cv = true;
                } else if (starts(s, "SS:")) {
                    sst = (uint8_t)s[a + 3];
                    const std::vector<long> v = ints_of(s, a + 4);
                    if (v.size() < 3) die(path + ": bad SS line at position " + std::to_string(m + 1));
                    for (int t = 0; t < 3; t++) s3[t] = (float)v[t] / fs;
                    have_ss = true;
                }
                i++;
            }
            if (!have_cv) die(path + ": no context vector at position " + std::to_string(m + 1));
            ss_any = ss_any || have_ss;
            P.cv.insert(P.cv.end(), cvv.begin(), cvv.end());
            P.cvprior.push_back(prior);
            P.cvnorm2.push_back(norm2);
            P.ss.insert(P.ss.end(), s3, s3 + 3);
            P.ssstate.push_back(sst >= 'a' && sst <= 'z' ? (uint8_t)(sst - 'a' + 'A') : sst);
        }
        while (i < n && !starts(L[i], "*")) i++;
        i++;
        P.desc = {desc};
        P.name = {file};
        P.has_ss = {(uint8_t)(ss_any ? 1 : 0)};
        all.append(P);
    }
    if (all.nprof() == 0) die(path + ": no COMER profile found");
    return all;
}

void ck_db(c2_status st, const char* err, const std::string& what)
{
    if (st != C2_OK) die(what + ": " + err);
}

// A database written by db2bin (<name>.bin): every profile's length and
// description, the profiles themselves read by range (read_db_range)
struct DbFile {
    std::string name, path;
    std::vector<int32_t> lengths;
    std::vector<std::string> desc;
    int64_t npos = 0;
    int nprof() const { return (int)lengths.size(); }
};

DbFile open_db(const std::string& name)
{
    DbFile F;
    F.name = name;
    std::string path = name;
    if (path.size() > 4 && path.compare(path.size() - 4, 4, ".prd") == 0) path = path.substr(0, path.size() - 4);
    if (path.size() < 4 || path.compare(path.size() - 4, 4, ".bin") != 0) path += ".bin";
    F.path = path;
    char err[512] = {0};
    int32_t P = 0;
    ck_db(c2_db2bin_info(path.c_str(), &P, &F.npos, err, sizeof err), err, path);
    F.lengths.resize(P);
    ck_db(c2_db2bin_lengths(path.c_str(), F.lengths.data(), err, sizeof err), err, path);
    size_t bytes = 0;
    ck_db(c2_db2bin_descriptions(path.c_str(), nullptr, &bytes, nullptr, err, sizeof err), err, path);
    std::vector<char> buf(bytes + 1, 0);
    std::vector<int64_t> off(P);
    ck_db(c2_db2bin_descriptions(path.c_str(), buf.data(), &bytes, off.data(), err, sizeof err), err, path);
    F.desc.resize(P);
    for (int k = 0; k < P; k++) F.desc[k] = std::string(buf.data() + off[k]);
    return F;
}

// Profiles [k0, k1) of a database file
Profiles read_db_range(const DbFile& F, int32_t k0, int32_t k1)
{
    int64_t N = 0;
    for (int k = k0; k < k1; k++) N += F.lengths[k];
    const int P = k1 - k0;
    char err[512] = {0};
    Profiles D;
    D.lengths.resize(P);
    D.offsets.resize(P);
    D.bkg.resize((size_t)P * 20);
    D.eno.resize(P);
    D.trn.resize((size_t)(N + P) * 7);
    D.trg.resize((size_t)N * 20);
    D.cv.resize((size_t)N * 19);
    D.cvprior.resize(N);
    D.cvnorm2.resize(N);
    D.ss.resize((size_t)N * 3);
    D.ssstate.resize(N);
    D.aa.resize(N);
    ck_db(c2_db2bin_read_range(F.path.c_str(), k0, k1, D.lengths.data(), D.offsets.data(), D.bkg.data(), D.eno.data(),
                               D.trn.data(), D.trg.data(), D.cv.data(), D.cvprior.data(), D.cvnorm2.data(),
                               D.ss.data(), D.ssstate.data(), D.aa.data(), err, sizeof err),
          err, F.path);
    D.desc.assign(F.desc.begin() + k0, F.desc.begin() + k1);
    D.name.resize(P);
    D.has_ss.resize(P);
    for (int k = 0; k < P; k++) {
        // db2bin writes ' ' as the SS state of profiles without predictions
        bool ss = false;
        for (int64_t j = D.offsets[k]; j < D.offsets[k] + D.lengths[k] && !ss; j++) ss = D.ssstate[j] != ' ';
        D.has_ss[k] = ss ? 1 : 0;
    }
    return D;
}

Profiles read_db(const std::string& name)
{
    const DbFile F = open_db(name);
    if (F.nprof() == 0) return Profiles{};
    return read_db_range(F, 0, F.nprof());
}

// The databases cut into chunks for the device: runs of consecutive profiles
// (pieces of one or more files) whose upload fits in `cap` bytes
// (c2_db_device_bytes); each chunk is uploaded with the totals of all
// databases and searched in turn.  A profile too large for cap alone makes a
// chunk of its own (its upload then reports the allocation failure).
struct Piece {
    int file;
    int32_t k0, k1;
};
struct Chunk {
    std::vector<Piece> pieces;
    int64_t gbase = 0;   // index of the chunk's first profile over all databases
    int32_t nprof = 0;
    int64_t npos = 0;
};

std::vector<Chunk> plan_chunks(c2_handle* h, const std::vector<DbFile>& F, uint64_t cap)
{
    std::vector<Chunk> C;
    Chunk cur;
    int32_t lmax = 0;
    int64_t g = 0;
    auto fits = [&](int64_t n, int32_t p, int32_t l) {
        uint64_t b = 0;
        if (c2_db_device_bytes(h, n, p, l, &b) != C2_OK) die("c2_db_device_bytes failed");
        return cap == 0 || b <= cap;
    };
    for (int f = 0; f < (int)F.size(); f++) {
        for (int32_t k = 0; k < F[f].nprof(); k++, g++) {
            const int32_t L = F[f].lengths[k];
            if (cur.nprof > 0 && !fits(cur.npos + L, cur.nprof + 1, std::max(lmax, L))) {
                C.push_back(cur);
                cur = Chunk{};
                lmax = 0;
            }
            if (cur.nprof == 0) cur.gbase = g;
            if (cur.pieces.empty() || cur.pieces.back().file != f) cur.pieces.push_back(Piece{f, k, k});
            cur.pieces.back().k1 = k + 1;
            cur.nprof++;
            cur.npos += L;
            lmax = std::max(lmax, L);
        }
    }
    if (cur.nprof > 0) C.push_back(cur);
    return C;
}

Profiles read_chunk(const std::vector<DbFile>& F, const Chunk& c)
{
    Profiles D;
    for (const Piece& p : c.pieces) D.append(read_db_range(F[p.file], p.k0, p.k1));
    return D;
}

std::string base_name(const std::string& p)
{
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? p : p.substr(s + 1);
}

void mkdirs(const std::string& d)
{
    std::string cur;
    for (size_t i = 0; i <= d.size(); i++) {
        if (i == d.size() || d[i] == '/') {
            if (!cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
                die("cannot create directory " + cur);
        }
        if (i < d.size()) cur += d[i];
    }
}

void usage(FILE* f, const char* prog)
{
    fprintf(f,
            "%s %s -- COMER2 profile-profile search on a B200 GPU\n\n"
            "Usage:\n"
            "%s -i <query> -d <database> [-o <output>] [-p <options>] [<other_options>]\n\n"
            "-i <query_profiles>         (stacked) profile(s) in COMER text format, or a\n"
            "                            database (extension .prd) made by makedb+db2bin.\n"
            "-d <database_name_list>     Database(s) made by makedb+db2bin, comma-separated.\n"
            "-o <output_directory>       Directory of output files for each query.\n"
            "-f <file_format>            Format of output files: 0, Plain; 1, JSON.  Default=0\n"
            "-p <options_file>           Input file of options (the format of options.txt).\n"
            "--dev-N=(<number>|,<id_list>) GPUs to use: a number, or a list starting with a comma;\n"
            "                            the database is split across them.  Default=1\n"
            "--dev-mem=<megabytes>       Maximum amount of GPU memory the search may use.\n"
            "-v [<level_number>]         Verbose mode.\n"
            "-h                          This text.\n",
            base_name(prog).c_str(), kVersion, base_name(prog).c_str());
}

struct Args {
    std::string query, dbs, outdir = ".", options;
    bool print_inputs = false;   // print the parsed parameters and profiles, search nothing
    int format = 0;
    std::vector<int> devices{0};   // --dev-N: GPUs to search on
    long long devmem_mb = 0;
};

Args parse_args(int argc, char** argv)
{
    Args a;
    for (int i = 1; i < argc; i++) {
        std::string s = argv[i];
        auto val = [&](const char* opt) -> std::string {
            if (i + 1 >= argc) die(std::string("option ") + opt + " needs a value");
            return argv[++i];
        };
        if (s == "-i") a.query = val("-i");
        else if (s == "-d") a.dbs = val("-d");
        else if (s == "-o") a.outdir = val("-o");
        else if (s == "-p") a.options = val("-p");
        else if (s == "-f") {
            a.format = atoi(val("-f").c_str());
            if (a.format != 0 && a.format != 1) die("-f: 0 (Plain) or 1 (JSON)");
        } else if (s == "-v") {
            g_verbose = 1;
            if (i + 1 < argc && isdigit((unsigned char)argv[i + 1][0])) g_verbose = atoi(argv[++i]);
        } else if (s == "-h") {
            usage(stdout, argv[0]);
            exit(0);
        } else if (s == "--print-inputs") {
            a.print_inputs = true;
        } else if (s.rfind("--dev-N=", 0) == 0) {
            const std::string v = s.substr(8);
            // ",<id>,<id>...": the listed GPUs; "<n>": GPUs 0 .. n-1 (at most
            // as many as there are)
            a.devices.clear();
            if (!v.empty() && v[0] == ',') {
                std::stringstream ds(v.substr(1));
                for (std::string id; std::getline(ds, id, ',');)
                    if (!id.empty()) a.devices.push_back(atoi(id.c_str()));
            } else {
                int32_t have = 0;
                c2_get_device_count(&have);
                const int n = std::max(1, std::min(atoi(v.c_str()), std::max(1, (int)have)));
                for (int d = 0; d < n; d++) a.devices.push_back(d);
            }
            if (a.devices.empty()) die("--dev-N: no GPU given");
        } else if (s.rfind("--dev-mem=", 0) == 0) {
            a.devmem_mb = atoll(s.c_str() + 10);
        } else if (s.rfind("--dev-", 0) == 0 || s.rfind("--io-", 0) == 0) {
            note(1, "option " + s + " has no effect in this implementation");
        } else {
            die("unknown argument " + s + " (-h for help)");
        }
    }
    if (a.query.empty() || a.dbs.empty()) die("both -i and -d are required (-h for help)");
    return a;
}

// The parsed inputs as text, every value with 9 significant digits (a check
// of the parsers against other readers of the same files)
void print_vec(const char* tag, const float* v, size_t n)
{
    printf("%s %zu", tag, n);
    for (size_t i = 0; i < n; i++) printf(" %.9g", v[i]);
    printf("\n");
}

void print_inputs(const Params& P, const Profiles& Q, const Profiles& D)
{
    const c2_params& p = P.p;
    const float sc[] = {p.ungapped_lambda, p.ungapped_K, p.ungapped_H, p.gapped_lambda, p.gapped_K, p.gapped_H,
                        p.gapped_alpha, p.gapped_beta, p.eval, p.ssswgt, p.cvswgt, p.minpp};
    print_vec("scalars", sc, 12);
    printf("ints %d %d %d %d %d\n", p.mapaln, p.x_uninf, p.ssemodel, p.ssss_card, p.cvs2s_shift);
    print_vec("ssss", P.ssss.data(), P.ssss.size());
    print_vec("cvkeys", P.cvkeys.data(), P.cvkeys.size());
    print_vec("cvvals", P.cvvals.data(), P.cvvals.size());
    print_vec("nnw", P.nnw.data(), P.nnw.size());
    for (const Profiles* S : {&Q, &D}) {
        const char* w = S == &Q ? "q" : "d";
        printf("%s.n %d %lld\n", w, S->nprof(), (long long)S->npos());
        std::vector<float> ln(S->lengths.begin(), S->lengths.end());
        const std::pair<const char*, const std::vector<float>*> f[] = {
            {"bkg", &S->bkg}, {"eno", &S->eno}, {"trn", &S->trn}, {"trg", &S->trg}, {"cv", &S->cv},
            {"cvprior", &S->cvprior}, {"cvnorm2", &S->cvnorm2}, {"ss", &S->ss}, {"lengths", &ln}};
        for (const auto& x : f) print_vec((std::string(w) + "." + x.first).c_str(), x.second->data(), x.second->size());
        printf("%s.aa %s\n", w, std::string(S->aa.begin(), S->aa.end()).c_str());
        printf("%s.ssstate %s\n", w, std::string(S->ssstate.begin(), S->ssstate.end()).c_str());
        for (int k = 0; k < S->nprof(); k++) printf("%s.desc %d %s\n", w, k, S->desc[k].c_str());
    }
}

void ck(c2_handle* h, c2_status st, const char* what)
{
    if (st == C2_OK) return;
    char buf[512] = {0};
    if (h) c2_last_error(h, buf, sizeof buf);
    die(std::string(what) + " failed (status " + std::to_string((int)st) + "): " + buf);
}

std::string params_path()
{
    if (const char* e = getenv("COMER2_PARAMS")) return e;
    // comer2_params.json in the package's data folder, next to the folder
    // holding this program
    char self[4096];
    const ssize_t n = readlink("/proc/self/exe", self, sizeof self - 1);
    if (n > 0) {
        self[n] = 0;
        std::string d(self);
        d = d.substr(0, d.find_last_of('/'));        // .../comer2_b200/_lib
        d = d.substr(0, d.find_last_of('/'));        // .../comer2_b200
        return d + "/data/comer2_params.json";
    }
    return "comer2_params.json";
}

int run(int argc, char** argv)
{
    const Args A = parse_args(argc, argv);
    Params P;
    load_params(params_path(), A.options, P);
    // queries
    Profiles Q;
    const std::string& qi = A.query;
    const bool qdb = qi.size() > 4 && (qi.compare(qi.size() - 4, 4, ".prd") == 0 || qi.compare(qi.size() - 4, 4, ".bin") == 0);
    Q = qdb ? read_db(qi) : read_text_profiles(qi);
    // databases, searched as one
    std::vector<DbFile> F;
    int64_t totN = 0, totP = 0;
    {
        std::stringstream ss(A.dbs);
        for (std::string nm; std::getline(ss, nm, ',');) {
            if (nm.empty()) continue;
            F.push_back(open_db(nm));
            totN += F.back().npos;
            totP += F.back().nprof();
        }
    }
    if (totP == 0) die("no database profiles");
    if (A.print_inputs) {
        Profiles D;
        for (const DbFile& f : F)
            if (f.nprof() > 0) D.append(read_db_range(f, 0, f.nprof()));
        print_inputs(P, Q, D);
        return 0;
    }
    note(1, "queries: " + std::to_string(Q.nprof()) + "; database: " + std::to_string(totP) + " profiles, " +
                std::to_string(totN) + " positions");
    // Device memory (per GPU): the --dev-mem limit, or what is free on the
    // device.  Half of what a handle does not hold yet goes to its database
    // chunk, the rest to the query and the phase-2 scratch (split into
    // candidate groups under the limit).  A database in more than one chunk
    // per GPU is double-buffered: two handles per GPU, each with half of the
    // memory, the next chunk read and uploaded on one while the other is
    // searched.  With several GPUs the chunks go round-robin to the GPUs.
    const int ndev = (int)A.devices.size();
    auto make_handle = [&](int dev, uint64_t lim) {
        c2_handle* hh = nullptr;
        const c2_status st = c2_create(dev, &P.p, &hh);
        if (st != C2_OK)
            die("c2_create on GPU " + std::to_string(dev) + " failed (status " + std::to_string((int)st) +
                "): check the GPU and the options (MAPALN 0 or 1, SSEMODEL 0..2, SS and CV weights >= 0)");
        if (A.devmem_mb > 0) ck(hh, c2_set_device_memory_limit(hh, lim), "c2_set_device_memory_limit");
        return hh;
    };
    c2_handle* h = make_handle(A.devices[0], (uint64_t)A.devmem_mb << 20);
    std::unique_ptr<c2_handle, c2_status (*)(c2_handle*)> guard(h, c2_destroy);
    uint64_t limit = 0, used0 = 0;
    if (A.devmem_mb > 0) {
        limit = (uint64_t)A.devmem_mb << 20;
    } else {
        uint64_t fr = 0, tot = 0;
        ck(h, c2_get_device_memory_info(h, &fr, &tot), "c2_get_device_memory_info");
        limit = fr;
    }
    ck(h, c2_get_device_memory_use(h, &used0), "c2_get_device_memory_use");
    if (limit <= used0) die("--dev-mem: the limit is below the memory the search's tables need");
    std::vector<Chunk> chunks = plan_chunks(h, F, (limit - used0) / 2);
    bool dbuf = false;   // two handles per GPU
    if (chunks.size() > 1 || ndev > 1) {
        if (limit / 2 <= used0) die("--dev-mem: the limit is below the memory two searches' tables need");
        uint64_t cap = (limit / 2 - used0) / 2;
        if (ndev > 1) {
            // at least one chunk per GPU
            int32_t lmax = 0;
            for (const auto& f : F)
                for (int32_t L : f.lengths) lmax = std::max(lmax, L);
            uint64_t all = 0;
            ck(h, c2_db_device_bytes(h, totN, (int32_t)totP, lmax, &all), "c2_db_device_bytes");
            cap = std::min<uint64_t>(cap, all / (uint64_t)ndev + 1);
        }
        chunks = plan_chunks(h, F, cap);
        dbuf = chunks.size() > (size_t)ndev;
        if (dbuf && A.devmem_mb > 0) ck(h, c2_set_device_memory_limit(h, limit / 2), "c2_set_device_memory_limit");
    }
    note(1, "database in " + std::to_string(chunks.size()) + " chunk(s) on " + std::to_string(ndev) + " GPU(s)");
    mkdirs(A.outdir);
    std::string qbase = base_name(qi);
    {
        const size_t pos = qbase.rfind('.');
        if (pos != std::string::npos && qbase.size() - pos <= 4) qbase = qbase.substr(0, pos);
    }
    // per query: the hits of every chunk (global profile indices), and the
    // search space and thresholds (the same for every chunk: they depend on
    // the query and the database totals only)
    struct QueryHits {
        std::vector<c2_hit> hits;
        std::vector<char> alns;
        uint64_t sspace = 0, dlen = 0;
        float thld = 0.f, logevthld = 0.f;
    };
    std::vector<QueryHits> acc(Q.nprof());
    std::mutex acc_mu;
    std::vector<const char*> dbn;
    for (const auto& f : F) dbn.push_back(f.name.c_str());
    std::vector<std::string> desc_all;
    std::vector<int32_t> len_all;
    std::vector<float> eno_all((size_t)totP);
    std::vector<uint8_t> ss_all((size_t)totP);
    for (const auto& f : F) {
        desc_all.insert(desc_all.end(), f.desc.begin(), f.desc.end());
        len_all.insert(len_all.end(), f.lengths.begin(), f.lengths.end());
    }
    std::vector<Profiles> queries;
    for (int qn = 0; qn < Q.nprof(); qn++) queries.push_back(Q.one(qn));
    // read a chunk from file and upload it to handle hh (with the totals of
    // all databases)
    auto load = [&](size_t ci, c2_handle* hh) {
        const Profiles D = read_chunk(F, chunks[ci]);
        const int64_t gb = chunks[ci].gbase;
        for (int k = 0; k < D.nprof(); k++) {
            eno_all[(size_t)(gb + k)] = D.eno[k];
            ss_all[(size_t)(gb + k)] = D.has_ss[k];
        }
        const c2_profiles dv = D.view();
        ck(hh, c2_upload_db(hh, &dv, (uint64_t)totN, (uint64_t)totP), "c2_upload_db");
    };
    // every query against the chunk uploaded to hh, through the batch call
    // (two workers, a query's phase 2 beside the next query's phase 1, unless
    // --dev-mem bounds the memory: the second worker's query and phase-2
    // buffers would come out of the chunk's budget); hits into acc with global
    // profile indices
    const int batch_workers = A.devmem_mb > 0 ? 1 : 2;
    const c2_profiles qall = Q.view();
    struct BatchCtx {
        std::vector<QueryHits>* acc;
        std::mutex* mu;
        int64_t gb;
        int failed_query = -1;
        c2_status failed = C2_OK;
    };
    auto on_query = [](void* user, int32_t q, c2_status st, const c2_hit* hits, int32_t nh, const char* alns,
                       size_t abytes) {
        BatchCtx* ctx = static_cast<BatchCtx*>(user);
        std::lock_guard<std::mutex> lk(*ctx->mu);
        if (st != C2_OK) {
            if (ctx->failed == C2_OK) { ctx->failed = st; ctx->failed_query = q; }
            return;
        }
        QueryHits& a = (*ctx->acc)[q];
        const int64_t base = (int64_t)a.alns.size();
        for (int i = 0; i < nh; i++) {
            c2_hit x = hits[i];
            x.profile += (int32_t)ctx->gb;
            x.aln_offset += base;
            a.hits.push_back(x);
        }
        a.alns.insert(a.alns.end(), alns, alns + abytes);
    };
    auto search_chunk = [&](size_t ci, c2_handle* hh) {
        BatchCtx ctx{&acc, &acc_mu, chunks[ci].gbase};
        const c2_status st = c2_search_batch(hh, &qall, batch_workers, on_query, &ctx);
        if (st != C2_OK || ctx.failed != C2_OK) {
            char buf[512] = {0};
            c2_last_error(hh, buf, sizeof buf);
            die("c2_search_batch failed (status " + std::to_string((int)(st != C2_OK ? st : ctx.failed)) +
                (ctx.failed_query >= 0 ? ", query " + std::to_string(ctx.failed_query) : std::string()) + "): " + buf);
        }
        note(2, "chunk " + std::to_string(ci + 1) + "/" + std::to_string(chunks.size()) + " searched");
    };
    // one worker per GPU over its chunks (ci = w, w + ndev, ...)
    auto worker = [&](int w) {
        std::vector<size_t> mine;
        for (size_t ci = (size_t)w; ci < chunks.size(); ci += (size_t)ndev) mine.push_back(ci);
        if (mine.empty()) return;
        const uint64_t lim = dbuf ? limit / 2 : limit;
        std::unique_ptr<c2_handle, c2_status (*)(c2_handle*)> h0(w == 0 ? nullptr : make_handle(A.devices[w], lim),
                                                                 c2_destroy);
        std::unique_ptr<c2_handle, c2_status (*)(c2_handle*)> h1(mine.size() > 1 ? make_handle(A.devices[w], lim)
                                                                                 : nullptr,
                                                                 c2_destroy);
        c2_handle* H[2] = {w == 0 ? h : h0.get(), h1.get()};
        load(mine[0], H[0]);
        for (size_t i = 0; i < mine.size(); i++) {
            std::exception_ptr up_err;
            std::thread up;
            if (i + 1 < mine.size())
                up = std::thread([&, i]() {
                    try {
                        load(mine[i + 1], H[(i + 1) & 1]);
                    } catch (...) {
                        up_err = std::current_exception();
                    }
                });
            std::exception_ptr err;
            try {
                search_chunk(mine[i], H[i & 1]);
            } catch (...) {
                err = std::current_exception();
            }
            if (up.joinable()) up.join();
            if (err) std::rethrow_exception(err);
            if (up_err) std::rethrow_exception(up_err);
        }
    };
    {
        std::vector<std::exception_ptr> errs(ndev);
        std::vector<std::thread> th;
        for (int w = 1; w < ndev; w++)
            th.emplace_back([&, w]() {
                try {
                    worker(w);
                } catch (...) {
                    errs[w] = std::current_exception();
                }
            });
        try {
            worker(0);
        } catch (...) {
            errs[0] = std::current_exception();
        }
        for (auto& t : th) t.join();
        for (auto& e : errs)
            if (e) std::rethrow_exception(e);
    }
    // search space and thresholds of every query (database totals; any
    // handle with a chunk uploaded has them)
    for (int qn = 0; qn < Q.nprof(); qn++) {
        QueryHits& a = acc[qn];
        ck(h, c2_get_query_limits(h, Q.lengths[qn], &a.sspace, &a.dlen, &a.thld, &a.logevthld),
           "c2_get_query_limits");
    }
    std::vector<const char*> ddesc;
    for (const auto& s : desc_all) ddesc.push_back(s.c_str());
    for (int qn = 0; qn < Q.nprof(); qn++) {
        const Profiles& q = queries[qn];
        QueryHits& a = acc[qn];
        // one list over the chunks in the order of a single search: by log
        // E-value, then profile index
        std::stable_sort(a.hits.begin(), a.hits.end(), [](const c2_hit& x, const c2_hit& y) {
            if (x.logE != y.logE) return x.logE < y.logE;
            return x.profile < y.profile;
        });
        const int32_t nh = (int32_t)a.hits.size();
        a.alns.push_back(0);
        c2_report_info r{};
        r.progname = "comer";
        r.progversion = kVersion;
        r.references = kReferences;
        r.query_desc = q.desc[0].c_str();
        r.query_length = q.lengths[0];
        r.query_eno = q.eno[0];
        r.query_has_ss = q.has_ss[0];
        r.db_names = dbn.data();
        r.n_db_names = (int32_t)dbn.size();
        r.db_positions = (uint64_t)totN;
        r.db_profiles = (uint64_t)totP;
        r.logevthld = a.logevthld;
        r.searchspace = (double)a.sspace;
        r.deltalen = (int32_t)a.dlen;
        r.ref_lambda = P.p.ungapped_lambda;
        r.ref_K = P.p.ungapped_K;
        r.gapped_lambda = P.p.gapped_lambda;
        r.gapped_K = P.p.gapped_K;
        r.print_ss = P.p.ssswgt > 0.f ? 1 : 0;
        r.dsclen = P.opt_int("DSCLEN", 1024);
        r.dscwidth = P.opt_int("DSCWIDTH", 60);
        r.alnwidth = P.opt_int("ALNWIDTH", 60);
        r.show = P.opt_int("SHOW", 1);
        r.nhits = P.opt_int("NOHITS", 700);
        r.nalns = P.opt_int("NOALNS", 700);
        r.db_desc = ddesc.data();
        r.db_lengths = len_all.data();
        r.db_eno = eno_all.data();
        r.db_has_ss = ss_all.data();
        if (a.hits.empty()) a.hits.resize(1);   // nh = 0: a valid pointer, nothing read
        const c2_hit* hp = a.hits.data();
        size_t obytes = 0;
        ck(h, c2_format_report(A.format, &r, hp, nh, a.alns.data(), nullptr, &obytes), "c2_format_report");
        std::vector<char> out(obytes + 1, 0);
        ck(h, c2_format_report(A.format, &r, hp, nh, a.alns.data(), out.data(), &obytes), "c2_format_report");
        const std::string fn = A.outdir + (A.outdir.empty() || A.outdir.back() == '/' ? "" : "/") + qbase + "__" +
                               std::to_string(qn) + (A.format == C2_REPORT_JSON ? ".json" : ".out");
        FILE* f = fopen(fn.c_str(), "wb");
        if (!f) die("cannot write " + fn);
        const size_t len = strlen(out.data());
        const bool ok = fwrite(out.data(), 1, len, f) == len;
        if (fclose(f) != 0 || !ok) die("write failed: " + fn);
        note(1, "query " + std::to_string(qn) + ": " + std::to_string(nh) + " hits -> " + fn);
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        fprintf(stderr, "[comer2] ERROR: %s\n", e.what());
        return 1;
    }
}
