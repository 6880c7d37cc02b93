// c2_report.cpp -- the reference's result files, Plain and JSON, from the
// hits of one query (c2_get_hits) and the run's details.
//
// Layouts, line by line, as the reference writes them:
//  * file frame: AlnWriter::WriteResultsPlain / WriteResultsJSON with
//    WritePrognamePlain/JSON, WriteQueryDescriptionPlain/JSON,
//    WriteSearchInformationPlain/JSON, WriteSummaryPlain/JSON
//    (src/libmycu/cualn/AlnWriterPlain.cpp:19-398, AlnWriterJSON.cpp:15-427);
//  * per hit: CuBatchProcessingFinalizer::CompressResultsPlain/JSON with
//    MakeAnnotation*, FormatScores*, FormatAlignment*, FormatFooter*
//    (src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:30-395,
//    CuBatchProcessingFinalizerJSON.cpp:30-380);
//  * description wrapping: FormatDescription / FormatDescriptionJSON
//    (src/liblib/fmtdescription.h:35-127);
//  * E-value, P-value and bit score: CuBatchProcessingFinalizer.h:179-188.
// Newlines are "\n" (the reference's NL on Unix, src/liblib/platform.h:34).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/comer2_b200.h"

namespace {

constexpr int kIndent = 13;        // OUTPUTINDENT
constexpr int kAnnotLen = 75;      // ANNOTATIONLEN
constexpr float kLogDpMax = 7.0978271289338397e+02f;
constexpr float kLn2 = 0.69314718055994530941723212146f;
const char* const NL = "\n";

void addf(std::string& o, const char* fmt, ...)
{
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    const int n = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (n > 0) o.append(buf, std::min(n, (int)sizeof buf - 1));
}

bool blank(char c) { return c == ' ' || c == '\t'; }

// Description copy with word wrapping at width (lines after the first start
// after indent spaces), at most maxoutlen characters, "..." over the last
// three when cut; addsep is written first when non-zero.
void fmt_desc(std::string& o, const char* desc, int maxoutlen, int indent, int width, int& outpos, int& linepos,
              char addsep)
{
    while (*desc && (blank(*desc) || *desc == '\n' || *desc == '\r')) desc++;
    if (addsep) {
        o.push_back(addsep);
        outpos++;
        linepos++;
    }
    while (*desc && outpos < maxoutlen) {
        if (blank(*desc)) {
            while (*desc && blank(*desc)) desc++;
            bool wrap = false;
            if (width < maxoutlen) {
                int loc = linepos + 1;
                for (const char* p = desc; *p && !blank(*p) && loc < width; p++, loc++) {}
                wrap = width <= loc;
            }
            if (wrap) {
                o += NL;
                outpos += (int)strlen(NL);
                o.append((size_t)indent, ' ');
                outpos += indent;
                linepos = indent;
            } else {
                o.push_back(' ');
                outpos++;
                linepos++;
            }
            continue;
        }
        o.push_back(*desc++);
        outpos++;
        linepos++;
    }
    if (maxoutlen <= outpos && 3 < maxoutlen)
        for (int i = 1; i <= 3 && (size_t)i <= o.size(); i++) o[o.size() - i] = '.';
}

// JSON string contents: blanks collapsed, '"', '\\' and '/' escaped, at most
// maxoutlen characters, "..." (over trailing escapes too) when cut
void fmt_desc_json(std::string& o, const char* desc, int maxoutlen, int& outpos)
{
    const size_t start = o.size();
    while (*desc && (blank(*desc) || *desc == '\n' || *desc == '\r')) desc++;
    while (*desc && outpos < maxoutlen) {
        if (blank(*desc)) {
            while (*desc && blank(*desc)) desc++;
            o.push_back(' ');
            outpos++;
            continue;
        }
        if (*desc == '"' || *desc == '\\' || *desc == '/') {
            o.push_back('\\');
            outpos++;
            if (maxoutlen <= outpos) break;
        }
        o.push_back(*desc++);
        outpos++;
    }
    if (maxoutlen <= outpos && 3 < maxoutlen) {
        const size_t n = o.size() - start;
        size_t i = 1;
        for (; i <= 3 && i <= n; i++) o[o.size() - i] = '.';
        for (; (int)i <= outpos && i <= n && o[o.size() - i] == '\\'; i++) o[o.size() - i] = '.';
    }
}

double evalue_of(float loge) { return kLogDpMax < loge ? 1.0e+308 : std::exp((double)loge); }
double pvalue_of(double e) { return e < 0.01 ? e : 1.0 - std::exp(-e); }
float bits_of(float sspace, float loge) { return sspace <= 0.0f ? 0.0f : (logf(sspace) - loge) / kLn2; }

struct Hit {
    const c2_hit* h;
    const char *q, *m, *t, *qs, *ts;   // alignment strings
};

Hit hit_at(const c2_hit* hits, const char* alns, int i)
{
    Hit x;
    x.h = hits + i;
    const int L = hits[i].alnlen;
    const char* b = alns + hits[i].aln_offset;
    x.q = b;
    x.m = b + (L + 1);
    x.t = b + 2 * (L + 1);
    x.qs = b + 3 * (L + 1);
    x.ts = b + 4 * (L + 1);
    return x;
}

const char* desc_of(const c2_report_info* r, int prof)
{
    return (r->db_desc && r->db_desc[prof]) ? r->db_desc[prof] : nullptr;
}

bool db_ss(const c2_report_info* r, int prof) { return !r->db_has_ss || r->db_has_ss[prof] != 0; }

// ---- Plain
void plain_annotation(std::string& o, const c2_report_info* r, const Hit& x)
{
    const size_t st = o.size();
    int outpos = 0, linepos = 0;
    if (const char* d = desc_of(r, x.h->profile)) fmt_desc(o, d, kAnnotLen, 0, kAnnotLen, outpos, linepos, 0);
    const int written = (int)(o.size() - st);
    if (written < kAnnotLen) o.append((size_t)(kAnnotLen - written), ' ');
    addf(o, " %7.0f %7.1g%s", x.h->score, evalue_of(x.h->logE), NL);
}

void plain_hit(std::string& o, const c2_report_info* r, const Hit& x, float sspace)
{
    const c2_hit& h = *x.h;
    const int prof = h.profile;
    const int width = kIndent < r->dscwidth ? r->dscwidth : 1;
    int outpos = 0, linepos = 0;
    if (const char* d = desc_of(r, prof)) fmt_desc(o, d, r->dsclen, kIndent, width, outpos, linepos, '>');
    o += NL;
    // scores
    const int alnlen = h.alnlen;
    const double ev = evalue_of(h.logE);
    addf(o, "  Length/ENO: Query = %d/%.1f, Sbjct = %d/%.1f%s%s", r->query_length, r->query_eno,
         r->db_lengths[prof], r->db_eno[prof], NL, NL);
    addf(o, " Score = %.2f (%.1f bits),  Expect = %.2g, P-value = %.2g%s", h.score, bits_of(sspace, h.logE), ev,
         pvalue_of(ev), NL);
    if (h.idts > 0) addf(o, " Identities = %d/%d (%d%%)", h.idts, alnlen, h.idts * 100 / alnlen);
    if (h.psts > 0) {
        if (h.idts) o += ",";
        addf(o, " Positives = %d/%d (%d%%)", h.psts, alnlen, h.psts * 100 / alnlen);
    }
    if (h.gaps > 0) {
        if (h.idts || h.psts) o += ",";
        addf(o, " Gaps = %d/%d (%d%%)", h.gaps, alnlen, h.gaps * 100 / alnlen);
    }
    addf(o, "%s%s", NL, NL);
    // alignment in fragments of alnwidth columns
    unsigned qb = (h.beg & 0xffffu) + 1, tb = (h.beg >> 16) + 1;
    const bool ss = r->print_ss && r->query_has_ss && db_ss(r, prof);
    const int w = r->alnwidth;
    for (int f = 0; f < alnlen; f += w) {
        const int nb = std::min(w, alnlen - f);
        if (ss) {
            addf(o, "%-13s", "struct");
            o.append(x.qs + f, (size_t)nb);
            o += NL;
        }
        {
            addf(o, "Query: %5u ", qb);
            o.append(x.q + f, (size_t)nb);
            const int g = (int)std::count(x.q + f, x.q + f + nb, '-');
            qb += nb - g;
            addf(o, " %-5d%s", nb <= g ? (int)qb : (int)qb - 1, NL);
        }
        addf(o, "%13c", ' ');
        o.append(x.m + f, (size_t)nb);
        o += NL;
        {
            addf(o, "Sbjct: %5u ", tb);
            o.append(x.t + f, (size_t)nb);
            const int g = (int)std::count(x.t + f, x.t + f + nb, '-');
            tb += nb - g;
            addf(o, " %-5d%s", nb <= g ? (int)tb : (int)tb - 1, NL);
        }
        if (ss) {
            addf(o, "%-13s", "struct");
            o.append(x.ts + f, (size_t)nb);
            o += NL;
        }
        o += NL;
    }
    if (r->show) {
        char kb[64], lb[64];
        const char *kp = "n/a", *lp = "n/a";
        addf(o, "%25c  %-6s   %-6s%s", ' ', "K", "Lambda", NL);
        if (h.E < 0.0f) {
            if (h.K > 0.0f) { snprintf(kb, sizeof kb, "%6.4f", h.K); kp = kb; }
            if (h.lambda > 0.0f) { snprintf(lb, sizeof lb, "%6.4f", h.lambda); lp = lb; }
        }
        addf(o, "%-25s  %6s   %6s%s", "Computed  ungapped,", kp, lp, NL);
        kp = lp = "n/a";
        if (h.E < 0.0f) {
            if (h.K_est > 0.0f) { snprintf(kb, sizeof kb, "%6.4f", h.K_est); kp = kb; }
            if (h.lambda_est > 0.0f) { snprintf(lb, sizeof lb, "%6.4f", h.lambda_est); lp = lb; }
        }
        addf(o, "%-25s  %6s   %6s%s", "Estimated gapped,", kp, lp, NL);
        addf(o, "Entropy, %6.4f; Expected, %6.4f; Min/Max, %.0f/%-.0f%s%s", h.H, h.E, (float)h.smin, (float)h.smax,
             NL, NL);
    }
    addf(o, "%s%s", NL, NL);
}

void summary_counts(const c2_report_info* r, int& effq, unsigned long long& effdb)
{
    effq = r->query_length;
    effdb = r->db_positions;
    if (r->deltalen < r->query_length) effq -= r->deltalen;
    if (r->db_profiles * (unsigned long long)r->deltalen < r->db_positions)
        effdb -= r->db_profiles * (unsigned long long)r->deltalen;
}

// The frame writers work against the reference's buffer budgets: the first
// three sections share a 4 KB writer buffer (the query description at most
// DSCLEN of it) and the database section a 1 KB one (AlnWriter.h:43-44);
// text beyond a budget is cut as the reference cuts it.
constexpr int kWriterBuffer = 4096, kTmpBuffer = 1024, kBufMax = 256;

// WritePrognamePlain: returns the bytes written
int plain_progname(std::string& o, const c2_report_info* r, int maxsize)
{
    const size_t st = o.size();
    if (r->progname) o += r->progname;
    if (r->progversion) addf(o, " %s", r->progversion);
    if (r->progname || r->progversion) addf(o, "%s%s", NL, NL);
    maxsize -= (int)(o.size() - st) + 3 * (int)strlen(NL) + 1;
    if (maxsize < 1) return (int)(o.size() - st);
    int outpos = 0, linepos = 0;
    for (int i = 0; r->references && r->references[i] && outpos < maxsize; i++) {
        fmt_desc(o, r->references[i], maxsize, 0, r->dscwidth, outpos, linepos, 0);
        o += NL;
        outpos += (int)strlen(NL);
        linepos = 0;
    }
    o += NL;
    return (int)(o.size() - st);
}

void plain_query(std::string& o, const c2_report_info* r, int maxsize)
{
    if (maxsize < 40) return;
    const size_t st = o.size();
    addf(o, "%s Query (%d positions):%s", NL, r->query_length, NL);
    maxsize -= (int)(o.size() - st);
    if (maxsize < 1) return;
    int outpos = 0, linepos = 0;
    if (r->query_desc) fmt_desc(o, r->query_desc, maxsize, 0, r->dscwidth, outpos, linepos, 0);
}

void plain_search_info(std::string& o, const c2_report_info* r, bool found)
{
    const int maxsize = kTmpBuffer;
    int size = 0;
    const char* dots = "...\n\n";
    auto over = [&](int delta) {
        if (maxsize < size + delta) {
            if (size + (int)strlen(dots) < maxsize) {
                o += dots;
                size += (int)strlen(dots);
            }
            return true;
        }
        return false;
    };
    auto put = [&](const std::string& t) {
        o += t;
        size += (int)t.size();
    };
    if (over(30)) return;
    put(std::string(NL) + NL + " Database(s):" + NL);
    for (int i = 0; i < r->n_db_names; i++) {
        const std::string nm = r->db_names[i] ? r->db_names[i] : "";
        const size_t n = std::min<size_t>(nm.size(), 100);
        if (over((int)n + 2)) return;
        std::string t = nm.substr(0, n);
        if (n < nm.size() && 3 < n)
            for (int k = 1; k <= 3; k++) t[t.size() - k] = '.';
        put(t + NL);
    }
    char buf[256];
    if (over(kIndent + 40)) return;
    snprintf(buf, sizeof buf, "%*s%llu profiles%s", kIndent, "", (unsigned long long)r->db_profiles, NL);
    put(buf);
    if (over(kIndent + 50)) return;
    snprintf(buf, sizeof buf, "%*s%llu total positions%s%s%s", kIndent, "", (unsigned long long)r->db_positions, NL,
             NL, NL);
    put(buf);
    if (over(kAnnotLen * 2)) return;
    if (found) {
        std::string t = " Profiles found below the e-value threshold:";
        while ((int)t.size() < kAnnotLen) t.push_back(' ');
        snprintf(buf, sizeof buf, " %7s %7s%s%s", "Score", "E-value", NL, NL);
        put(t + buf);
    } else {
        snprintf(buf, sizeof buf, " No profiles found below an e-value threshold of %g.%s%s%s",
                 std::exp(r->logevthld), NL, NL, NL);
        put(buf);
    }
}

void plain_file(std::string& o, const c2_report_info* r, const c2_hit* hits, int nhits, const char* alns)
{
    const float sspace = (float)r->searchspace;
    const int used = plain_progname(o, r, kWriterBuffer);
    plain_query(o, r, std::min(kWriterBuffer - used, r->dsclen));
    plain_search_info(o, r, nhits > 0);
    if (nhits > 0) {
        for (int i = 0; i < nhits && i < r->nhits; i++) plain_annotation(o, r, hit_at(hits, alns, i));
        addf(o, "%s%s%s", NL, NL, NL);
        for (int i = 0; i < nhits && i < r->nalns; i++) plain_hit(o, r, hit_at(hits, alns, i), sspace);
    }
    // summary
    int effq;
    unsigned long long effdb;
    summary_counts(r, effq, effdb);
    addf(o, "%-20s  %-6s   %-6s%s", "Reference values of", "K", "Lambda", NL);
    addf(o, "%-20s  %6.4f   %6.4f%s", "Ungapped", r->ref_K, r->ref_lambda, NL);
    addf(o, "%-20s  %6.4f   %6.4f%s%s", "Gapped", r->gapped_K, r->gapped_lambda, NL, NL);
    addf(o, "Length of query, %d%s", r->query_length, NL);
    addf(o, "Length of database, %llu%s", (unsigned long long)r->db_positions, NL);
    addf(o, "Effective length of query, %d%s", effq, NL);
    addf(o, "Effective length of database, %llu%s", effdb, NL);
    addf(o, "Effective search space, %llu%s%s", (unsigned long long)(size_t)sspace, NL, NL);
}

// ---- JSON
void json_annotation(std::string& o, const c2_report_info* r, const Hit& x)
{
    addf(o, "    {\"summary_entry\": {%s      \"description\": \"", NL);
    int outpos = 0;
    if (const char* d = desc_of(r, x.h->profile)) fmt_desc_json(o, d, kAnnotLen, outpos);
    addf(o, "\",%s", NL);
    addf(o, "      \"score\": %.0f,%s      \"evalue\": %.2g%s    }}", x.h->score, NL, evalue_of(x.h->logE), NL);
}

void json_hit(std::string& o, const c2_report_info* r, const Hit& x, float sspace)
{
    const c2_hit& h = *x.h;
    const int prof = h.profile;
    addf(o, "    {\"hit_record\": {%s      \"target_description\": \"", NL);
    int outpos = 0;
    if (const char* d = desc_of(r, prof)) fmt_desc_json(o, d, r->dsclen, outpos);
    addf(o, "\",%s", NL);
    addf(o,
         "      \"query_length\": %d,%s      \"query_eno\": %.1f,%s      \"target_length\": %d,%s"
         "      \"target_eno\": %.1f,%s      \"alignment\": {%s",
         r->query_length, NL, r->query_eno, NL, r->db_lengths[prof], NL, r->db_eno[prof], NL, NL);
    const int alnlen = h.alnlen;
    const double ev = evalue_of(h.logE);
    addf(o,
         "        \"score\": %.2f,%s        \"bit_score\": %.1f,%s        \"evalue\": %.2g,%s"
         "        \"pvalue\": %.2g,%s",
         h.score, NL, bits_of(sspace, h.logE), NL, ev, NL, pvalue_of(ev), NL);
    addf(o,
         "        \"n_identities\": %d,%s        \"n_positives\": %d,%s        \"n_gaps\": %d,%s"
         "        \"aln_length\": %d,%s",
         h.idts, NL, h.psts, NL, h.gaps, NL, alnlen, NL);
    const unsigned qb = (h.beg & 0xffffu) + 1, tb = (h.beg >> 16) + 1;
    const int gq = (int)std::count(x.q, x.q + alnlen, '-'), gt = (int)std::count(x.t, x.t + alnlen, '-');
    const unsigned qe = qb + alnlen - gq, te = tb + alnlen - gt;
    const int ss = (r->query_has_ss && db_ss(r, prof)) ? 1 : 0;
    addf(o,
         "        \"query_from\": %u,%s        \"query_to\": %u,%s        \"target_from\": %u,%s"
         "        \"target_to\": %u,%s",
         qb, NL, alnlen <= gq ? qe : qe - 1, NL, tb, NL, alnlen <= gt ? te : te - 1, NL);
    addf(o, "        \"query_secstr_available\": %d,%s        \"target_secstr_available\": %d,%s"
            "        \"query_secstr\": \"", ss, NL, ss, NL);
    if (ss) o.append(x.qs, (size_t)alnlen);
    addf(o, "\",%s        \"target_secstr\": \"", NL);
    if (ss) o.append(x.ts, (size_t)alnlen);
    addf(o, "\",%s        \"query_aln\": \"", NL);
    o.append(x.q, (size_t)alnlen);
    addf(o, "\",%s        \"target_aln\": \"", NL);
    o.append(x.t, (size_t)alnlen);
    addf(o, "\",%s        \"middle\": \"", NL);
    o.append(x.m, (size_t)alnlen);
    addf(o, "\",%s", NL);
    char kb[64], lb[64];
    const char *kp = "NA", *lp = "NA";
    if (h.E < 0.0f) {
        if (h.K > 0.0f) { snprintf(kb, sizeof kb, "%6.4f", h.K); kp = kb; }
        if (h.lambda > 0.0f) { snprintf(lb, sizeof lb, "%6.4f", h.lambda); lp = lb; }
    }
    addf(o, "        \"computed_K_ungapped\": \"%s\",%s        \"computed_lambda_ungapped\": \"%s\",%s", kp, NL, lp,
         NL);
    kp = lp = "NA";
    if (h.E < 0.0f) {
        if (h.K_est > 0.0f) { snprintf(kb, sizeof kb, "%6.4f", h.K_est); kp = kb; }
        if (h.lambda_est > 0.0f) { snprintf(lb, sizeof lb, "%6.4f", h.lambda_est); lp = lb; }
    }
    addf(o,
         "        \"estimated_K_gapped\": \"%s\",%s        \"estimated_lambda_gapped\": \"%s\",%s"
         "        \"entropy\": %.4f,%s        \"expected_score\": %.4f,%s        \"min_score\": %.0f,%s"
         "        \"max_score\": %.0f%s",
         kp, NL, lp, NL, h.H, NL, h.E, NL, (float)h.smin, NL, (float)h.smax, NL);
    addf(o, "      }%s    }}", NL);
}

int json_progname(std::string& o, const c2_report_info* r, int maxsize)
{
    const size_t st = o.size();
    addf(o, "{\"comer_search\": {%s  \"program\": \"%s\",%s  \"version\": \"%s\",%s", NL,
         r->progname ? r->progname : "", NL, r->progversion ? r->progversion : "", NL);
    maxsize -= (int)(o.size() - st) + 1024;
    if (maxsize < 1) return (int)(o.size() - st);
    addf(o, "  \"references\": [%s", NL);
    const int maxref = 1024 - 60;
    int tot = 0;
    bool wr = true;
    const char* const* refs = r->references;
    for (int i = 0; !i || (wr && refs && refs[i]); i++) {
        const char* s = refs ? refs[i] : nullptr;
        tot += s ? (int)strlen(s) : 0;
        wr = tot < maxref;
        addf(o, "    \"%s\"%s%s", (wr && s) ? s : "", (wr && s && refs[i + 1]) ? "," : "", NL);
    }
    addf(o, "  ],%s", NL);
    return (int)(o.size() - st);
}

void json_query(std::string& o, const c2_report_info* r, int maxsize)
{
    if (maxsize < 60) return;
    const size_t st = o.size();
    addf(o, "  \"query\": {%s    \"length\": %d,%s", NL, r->query_length, NL);
    maxsize -= (int)(o.size() - st) + kBufMax;
    if (maxsize < 1) return;
    int outpos = 0;
    const size_t a = o.size();
    o += "    \"name\": \"";
    addf(o, "\",%s", NL);
    o += "    \"description\": \"";
    outpos += (int)(o.size() - a);
    if (r->query_desc) fmt_desc_json(o, r->query_desc, maxsize, outpos);
    addf(o, "\"%s  },%s", NL, NL);
}

void json_search_info(std::string& o, const c2_report_info* r, bool found)
{
    int maxsize = kTmpBuffer;
    auto over = [&](int delta) {
        maxsize -= delta;
        return maxsize < 1;
    };
    if (over(40 * 7)) return;
    addf(o, "  \"database\": {%s    \"names\": [%s", NL, NL);
    for (int i = 0; i < r->n_db_names; i++) {
        const char* nm = r->db_names[i] ? r->db_names[i] : "";
        const int n = (int)std::min<size_t>(strlen(nm), 99);
        if (over(n + 15)) {
            o += "      \"...\"";
            o += NL;
            break;
        }
        o += "      \"";
        int outpos = 0;
        fmt_desc_json(o, nm, n + 1, outpos);
        if (i + 1 < r->n_db_names) addf(o, "\",%s", NL);
        else addf(o, "\"%s", NL);
    }
    addf(o, "    ],%s    \"number_of_profiles\": %llu,%s    \"number_of_positions\": %llu%s  },%s", NL,
         (unsigned long long)r->db_profiles, NL, (unsigned long long)r->db_positions, NL, NL);
    if (over(90 * 4)) return;
    if (found) addf(o, "  \"message\": \"Profiles found below the e-value threshold:\",%s", NL);
    else addf(o, "  \"message\": \"No profiles found below an e-value threshold of %g\",%s", std::exp(r->logevthld), NL);
}

void json_file(std::string& o, const c2_report_info* r, const c2_hit* hits, int nhits, const char* alns)
{
    const float sspace = (float)r->searchspace;
    const int used = json_progname(o, r, kWriterBuffer);
    json_query(o, r, std::min(kWriterBuffer - used, r->dsclen));
    json_search_info(o, r, nhits > 0);
    addf(o, "  \"search_summary\": [%s", NL);
    for (int i = 0; i < nhits && i < r->nhits; i++) {
        json_annotation(o, r, hit_at(hits, alns, i));
        const bool last = !(i + 1 < nhits && i + 1 < r->nhits);
        o += last ? NL : ",\n";
    }
    addf(o, "  ],%s  \"search_hits\": [%s", NL, NL);
    // the separator after an alignment record tests the hit-list bound, as the
    // reference's writer does (AlnWriterJSON.cpp:108)
    for (int i = 0; i < nhits && i < r->nalns; i++) {
        json_hit(o, r, hit_at(hits, alns, i), sspace);
        const bool last = !(i + 1 < nhits && i + 1 < r->nhits);
        o += last ? NL : ",\n";
    }
    addf(o, "  ],%s", NL);
    int effq;
    unsigned long long effdb;
    summary_counts(r, effq, effdb);
    addf(o,
         "  \"search_statistics\": {%s    \"reference_K_ungapped\": %.4f,%s    \"reference_lambda_ungapped\": %.4f,%s"
         "    \"reference_K_gapped\": %.4f,%s    \"reference_lambda_gapped\": %.4f,%s    \"query_length\": %d,%s"
         "    \"database_size\": %llu,%s    \"effective_query_length\": %d,%s"
         "    \"effective_database_size\": %llu,%s    \"effective_search_space\": %llu%s  }%s}}%s",
         NL, r->ref_K, NL, r->ref_lambda, NL, r->gapped_K, NL, r->gapped_lambda, NL, r->query_length, NL,
         (unsigned long long)r->db_positions, NL, effq, NL, effdb, NL, (unsigned long long)(size_t)sspace, NL, NL, NL);
}

}  // namespace

extern "C" c2_status c2_format_report(int32_t format, const c2_report_info* info, const c2_hit* hits, int32_t nhits,
                                      const char* alns, char* out, size_t* out_bytes)
{
    if (!info || !out_bytes || nhits < 0 || (nhits > 0 && (!hits || !alns || !info->db_lengths || !info->db_eno)))
        return C2_ERR_ARG;
    if (format != C2_REPORT_PLAIN && format != C2_REPORT_JSON) return C2_ERR_ARG;
    if (info->alnwidth < 1 || info->dsclen < 1 || info->dscwidth < 1 || info->nhits < 0 || info->nalns < 0)
        return C2_ERR_ARG;
    for (int i = 0; i < nhits; i++)
        if (hits[i].profile < 0 || hits[i].alnlen < 0) return C2_ERR_ARG;
    std::string o;
    if (format == C2_REPORT_PLAIN) plain_file(o, info, hits, nhits, alns);
    else json_file(o, info, hits, nhits, alns);
    if (!out) {
        *out_bytes = o.size() + 1;
        return C2_OK;
    }
    if (*out_bytes < o.size() + 1) {
        *out_bytes = o.size() + 1;
        return C2_ERR_ARG;
    }
    memcpy(out, o.c_str(), o.size() + 1);
    *out_bytes = o.size() + 1;
    return C2_OK;
}
