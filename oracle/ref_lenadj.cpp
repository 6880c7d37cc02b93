// TEST INFRASTRUCTURE ONLY (never part of the product): drives the
// reference's own length adjustment, AbstractScoreMatrix::ComputeLengthAdjustment
// (src/libpro/srcsco/AbstractScoreMatrix.cpp:247-380, Gertz 2005), compiled
// from the reference tree by oracle/Makefile into oracle/_ref/ref_lenadj.
// It pins the oracle's length_adjustment, and through the GPU test the
// search space that c2_set_query computes.
//
// usage: ref_lenadj lambda K alpha beta < lines "m n N" > lines "searchspace deltalen"
#include <cstdio>
#include <cstdlib>

#include "libpro/srcsco/AbstractScoreMatrix.h"

namespace {
// the abstract class with its pure virtuals stubbed: only the statistics
// members of the base are used
struct LenAdj : public AbstractScoreMatrix<float> {
    explicit LenAdj(Configuration* c) : AbstractScoreMatrix<float>(CuBatchLSO, c, StatisticsGiven) {}
    float GetScore(int, int) const override { return 0.f; }
    float GetModScore(int, int) const override { return 0.f; }
    void ComputeScoreMatrix(bool) override {}
    float GetFinalScore(float v) const override { return v; }
    void ScaleScoreMatrix() override {}
    void ComputeStatisticalParameters(bool) override {}
    void ComputeScoreProbabilities(ScoresAttr<float>*) override {}
    void PrintParameterTable(TPrintFunction, void*) const override {}
    void SetScore(int, int, float) override {}
    void SetModScore(int, int, float) override {}
    bool GetAllNegatives() const override { return false; }
    void SetAllNegatives(bool) override {}
    const float** GetScores() const override { return nullptr; }
};
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 5) {
        fprintf(stderr, "usage: %s lambda K alpha beta < \"m n N\" lines\n", argv[0]);
        return 2;
    }
    Configuration cfg[NoCTypes];
    for (int t = 0; t < NoCTypes; t++) {
        cfg[t].SetLambda((float)atof(argv[1]));
        cfg[t].SetK((float)atof(argv[2]));
        cfg[t].SetH(1.f);
        cfg[t].SetAlpha((float)atof(argv[3]));
        cfg[t].SetBeta((float)atof(argv[4]));
    }
    unsigned long long m, n, N;
    while (scanf("%llu %llu %llu", &m, &n, &N) == 3) {
        LenAdj h(cfg);   // a fresh object: the reference caches results per query length
        h.ComputeLengthAdjustment((size_t)m, (uint64_mt)n, (size_t)N);
        printf("%llu %llu\n", (unsigned long long)h.GetSearchSpace(), (unsigned long long)h.GetDeltaLength());
    }
    return 0;
}
