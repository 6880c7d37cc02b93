// TEST INFRASTRUCTURE ONLY (never part of the product): reads the reference's
// SS score table and CV score map with its own readers, SSSScores::ReadScores
// and CVS2Scores::ReadScores (src/libpro/srcpro/SSSScores.cpp,
// CVS2Scores.cpp: keys, smoothing, shift), compiled from the reference tree
// by oracle/Makefile into oracle/_ref/ref_tables, and prints what they hold.
// It pins the tables the parameter loader hands to the kernels.
//
// usage: ref_tables [<ssss file> <cvs2s file>]  (default: the reference tree's
// src/env files, whose directory the build passes as REF_ENV)
//   ssss <card> <n> v1 .. vn            (table 0 of probability level 0)
//   cvs2s <nlevels> <shift> <n> k1 s1 .. kn sn   (level 0, after smoothing)
//   cvconst <1/kappa0> <PowerNU0> <CTERM>        (the _TCTXVECT constants,
//                                                 src/libpro/srcpro/TCTXVECT.cpp)
#include <cstdio>

#include "libpro/srcpro/CVS2Scores.h"
#include "libpro/srcpro/SSSScores.h"
#include "libpro/srcpro/TCTXVECT.h"

#ifndef REF_ENV
#define REF_ENV "."
#endif

int main(int argc, char** argv)
{
    if (argc != 1 && argc != 3) {
        fprintf(stderr, "usage: %s [ssss cvs2s]\n", argv[0]);
        return 2;
    }
    const char* fss = argc == 3 ? argv[1] : REF_ENV "/ssss";
    const char* fcv = argc == 3 ? argv[2] : REF_ENV "/cvs2s";
    try {
        SSSScores sss;
        sss.ReadScores(fss);
        const extspsl::Pslvector* t = sss.GetScores()[0][0];
        printf("ssss %d %d", sss.GetCardinality(), t->GetSize());
        for (int i = 0; i < t->GetSize(); i++) printf(" %.9g", t->GetValueAt(i));
        printf("\n");
        CVS2Scores cvs;
        cvs.ReadScores(fcv);
        const CVS2Scores& cc = cvs;   // the public const accessors
        const extspsl::Pslvector* k = cc.GetKeys(0);
        const extspsl::Pslvector* s = cc.GetScores(0);
        printf("cvs2s %d %d %d", cc.GetNoTables(), cc.GetShift(0), k->GetSize());
        for (int i = 0; i < k->GetSize(); i++) printf(" %.9g %.9g", k->GetValueAt(i), s->GetValueAt(i));
        printf("\n");
        printf("cvconst %.9g %.9g %.9g\n", CVS.loKAPPA0, CVS.PowerNU0, CVS.CTERM);
    } catch (...) {
        fprintf(stderr, "reading the tables failed\n");
        return 1;
    }
    return 0;
}
