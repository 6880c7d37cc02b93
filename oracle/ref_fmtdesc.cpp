// TEST INFRASTRUCTURE (not part of the product): runs the reference's own
// description formatters, FormatDescription and FormatDescriptionJSON
// (src/liblib/fmtdescription.h, included from the reference tree at build
// time), on cases read from stdin, so that the tests can pin the report
// writer's restatement (comer2_b200/csrc/c2_report.cpp) to them.
//
// Input, one case per line:  mode maxoutlen indent width addsep<TAB>description
//   mode 0: FormatDescription(out, desc, maxoutlen, indent, width, 0, 0, addsep)
//   mode 1: FormatDescriptionJSON(out, desc, maxoutlen, 0)
// Output per case: the formatted bytes, then the record separator 0x1e '\n'.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "liblib/fmtdescription.h"

int main()
{
    static char line[1 << 20];
    while (fgets(line, sizeof line, stdin)) {
        size_t n = strlen(line);
        if (n && line[n - 1] == '\n') line[--n] = 0;
        char* tab = strchr(line, '\t');
        if (!tab) return 2;
        *tab = 0;
        int mode = 0, maxoutlen = 0, indent = 0, width = 0, addsep = 0;
        if (sscanf(line, "%d %d %d %d %d", &mode, &maxoutlen, &indent, &width, &addsep) != 5) return 2;
        const char* desc = tab + 1;
        std::vector<char> buf((size_t)maxoutlen * 4 + strlen(desc) * 4 + 4096, 0);
        char* start = buf.data() + 16;   // room for the "..." overwrite before the start
        char* out = start;
        int outpos = 0, linepos = 0;
        if (mode == 0) FormatDescription(out, desc, maxoutlen, indent, width, outpos, linepos, (char)addsep);
        else FormatDescriptionJSON(out, desc, maxoutlen, outpos);
        fwrite(start, 1, (size_t)(out - start), stdout);
        fputs("\x1e\n", stdout);
    }
    return 0;
}
