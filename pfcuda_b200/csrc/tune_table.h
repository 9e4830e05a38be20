// tune_table.h -- generated by pfcuda_b200/build.py from pfcuda_b200/tune_table.json
// (the table pfcuda_b200/tune.py measures); do not edit.
#pragma once
#include <stdint.h>

#include "../../include/pfb200.h"

namespace pfb {

struct TuneEntry {
    int cplx, split, n_min, n_max;
    long long batch_min, batch_max;
    int panel, slices, ranges, epilogue;
};

static const TuneEntry kTuneTable[] = {
    {-1, -1, 0, 0, 0LL, 0LL, 0, 0, 0, 0},  // (no measured entries)
};

// The first entry for this dtype class and mode whose order and batch bins
// hold (n, batch), else the defaults.
inline pfb_slog_config tuned_config(int dtype, int n, int64_t batch, bool split)
{
    const int cplx = (dtype == PFB_C64 || dtype == PFB_C128) ? 1 : 0;
    for (const TuneEntry &e : kTuneTable)
        if (e.cplx == cplx && e.split == (split ? 1 : 0) && n >= e.n_min && n <= e.n_max &&
            batch >= e.batch_min && batch <= e.batch_max)
            return pfb_slog_config{e.panel, e.slices, e.ranges, e.epilogue};
    return pfb_slog_config{1, 7, 2, 1};
}

}  // namespace pfb
