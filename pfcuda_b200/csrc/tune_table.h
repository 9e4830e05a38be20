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
    {0, 1, 34, 544, 1LL, 1LL, 1, 7, 2, 1},  // n=512 batch=1: 1.044 ms
    {0, 0, 34, 544, 1LL, 1LL, 1, 7, 2, 1},  // n=512 batch=1: 1.028 ms
    {0, 1, 34, 544, 2LL, 221LL, 1, 7, 2, 2},  // n=512 batch=74: 1.228 ms
    {0, 0, 34, 544, 2LL, 221LL, 1, 7, 1, 1},  // n=512 batch=74: 1.243 ms
    {0, 1, 34, 544, 222LL, 1099511627776LL, 2, 7, 1, 2},  // n=512 batch=296: 2.537 ms
    {0, 0, 34, 544, 222LL, 1099511627776LL, 2, 7, 1, 1},  // n=512 batch=296: 2.728 ms
    {0, 1, 546, 1056, 1LL, 1LL, 1, 7, 2, 1},  // n=1024 batch=1: 2.130 ms
    {0, 0, 546, 1056, 1LL, 1LL, 1, 7, 1, 1},  // n=1024 batch=1: 2.101 ms
    {0, 1, 546, 1056, 2LL, 98LL, 1, 7, 2, 2},  // n=1024 batch=33: 2.667 ms
    {0, 0, 546, 1056, 2LL, 98LL, 1, 7, 1, 1},  // n=1024 batch=33: 2.831 ms
    {0, 1, 546, 1056, 99LL, 1099511627776LL, 2, 7, 2, 2},  // n=1024 batch=132: 5.783 ms
    {0, 0, 546, 1056, 99LL, 1099511627776LL, 2, 7, 1, 1},  // n=1024 batch=132: 6.639 ms
    {0, 1, 1058, 2080, 1LL, 1LL, 1, 7, 2, 1},  // n=2048 batch=1: 4.333 ms
    {0, 0, 1058, 2080, 1LL, 1LL, 1, 7, 1, 1},  // n=2048 batch=1: 4.253 ms
    {0, 1, 1058, 2080, 2LL, 44LL, 1, 7, 2, 2},  // n=2048 batch=15: 5.947 ms
    {0, 0, 1058, 2080, 2LL, 44LL, 1, 7, 2, 1},  // n=2048 batch=15: 6.751 ms
    {0, 1, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 1, 2},  // n=2048 batch=60: 14.519 ms
    {0, 0, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 2, 1},  // n=2048 batch=60: 17.550 ms
    {0, 1, 2082, 4160, 1LL, 1LL, 1, 7, 2, 1},  // n=4096 batch=1: 9.256 ms
    {0, 0, 2082, 4160, 1LL, 1LL, 1, 7, 1, 1},  // n=4096 batch=1: 9.453 ms
    {0, 1, 2082, 4160, 2LL, 20LL, 1, 7, 1, 2},  // n=4096 batch=7: 13.873 ms
    {0, 0, 2082, 4160, 2LL, 20LL, 1, 7, 2, 1},  // n=4096 batch=7: 17.717 ms
    {0, 1, 2082, 4160, 21LL, 1099511627776LL, 2, 7, 2, 2},  // n=4096 batch=28: 34.758 ms
    {0, 0, 2082, 4160, 21LL, 1099511627776LL, 2, 7, 1, 1},  // n=4096 batch=28: 50.672 ms
    {0, 1, 4162, 8224, 1LL, 1LL, 1, 7, 1, 2},  // n=6144 batch=1: 20.188 ms
    {0, 0, 4162, 8224, 1LL, 1LL, 1, 7, 1, 1},  // n=6144 batch=1: 19.664 ms
    {0, 1, 4162, 8224, 2LL, 20LL, 1, 7, 2, 1},  // n=6144 batch=7: 44.561 ms
    {0, 0, 4162, 8224, 2LL, 20LL, 1, 7, 1, 1},  // n=6144 batch=7: 56.813 ms
    {0, 1, 4162, 8224, 21LL, 1099511627776LL, 1, 7, 1, 1},  // n=6144 batch=13: 72.602 ms
    {0, 0, 4162, 8224, 21LL, 1099511627776LL, 1, 7, 1, 1},  // n=6144 batch=13: 98.274 ms
    {1, 1, 34, 544, 1LL, 1LL, 2, 7, 1, 1},  // n=512 batch=1: 1.547 ms
    {1, 0, 34, 544, 1LL, 1LL, 2, 7, 2, 1},  // n=512 batch=1: 1.336 ms
    {1, 1, 34, 544, 2LL, 221LL, 2, 7, 1, 2},  // n=512 batch=74: 2.144 ms
    {1, 0, 34, 544, 2LL, 221LL, 2, 7, 2, 1},  // n=512 batch=74: 1.963 ms
    {1, 1, 34, 544, 222LL, 1099511627776LL, 2, 7, 2, 2},  // n=512 batch=296: 5.421 ms
    {1, 0, 34, 544, 222LL, 1099511627776LL, 2, 7, 2, 1},  // n=512 batch=296: 4.764 ms
    {1, 1, 546, 1056, 1LL, 1LL, 2, 7, 2, 1},  // n=1024 batch=1: 3.154 ms
    {1, 0, 546, 1056, 1LL, 1LL, 2, 7, 1, 1},  // n=1024 batch=1: 2.718 ms
    {1, 1, 546, 1056, 2LL, 98LL, 2, 7, 2, 2},  // n=1024 batch=33: 5.171 ms
    {1, 0, 546, 1056, 2LL, 98LL, 2, 7, 2, 1},  // n=1024 batch=33: 4.813 ms
    {1, 1, 546, 1056, 99LL, 1099511627776LL, 2, 7, 1, 1},  // n=1024 batch=132: 13.993 ms
    {1, 0, 546, 1056, 99LL, 1099511627776LL, 2, 7, 1, 1},  // n=1024 batch=132: 12.681 ms
    {1, 1, 1058, 2080, 1LL, 1LL, 2, 7, 2, 1},  // n=2048 batch=1: 6.551 ms
    {1, 0, 1058, 2080, 1LL, 1LL, 2, 7, 2, 1},  // n=2048 batch=1: 5.858 ms
    {1, 1, 1058, 2080, 2LL, 44LL, 2, 7, 2, 2},  // n=2048 batch=15: 13.028 ms
    {1, 0, 1058, 2080, 2LL, 44LL, 2, 7, 2, 1},  // n=2048 batch=15: 12.805 ms
    {1, 1, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 1, 1},  // n=2048 batch=59: 40.786 ms
    {1, 0, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 1, 1},  // n=2048 batch=59: 36.973 ms
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
