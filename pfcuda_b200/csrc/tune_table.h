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
    {0, 1, 34, 544, 1LL, 1LL, 1, 7, 2, 1},  // n=512 batch=1: 1.033 ms
    {0, 0, 34, 544, 1LL, 1LL, 1, 7, 2, 1},  // n=512 batch=1: 1.013 ms
    {0, 1, 34, 544, 2LL, 221LL, 1, 7, 2, 1},  // n=512 batch=74: 1.238 ms
    {0, 0, 34, 544, 2LL, 221LL, 1, 7, 2, 1},  // n=512 batch=74: 1.243 ms
    {0, 1, 34, 544, 222LL, 1099511627776LL, 2, 7, 2, 1},  // n=512 batch=296: 2.590 ms
    {0, 0, 34, 544, 222LL, 1099511627776LL, 2, 7, 2, 1},  // n=512 batch=296: 2.726 ms
    {0, 1, 546, 1056, 1LL, 1LL, 1, 7, 2, 1},  // n=1024 batch=1: 2.101 ms
    {0, 0, 546, 1056, 1LL, 1LL, 1, 7, 1, 1},  // n=1024 batch=1: 2.074 ms
    {0, 1, 546, 1056, 2LL, 98LL, 1, 7, 1, 1},  // n=1024 batch=33: 2.729 ms
    {0, 0, 546, 1056, 2LL, 98LL, 1, 7, 1, 1},  // n=1024 batch=33: 2.833 ms
    {0, 1, 546, 1056, 99LL, 1099511627776LL, 2, 7, 1, 1},  // n=1024 batch=132: 5.967 ms
    {0, 0, 546, 1056, 99LL, 1099511627776LL, 2, 7, 2, 1},  // n=1024 batch=132: 6.638 ms
    {0, 1, 1058, 2080, 1LL, 1LL, 1, 7, 2, 1},  // n=2048 batch=1: 4.300 ms
    {0, 0, 1058, 2080, 1LL, 1LL, 1, 7, 1, 1},  // n=2048 batch=1: 4.241 ms
    {0, 1, 1058, 2080, 2LL, 44LL, 1, 7, 2, 1},  // n=2048 batch=15: 6.163 ms
    {0, 0, 1058, 2080, 2LL, 44LL, 1, 7, 1, 1},  // n=2048 batch=15: 6.756 ms
    {0, 1, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 1, 1},  // n=2048 batch=60: 15.238 ms
    {0, 0, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 1, 1},  // n=2048 batch=60: 17.536 ms
    {0, 1, 2082, 4160, 1LL, 1LL, 1, 7, 1, 1},  // n=4096 batch=1: 9.236 ms
    {0, 0, 2082, 4160, 1LL, 1LL, 1, 7, 1, 1},  // n=4096 batch=1: 9.473 ms
    {0, 1, 2082, 4160, 2LL, 20LL, 1, 7, 2, 1},  // n=4096 batch=7: 14.501 ms
    {0, 0, 2082, 4160, 2LL, 20LL, 1, 7, 2, 1},  // n=4096 batch=7: 17.729 ms
    {0, 1, 2082, 4160, 21LL, 1099511627776LL, 2, 7, 2, 1},  // n=4096 batch=22: 32.936 ms
    {0, 0, 2082, 4160, 21LL, 1099511627776LL, 2, 7, 2, 1},  // n=4096 batch=22: 41.878 ms
    {0, 1, 4162, 8224, 1LL, 1LL, 1, 7, 2, 1},  // n=6144 batch=1: 20.481 ms
    {0, 0, 4162, 8224, 1LL, 1LL, 1, 7, 1, 1},  // n=6144 batch=1: 19.619 ms
    {0, 1, 4162, 8224, 2LL, 20LL, 1, 7, 2, 1},  // n=6144 batch=7: 47.834 ms
    {0, 0, 4162, 8224, 2LL, 20LL, 1, 7, 1, 1},  // n=6144 batch=7: 56.190 ms
    {0, 1, 4162, 8224, 21LL, 1099511627776LL, 1, 7, 1, 1},  // n=6144 batch=9: 59.160 ms
    {0, 0, 4162, 8224, 21LL, 1099511627776LL, 1, 7, 1, 1},  // n=6144 batch=9: 70.097 ms
    {1, 1, 34, 544, 1LL, 1LL, 2, 7, 1, 1},  // n=512 batch=1: 1.522 ms
    {1, 0, 34, 544, 1LL, 1LL, 2, 7, 2, 1},  // n=512 batch=1: 1.318 ms
    {1, 1, 34, 544, 2LL, 221LL, 2, 7, 1, 1},  // n=512 batch=74: 2.221 ms
    {1, 0, 34, 544, 2LL, 221LL, 2, 7, 1, 1},  // n=512 batch=74: 1.961 ms
    {1, 1, 34, 544, 222LL, 1099511627776LL, 2, 7, 2, 1},  // n=512 batch=296: 5.547 ms
    {1, 0, 34, 544, 222LL, 1099511627776LL, 2, 7, 2, 1},  // n=512 batch=296: 4.763 ms
    {1, 1, 546, 1056, 1LL, 1LL, 2, 7, 2, 1},  // n=1024 batch=1: 3.129 ms
    {1, 0, 546, 1056, 1LL, 1LL, 2, 7, 1, 1},  // n=1024 batch=1: 2.699 ms
    {1, 1, 546, 1056, 2LL, 98LL, 2, 7, 1, 1},  // n=1024 batch=33: 5.384 ms
    {1, 0, 546, 1056, 2LL, 98LL, 2, 7, 1, 1},  // n=1024 batch=33: 4.819 ms
    {1, 1, 546, 1056, 99LL, 1099511627776LL, 2, 7, 2, 1},  // n=1024 batch=132: 14.233 ms
    {1, 0, 546, 1056, 99LL, 1099511627776LL, 2, 7, 2, 1},  // n=1024 batch=132: 12.683 ms
    {1, 1, 1058, 2080, 1LL, 1LL, 2, 7, 2, 1},  // n=2048 batch=1: 6.554 ms
    {1, 0, 1058, 2080, 1LL, 1LL, 2, 7, 1, 1},  // n=2048 batch=1: 5.833 ms
    {1, 1, 1058, 2080, 2LL, 44LL, 2, 7, 2, 1},  // n=2048 batch=15: 13.602 ms
    {1, 0, 1058, 2080, 2LL, 44LL, 2, 7, 2, 1},  // n=2048 batch=15: 12.804 ms
    {1, 1, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 2, 1},  // n=2048 batch=44: 29.985 ms
    {1, 0, 1058, 2080, 45LL, 1099511627776LL, 2, 7, 2, 1},  // n=2048 batch=44: 28.418 ms
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
