// ref_cpu_shim.cpp -- C entry points over the reference's own CPU Pfaffian.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  This file
// is compiled together with the UNMODIFIED reference source
// src/pfaffian_cpu.cpp (read where it lies, never copied) into
// oracle/_ref/libref_cpu.so; see oracle/Makefile.
//
// The reference function is `double pfaffian(double* A, const int n)`
// (include/pfaffian_cpu.h:5, src/pfaffian_cpu.cpp:7): row-major float64, works
// in place and returns the plain product of pivots.  The pybind11 wrapper that
// the reference ships (bindings/pybind_bindings.cpp:8-25) only adds shape checks;
// these entry points add a batch driver that spreads matrices over std::thread,
// each thread on its own scratch copy because the reference overwrites its input.
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <atomic>

double pfaffian(double* A, const int n);   // src/pfaffian_cpu.cpp:7

extern "C" double refcpu_pfaffian(double* A, int n) { return pfaffian(A, n); }

// B contiguous row-major n x n matrices; out[b] = reference Pf.  Returns the
// number of threads used.
extern "C" int refcpu_pfaffian_batch(const double* A, int64_t B, int n, double* out, int threads)
{
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    if ((int64_t)threads > B) threads = (int)(B > 0 ? B : 1);
    const size_t nn = (size_t)n * (size_t)n;
    std::atomic<int64_t> next(0);
    auto work = [&]() {
        std::vector<double> S(nn ? nn : 1);
        for (;;) {
            int64_t b = next.fetch_add(1);
            if (b >= B) break;
            std::memcpy(S.data(), A + (size_t)b * nn, nn * sizeof(double));
            out[b] = pfaffian(S.data(), n);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    return threads;
}
