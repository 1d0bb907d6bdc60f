// host_par.h — contiguous-chunk parallel loops for the host-side topology and analysis passes.
#pragma once
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace ifea {

// Number of chunks par_chunks splits [0, n) into: the host's threads (at most 16) for n >= 8192, else one.
inline int par_chunk_count(int n)
{
    return n >= 8192 ? (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency())) : 1;
}

// f(t, begin, end) over par_chunk_count(n) contiguous chunks of [0, n), chunk t on its own thread (one chunk on
// this thread when n is small); the chunks' bounds depend on n alone, so two calls with the same n split alike.
// A pass that writes only its own chunk's outputs, or per-chunk buffers joined in chunk order afterwards, gives
// the serial loop's result.
template <class F>
int par_chunks(int n, F &&f)
{
    const int nt = par_chunk_count(n);
    if (nt == 1) {
        f(0, 0, n);
        return 1;
    }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t] { f(t, (int)((int64_t)n * t / nt), (int)((int64_t)n * (t + 1) / nt)); });
    for (auto &x : th) x.join();
    return nt;
}

}  // namespace ifea
