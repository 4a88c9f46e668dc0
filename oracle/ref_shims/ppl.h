// Shim for building the reference's CPU code with g++ (TEST INFRASTRUCTURE ONLY).
// concurrency::parallel_for runs as an OpenMP loop.
#pragma once
#include <cstddef>
namespace concurrency {
template <class I, class F>
inline void parallel_for(I first, I last, const F& f)
{
#pragma omp parallel for schedule(static)
    for (long long i = (long long)first; i < (long long)last; ++i) f((I)i);
}
}  // namespace concurrency
