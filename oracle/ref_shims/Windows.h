// Shim for building the reference's CPU code with g++ (TEST INFRASTRUCTURE ONLY).
// The Win32 interlocked calls map onto GCC atomics; LONG is 32-bit as on Windows.
#pragma once
#include <cstdint>
typedef int32_t LONG;
inline uint32_t InterlockedExchange(uint32_t* target, uint32_t value) { return __atomic_exchange_n(target, value, __ATOMIC_SEQ_CST); }
inline LONG InterlockedCompareExchange(volatile LONG* dst, LONG exchange, LONG comparand)
{
    LONG expected = comparand;
    __atomic_compare_exchange_n((LONG*)dst, &expected, exchange, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return expected;
}
inline LONG InterlockedIncrement(volatile LONG* p) { return __atomic_add_fetch((LONG*)p, 1, __ATOMIC_SEQ_CST); }
