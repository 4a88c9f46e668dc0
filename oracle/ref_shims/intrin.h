// Shim for building the reference's CPU code with g++ (TEST INFRASTRUCTURE ONLY).
// Provides the MSVC bit-count intrinsics the reference headers call.
#pragma once
#include <cstdint>
#include <cstdlib>
inline unsigned int __lzcnt(unsigned int x) { return x == 0 ? 32u : (unsigned int)__builtin_clz(x); }
inline unsigned long long _lzcnt_u64(unsigned long long x) { return x == 0 ? 64ull : (unsigned long long)__builtin_clzll(x); }
inline unsigned int _tzcnt_u32(unsigned int x) { return x == 0 ? 32u : (unsigned int)__builtin_ctz(x); }
inline unsigned long long _tzcnt_u64(unsigned long long x) { return x == 0 ? 64ull : (unsigned long long)__builtin_ctzll(x); }
inline void __debugbreak() { abort(); }
