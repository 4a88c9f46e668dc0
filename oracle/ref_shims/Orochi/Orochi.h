// Shim for building the reference's CPU code with g++ (TEST INFRASTRUCTURE ONLY).
// The handful of Orochi runtime calls reached by the host-side headers are backed by
// host memory: "device" buffers are plain malloc'd arrays.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <cstring>
typedef void* oroDeviceptr;
typedef void* oroStream;
typedef int oroError;
enum oroMemcpyKind { oroMemcpyHostToHost = 0, oroMemcpyHostToDevice = 1, oroMemcpyDeviceToHost = 2, oroMemcpyDeviceToDevice = 3 };
inline oroError oroMalloc(oroDeviceptr* p, size_t n) { *p = malloc(n ? n : 1); return 0; }
inline oroError oroFree(oroDeviceptr p) { free(p); return 0; }
inline oroError oroMemcpy(void* dst, oroDeviceptr src, size_t n, oroMemcpyKind) { memcpy(dst, src, n); return 0; }
inline oroError oroMemsetD32(oroDeviceptr p, uint32_t v, size_t count) { uint32_t* q = (uint32_t*)p; for (size_t i = 0; i < count; i++) q[i] = v; return 0; }
inline oroError oroMemsetD32Async(oroDeviceptr p, uint32_t v, size_t count, oroStream) { return oroMemsetD32(p, v, count); }
