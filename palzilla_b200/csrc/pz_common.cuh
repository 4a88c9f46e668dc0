// pz_common.cuh -- shared device-side definitions for the Palzilla B200 kernels.
//
// Data layouts follow the reference's structs bit for bit (minimum_lbvh.h:207-291,
// pk.h:74-86) because they cross the drop-in boundary.  Vector arithmetic keeps
// the reference's operation order; translation units whose results must be
// bit-exact with the CPU restatement (traversal, photons, eye pass) are built with
// -fmad=false, and the ray/box and ray/triangle tests below use explicit
// round-to-nearest intrinsics so that they stay exact in every unit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/palzilla_b200.h"

#define PZ_HD __host__ __device__ __forceinline__
#define PZ_D __device__ __forceinline__

namespace pz {

constexpr float kFltMax = 3.402823466e+38F;
constexpr float kPi = 3.14159265358979323846f;
constexpr uint32_t kInvalidNode = 0x7FFFFFFFu;
constexpr int kMaxDevices = 64;

// SM count of the current device, looked up once per device ordinal: persistent and
// grid-stride launches are sized in multiples of it (148 on a B200).
inline int num_sms()
{
    static std::atomic<int> cache[kMaxDevices];  // 0 = not looked up yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

struct Tri { float3 v0, v1, v2; };                        // 36 B, minimum_lbvh.h:207
struct Attrib { int32_t material; float3 n0, n1, n2; };   // 40 B, pk.h:74
struct Box { float3 lo, hi; };                            // 24 B, minimum_lbvh.h:220
struct Node {                                             // 64 B, minimum_lbvh.h:285
    uint32_t children[2];
    Box boxes[2];
    uint32_t parent;
    uint32_t context;
};
static_assert(sizeof(Tri) == 36, "Triangle layout");
static_assert(sizeof(Attrib) == 40, "TriangleAttrib layout");
static_assert(sizeof(Node) == 64, "InternalNode layout");

enum : int32_t { kDiffuse = 0, kMirror = 1, kDielectric = 2 };

PZ_HD uint32_t make_node(uint32_t idx, bool leaf) { return (idx & 0x7FFFFFFFu) | (leaf ? 0x80000000u : 0u); }
PZ_HD bool is_leaf(uint32_t n) { return (n >> 31) != 0; }
PZ_HD uint32_t node_idx(uint32_t n) { return n & 0x7FFFFFFFu; }

// ---------------------------------------------------------------- float3 math
PZ_HD float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
PZ_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
PZ_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
PZ_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
PZ_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
PZ_HD float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
PZ_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
PZ_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
PZ_HD float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
PZ_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PZ_HD float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PZ_HD float3 vmin(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
PZ_HD float3 vmax(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
PZ_HD float3 vabs(float3 a) { return make_float3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
PZ_HD float lerpf(float a, float b, float t) { return a + t * (b - a); }
PZ_HD float3 lerp3(float3 a, float3 b, float t) { return a + t * (b - a); }
PZ_HD float length(float3 v) { return sqrtf(dot(v, v)); }
// 1/sqrt with correctly rounded divide and square root: the reference's host
// definition of rsqrtf, which the CPU oracle reproduces bit for bit.
PZ_D float3 normalize(float3 v)
{
    float inv = __fdiv_rn(1.0f, __fsqrt_rn(dot(v, v)));
    return v * inv;
}

PZ_HD Box box_empty() { return Box{mk3(kFltMax, kFltMax, kFltMax), mk3(-kFltMax, -kFltMax, -kFltMax)}; }
PZ_HD void box_extend(Box& b, float3 p) { b.lo = vmin(b.lo, p); b.hi = vmax(b.hi, p); }
PZ_HD void box_extend(Box& b, const Box& o) { b.lo = vmin(b.lo, o.lo); b.hi = vmax(b.hi, o.hi); }

// ---------------------------------------------------------------- exact ray tests
// Explicit round-to-nearest operations: never contracted into FMA, so the hit
// decisions agree bit for bit with the CPU restatement whatever -fmad says.
namespace ex {
PZ_D float mul(float a, float b) { return __fmul_rn(a, b); }
PZ_D float add(float a, float b) { return __fadd_rn(a, b); }
PZ_D float sub(float a, float b) { return __fsub_rn(a, b); }
PZ_D float3 add3(float3 a, float3 b) { return mk3(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)); }
PZ_D float3 sub3(float3 a, float3 b) { return mk3(sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)); }
PZ_D float3 mul3(float3 a, float s) { return mk3(mul(a.x, s), mul(a.y, s), mul(a.z, s)); }
PZ_D float3 mulv(float3 a, float3 b) { return mk3(mul(a.x, b.x), mul(a.y, b.y), mul(a.z, b.z)); }
PZ_D float dot(float3 a, float3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
PZ_D float3 cross(float3 a, float3 b)
{
    return mk3(sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x)));
}
}  // namespace ex

// minimum_lbvh.h:913-916
PZ_D float3 inv_rd(float3 rd)
{
    float3 r = mk3(__fdiv_rn(1.0f, rd.x), __fdiv_rn(1.0f, rd.y), __fdiv_rn(1.0f, rd.z));
    return mk3(fmaxf(-kFltMax, fminf(r.x, kFltMax)), fmaxf(-kFltMax, fminf(r.y, kFltMax)),
               fmaxf(-kFltMax, fminf(r.z, kFltMax)));
}

// slabs, minimum_lbvh.h:82-96; returns true when [rmin, rmax] is non-empty.
PZ_D bool slab_hit(float3 ro, float3 inv, float3 lo, float3 hi, float tmax, float* rmin)
{
    float3 t0 = ex::mulv(ex::sub3(lo, ro), inv);
    float3 t1 = ex::mulv(ex::sub3(hi, ro), inv);
    float3 tn = vmin(t0, t1), tf = vmax(t0, t1);
    float a = fmaxf(fmaxf(fmaxf(tn.x, tn.y), tn.z), 0.0f);
    float b = fminf(ex::mul(fminf(fminf(tf.x, tf.y), tf.z), 1.00000024f), tmax);
    *rmin = a;
    return a <= b;
}

// intersectRayTriangle, minimum_lbvh.h:372-422 (watertight Pluecker volumes)
PZ_D bool ray_triangle(float* tOut, float* uOut, float* vOut, float3* ngOut, float t_min, float t_max, float3 ro,
                       float3 rd, float3 v0, float3 v1, float3 v2)
{
    float3 e0 = ex::sub3(v1, v0);
    float3 e1 = ex::sub3(v2, v1);
    float3 ng = ex::cross(e0, e1);
    float t = __fdiv_rn(ex::dot(ex::sub3(v0, ro), ng), ex::dot(ng, rd));
    if (t_min <= t && t <= t_max) {
        float3 e2 = ex::sub3(v0, v2);
        float3 ro2 = ex::mul3(ro, 2.0f);
        float u_vol = ex::dot(ex::cross(e2, ex::sub3(ex::add3(v0, v2), ro2)), rd);
        float v_vol = ex::dot(ex::cross(e0, ex::sub3(ex::add3(v1, v0), ro2)), rd);
        float w_vol = ex::dot(ex::cross(e1, ex::sub3(ex::add3(v2, v1), ro2)), rd);
        if (fminf(fminf(u_vol, v_vol), w_vol) < 0.0f && 0.0f < fmaxf(fmaxf(u_vol, v_vol), w_vol)) return false;
        float vol = ex::add(ex::add(u_vol, v_vol), w_vol);
        *tOut = t;
        *uOut = __fdiv_rn(u_vol, vol);
        *vOut = __fdiv_rn(v_vol, vol);
        *ngOut = ng;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------- hashing / Sobol (sobol.h)
PZ_HD uint32_t lk_perm(uint32_t x, uint32_t seed)
{
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
PZ_D uint32_t nus(uint32_t x, uint32_t seed) { return __brev(lk_perm(__brev(x), seed)); }
PZ_HD uint32_t pascal_P(uint32_t v)
{
    v ^= v << 16;
    v ^= (v & 0x00FF00FFu) << 8;
    v ^= (v & 0x0F0F0F0Fu) << 4;
    v ^= (v & 0x33333333u) << 2;
    v ^= (v & 0x55555555u) << 1;
    return v;
}
PZ_HD float random_float(uint32_t u) { return (float)(u >> 8) * (1.0f / 16777216.0f); }
PZ_HD uint32_t hash_pcg(uint32_t v)
{
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
PZ_D void sobol2d(float* x, float* y, uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2)
{
    uint32_t vx = p0 * 1664525u + 1013904223u, vy = p1 * 1664525u + 1013904223u, vz = p2 * 1664525u + 1013904223u;
    vx += vy * vz; vy += vz * vx; vz += vx * vy;
    vx ^= vx >> 16; vy ^= vy >> 16; vz ^= vz >> 16;
    vx += vy * vz; vy += vz * vx; vz += vx * vy;
    uint32_t v = lk_perm(__brev(index), vx);
    *x = random_float(nus(v, vy));
    *y = random_float(nus(pascal_P(v), vz));
}
PZ_HD uint32_t hash_combine(uint32_t seed, uint32_t h) { return h + 0x9e3779b9u + (seed << 6) + (seed >> 2); }
PZ_HD uint32_t hash_of_iP(int x, int y, int z)
{
    uint32_t h = 12345;
    h = hash_combine(h, (uint32_t)x * 2654435761u);
    h = hash_combine(h, (uint32_t)y * 805459861u);
    h = hash_combine(h, (uint32_t)z * 3674653429u);
    return h | 1u;
}

// ---------------------------------------------------------------- device error word
// Bit flags OR-ed into a caller-visible status word instead of trapping.
enum : uint32_t {
    kErrSpinLimit = 1u << 0,      // a bounded spin wait gave up
    kErrCapacity = 1u << 1,       // an output queue or table overflowed
    kErrStackOverflow = 1u << 2,  // a traversal stack would have overflowed
    kErrBadInput = 1u << 3,
};
PZ_D void raise_error(uint32_t* status, uint32_t bits)
{
    if (status) atomicOr(status, bits);
}

}  // namespace pz
