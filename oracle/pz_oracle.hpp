// pz_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of Palzilla's caustics hot path, used as the parity checker
// for the CUDA kernels in palzilla_b200/csrc.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load the library built from this file;
// the product path never calls it.
//
// Every function states the reference file:line it restates.  In float mode the
// arithmetic follows the reference's operation order exactly (no FMA contraction:
// the library is built with -ffp-contract=off), so Morton keys, sort order,
// LBVH topology, traversal hits and photon tuples are bit-exact against both
// the reference's own CPU code (oracle/_ref, built by oracle/build_ref.sh) and
// the CUDA kernels.  The solver, throughput, dAdw and interval code are templated
// on the scalar type so the same restatement also gives the FP64 reference.
//
// Known, intentional differences from the reference (each documented at the
// function): normalize() uses 1/sqrt(x) (the reference's host definition;
// the reference GPU build uses the approximate rsqrtf), the CIE functions use
// the accurate exp/log, and the LBVH launch bug for n == 1 (mod 256) is absent.
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace pzo {

// ----------------------------------------------------------------------------
// small vector math (restates the operators of the reference's vector header;
// operation order matters for bit-exactness)
// ----------------------------------------------------------------------------
template <class T> struct V3 { T x, y, z; };
using F3 = V3<float>;
using D3 = V3<double>;

template <class T> inline V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> splat(T s) { return V3<T>{s, s, s}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline T length(V3<T> v) { return std::sqrt(dot(v, v)); }
// normalize = v * (1 / sqrt(|v|^2)): the reference's host definition of rsqrtf.
template <class T> inline V3<T> normalize(V3<T> v) { T inv = T(1) / std::sqrt(dot(v, v)); return v * inv; }
template <class T> inline V3<T> vmin(V3<T> a, V3<T> b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
template <class T> inline V3<T> vmax(V3<T> a, V3<T> b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
template <class T> inline V3<T> vabs(V3<T> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
template <class T> inline T lerp(T a, T b, T t) { return a + t * (b - a); }
template <class T> inline V3<T> lerp3(V3<T> a, V3<T> b, T t) { return a + t * (b - a); }
template <class T> inline V3<T> to(F3 a) { return V3<T>{T(a.x), T(a.y), T(a.z)}; }

constexpr float kFltMax = 3.402823466e+38F;
constexpr float kPi = 3.14159265358979323846f;

// ----------------------------------------------------------------------------
// scene / BVH data types -- binary layout of minimum_lbvh.h:207-291, pk.h:74-78
// ----------------------------------------------------------------------------
struct Triangle { F3 vs[3]; };                                   // minimum_lbvh.h:207-210
struct TriangleAttrib { int32_t material; F3 shadingNormals[3]; }; // pk.h:74-78
enum Material : int32_t { kDiffuse = 0, kMirror = 1, kDielectric = 2 }; // pk.h:67-72
struct AABB { F3 lower, upper; };                                 // minimum_lbvh.h:220-261
// NodeIndex (minimum_lbvh.h:263-274) is a u32 bit field: index in bits 0..30, leaf flag in bit 31.
struct InternalNode {                                             // minimum_lbvh.h:285-291
    uint32_t children[2];
    AABB aabbs[2];
    uint32_t parent;
    uint32_t context;
};
static_assert(sizeof(Triangle) == 36, "Triangle layout");
static_assert(sizeof(TriangleAttrib) == 40, "TriangleAttrib layout");
static_assert(sizeof(InternalNode) == 64, "InternalNode layout");

constexpr uint32_t kInvalidNode = 0x7FFFFFFFu;  // NodeIndex::invalid(), minimum_lbvh.h:270-273
inline uint32_t make_node(uint32_t index, bool leaf) { return (index & 0x7FFFFFFFu) | (leaf ? 0x80000000u : 0u); }
inline bool node_is_leaf(uint32_t n) { return (n >> 31) != 0; }
inline uint32_t node_idx(uint32_t n) { return n & 0x7FFFFFFFu; }

inline AABB aabb_empty() { return AABB{splat(kFltMax), splat(-kFltMax)}; }  // minimum_lbvh.h:225-236
inline void aabb_extend(AABB& b, F3 p) { b.lower = vmin(b.lower, p); b.upper = vmax(b.upper, p); } // :237-241
inline void aabb_extend(AABB& b, const AABB& o) { b.lower = vmin(b.lower, o.lower); b.upper = vmax(b.upper, o.upper); } // :243-247
inline float aabb_surface_area(const AABB& b)  // minimum_lbvh.h:256-260
{
    F3 s = b.upper - b.lower;
    return (s.x * s.y + s.y * s.z + s.z * s.x) * 2.0f;
}

// float -> int with round-toward-zero and the saturating / NaN->0 semantics of
// the GPU conversion instruction.  The reference relies on a plain C cast
// (minimum_lbvh.h:251); the two agree for every in-range value, which is all
// the Morton encoder ever sees.
inline int f2i_rz(float q)
{
    if (q != q) return 0;
    if (q >= 2147483648.0f) return 0x7FFFFFFF;
    if (q <= -2147483648.0f) return (int)0x80000000;
    return (int)q;
}

// minimum_lbvh.h:173-182
inline uint64_t splat3(uint32_t a)
{
    uint64_t x = a & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
// minimum_lbvh.h:190-195
inline uint64_t encode_morton(uint32_t x, uint32_t y, uint32_t z) { return splat3(x) | splat3(y) << 1 | splat3(z) << 2; }
// AABB::encodeMortonCode, minimum_lbvh.h:249-254
inline uint64_t aabb_encode_morton(const AABB& b, F3 p)
{
    F3 q = (p - b.lower) / (b.upper - b.lower) * 2097152.0f;  // (MORTON_MAX_VALUE_3D + 1)
    int cx = std::max(0, std::min(f2i_rz(q.x), 0x1FFFFF));
    int cy = std::max(0, std::min(f2i_rz(q.y), 0x1FFFFF));
    int cz = std::max(0, std::min(f2i_rz(q.z), 0x1FFFFF));
    return encode_morton((uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
}
inline int clz32(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }
inline int delta32(uint32_t a, uint32_t b) { return 32 - clz32(a ^ b); }  // minimum_lbvh.h:140-143

constexpr uint32_t BUILD_OPTION_USE_NORMAL = 1;  // minimum_lbvh.h:42-46
constexpr uint32_t BUILD_OPTION_CPU_PARALLEL = 2;

inline F3 unnormalized_normal(const Triangle& t) { return cross(t.vs[1] - t.vs[0], t.vs[2] - t.vs[0]); } // :211-214

// getSceneAABB, minimum_lbvh.cu:38-66 (min/max are exact, so reduction order is irrelevant)
inline AABB scene_aabb(const Triangle* tris, int n)
{
    AABB b = aabb_empty();
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) aabb_extend(b, tris[i].vs[j]);
    return b;
}

// buildMortons, minimum_lbvh.cu:68-92 (GPU key packing for USE_NORMAL, :85)
inline uint32_t morton_key(const Triangle& tri, const AABB& scene, uint32_t buildOption)
{
    F3 center = (tri.vs[0] + tri.vs[1] + tri.vs[2]) / 3.0f;
    if (buildOption & BUILD_OPTION_USE_NORMAL) {
        F3 ng = normalize(unnormalized_normal(tri));
        AABB unit{mk(-1.f, -1.f, -1.f), mk(1.f, 1.f, 1.f)};
        uint32_t nMorton = (uint32_t)(aabb_encode_morton(unit, ng) >> 31);
        uint32_t pMorton = (uint32_t)(aabb_encode_morton(scene, center) >> 31);
        return (nMorton & 0xFFFFFFC0u) | (pMorton >> 26);
    }
    return (uint32_t)(aabb_encode_morton(scene, center) >> 31);  // upper 32 of 63 bits
}

struct IndexedMorton { uint32_t morton; uint32_t index; };  // minimum_lbvh.h:511-515

// build_lbvh, minimum_lbvh.h:293-370 (sequential form: the exchange is a plain swap)
inline void build_lbvh_leaf(uint32_t* rootNode, InternalNode* internals, const Triangle* triangles, int nTriangles,
                            const uint8_t* deltas, uint32_t i_leaf, uint32_t triangleIndex)
{
    uint32_t nInternals = (uint32_t)(nTriangles - 1);
    uint32_t nDeltas = nInternals;
    uint32_t leaf_lower = i_leaf, leaf_upper = i_leaf;
    uint32_t node = make_node(triangleIndex, true);
    AABB aabb = aabb_empty();
    if (triangles)
        for (int j = 0; j < 3; j++) aabb_extend(aabb, triangles[triangleIndex].vs[j]);
    bool isRoot = true;
    while (leaf_upper - leaf_lower < nInternals) {
        uint32_t deltaL = 0 < leaf_lower ? deltas[leaf_lower - 1] : 0xFFFFFFFFu;
        uint32_t deltaR = leaf_upper < nDeltas ? deltas[leaf_upper] : 0xFFFFFFFFu;
        int goLeft = deltaL < deltaR ? 1 : 0;
        uint32_t parent = goLeft ? (leaf_lower - 1) : leaf_upper;
        internals[parent].children[goLeft] = node;
        internals[parent].aabbs[goLeft] = aabb;
        if (!node_is_leaf(node)) internals[node_idx(node)].parent = make_node(parent, false);
        uint32_t index = goLeft ? leaf_upper : leaf_lower;
        std::swap(index, internals[parent].context);
        if (index == 0xFFFFFFFFu) { isRoot = false; break; }
        leaf_lower = std::min(leaf_lower, index);
        leaf_upper = std::max(leaf_upper, index);
        internals[parent].context = leaf_upper < nInternals ? leaf_upper : 0xFFFFFFFFu;
        node = make_node(parent, false);
        aabb_extend(aabb, internals[parent].aabbs[goLeft ^ 1]);
    }
    if (isRoot) {
        *rootNode = node;
        if (nInternals > 0) internals[node_idx(node)].parent = kInvalidNode;  // n == 1 has no internal node
    }
}

// Whole GPU builder pipeline (minimum_lbvh.h:798-886) in sequential form with a
// STABLE sort, i.e. the order the GPU onesweep radix sort produces.
struct LBVH {
    uint32_t root = kInvalidNode;
    std::vector<InternalNode> nodes;
    std::vector<uint8_t> deltas;
    std::vector<IndexedMorton> sorted;
    AABB scene{};
};
inline void build_bvh(LBVH& out, const Triangle* tris, int n, uint32_t buildOption)
{
    out.nodes.assign(n > 1 ? n - 1 : 0, InternalNode{});
    for (auto& nd : out.nodes) std::memset(&nd, 0xFF, sizeof(nd));
    out.deltas.assign(n > 1 ? n - 1 : 0, 0);
    out.root = kInvalidNode;
    out.sorted.resize(n);
    if (n <= 0) return;
    out.scene = scene_aabb(tris, n);
    for (int i = 0; i < n; i++) out.sorted[i] = IndexedMorton{morton_key(tris[i], out.scene, buildOption), (uint32_t)i};
    std::stable_sort(out.sorted.begin(), out.sorted.end(),
                     [](IndexedMorton a, IndexedMorton b) { return a.morton < b.morton; });
    for (int i = 0; i + 1 < n; i++) out.deltas[i] = (uint8_t)delta32(out.sorted[i].morton, out.sorted[i + 1].morton);
    for (int i = 0; i < n; i++)
        build_lbvh_leaf(&out.root, out.nodes.data(), tris, n, out.deltas.data(), (uint32_t)i, out.sorted[i].index);
}

// validate_lbvh, minimum_lbvh.h:424-435 (returns false instead of aborting)
inline bool validate_lbvh(uint32_t node, const InternalNode* internals, const uint8_t* deltas, int maxDelta)
{
    if (node_is_leaf(node)) return true;
    int d = deltas[node_idx(node)];
    if (d > maxDelta) return false;
    return validate_lbvh(internals[node_idx(node)].children[0], internals, deltas, d) &&
           validate_lbvh(internals[node_idx(node)].children[1], internals, deltas, d);
}

// ----------------------------------------------------------------------------
// ray queries -- minimum_lbvh.h:82-96, 372-422, 905-1152
// ----------------------------------------------------------------------------
struct Hit {  // minimum_lbvh.h:905-911
    float t = kFltMax;
    float u = 0, v = 0;
    F3 ng{0, 0, 0};
    uint32_t triangleIndex = 0xFFFFFFFFu;
};

inline void slabs(float* rmin, float* rmax, F3 ro, F3 one_over_rd, F3 lower, F3 upper, float knownHitT)
{
    F3 t0 = (lower - ro) * one_over_rd;
    F3 t1 = (upper - ro) * one_over_rd;
    F3 tmin = vmin(t0, t1), tmax = vmax(t0, t1);
    float region_min = std::fmax(std::fmax(tmin.x, tmin.y), tmin.z);
    float region_max = std::fmin(std::fmin(tmax.x, tmax.y), tmax.z) * 1.00000024f;
    region_min = std::fmax(region_min, 0.0f);
    region_max = std::fmin(region_max, knownHitT);
    *rmin = region_min;
    *rmax = region_max;
}

inline F3 inv_rd(F3 rd)  // minimum_lbvh.h:913-916
{
    F3 r = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    return mk(std::fmax(-kFltMax, std::fmin(r.x, kFltMax)), std::fmax(-kFltMax, std::fmin(r.y, kFltMax)),
              std::fmax(-kFltMax, std::fmin(r.z, kFltMax)));
}

inline bool intersect_ray_triangle(float* tOut, float* uOut, float* vOut, F3* ngOut, float t_min, float t_max, F3 ro,
                                   F3 rd, F3 v0, F3 v1, F3 v2)
{
    F3 e0 = v1 - v0;
    F3 e1 = v2 - v1;
    F3 ng = cross(e0, e1);
    float t = dot(v0 - ro, ng) / dot(ng, rd);
    if (t_min <= t && t <= t_max) {
        F3 e2 = v0 - v2;
        float u_vol = dot(cross(e2, v0 + v2 - ro * 2.0f), rd);
        float v_vol = dot(cross(e0, v1 + v0 - ro * 2.0f), rd);
        float w_vol = dot(cross(e1, v2 + v1 - ro * 2.0f), rd);
        if (std::fmin(std::fmin(u_vol, v_vol), w_vol) < 0.0f && 0.0f < std::fmax(std::fmax(u_vol, v_vol), w_vol))
            return false;
        float vol = u_vol + v_vol + w_vol;
        *tOut = t;
        *uOut = u_vol / vol;
        *vOut = v_vol / vol;
        *ngOut = ng;
        return true;
    }
    return false;
}

// intersect_stackfull, minimum_lbvh.h:927-988 (near-first, LIFO stack)
inline void intersect_stackfull(Hit* hit, const InternalNode* nodes, const Triangle* triangles, uint32_t root, F3 ro,
                                F3 rd, F3 one_over_rd)
{
    uint32_t stack[256];
    int sp = 0;
    uint32_t node = root;
    while (node != kInvalidNode) {
        if (node_is_leaf(node)) {
            float t, u, v;
            F3 ng;
            const Triangle& tri = triangles[node_idx(node)];
            if (intersect_ray_triangle(&t, &u, &v, &ng, 0.0f, hit->t, ro, rd, tri.vs[0], tri.vs[1], tri.vs[2])) {
                hit->t = t;
                hit->u = u;
                hit->v = v;
                hit->ng = ng;
                hit->triangleIndex = node_idx(node);
            }
            node = sp == 0 ? kInvalidNode : stack[--sp];
            continue;
        }
        const InternalNode& nd = nodes[node_idx(node)];
        float lx, ly, rx, ry;
        slabs(&lx, &ly, ro, one_over_rd, nd.aabbs[0].lower, nd.aabbs[0].upper, hit->t);
        slabs(&rx, &ry, ro, one_over_rd, nd.aabbs[1].lower, nd.aabbs[1].upper, hit->t);
        bool hitL = lx <= ly, hitR = rx <= ry;
        if (hitL && hitR) {
            uint32_t near_node = nd.children[0], far_node = nd.children[1];
            if (rx < lx) std::swap(near_node, far_node);
            node = near_node;
            stack[sp++] = far_node;
        } else if (hitL || hitR) {
            node = nd.children[hitL ? 0 : 1];
        } else {
            node = sp == 0 ? kInvalidNode : stack[--sp];
        }
    }
}

// intersect_escape_link, minimum_lbvh.h:1078-1152 (stackless, uses parent and context links)
inline void intersect_escape_link(Hit* hit, const InternalNode* nodes, const Triangle* triangles, uint32_t root, F3 ro,
                                  F3 rd, F3 one_over_rd, bool anyHit)
{
    uint32_t curr = root, prev = kInvalidNode;
    while (curr != kInvalidNode) {
        if (node_is_leaf(curr)) {
            float t, u, v;
            F3 ng;
            const Triangle& tri = triangles[node_idx(curr)];
            if (intersect_ray_triangle(&t, &u, &v, &ng, 0.0f, hit->t, ro, rd, tri.vs[0], tri.vs[1], tri.vs[2])) {
                hit->t = t;
                hit->u = u;
                hit->v = v;
                hit->triangleIndex = node_idx(curr);
                hit->ng = ng;
                if (anyHit) break;
            }
            if (nodes[node_idx(prev)].children[0] == curr) {
                std::swap(curr, prev);
                continue;
            }
            uint32_t ioi = nodes[node_idx(prev)].context;
            uint32_t next = ioi != 0xFFFFFFFFu ? make_node(ioi, false) : kInvalidNode;
            prev = curr;
            curr = next;
            continue;
        }
        const InternalNode& nd = nodes[node_idx(curr)];
        uint32_t parent = nd.parent;
        AABB box;
        uint32_t hitChild, miss;
        if (prev == parent) {
            box = nd.aabbs[0];
            hitChild = nd.children[0];
            miss = curr;
        } else {
            box = nd.aabbs[1];
            hitChild = nd.children[1];
            miss = nd.context != 0xFFFFFFFFu ? make_node(nd.context, false) : kInvalidNode;
        }
        float a, b;
        slabs(&a, &b, ro, one_over_rd, box.lower, box.upper, hit->t);
        uint32_t next = a <= b ? hitChild : miss;
        prev = curr;
        curr = next;
    }
}

// ----------------------------------------------------------------------------
// hashing and Sobol -- sobol.h:18-129, minimum_lbvh.h:919-924, pk.h:207-225
// ----------------------------------------------------------------------------
inline uint32_t reverse_bits(uint32_t v)
{
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
    v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
    return (v >> 16) | (v << 16);
}
inline uint32_t lk_permutation(uint32_t x, uint32_t seed)
{
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
inline uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) { return reverse_bits(lk_permutation(reverse_bits(x), seed)); }
inline uint32_t pascal_P(uint32_t v)
{
    v ^= v << 16;
    v ^= (v & 0x00FF00FFu) << 8;
    v ^= (v & 0x0F0F0F0Fu) << 4;
    v ^= (v & 0x33333333u) << 2;
    v ^= (v & 0x55555555u) << 1;
    return v;
}
inline float random_float(uint32_t u) { return (float)(u >> 8) / 16777216.0f; }
inline uint32_t hash_pcg(uint32_t v)
{
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
inline void pcg3d(uint32_t* x, uint32_t* y, uint32_t* z)
{
    uint32_t vx = *x * 1664525u + 1013904223u, vy = *y * 1664525u + 1013904223u, vz = *z * 1664525u + 1013904223u;
    vx += vy * vz; vy += vz * vx; vz += vx * vy;
    vx ^= vx >> 16; vy ^= vy >> 16; vz ^= vz >> 16;
    vx += vy * vz; vy += vz * vx; vz += vx * vy;
    *x = vx; *y = vy; *z = vz;
}
inline void sobol2d(float* x, float* y, uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2)
{
    pcg3d(&p0, &p1, &p2);
    uint32_t v = lk_permutation(reverse_bits(index), p0);
    *x = random_float(nested_uniform_scramble(v, p1));
    *y = random_float(nested_uniform_scramble(pascal_P(v), p2));
}
inline uint32_t hash_combine(uint32_t seed, uint32_t h) { return h + 0x9e3779b9u + (seed << 6) + (seed >> 2); }
inline uint32_t hash_of_iP(int x, int y, int z)
{
    uint32_t h = 12345;
    h = hash_combine(h, (uint32_t)x * 2654435761u);
    h = hash_combine(h, (uint32_t)y * 805459861u);
    h = hash_combine(h, (uint32_t)z * 3674653429u);
    return h | 1u;
}
inline int floor_i(float f) { return f2i_rz(std::floor(f)); }
inline uint32_t spacial_hash(F3 p, float step)
{
    F3 idx = p / step;
    return hash_of_iP(floor_i(idx.x), floor_i(idx.y), floor_i(idx.z));
}

// ----------------------------------------------------------------------------
// optics -- pk.h:43-65, 165-205, 405-459
// ----------------------------------------------------------------------------
inline float ray_offset_scale(F3 p)
{
    p = vabs(p);
    float m = std::fmax(std::fmax(std::fmax(p.x, p.y), p.z), 1.0f);
    return m * 1.192092896e-07F * 128.0f;
}
inline void sph_intersect(float* t0, float* t1, F3 ro, F3 rd, F3 ce, float ra)
{
    float len2rd = dot(rd, rd);
    F3 oc = ro - ce;
    float b = dot(oc, rd) / len2rd;
    float c = dot(oc, oc) - ra * ra;
    float h = b * b - c / len2rd;
    if (h < 0.0f) { *t0 = -1.0f; *t1 = -1.0f; return; }
    h = std::sqrt(h);
    *t0 = -b - h;
    *t1 = -b + h;
}
inline void square2triangle(float* x, float* y)
{
    if (*y > *x) { *x *= 0.5f; *y -= *x; }
    else { *y *= 0.5f; *x -= *y; }
}
template <class T> inline bool refraction_norm_free(V3<T>* wo, V3<T> wi, V3<T> n, T eta)
{
    T NoN = dot(n, n);
    T WIoN = dot(wi, n);
    if (WIoN < T(0)) { WIoN = -WIoN; n = -n; eta = T(1) / eta; }
    T WIoWI = dot(wi, wi);
    T k = NoN * WIoWI * (eta * eta - T(1)) + WIoN * WIoN;
    if (k < T(0)) return false;
    *wo = -wi * NoN + (WIoN - std::sqrt(k)) * n;
    return true;
}
template <class T> inline V3<T> reflection(V3<T> wi, V3<T> n) { return n * dot(wi, n) * T(2) / dot(n, n) - wi; }
template <class T> inline T fresnel_exact_norm_free(V3<T> wi, V3<T> n, T eta)
{
    T nn = dot(n, n), wiwi = dot(wi, wi), C = dot(n, wi);
    if (C < T(0)) { C = -C; n = -n; eta = T(1) / eta; }
    T K = nn * wiwi * (eta * eta - T(1)) + C * C;
    if (K < T(0)) return T(1);
    T G = std::sqrt(K);
    T GmC = G - C, GpC = G + C;
    T a = GmC / GpC, b = (C * GpC - nn * wiwi) / (C * GmC + nn * wiwi);
    return T(0.5) * (a * a) * (T(1) + b * b);
}

struct EventDescriptor {  // pk.h:117-162; u32 = events (bits 0..23) | size << 24
    uint32_t bits = 0;
    int size() const { return (int)(bits >> 24); }
    bool isT(int i) const { return (bits >> i) & 1u; }
    void push_back(bool T) { int s = size(); uint32_t ev = bits & 0xFFFFFFu; ev &= ~(1u << s); if (T) ev |= 1u << s; bits = ev | ((uint32_t)(s + 1) << 24); }
};

// occluded, pk.h:88-115
inline bool occluded(const InternalNode* nodes, const Triangle* tris, uint32_t root, F3 from, F3 from_n, F3 to_, F3 to_n)
{
    if (dot(to_ - from, from_n) < 0.0f) from_n = -from_n;
    if (dot(from - to_, to_n) < 0.0f) to_n = -to_n;
    F3 from_safe = from + from_n * ray_offset_scale(from);
    F3 to_safe = to_ + to_n * ray_offset_scale(to_);
    F3 rd = to_safe - from_safe;
    Hit hit;
    hit.t = 1.0f;
    intersect_escape_link(&hit, nodes, tris, root, from_safe, rd, inv_rd(rd), true);
    return hit.t < 1.0f;
}

// ----------------------------------------------------------------------------
// PathCache -- pk.h:227-402 (host form; insertion order = caller order)
// ----------------------------------------------------------------------------
struct PathCache {
    uint32_t capacity = 1u << 22;
    float step = 0.01f;
    std::vector<uint32_t> hashOfPath;  // 0 = empty
    std::vector<uint32_t> cellHash;    // TrianglePath::hashOfP
    std::vector<uint32_t> events;      // EventDescriptor::asU32
    std::vector<int32_t> tris;         // 4 per slot
    std::vector<float> params;         // 8 per slot
    uint32_t count = 0;
    void init(uint32_t cap, float s)
    {
        capacity = cap; step = s;
        hashOfPath.assign(cap, 0); cellHash.assign(cap, 0); events.assign(cap, 0);
        tris.assign((size_t)cap * 4, 0); params.assign((size_t)cap * 8, 0.f);
        count = 0;
    }
    static uint32_t path_hash(uint32_t ev, const int32_t* t)
    {
        uint32_t h = ev;
        for (int d = 0; d < (int)(ev >> 24); d++) h = hash_pcg(h + (uint32_t)t[d]);
        return h | 1u;
    }
    bool store(F3 pos, const int32_t* t, const float* prm, uint32_t ev)
    {
        uint32_t hp = path_hash(ev, t);
        int K = (int)(ev >> 24);
        bool success = false;
        F3 idx = pos / step;
        int x = floor_i(idx.x), y = floor_i(idx.y), z = floor_i(idx.z);
        int dx = idx.x - (float)x < 0.5f ? -1 : 1;
        int dy = idx.y - (float)y < 0.5f ? -1 : 1;
        int dz = idx.z - (float)z < 0.5f ? -1 : 1;
        for (int iz = 0; iz < 2; iz++)
            for (int iy = 0; iy < 2; iy++)
                for (int ix = 0; ix < 2; ix++) {
                    uint32_t hP = hash_of_iP(x + ix * dx, y + iy * dy, z + iz * dz);
                    uint32_t home = hP % capacity;
                    for (uint32_t off = 0; off < capacity; off++) {
                        uint32_t i = (home + off) % capacity;
                        uint32_t old = hashOfPath[i];
                        if (old == 0) {
                            hashOfPath[i] = hp;
                            cellHash[i] = hP;
                            events[i] = ev;
                            for (int d = 0; d < K; d++) tris[(size_t)i * 4 + d] = t[d];
                            for (int d = 0; d < 2 * K; d++) params[(size_t)i * 8 + d] = prm[d];
                            success = true;
                            count++;
                            break;
                        } else if (old == hp) {
                            break;
                        }
                    }
                }
        return success;
    }
    template <class F> void lookup(F3 p, uint32_t ev, F f) const  // pk.h:374-396
    {
        uint32_t hP = spacial_hash(p, step);
        uint32_t home = hP % capacity;
        for (uint32_t off = 0; off < capacity; off++) {
            uint32_t i = (home + off) % capacity;
            if (hashOfPath[i] == 0) break;
            if (cellHash[i] != hP) continue;
            if (events[i] != ev) continue;
            f(i);
        }
    }
};

// photonTrace, main_gpu.cu:56-211, for one (triangle, photon).  Returns true and
// fills the record when the path lands on a diffuse surface with throughput
// above minThroughput (the condition of main_gpu.cu:198).
struct PhotonRecord { uint32_t ev; int32_t tris[4]; float params[8]; F3 p_final; };
inline bool photon_trace_one(PhotonRecord* rec, const InternalNode* nodes, uint32_t root, const Triangle* tris,
                             const TriangleAttrib* attribs, int iTri, uint32_t photon, F3 p_light, float eta_min,
                             float eta_max, int iteration, float minThroughput)
{
    if (attribs[iTri].material == kDiffuse) return false;
    const Triangle tri = tris[iTri];
    F3 ng0 = unnormalized_normal(tri);
    F3 ns0 = attribs[iTri].shadingNormals[0];
    ng0 = ng0 * dot(ng0, ns0);
    if (dot(ng0, p_light - tri.vs[0]) < 0.0f) return false;
    const int K = 4;
    float px, py;
    sobol2d(&px, &py, photon, (uint32_t)iteration, (uint32_t)iTri, 789u);
    square2triangle(&px, &py);
    float er_x, er_y;
    sobol2d(&er_x, &er_y, photon, (uint32_t)iteration, (uint32_t)iTri, 178u);
    float eta = lerp(eta_min, eta_max, er_x);
    F3 e0 = tri.vs[1] - tri.vs[0];
    F3 e1 = tri.vs[2] - tri.vs[0];
    F3 p = tri.vs[0] + e0 * px + e1 * py;
    F3 ro = p_light;
    F3 rd = p - p_light;
    EventDescriptor ed;
    bool admissible = false;
    float throughput = 1.0f;
    F3 p_final{0, 0, 0};
    int32_t triIdx[4] = {0, 0, 0, 0};
    float prm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int d = 0; d < K + 1; d++) {
        Hit hit;
        intersect_stackfull(&hit, nodes, tris, root, ro, rd, inv_rd(rd));
        if (hit.t == kFltMax) break;
        const TriangleAttrib& at = attribs[hit.triangleIndex];
        int m = at.material;
        F3 p_hit = ro + rd * hit.t;
        F3 ns = at.shadingNormals[0] + (at.shadingNormals[1] - at.shadingNormals[0]) * hit.u +
                (at.shadingNormals[2] - at.shadingNormals[0]) * hit.v;
        if (m == kDiffuse) {
            if (d == 0) break;
            admissible = true;
            p_final = p_hit;
            break;
        }
        if (d == K) break;
        F3 wi = -rd;
        triIdx[d] = (int32_t)hit.triangleIndex;
        prm[d * 2] = hit.u;
        prm[d * 2 + 1] = hit.v;
        float rx, ry;
        sobol2d(&rx, &ry, photon, (uint32_t)d, (uint32_t)iTri, (uint32_t)iteration);
        float reflectance = fresnel_exact_norm_free(wi, ns, eta);
        bool isT = false;
        if (m == kMirror) isT = false;
        else if (m == kDielectric) isT = !(rx < reflectance);
        ed.push_back(isT);
        float sign = 1.0f;
        F3 wo;
        if (!isT) {
            wo = reflection(wi, ns);
            if (m == kDielectric) throughput *= reflectance;
        } else {
            if (!refraction_norm_free(&wo, wi, ns, eta)) break;
            sign = -1.0f;
            throughput *= 1.0f - reflectance;
        }
        if (0.0f < dot(hit.ng, wi) * dot(hit.ng, wo) * sign) {
            F3 offset_dir = normalize(hit.ng * dot(hit.ng, wo));
            ro = p_hit + offset_dir * ray_offset_scale(p_hit);
            rd = wo;
            continue;
        }
        break;
    }
    if (admissible && minThroughput < throughput) {
        rec->ev = ed.bits;
        std::memcpy(rec->tris, triIdx, sizeof(triIdx));
        std::memcpy(rec->params, prm, sizeof(prm));
        rec->p_final = p_final;
        return true;
    }
    return false;
}

// ----------------------------------------------------------------------------
// camera -- camera.h:4-41
// ----------------------------------------------------------------------------
struct RayGenerator { F3 origin{0, 0, 0}, right{1, 0, 0}, up{0, 1, 0}; };
inline RayGenerator lookat(F3 eye, F3 center, F3 upv, float fovy, int w, int h)
{
    F3 f = normalize(center - eye);
    F3 s = normalize(cross(f, upv));
    F3 u = cross(s, f);
    // camera.h:16 calls the unqualified C tan(), i.e. the double-precision function.
    float ty = (float)std::tan((double)(fovy * 0.5f));
    float tx = ty / (float)h * (float)w;
    return RayGenerator{eye, s * tx, u * ty};
}
inline void shoot(const RayGenerator& g, F3* ro, F3* rd, float u, float v)
{
    F3 from = g.origin;
    F3 forward = normalize(cross(g.up, g.right));
    F3 to_ = g.origin + forward + lerp3(-g.right, g.right, u) + lerp3(g.up, -g.up, v);
    *ro = from;
    *rd = to_ - from;
}

// ----------------------------------------------------------------------------
// spectral model -- pk.h:932-1033.  Accurate exp/log (the reference device build uses
// the fast approximations; its host build uses std::expf as here).
// ----------------------------------------------------------------------------
inline float cauchy(float A, float B, float nm) { return A + B / (nm * nm); }
inline float asym_gauss(float x, float mean, float sigma, float a)
{
    float denom = sigma + a * (x - mean);
    if (denom < 1.0e-15f) denom = 1.0e-15f;
    if (sigma * 2.0f < denom) denom = sigma * 2.0f;
    float k = (x - mean) / denom;
    return std::exp(-k * k);
}
inline float cmf_x(float x)
{
    float a = 0.42f * asym_gauss(x, 445.5849609375f, 31.146467208862305f, 0.06435633450746536f);
    float b = 1.16f * asym_gauss(x, 594.5570068359375f, 48.602108001708984f, -0.04772702232003212f);
    return (a + b - a * b * 42.559776306152344f) * 1.0008530432426956f;
}
inline float cmf_y(float x) { return 1.0f * asym_gauss(x, 556.8383178710938f, 66.54190826416016f, -0.026492968201637268f) * 1.004315086937574f; }
inline float cmf_z(float x) { return 2.146832f * asym_gauss(x, 445.9251708984375f, 30.91781997680664f, 0.08379141241312027f) * 0.9975112815948937f; }
inline float logistic_pdf(float x, float s)
{
    float k = std::exp(-std::fabs(x) / s);
    return (float)(k / ((1.0 + k) * (1.0 + k) * s));
}
inline float logistic_cdf(float x, float s) { return 1.0f / (1.0f + std::exp(-x / s)); }
inline float inverse_logistic_cdf(float u, float s)
{
    if (0.99999994f < u) u = 0.99999994f;
    if (u < 1.175494351e-38f) u = 1.175494351e-38f;
    return -s * std::log(1.0f / u - 1.0f);
}
inline float cmf_y_pdf(float x)
{
    float sx = x - 554.270751953125f, s = 26.879621505737305f;
    return logistic_pdf(sx, s) / (logistic_cdf(275.729248046875f, s) - logistic_cdf(-164.270751953125f, s));
}
inline float cmf_y_sample(float u)
{
    float s = 26.879621505737305f;
    float Pa = logistic_cdf(-164.270751953125f, s), Pb = logistic_cdf(275.729248046875f, s);
    return inverse_logistic_cdf(Pa + (Pb - Pa) * u, s) + 554.270751953125f;
}
inline F3 xyz2srgblinear(F3 xyz)
{
    return mk(dot(mk(3.2406f, -1.5372f, -0.4986f), xyz), dot(mk(-0.9689f, 1.8758f, 0.0415f), xyz),
              dot(mk(0.0557f, -0.204f, 1.057f), xyz));
}
inline float srgb_oetf(float r)
{
    r = std::fmax(r, 0.0f);
    if (r <= 0.003130f) return 12.92f * r;
    return 1.055f * std::pow(r, 1.0f / 2.4f) - 0.055f;
}
constexpr float kIntegralCmfY = 118.51810464018001f;
inline uint32_t pack_rgba(float r, float g, float b, float a)  // main_gpu.cu:9-14
{
    auto q = [](float c) { int i = f2i_rz(c * 255.0f + 0.5f); return std::max(0, std::min(i, 255)); };
    return 0xFF000000u | ((uint32_t)q(b) << 16) | ((uint32_t)q(g) << 8) | (uint32_t)q(r);
}

// ----------------------------------------------------------------------------
// forward-mode duals -- restates saka.h:11-202
// ----------------------------------------------------------------------------
template <class T> struct Dual { T v, g; };
template <class T> inline Dual<T> dc(T v) { return Dual<T>{v, T(0)}; }
template <class T> inline Dual<T> operator+(Dual<T> a, Dual<T> b) { return {a.v + b.v, a.g * T(1) + b.g * T(1)}; }
template <class T> inline Dual<T> operator-(Dual<T> a, Dual<T> b) { return {a.v - b.v, a.g * T(1) + b.g * T(-1)}; }
template <class T> inline Dual<T> operator-(Dual<T> a) { return {-a.v, a.g * T(-1)}; }
template <class T> inline Dual<T> operator*(Dual<T> a, Dual<T> b) { return {a.v * b.v, a.g * b.v + b.g * a.v}; }
template <class T> inline Dual<T> operator/(Dual<T> a, Dual<T> b) { return {a.v / b.v, a.g * (T(1) / b.v) + b.g * (-a.v / (b.v * b.v))}; }
template <class T> inline Dual<T> dsqrt(Dual<T> a) { return {std::sqrt(a.v), a.g * (T(0.5) / std::sqrt(a.v))}; }
template <class T> struct Dual3 { Dual<T> x, y, z; };
template <class T> inline Dual3<T> d3(V3<T> v) { return {dc(v.x), dc(v.y), dc(v.z)}; }
template <class T> inline Dual3<T> operator+(Dual3<T> a, Dual3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline Dual3<T> operator-(Dual3<T> a, Dual3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline Dual3<T> operator-(Dual3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline Dual3<T> operator*(Dual3<T> a, Dual<T> s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline Dual3<T> operator/(Dual3<T> a, Dual<T> s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline Dual<T> ddot(Dual3<T> a, Dual3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline Dual3<T> dcross(Dual3<T> a, Dual3<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline Dual3<T> dreflection(Dual3<T> wi, Dual3<T> n)
{
    return n * ddot(wi, n) * dc(T(2)) / ddot(n, n) - wi;
}
template <class T> inline Dual3<T> drefraction(Dual3<T> wi, Dual3<T> n, T eta)
{
    Dual<T> NoN = ddot(n, n), WIoN = ddot(wi, n), WoW = ddot(wi, wi);
    Dual<T> k = NoN * WoW * dc(eta * eta - T(1)) + WIoN * WIoN;
    if (k.v < T(0)) return d3(V3<T>{0, 0, 0});
    return -wi * NoN + n * (WIoN - dsqrt(k));
}

// ----------------------------------------------------------------------------
// Householder QR least squares -- restates sen.h:658-747 (column-major R x C)
// ----------------------------------------------------------------------------
template <class T, int R, int C> struct Mat {
    T m[R * C];
    T& operator()(int r, int c) { return m[c * R + r]; }
    const T& operator()(int r, int c) const { return m[c * R + r]; }
};
template <class T, int R, int C> inline void solve_qr_overdetermined(Mat<T, R, C> A, const T* b_in, T* x)
{
    constexpr int NH = (C < R - 1) ? C : R - 1;
    T vs[R * (NH > 0 ? NH : 1)];
    for (int i = 0; i < NH; i++) {
        for (int j = 0; j < R; j++) vs[i * R + j] = j < i ? T(0) : -A(j, i);
        T sgn = T(0) < vs[i * R + i] ? T(1) : T(-1);
        T cd = T(0);
        for (int r = 0; r < R; r++) cd += vs[i * R + r] * vs[i * R + r];
        T x_len = std::sqrt(cd);
        vs[i * R + i] += sgn * x_len;
        T v_len2 = T(2) * x_len * (x_len + std::fabs(A(i, i)));
        A(i, i) = sgn * x_len;
        for (int r = i + 1; r < R; r++) A(r, i) = T(0);
        for (int c = i + 1; c < C; c++) {
            T vdc = T(0);
            for (int r = i; r < R; r++) vdc += vs[i * R + r] * A(r, c);
            T k = T(2) * vdc / v_len2;
            for (int r = i; r < R; r++) A(r, c) -= k * vs[i * R + r];
        }
    }
    T b[R];
    for (int r = 0; r < R; r++) b[r] = b_in[r];
    for (int i = 0; i < NH; i++) {
        T vdc = T(0), vdv = T(0);
        for (int r = i; r < R; r++) { T v = vs[i * R + r]; vdc += v * b[r]; vdv += v * v; }
        T k = T(2) * vdc / vdv;
        for (int r = i; r < R; r++) b[r] -= k * vs[i * R + r];
    }
    for (int r = C - 1; 0 <= r; r--) {
        T sum = T(0);
        for (int i = r + 1; i < C; i++) sum += A(r, i) * x[i];
        x[r] = (b[r] - sum) / A(r, r);
    }
}

// ----------------------------------------------------------------------------
// specular constraint solver -- solveConstraints<K>, pk.h:466-592
// parameters: 2K barycentrics (in: initial guess, out: root)
// ----------------------------------------------------------------------------
template <class T, int K>
inline bool solve_constraints(T* parameters, V3<T> p_beg, V3<T> p_end, const Triangle* tris, const TriangleAttrib* attribs,
                              T eta, uint32_t events, int maxIterations, T costTolerance, int earlyTermWarmUp,
                              int* iterationsOut = nullptr)
{
    const int NP = 2 * K;
    T edge_eps = T(0.25);
    for (int iter = 0; iter < maxIterations; iter++) {
        Mat<T, 3 * K, 2 * K> A;
        T b[3 * K];
        T cost = T(0);
        for (int i = 0; i < NP; i++) {
            Dual3<T> vertices[K + 2];
            vertices[0] = d3(p_beg);
            vertices[K + 1] = d3(p_end);
            Dual3<T> sn[K];
            for (int k = 0; k < K; k++) {
                Dual<T> pu{parameters[k * 2 + 0], T(k * 2 + 0 == i ? 1 : 0)};
                Dual<T> pv{parameters[k * 2 + 1], T(k * 2 + 1 == i ? 1 : 0)};
                V3<T> v0 = to<T>(tris[k].vs[0]);
                V3<T> e0 = to<T>(tris[k].vs[1] - tris[k].vs[0]);
                V3<T> e1 = to<T>(tris[k].vs[2] - tris[k].vs[0]);
                vertices[k + 1] = d3(v0) + d3(e0) * pu + d3(e1) * pv;
                V3<T> n0 = to<T>(attribs[k].shadingNormals[0]);
                V3<T> ne0 = to<T>(attribs[k].shadingNormals[1] - attribs[k].shadingNormals[0]);
                V3<T> ne1 = to<T>(attribs[k].shadingNormals[2] - attribs[k].shadingNormals[0]);
                sn[k] = d3(n0) + d3(ne0) * pu + d3(ne1) * pv;
            }
            for (int k = 0; k < K; k++) {
                Dual3<T> wi = vertices[k] - vertices[k + 1];
                Dual3<T> wo = vertices[k + 2] - vertices[k + 1];
                Dual3<T> n = sn[k];
                if (ddot(wi, n).v < T(0)) std::swap(wi, wo);
                Dual3<T> wo_opt = ((events >> k) & 1u) ? drefraction(wi, n, eta) : dreflection(wi, n);
                Dual3<T> c = dcross(wo, wo_opt);
                A(k * 3 + 0, i) = c.x.g; A(k * 3 + 1, i) = c.y.g; A(k * 3 + 2, i) = c.z.g;
                b[k * 3 + 0] = c.x.v; b[k * 3 + 1] = c.y.v; b[k * 3 + 2] = c.z.v;
                if (i == 0) cost += ddot(c, c).v;
            }
        }
        if (cost < costTolerance) { if (iterationsOut) *iterationsOut = iter; return true; }
        T dp[2 * K];
        solve_qr_overdetermined<T, 3 * K, 2 * K>(A, b, dp);
        for (int i = 0; i < NP; i++) parameters[i] = parameters[i] - dp[i];
        if (earlyTermWarmUp <= iter) {
            for (int k = 0; k < K; k++) {
                T u = parameters[k * 2 + 0], v = parameters[k * 2 + 1];
                if (-edge_eps < u && -edge_eps < v && u + v < T(1) + edge_eps) continue;
                if (iterationsOut) *iterationsOut = iter + 1;
                return false;
            }
            edge_eps *= edge_eps;
        }
    }
    if (iterationsOut) *iterationsOut = maxIterations;
    return false;
}

template <class T> inline V3<T> get_vertex(int k, const Triangle* tris, const T* params)  // pk.h:752-758
{
    V3<T> v0 = to<T>(tris[k].vs[0]);
    V3<T> e0 = to<T>(tris[k].vs[1] - tris[k].vs[0]);
    V3<T> e1 = to<T>(tris[k].vs[2] - tris[k].vs[0]);
    return v0 + e0 * params[k * 2 + 0] + e1 * params[k * 2 + 1];
}

// contributableThroughput<K>, pk.h:760-842.  Visibility runs in float against the
// float BVH (as the reference); the rest in T.
template <class T, int K>
inline T contributable_throughput(const T* params, V3<T> p_beg, V3<T> p_end, const Triangle* tris, const TriangleAttrib* attribs,
                                  uint32_t events, const InternalNode* nodes, const Triangle* sceneTris, uint32_t root, T eta)
{
    V3<T> vertices[K + 2];
    V3<T> sn[K + 2];
    vertices[0] = p_beg;
    vertices[K + 1] = p_end;
    for (int k = 0; k < K; k++) {
        T u = params[k * 2 + 0], v = params[k * 2 + 1];
        if (u < T(0) || v < T(0) || T(1) < u + v) return T(0);
        vertices[k + 1] = get_vertex<T>(k, tris, params);
        V3<T> n0 = to<T>(attribs[k].shadingNormals[0]);
        V3<T> ne0 = to<T>(attribs[k].shadingNormals[1] - attribs[k].shadingNormals[0]);
        V3<T> ne1 = to<T>(attribs[k].shadingNormals[2] - attribs[k].shadingNormals[0]);
        sn[k + 1] = normalize(n0 + ne0 * u + ne1 * v);
    }
    sn[0] = normalize(vertices[1] - vertices[0]);
    sn[K + 1] = normalize(vertices[K] - vertices[K + 1]);
    T thr = T(1);
    for (int k = 0; k < K; k++) {
        V3<T> wi = vertices[k] - vertices[k + 1];
        V3<T> wo = vertices[k + 2] - vertices[k + 1];
        V3<T> n = sn[k + 1];
        bool eR = T(0) < dot(wi, n) * dot(wo, n);
        if (((events >> k) & 1u) == (eR ? 1u : 0u)) return T(0);  // event mismatch
        V3<T> ng = to<T>(unnormalized_normal(tris[k]));
        bool egR = T(0) < dot(wi, ng) * dot(wo, ng);
        if (eR != egR) return T(0);
        if (attribs[k].material == kDielectric) {
            T r = fresnel_exact_norm_free(wi, n, eta);
            thr *= eR ? r : T(1) - r;
        }
    }
    for (int i = 0; i < K + 1; i++) {
        V3<T> d = vertices[i] - vertices[i + 1];
        if (dot(d, d) < T(1.0e-5f)) return T(0);
    }
    for (int i = 0; i < K + 1; i++) {
        F3 a = mk((float)vertices[i].x, (float)vertices[i].y, (float)vertices[i].z);
        F3 b = mk((float)vertices[i + 1].x, (float)vertices[i + 1].y, (float)vertices[i + 1].z);
        F3 na = mk((float)sn[i].x, (float)sn[i].y, (float)sn[i].z);
        F3 nb = mk((float)sn[i + 1].x, (float)sn[i + 1].y, (float)sn[i + 1].z);
        if (occluded(nodes, sceneTris, root, a, na, b, nb)) return T(0);
    }
    return thr;
}

// GetOrthonormalBasis, pk.h:453-459
template <class T> inline void orthonormal_basis(V3<T> z, V3<T>* x, V3<T>* y)
{
    const T sign = std::copysign(T(1), z.z);
    const T a = T(-1) / (sign + z.z);
    const T b = z.x * z.y * a;
    *x = V3<T>{T(1) + sign * z.x * z.x * a, sign * b, -sign * z.x};
    *y = V3<T>{b, sign + z.y * z.y * a, -z.y};
}
template <class T> inline Dual3<T> ray_plane(Dual3<T> ro, Dual3<T> rd, Dual3<T> ng, Dual3<T> v0)  // pk.h:594-598
{
    Dual<T> t = ddot(v0 - ro, ng) / ddot(ng, rd);
    return ro + rd * t;
}

// dAdw, pk.h:844-930 (generalized geometry term by ray differentials)
template <class T>
inline T dAdw(V3<T> ro, V3<T> rd, V3<T> p_end, const Triangle* tris, const TriangleAttrib* attribs, uint32_t events, T eta)
{
    rd = normalize(rd);
    int K = (int)(events >> 24);
    V3<T> dAxis[2];
    for (int i = 0; i < 2; i++) {
        Dual<T> dif[2] = {dc(T(0)), dc(T(0))};
        dif[i].g = T(1);
        Dual3<T> ro_j = d3(ro);
        V3<T> T0, T1;
        orthonormal_basis(rd, &T0, &T1);
        Dual3<T> rd_j = d3(rd) + d3(T0) * dif[0] + d3(T1) * dif[1];
        for (int j = 0; j < K; j++) {
            const Triangle& tri = tris[j];
            V3<T> ng = to<T>(unnormalized_normal(tri));
            Dual3<T> p = ray_plane(ro_j, rd_j, d3(ng), d3(to<T>(tri.vs[0])));
            V3<T> tv0 = to<T>(tri.vs[0]), tv1 = to<T>(tri.vs[1]), tv2 = to<T>(tri.vs[2]);
            Dual<T> v = ddot(p - d3(tv1), d3(cross(ng, tv1 - tv0)));
            Dual<T> w = ddot(p - d3(tv2), d3(cross(ng, tv2 - tv1)));
            Dual<T> u = ddot(p - d3(tv0), d3(cross(ng, tv0 - tv2)));
            Dual<T> area = u + v + w;
            u = u / area; v = v / area; w = w / area;
            Dual3<T> n = d3(to<T>(attribs[j].shadingNormals[0])) * w + d3(to<T>(attribs[j].shadingNormals[1])) * u +
                         d3(to<T>(attribs[j].shadingNormals[2])) * v;
            Dual3<T> wi = -rd_j;
            Dual3<T> wo;
            if ((events >> j) & 1u) {
                if (ddot(wi, n).v < T(0)) {
                    wo = drefraction(wi, -n, T(1) / eta);
                    if (wo.x.v == T(0) && wo.y.v == T(0) && wo.z.v == T(0)) return T(3.402823466e+38f);
                } else {
                    wo = drefraction(wi, n, eta);
                }
            } else {
                wo = dreflection(wi, n);
            }
            ro_j = p;
            rd_j = wo;
        }
        V3<T> p_last{ro_j.x.v, ro_j.y.v, ro_j.z.v};
        Dual3<T> pf = ray_plane(ro_j, rd_j, d3(p_last - p_end), d3(p_end));
        dAxis[i] = V3<T>{pf.x.g, pf.y.g, pf.z.g};
    }
    T len0 = length(dAxis[0]), len1 = length(dAxis[1]);
    T sinTheta = length(cross(dAxis[0] / len0, dAxis[1] / len1));
    return len0 * len1 * std::fmax(sinTheta, T(0.01));
}

// ----------------------------------------------------------------------------
// interval arithmetic, round-to-nearest -- restates interval.h:34-713
// ----------------------------------------------------------------------------
struct Intr { float l, u; };
inline Intr ival(float v) { return Intr{v, v}; }
inline Intr operator-(Intr a) { return {-a.u, -a.l}; }
inline Intr operator+(Intr a, Intr b) { return {a.l + b.l, a.u + b.u}; }
inline Intr operator-(Intr a, Intr b) { return {a.l - b.u, a.u - b.l}; }
inline float smin(float a, float b) { return a < b ? a : b; }
inline float smax(float a, float b) { return a > b ? a : b; }
inline Intr operator*(Intr a, Intr b)
{
    float p0 = a.l * b.l, p1 = a.l * b.u, p2 = a.u * b.l, p3 = a.u * b.u;
    return {smin(p0, smin(p1, smin(p2, p3))), smax(p0, smax(p1, smax(p2, p3)))};
}
inline Intr operator/(Intr a, Intr b) { return a * Intr{1.0f / b.l, 1.0f / b.u}; }
inline Intr isqrt(Intr x) { return {std::sqrt(x.l), std::sqrt(x.u)}; }
inline Intr isquare(Intr x)
{
    float l2 = x.l * x.l, u2 = x.u * x.u;
    float larger = smax(l2, u2);
    if (x.l <= 0.0f && 0.0f <= x.u) return {0.0f, larger};
    return {smin(l2, u2), larger};
}
struct Intr3 { Intr x, y, z; };
inline Intr3 i3(F3 v) { return {ival(v.x), ival(v.y), ival(v.z)}; }
inline Intr3 i3(const AABB& b) { return {{b.lower.x, b.upper.x}, {b.lower.y, b.upper.y}, {b.lower.z, b.upper.z}}; }
inline Intr3 operator-(Intr3 a) { return {-a.x, -a.y, -a.z}; }
inline Intr3 operator+(Intr3 a, Intr3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Intr3 operator-(Intr3 a, Intr3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Intr3 operator*(Intr3 a, Intr s) { return {a.x * s, a.y * s, a.z * s}; }
inline Intr idot(Intr3 a, Intr3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Intr3 icross(Intr3 a, Intr3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline Intr ilength_sq(Intr3 v) { return isquare(v.x) + isquare(v.y) + isquare(v.z); }
inline bool zero_included(Intr3 v) { return v.x.l * v.x.u <= 0.0f && v.y.l * v.y.u <= 0.0f && v.z.l * v.z.u <= 0.0f; }
inline bool intersects(Intr3 a, Intr3 b, float eps)
{
    if (a.x.u + eps < b.x.l || b.x.u + eps < a.x.l) return false;
    if (a.y.u + eps < b.y.l || b.y.u + eps < a.y.l) return false;
    if (a.z.u + eps < b.z.l || b.z.u + eps < a.z.l) return false;
    return true;
}
inline Intr3 ireflection(Intr3 wi, Intr3 n)  // interval.h:229-252
{
    const float eps = 1.0e-10f;
    Intr nxx = isquare(n.x), nyy = isquare(n.y), nzz = isquare(n.z);
    Intr nn = nxx + nyy + nzz;
    Intr s{2.0f / smax(nn.u, eps), 2.0f / smax(nn.l, eps)};
    Intr m11 = s * nxx - ival(1.0f), m12 = s * n.x * n.y, m13 = s * n.x * n.z;
    Intr m21 = m12, m22 = s * nyy - ival(1.0f), m23 = s * n.y * n.z;
    Intr m31 = m13, m32 = m23, m33 = s * nzz - ival(1.0f);
    return {m11 * wi.x + m12 * wi.y + m13 * wi.z, m21 * wi.x + m22 * wi.y + m23 * wi.z,
            m31 * wi.x + m32 * wi.y + m33 * wi.z};
}
inline Intr3 irefraction_normal(Intr3 wi, Intr3 wo, float eta)  // interval.h:254-259
{
    Intr lenWi = isqrt(ilength_sq(wi));
    Intr lenWo = isqrt(ilength_sq(wo));
    return -(wo * lenWi * ival(eta) + wi * lenWo);
}
inline bool irefraction_norm_free(Intr3* wo, Intr3 wi, Intr3 n, float eta)  // interval.h:398-418
{
    Intr NoN = ilength_sq(n);
    Intr WIoN = idot(wi, n);
    if (WIoN.u < 0.0f) return false;
    WIoN.l = smax(WIoN.l, 0.0f);
    Intr WIoWI = ilength_sq(wi);
    Intr k = NoN * WIoWI * ival(eta * eta - 1.0f) + isquare(WIoN);
    if (k.u < 0.0f) return false;
    k.l = smax(k.l, 0.0f);
    *wo = -wi * NoN + n * (WIoN - isqrt(k));
    return true;
}
inline Intr3 inormalize(Intr3 p)  // interval.h:479-679 (the live branch)
{
    const float eps = 1.0e-10f;
    if (p.x.l * p.x.u <= 0.0f && p.y.l * p.y.u <= 0.0f && p.z.l * p.z.u <= 0.0f)
        return {{-1.0f, 1.0f}, {-1.0f, 1.0f}, {-1.0f, 1.0f}};
    float vs[3][2] = {{p.x.l, p.x.u}, {p.y.l, p.y.u}, {p.z.l, p.z.u}};
    float bd[3][2] = {{2.0f, -2.0f}, {2.0f, -2.0f}, {2.0f, -2.0f}};
    for (int iz = 0; iz < 2; iz++)
        for (int iy = 0; iy < 2; iy++)
            for (int ix = 0; ix < 2; ix++) {
                float x = vs[0][ix], y = vs[1][iy], z = vs[2][iz];
                float len = smax(std::sqrt(x * x + y * y + z * z), eps);
                float nx = x / len, ny = y / len, nz = z / len;
                bd[0][0] = smin(bd[0][0], nx); bd[1][0] = smin(bd[1][0], ny); bd[2][0] = smin(bd[2][0], nz);
                bd[0][1] = smax(bd[0][1], nx); bd[1][1] = smax(bd[1][1], ny); bd[2][1] = smax(bd[2][1], nz);
            }
    if (0.0f < vs[0][0] * vs[0][1] && 0.0f < vs[1][0] * vs[1][1] && 0.0f < vs[2][0] * vs[2][1])
        return {{bd[0][0], bd[0][1]}, {bd[1][0], bd[1][1]}, {bd[2][0], bd[2][1]}};
    for (int axis = 0; axis < 3; axis++) {
        int ab = (axis + 1) % 3, ac = (axis + 2) % 3;
        if (0.0f < vs[axis][0] * vs[axis][1]) {
            float nz = 0.0f < vs[axis][0] ? vs[axis][0] : vs[axis][1];
            float nzz = nz * nz;
            bool zx = vs[ab][0] * vs[ab][1] <= 0.0f;
            bool zy = vs[ac][0] * vs[ac][1] <= 0.0f;
            if (zy) {
                float lo = vs[ab][0], up = vs[ab][1];
                float ll = smax(std::sqrt(nzz + lo * lo), eps), ul = smax(std::sqrt(nzz + up * up), eps);
                bd[ab][0] = smin(bd[ab][0], lo / ll);
                bd[ab][1] = smax(bd[ab][1], up / ul);
            }
            if (zx) {
                float lo = vs[ac][0], up = vs[ac][1];
                float ll = smax(std::sqrt(nzz + lo * lo), eps), ul = smax(std::sqrt(nzz + up * up), eps);
                bd[ac][0] = smin(bd[ac][0], lo / ll);
                bd[ac][1] = smax(bd[ac][1], up / ul);
            }
            if (zx && zy) {
                if (0.0f <= vs[axis][1]) bd[axis][1] = 1.0f;
                else bd[axis][0] = -1.0f;
            }
        }
    }
    return {{bd[0][0], bd[0][1]}, {bd[1][0], bd[1][1]}, {bd[2][0], bd[2][1]}};
}

// ----------------------------------------------------------------------------
// Path Cuts -- InternalNormalBound (pk.h:1705-1709), normal bounds (main.cpp:250-295),
// traverseAdmissibleNodes<K> (pk.h:1760-2220, live branch)
// ----------------------------------------------------------------------------
struct InternalNormalBound { AABB normalBounds[2]; uint32_t counter; };

inline void build_normal_bounds(std::vector<InternalNormalBound>& out, const InternalNode* internals, int nInternals,
                                const Triangle* tris, const TriangleAttrib* attribs)
{
    out.assign(nInternals, InternalNormalBound{});
    for (auto& b : out) { b.normalBounds[0] = AABB{}; b.normalBounds[1] = AABB{}; b.counter = 0; }
    for (int i = 0; i < nInternals; i++) {
        for (int j = 0; j < 2; j++) {
            uint32_t me = internals[i].children[j];
            if (!node_is_leaf(me)) continue;
            uint32_t parent = make_node((uint32_t)i, false);
            AABB nb = aabb_empty();
            for (int k = 0; k < 3; k++) aabb_extend(nb, attribs[node_idx(me)].shadingNormals[k]);
            while (parent != kInvalidNode) {
                int ci = internals[node_idx(parent)].children[0] == me ? 0 : 1;
                out[node_idx(parent)].normalBounds[ci] = nb;
                uint32_t v = out[node_idx(parent)].counter++;
                if (v == 0) break;
                aabb_extend(nb, out[node_idx(parent)].normalBounds[ci ^ 1]);
                me = parent;
                parent = internals[node_idx(me)].parent;
            }
        }
    }
}

inline AABB node_aabb(const InternalNode& n) { AABB b = n.aabbs[0]; aabb_extend(b, n.aabbs[1]); return b; }

template <int K, class CB>
inline void traverse_admissible_nodes(uint32_t events, float eta, F3 p_beg, F3 p_end, const InternalNode* internals,
                                      const InternalNormalBound* nbs, const Triangle* tris, const TriangleAttrib* attribs,
                                      uint32_t root, CB admissibles, uint64_t* nodeTuplesVisited = nullptr)
{
    struct Tup { uint32_t n[K]; };
    Intr3 pb = i3(p_beg), pe = i3(p_end);
    std::vector<Tup> stack;
    Tup inv;
    for (int i = 0; i < K; i++) inv.n[i] = kInvalidNode;
    stack.push_back(inv);
    Tup cur;
    for (int i = 0; i < K; i++) cur.n[i] = root;
    while (cur.n[0] != kInvalidNode) {
        if (nodeTuplesVisited) (*nodeTuplesVisited)++;
        int cut = -1;
        float maxSA = -1.0f;
        for (int i = 0; i < K; i++) {
            if (node_is_leaf(cur.n[i])) continue;
            float sa = aabb_surface_area(node_aabb(internals[node_idx(cur.n[i])]));
            if (maxSA < sa) { cut = i; maxSA = sa; }
        }
        if (cut == -1) {
            int idx[K];
            for (int i = 0; i < K; i++) idx[i] = (int)node_idx(cur.n[i]);
            bool invalid = false;
            for (int i = 0; i < K - 1; i++)
                if (idx[i] == idx[i + 1]) { invalid = true; break; }
            {
                const Triangle& tb = tris[idx[0]];
                F3 ng = unnormalized_normal(tb);
                ng = ng * dot(ng, attribs[idx[0]].shadingNormals[0]);
                if (dot(ng, p_beg) < dot(ng, tb.vs[0])) invalid = true;
            }
            {
                const Triangle& te = tris[idx[K - 1]];
                F3 ng = unnormalized_normal(te);
                ng = ng * dot(ng, attribs[idx[K - 1]].shadingNormals[0]);
                if (dot(ng, p_end) < dot(ng, te.vs[0])) invalid = true;
            }
            if (!invalid) admissibles(idx);
        } else {
            for (int i = 0; i < 2; i++) {
                Intr3 vertices[K + 2];
                Intr3 normals[K];
                vertices[0] = pb;
                vertices[K + 1] = pe;
                for (int k = 0; k < K; k++) {
                    uint32_t nd = cur.n[k];
                    if (k == cut) {
                        vertices[k + 1] = i3(internals[node_idx(nd)].aabbs[i]);
                        normals[k] = i3(nbs[node_idx(nd)].normalBounds[i]);
                    } else if (node_is_leaf(nd)) {
                        AABB b = aabb_empty();
                        for (int q = 0; q < 3; q++) aabb_extend(b, tris[node_idx(nd)].vs[q]);
                        vertices[k + 1] = i3(b);
                        AABB nb = aabb_empty();
                        for (int q = 0; q < 3; q++) aabb_extend(nb, attribs[node_idx(nd)].shadingNormals[q]);
                        normals[k] = i3(nb);
                    } else {
                        vertices[k + 1] = i3(node_aabb(internals[node_idx(nd)]));
                        AABB nb = aabb_empty();
                        aabb_extend(nb, nbs[node_idx(nd)].normalBounds[0]);
                        aabb_extend(nb, nbs[node_idx(nd)].normalBounds[1]);
                        normals[k] = i3(nb);
                    }
                }
                bool admissible = true;
                bool inMedium = false;
                Intr3 wi = vertices[0] - vertices[1];
                for (int k = 0; k < K; k++) {
                    Intr3 wo = vertices[k + 2] - vertices[k + 1];
                    Intr3 nrm = normals[k];
                    Intr3 wo_next;
                    if (!((events >> k) & 1u)) {
                        wo_next = ireflection(wi, nrm);
                    } else {
                        float e = inMedium ? 1.0f / eta : eta;
                        Intr3 wiv = vertices[k] - vertices[k + 1];
                        Intr3 ht = irefraction_normal(wiv, wo, e);
                        if (!zero_included(icross(nrm, ht))) { admissible = false; break; }
                        if (!irefraction_norm_free(&wo_next, wi, inMedium ? -nrm : nrm, e)) { admissible = false; break; }
                    }
                    if (!zero_included(icross(wo_next, wo))) { admissible = false; break; }
                    inMedium = !inMedium;
                    wi = -wo_next;
                }
                if (admissible) {
                    Tup nt = cur;
                    nt.n[cut] = internals[node_idx(cur.n[cut])].children[i];
                    stack.push_back(nt);
                }
            }
        }
        cur = stack.back();
        stack.pop_back();
    }
}

}  // namespace pzo
