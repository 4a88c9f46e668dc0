// pz_cache.cuh -- PathCache on the device (pk.h:227-402), structure-of-arrays layout.
//
// Semantics follow the reference: a landing photon's path {events, triangles,
// barycentrics} is inserted into the 8 cells nearest to its landing point, each by
// linear probing from the cell hash with a CAS on the path hash; an existing equal
// path hash stops the probe.  Lookups scan a cell's probe chain until an empty slot
// and report slots whose cell hash and event descriptor match.  Differences: the
// record fields live in separate arrays (probing reads 12 B per slot instead of a
// 56-byte record), the capacity is any power of two, and a probe that exceeds
// kMaxProbe slots stops with PZ_DEVICE_ERR_CAPACITY instead of scanning the whole
// table.
#pragma once
#include "pz_common.cuh"

namespace pz {

constexpr uint32_t kMaxProbe = 1u << 16;

struct CacheHeader {
    uint32_t status;
    uint32_t count;      // stored (path, cell) entries
    uint32_t capacity;   // power of two
    float step;          // cell size
    uint32_t pad[60];
};
static_assert(sizeof(CacheHeader) == 256, "cache header");

struct CacheView {
    CacheHeader* h;
    uint32_t* hash;   // path hash, 0 = empty
    uint32_t* cell;   // cell hash (TrianglePath::hashOfP)
    uint32_t* event;  // EventDescriptor::asU32
    int4* tris;       // up to 4 triangle indices
    float4* params;   // 2 float4 per slot: barycentrics of up to 4 vertices
    uint32_t capacity;
    float step;
};

inline size_t cache_bytes(uint32_t capacity) { return 256 + (size_t)capacity * (4 + 4 + 4 + 16 + 32); }

inline CacheView cache_view(void* base, uint32_t capacity, float step)
{
    CacheView c;
    char* p = static_cast<char*>(base);
    c.h = reinterpret_cast<CacheHeader*>(p);
    p += 256;
    c.tris = reinterpret_cast<int4*>(p);
    p += (size_t)capacity * 16;
    c.params = reinterpret_cast<float4*>(p);
    p += (size_t)capacity * 32;
    c.hash = reinterpret_cast<uint32_t*>(p);
    p += (size_t)capacity * 4;
    c.cell = reinterpret_cast<uint32_t*>(p);
    p += (size_t)capacity * 4;
    c.event = reinterpret_cast<uint32_t*>(p);
    c.capacity = capacity;
    c.step = step;
    return c;
}

// hashOfPath, pk.h:293-298
PZ_HD uint32_t path_hash(uint32_t ev, const int* tris)
{
    uint32_t h = ev;
    const int K = (int)(ev >> 24);
    for (int d = 0; d < K; d++) h = hash_pcg(h + (uint32_t)tris[d]);
    return h | 1u;
}

// spacial_hash, pk.h:219-225
PZ_D uint32_t spacial_hash(float3 p, float step)
{
    float3 idx = p / step;
    return hash_of_iP(__float2int_rz(floorf(idx.x)), __float2int_rz(floorf(idx.y)), __float2int_rz(floorf(idx.z)));
}

// PathCache::store, pk.h:291-349
PZ_D bool cache_store(const CacheView& c, float3 pos, const int* tris, const float* params, uint32_t ev)
{
    const uint32_t hp = path_hash(ev, tris);
    const int K = (int)(ev >> 24);
    const uint32_t mask = c.capacity - 1u;
    bool success = false;
    float3 idx = pos / c.step;
    int x = __float2int_rz(floorf(idx.x)), y = __float2int_rz(floorf(idx.y)), z = __float2int_rz(floorf(idx.z));
    int dx = idx.x - (float)x < 0.5f ? -1 : 1;
    int dy = idx.y - (float)y < 0.5f ? -1 : 1;
    int dz = idx.z - (float)z < 0.5f ? -1 : 1;
    for (int iz = 0; iz < 2; iz++)
        for (int iy = 0; iy < 2; iy++)
            for (int ix = 0; ix < 2; ix++) {
                const uint32_t hP = hash_of_iP(x + ix * dx, y + iy * dy, z + iz * dz);
                const uint32_t home = hP & mask;
                uint32_t off = 0;
                for (; off < kMaxProbe; off++) {
                    const uint32_t i = (home + off) & mask;
                    const uint32_t old = atomicCAS(c.hash + i, 0u, hp);
                    if (old == 0u) {
                        c.cell[i] = hP;
                        c.event[i] = ev;
                        c.tris[i] = make_int4(tris[0], K > 1 ? tris[1] : 0, K > 2 ? tris[2] : 0, K > 3 ? tris[3] : 0);
                        float p[8];
                        for (int d = 0; d < 8; d++) p[d] = d < 2 * K ? params[d] : 0.0f;
                        c.params[2 * i] = make_float4(p[0], p[1], p[2], p[3]);
                        c.params[2 * i + 1] = make_float4(p[4], p[5], p[6], p[7]);
                        success = true;
                        atomicAdd(&c.h->count, 1u);
                        break;
                    } else if (old == hp) {
                        break;
                    }
                }
                if (off == kMaxProbe) raise_error(&c.h->status, kErrCapacity);
            }
    return success;
}

}  // namespace pz
