// pz_cache.cuh -- PathCache on the device (pk.h:227-402), structure-of-arrays layout.
//
// Semantics follow the reference: a landing photon's path {events, triangles,
// barycentrics} is inserted into the 8 cells nearest to its landing point, each by
// linear probing from the cell hash with a CAS on the path hash; an existing equal
// path hash stops the probe.  Lookups scan a cell's probe chain until an empty slot
// and report slots whose cell hash and event descriptor match.  Differences: the
// record fields live in separate arrays (probing reads 4 B of path hash per slot
// instead of a 56-byte record), a slot is read before it is claimed with the CAS (the
// probe stops on the same slot), the capacity is any power of two, and a probe that
// exceeds kMaxProbe slots stops with PZ_DEVICE_ERR_CAPACITY instead of scanning the
// whole table.
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

// The hash of the k-th (0..7) of the 8 cells nearest to pos, in the reference's order
// (x fastest, then y, then z; pk.h:302-313).
PZ_D uint32_t cache_cell_hash(const CacheView& c, float3 pos, int k)
{
    const float3 idx = pos / c.step;
    const int x = __float2int_rz(floorf(idx.x)), y = __float2int_rz(floorf(idx.y)), z = __float2int_rz(floorf(idx.z));
    const int dx = idx.x - (float)x < 0.5f ? -1 : 1;
    const int dy = idx.y - (float)y < 0.5f ? -1 : 1;
    const int dz = idx.z - (float)z < 0.5f ? -1 : 1;
    return hash_of_iP(x + (k & 1) * dx, y + ((k >> 1) & 1) * dy, z + (k >> 2) * dz);
}

// A claimed slot receives the tuple (pk.h:320-339) and counts as a stored entry.
PZ_D void cache_fill_slot(const CacheView& c, uint32_t i, uint32_t hP, uint32_t ev, int4 t, float4 p0, float4 p1)
{
    c.cell[i] = hP;
    c.event[i] = ev;
    c.tris[i] = t;
    c.params[2 * i] = p0;
    c.params[2 * i + 1] = p1;
    atomicAdd(&c.h->count, 1u);
}

// One cell of PathCache::store (pk.h:313-345), probing from slot i at probe offset off
// (the home slot, the cell hash & mask, is offset 0) for at most `steps` slots.  It visits
// the same slots in the same order and stops on the same conditions as the reference's
// CAS-per-slot loop, but reads each slot from L2 first (atomics live there): a slot
// holding this path hash ends the probe, one holding another hash is passed, and only a
// slot that reads empty is claimed with the CAS, whose answer is then handled like the
// reference's.  Slots go from empty to a path hash once and never change while photons
// are stored, so a read that saw a hash sees what the CAS would have returned.  t and
// p0/p1 are the tuple's triangle indices and barycentrics, zero past its length.
// Returns true while the probe is unfinished (i and off then name the next slot).
PZ_D bool cache_probe(const CacheView& c, uint32_t hP, uint32_t hp, uint32_t ev, int4 t, float4 p0, float4 p1,
                      uint32_t& i, uint32_t& off, uint32_t steps)
{
    const uint32_t mask = c.capacity - 1u;
    for (uint32_t k = 0; k < steps; k++) {
        if (off >= kMaxProbe) {
            raise_error(&c.h->status, kErrCapacity);
            return false;
        }
        const uint32_t seen = __ldcg(c.hash + i);
        if (seen == hp) return false;
        if (seen == 0u) {
            const uint32_t old = atomicCAS(c.hash + i, 0u, hp);
            if (old == 0u) {
                cache_fill_slot(c, i, hP, ev, t, p0, p1);
                return false;
            }
            if (old == hp) return false;
        }
        i = (i + 1u) & mask;
        off++;
    }
    if (off >= kMaxProbe) {
        raise_error(&c.h->status, kErrCapacity);
        return false;
    }
    return true;
}

}  // namespace pz
