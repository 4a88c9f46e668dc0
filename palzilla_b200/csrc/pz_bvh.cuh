// pz_bvh.cuh -- LBVH builder interface (see pz_bvh.cu).
#pragma once
#include "pz_sort.cuh"

namespace pz {
namespace bvh {

// Builder scratch header: the sort header followed by the scene AABB, stored as
// order-preserving integers (lower bounds complemented) so that zero is "empty".
struct Scratch {
    sort::Header sort;
    uint32_t aabb_enc[8];
};

struct Layout {
    Scratch* s;
    unsigned long long* lookback;
    unsigned long long* keys;  // sorted {morton (low 32), triangle index (high 32)}
    unsigned long long* tmp;
    uint8_t* deltas;
    uint32_t* flags;
    float4* pending;  // per internal node, one 32-byte slot per side: an arriver's child and box
};

enum class Stage { kKeys, kSorted, kAll };

size_t scratch_bytes(uint32_t n);
Layout layout(void* scratch, uint32_t n);
cudaError_t build(const Tri* tris, uint32_t n, uint32_t opt, Node* nodes, uint32_t* root, void* scratch,
                  cudaStream_t st, Stage stopAfter = Stage::kAll);

}  // namespace bvh
}  // namespace pz
