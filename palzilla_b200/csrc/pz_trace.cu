// pz_trace.cu -- batch ray queries over the LBVH (closest hit and any hit), used for
// the traversal parity tests and the rays/s measurement.  Compiled with -fmad=false.
#include "pz_trace.cuh"
#include "pz_trace_api.cuh"

namespace pz {

__global__ void __launch_bounds__(256) k_trace_closest(const Node* __restrict__ nodes, const uint32_t* __restrict__ root,
                                                       const Tri* __restrict__ tris, uint32_t n,
                                                       const float* __restrict__ ro, const float* __restrict__ rd,
                                                       float* __restrict__ tOut, float* __restrict__ uvOut,
                                                       uint32_t* __restrict__ triOut, float* __restrict__ ngOut,
                                                       uint32_t* status)
{
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float3 o = mk3(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]);
    const float3 d = mk3(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]);
    Hit h = make_miss();
    closest_hit(h, nodes, tris, __ldg(root), o, d, status);
    tOut[i] = h.t;
    if (uvOut) { uvOut[2 * i] = h.u; uvOut[2 * i + 1] = h.v; }
    if (triOut) triOut[i] = h.tri;
    if (ngOut) { ngOut[3 * i] = h.ng.x; ngOut[3 * i + 1] = h.ng.y; ngOut[3 * i + 2] = h.ng.z; }
}

__global__ void __launch_bounds__(256) k_trace_any(const Node* __restrict__ nodes, const uint32_t* __restrict__ root,
                                                   const Tri* __restrict__ tris, uint32_t n,
                                                   const float* __restrict__ ro, const float* __restrict__ rd,
                                                   const float* __restrict__ tmax, uint8_t* __restrict__ hitOut)
{
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float3 o = mk3(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]);
    const float3 d = mk3(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]);
    const float tm = tmax[i];
    hitOut[i] = any_hit(nodes, tris, __ldg(root), o, d, tm) < tm ? 1 : 0;
}

cudaError_t launch_trace_closest(const Node* nodes, const uint32_t* root, const Tri* tris, uint32_t n, const float* ro,
                                 const float* rd, float* t, float* uv, uint32_t* tri, float* ng, uint32_t* status,
                                 cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_trace_closest<<<(n + 255) / 256, 256, 0, s>>>(nodes, root, tris, n, ro, rd, t, uv, tri, ng, status);
    return cudaGetLastError();
}

cudaError_t launch_trace_any(const Node* nodes, const uint32_t* root, const Tri* tris, uint32_t n, const float* ro,
                             const float* rd, const float* tmax, uint8_t* hit, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_trace_any<<<(n + 255) / 256, 256, 0, s>>>(nodes, root, tris, n, ro, rd, tmax, hit);
    return cudaGetLastError();
}

}  // namespace pz
