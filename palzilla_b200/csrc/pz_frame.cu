// pz_frame.cu -- eye pass and (pixel, tuple) work-list construction.
//
// k_primary:  solvePrimary (main_gpu.cu:213-371): one jittered camera ray per pixel,
//             optional thick lens (pk.h:1042-1073), up to 32 specular bounces with
//             Fresnel-sampled events to the first diffuse hit, point-light direct light
//             with a shadow ray; writes FirstDiffuse {p, n, R, lambda} and adds to the
//             float4 accumulator.  The albedo of the diffuse hit is the floor texture sampled
//             at its (x, z) (Texture8RGBX, pk.h:1075-1098; main_gpu.cu:343) or a constant.
//             Bit-exact with the CPU oracle except lambda, which goes through expf/logf,
//             and the texture's gamma decode, which goes through powf.
// k_lookup:   lookupFlatten (main_gpu.cu:373-416): per pixel, the PathCache slots of the
//             pixel's cell with the requested event string, appended to the work list as
//             SpecularPath {pixel, slot} and IndexedSpecularPath {path hash, index}.
// k_reorder:  reorderSpecularPath (main_gpu.cu:515-525).
// This unit is compiled with -fmad=false.
#include "pz_cache.cuh"
#include "pz_frame.cuh"
#include "pz_optics.cuh"
#include "pz_trace.cuh"

namespace pz {

// sphIntersect, pk.h:52-65 (nearest root)
PZ_D float sph_intersect_near(float3 ro, float3 rd, float3 ce, float ra)
{
    float len2rd = dot(rd, rd);
    float3 oc = ro - ce;
    float b = dot(oc, rd) / len2rd;
    float c = dot(oc, oc) - ra * ra;
    float h = b * b - c / len2rd;
    if (h < 0.0f) return -1.0f;
    h = sqrtf(h);
    return -b - h;
}

__global__ void __launch_bounds__(256) k_primary(float4* __restrict__ accum, FirstDiffuse* __restrict__ fds, int W,
                                                 int H, RayGen g, Lens lens, const Node* __restrict__ nodes,
                                                 const uint32_t* __restrict__ rootPtr, const Tri* __restrict__ tris,
                                                 const Attrib* __restrict__ attribs, float3 p_light,
                                                 float lightIntensity, float radianceClamp, float cauchyA,
                                                 float cauchyB, float3 albedo, Tex tex, int iteration,
                                                 uint32_t* status)
{
    const int xi = blockIdx.x * 16 + (threadIdx.x & 15);
    const int yi = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (xi >= W || yi >= H) return;
    const int pixel = xi + yi * W;
    const uint32_t root = __ldg(rootPtr);

    float2 jit;
    sobol2d(&jit.x, &jit.y, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, 0u);
    // RayGenerator::shoot, camera.h:24-31
    const float3 forward = normalize(cross(g.up, g.right));
    const float u = ((float)xi + jit.x) / (float)W, v = ((float)yi + jit.y) / (float)H;
    const float3 to = g.origin + forward + lerp3(-g.right, g.right, u) + lerp3(g.up, -g.up, v);
    float3 ro = g.origin, rd = to - g.origin;

    float2 lr;
    sobol2d(&lr.x, &lr.y, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, 1u);
    const float lambda = cmf_y_sample(lr.x);
    const float p_lambda = cmf_y_pdf(lambda);
    const float eta = cauchyA + cauchyB / (lambda * lambda);

    if (lens.R > 0.0f) {  // solveLens, pk.h:1042-1073
        const float3 lo = g.origin + forward * lens.distance;
        const float3 c1 = lo + forward * (lens.R - lens.thickness * 0.5f);
        const float3 c2 = lo - forward * (lens.R - lens.thickness * 0.5f);
        const float t1 = sph_intersect_near(ro, rd, c1, lens.R);
        if (!(t1 < 0.0f)) {
            const float3 hit1 = ro + rd * t1;
            float3 wo = rd;
            refraction_norm_free(&wo, -rd, hit1 - c1, eta);
            rd = wo;
            ro = hit1;
            const float t2 = sph_intersect_near(ro, rd, c2, lens.R);
            const float3 hit2 = ro + rd * t2;
            if (refraction_norm_free(&wo, -rd, hit2 - c2, eta)) {
                rd = wo;
                ro = hit2;
            }
        }
    }

    bool hasDiffuse = false;
    Hit last = make_miss();
    uint32_t dim = 2;
    for (int d = 0; d < 32; d++) {
        Hit hit = make_miss();
        closest_hit(hit, nodes, tris, root, ro, rd, status);
        if (hit.t == kFltMax) {
            last = hit;
            break;
        }
        const Attrib* A = attribs + hit.tri;
        const int32_t m = __ldg(&A->material);
        float2 rnd;
        sobol2d(&rnd.x, &rnd.y, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, dim++);
        if (m == kDiffuse) {
            hasDiffuse = true;
            last = hit;
            break;
        }
        const float3 p_hit = ro + rd * hit.t;
        const float* sn = reinterpret_cast<const float*>(A) + 1;
        const float3 n0 = mk3(__ldg(sn + 0), __ldg(sn + 1), __ldg(sn + 2));
        const float3 n1 = mk3(__ldg(sn + 3), __ldg(sn + 4), __ldg(sn + 5));
        const float3 n2 = mk3(__ldg(sn + 6), __ldg(sn + 7), __ldg(sn + 8));
        const float3 ns = n0 + (n1 - n0) * hit.u + (n2 - n0) * hit.v;
        const float3 wi = -rd;
        const bool isT = (m == kDielectric) && !(rnd.x < fresnel_exact_norm_free(wi, ns, eta));
        float sign = 1.0f;
        float3 wo;
        if (!isT) {
            wo = reflection(wi, ns);
        } else {
            if (!refraction_norm_free(&wo, wi, ns, eta)) break;
            sign = -1.0f;
        }
        if (0.0f < dot(hit.ng, wi) * dot(hit.ng, wo) * sign) {
            const float3 od = normalize(hit.ng * dot(hit.ng, wo));
            ro = p_hit + od * ray_offset_scale(p_hit);
            rd = wo;
            continue;
        }
        break;
    }
    FirstDiffuse* fd = fds + pixel;
    float4 acc = accum[pixel];
    if (!hasDiffuse) {
        acc.w += 1.0f;
        accum[pixel] = acc;
        fd->R = mk3(0.f, 0.f, 0.f);
        return;
    }
    const float3 p = ro + rd * last.t;
    float3 n = normalize(last.ng);
    if (0.0f < dot(n, rd)) n = -n;
    const float3 toL = p_light - p;
    const float d2 = dot(toL, toL);
    const float3 R = tex.texels ? sample_point(tex, p.x, p.z) : albedo;
    float3 L = mk3(0.f, 0.f, 0.f);
    if (!occluded(nodes, tris, root, p, n, p_light, mk3(0.f, 0.f, 0.f))) {
        float contrib = lightIntensity / d2 * fmaxf(dot(normalize(toL), n), 0.0f);
        contrib = fminf(contrib, radianceClamp);
        L = L + (R / kPi) * lambda_to_srgb(lambda) * contrib / p_lambda;
    }
    fd->p = p;
    fd->ng = n;
    fd->R = R;
    fd->lambda = lambda;
    acc.x += L.x;
    acc.y += L.y;
    acc.z += L.z;
    acc.w += 1.0f;
    accum[pixel] = acc;
}

__global__ void __launch_bounds__(256) k_lookup(uint32_t ev, SpecularPath* __restrict__ paths,
                                                unsigned long long* __restrict__ indexed, uint32_t* counter,
                                                uint32_t capacity, const FirstDiffuse* __restrict__ fds, int nPixels,
                                                CacheView cache)
{
    const int pixel = blockIdx.x * 256 + threadIdx.x;
    if (pixel >= nPixels) return;
    const FirstDiffuse& fd = fds[pixel];
    const float3 R = fd.R;
    if (R.x == 0.0f && R.y == 0.0f && R.z == 0.0f) return;
    const uint32_t hP = spacial_hash(fd.p, cache.step);
    const uint32_t mask = cache.capacity - 1u;
    const uint32_t home = hP & mask;
    uint32_t count = 0, off = 0;
    for (; off < kMaxProbe; off++) {
        const uint32_t i = (home + off) & mask;
        if (cache.hash[i] == 0u) break;
        if (cache.cell[i] != hP || cache.event[i] != ev) continue;
        count++;
    }
    if (off == kMaxProbe) raise_error(&cache.h->status, kErrCapacity);
    if (count == 0) return;
    const uint32_t head = atomicAdd(counter, count);
    if (head + count > capacity) {  // main_gpu.cu:399-403 drops the pixel; the status says so
        raise_error(&cache.h->status, kErrCapacity);
        return;
    }
    uint32_t k = 0;
    for (off = 0; off < kMaxProbe && k < count; off++) {
        const uint32_t i = (home + off) & mask;
        if (cache.hash[i] == 0u) break;
        if (cache.cell[i] != hP || cache.event[i] != ev) continue;
        const uint32_t dst = head + k++;
        paths[dst] = SpecularPath{pixel, (int)i};
        indexed[dst] = (unsigned long long)cache.hash[i] | ((unsigned long long)dst << 32);
    }
}

__global__ void k_reorder(const unsigned long long* __restrict__ indexed, SpecularPath* __restrict__ dst,
                          const SpecularPath* __restrict__ src, uint32_t n)
{
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    dst[i] = src[(uint32_t)(indexed[i] >> 32)];
}

cudaError_t launch_primary(float4* accum, FirstDiffuse* fds, int W, int H, const RayGen& g, const Lens& lens,
                           const Node* nodes, const uint32_t* root, const Tri* tris, const Attrib* attribs,
                           float3 p_light, float lightIntensity, float radianceClamp, float cauchyA, float cauchyB,
                           float3 albedo, const Tex& tex, int iteration, uint32_t* status, cudaStream_t s)
{
    dim3 grid((W + 15) / 16, (H + 15) / 16);
    k_primary<<<grid, 256, 0, s>>>(accum, fds, W, H, g, lens, nodes, root, tris, attribs, p_light, lightIntensity,
                                   radianceClamp, cauchyA, cauchyB, albedo, tex, iteration, status);
    return cudaGetLastError();
}

cudaError_t launch_lookup(uint32_t ev, SpecularPath* paths, unsigned long long* indexed, uint32_t* counter,
                          uint32_t capacity, const FirstDiffuse* fds, int nPixels, const CacheView& cache,
                          cudaStream_t s)
{
    if (nPixels <= 0) return cudaSuccess;
    k_lookup<<<(nPixels + 255) / 256, 256, 0, s>>>(ev, paths, indexed, counter, capacity, fds, nPixels, cache);
    return cudaGetLastError();
}

cudaError_t launch_reorder(const unsigned long long* indexed, SpecularPath* dst, const SpecularPath* src, uint32_t n,
                           cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_reorder<<<(n + 255) / 256, 256, 0, s>>>(indexed, dst, src, n);
    return cudaGetLastError();
}

}  // namespace pz
