// palzilla_b200.hpp -- C++ facade over the C ABI (palzilla_b200.h) with the reference's
// host classes, names and argument meaning, for C++ callers of the caustics path:
//   OnesweepSort   tinyhiponesweep::OnesweepSort (tinyhiponesweep.h:562-668)
//   BVHGPUBuilder  minimum_lbvh::BVHGPUBuilder   (minimum_lbvh.h:741-900)
//   RayGenerator   RayGenerator                  (camera.h:4-41)
//   PKRenderer     PKRenderer subset             (pk.h:1228-1702): setup / loadFrame (scene
//                  from arrays instead of an Alembic archive) / allocate / step / clear /
//                  resolve, with the reference's public tunables.
// Like the reference's classes, these own their device buffers (RAII over cudaMalloc);
// every kernel runs in libpalzilla_b200.so.  Errors throw palzilla_b200::Error with the
// library's message.  Header only; link with -lpalzilla_b200 -lcudart.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "palzilla_b200.h"

namespace palzilla_b200 {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char* where)
{
    if (rc != PZ_OK) throw Error(rc, std::string(where) + ": " + pz_last_error());
}
inline void check_cuda(cudaError_t e, const char* where)
{
    if (e != cudaSuccess) throw Error(PZ_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Device buffer of T (TypedBuffer<T> with TYPED_BUFFER_DEVICE, typedbuffer.h).
template <class T> class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { allocate(n); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : m_p(o.m_p), m_n(o.m_n) { o.m_p = nullptr; o.m_n = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
    {
        if (this != &o) {
            release();
            m_p = o.m_p;
            m_n = o.m_n;
            o.m_p = nullptr;
            o.m_n = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void allocate(size_t n)
    {
        if (n == m_n && m_p) return;
        release();
        if (n) check_cuda(cudaMalloc(reinterpret_cast<void**>(&m_p), n * sizeof(T)), "cudaMalloc");
        m_n = n;
    }
    void release()
    {
        if (m_p) cudaFree(m_p);
        m_p = nullptr;
        m_n = 0;
    }
    void upload(const std::vector<T>& v, cudaStream_t s = 0)
    {
        allocate(v.size());
        if (!v.empty()) check_cuda(cudaMemcpyAsync(m_p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    }
    void download(std::vector<T>& v, cudaStream_t s = 0) const
    {
        v.resize(m_n);
        if (m_n) check_cuda(cudaMemcpyAsync(v.data(), m_p, m_n * sizeof(T), cudaMemcpyDeviceToHost, s), "download");
        check_cuda(cudaStreamSynchronize(s), "download");
    }
    T* data() const { return m_p; }
    size_t size() const { return m_n; }
    size_t bytes() const { return m_n * sizeof(T); }

private:
    T* m_p = nullptr;
    size_t m_n = 0;
};

// tinyhiponesweep::KeyValueSoA32 / KeyValueSoA64 (tinyhiponesweep.h:562-570)
struct KeyValueSoA32 { uint32_t* key; uint32_t* value; };
struct KeyValueSoA64 { uint64_t* key; uint32_t* value; };

class OnesweepSort {
public:
    explicit OnesweepSort(int device = 0) { check_cuda(cudaSetDevice(device), "OnesweepSort"); }
    // Stable sort of n keys on bits [startBit, endBit); the result ends in `elements`.
    void sort(KeyValueSoA64 elements, KeyValueSoA64 tmp, uint32_t n, int startBit, int endBit, cudaStream_t stream)
    {
        run(elements.key, elements.value, tmp.key, tmp.value, n, 8, startBit, endBit, stream);
    }
    void sort(KeyValueSoA32 elements, KeyValueSoA32 tmp, uint32_t n, int startBit, int endBit, cudaStream_t stream)
    {
        run(elements.key, elements.value, tmp.key, tmp.value, n, 4, startBit, endBit, stream);
    }
    uint32_t status(cudaStream_t stream = 0) const
    {
        uint32_t st = 0;
        if (m_scratch.data()) check(pz_scratch_status(m_scratch.data(), &st, (pz_stream_t)stream), "OnesweepSort::status");
        return st;
    }

private:
    void run(void* k, uint32_t* v, void* tk, uint32_t* tv, uint32_t n, int kb, int sb, int eb, cudaStream_t s)
    {
        const size_t need = pz_onesweep_scratch_bytes(n);
        if (m_scratch.bytes() < need) m_scratch.allocate(need);
        check(pz_onesweep_sort(k, v, tk, tv, n, kb, sb, eb, m_scratch.data(), m_scratch.bytes(), (pz_stream_t)s),
              "OnesweepSort::sort");
    }
    DeviceBuffer<uint8_t> m_scratch;
};

class BVHGPUBuilder {
public:
    // (kernelPath, includeDir) of the reference are not needed: the kernels are compiled in.
    BVHGPUBuilder() { m_root.allocate(1); }
    void build(const pz_triangle* trianglesDevice, int n, uint32_t buildOption, OnesweepSort& /*sorter*/,
               cudaStream_t stream)
    {
        m_nTriangles = n;
        m_internalsBuf.allocate(n > 1 ? (size_t)n - 1 : 1);
        const size_t need = pz_bvh_scratch_bytes(n);
        if (m_scratch.bytes() < need) m_scratch.allocate(need);
        check(pz_bvh_build(trianglesDevice, n, buildOption, m_internalsBuf.data(), m_root.data(), m_scratch.data(),
                           m_scratch.bytes(), (pz_stream_t)stream),
              "BVHGPUBuilder::build");
        m_internals = m_internalsBuf.data();
        m_rootNode = m_root.data();
    }
    pz_internal_node* m_internals = nullptr;  // n - 1 nodes
    uint32_t* m_rootNode = nullptr;           // device NodeIndex
    int m_nTriangles = 0;

private:
    DeviceBuffer<pz_internal_node> m_internalsBuf;
    DeviceBuffer<uint32_t> m_root;
    DeviceBuffer<uint8_t> m_scratch;
};

// camera.h:4-41
struct RayGenerator {
    pz_ray_generator g{};
    void lookat(pz_float3 eye, pz_float3 center, pz_float3 up, float fovy, int width, int height)
    {
        pz_ray_generator_lookat(&g, eye, center, up, fovy, width, height);
    }
};

// No reference counterpart (the reference has a point light).  Sample `iteration` of a
// downward-facing square light of extent (size_x, size_z) centred on `center`: the R2
// sequence (Roberts 2018: x_i = frac(1/2 + i / g), y_i = frac(1/2 + i / g^2), g the
// plastic number), in double, rounded to float.  Iteration 0 is the centre; a light of
// size zero is its centre.
inline pz_float3 light_point(pz_float3 center, float size_x, float size_z, int iteration)
{
    if (size_x == 0.0f && size_z == 0.0f) return center;
    const double g = 1.32471795724474602596;
    const double u = std::fmod(0.5 + iteration / g, 1.0), v = std::fmod(0.5 + iteration / (g * g), 1.0);
    return pz_float3{(float)((double)center.x + (u - 0.5) * (double)size_x), center.y,
                     (float)((double)center.z + (v - 0.5) * (double)size_z)};
}

// The reference's event descriptor (pk.h:122-162): bit k set = transmission at vertex k.
inline uint32_t event_descriptor(const std::string& events)
{
    uint32_t e = 0;
    for (size_t k = 0; k < events.size(); k++)
        if (events[k] == 'T') e |= 1u << k;
    return e | ((uint32_t)events.size() << 24);
}

class PKRenderer {
public:
    // tunables, as the reference's members (pk.h:1683-1701)
    pz_float3 m_p_light = {0.0f, 3.0f, 0.0f};
    float m_lightSize[2] = {0.0f, 0.0f};  // area light extent along x and z (0: point light)
    float m_lightIntencity = 16.0f;
    float m_minThroughput = 0.05f;
    float m_radianceClamp = 12.0f;
    pz_lens_params m_lensParams = {0.6f, 0.05f, 0.0f};
    float m_cauchyA = 1.5f, m_cauchyB = 4200.0f;  // CauchyDispersion(1.5, 4200), lambda in nm
    pz_float3 m_albedo = {0.75f, 0.75f, 0.75f};
    RayGenerator m_camera;
    int m_photonsPerTriangle = 256;              // PHOTON_BLOCK_SIZE (pk.h:32)
    uint32_t m_maxSpecularPaths = 1u << 25;      // MAX_SPECULAR_PATH_COUNT
    int m_iteration = 0;

    void setup(int device)
    {
        check_cuda(cudaSetDevice(device), "PKRenderer::setup");
        m_onesweep = OnesweepSort(device);
    }
    // Floor texture (the reference's Texture8RGBX, pk.h:1075-1098, loaded from an image file at
    // setup): RGBX texels, row-major, width x height, sampled at a diffuse hit's (x, z).  An
    // empty vector removes it (the diffuse hits then take m_albedo).
    void setFloorTexture(const std::vector<uint8_t>& rgbx, int width, int height)
    {
        if (rgbx.empty()) {
            m_floorTexture.release();
            return;
        }
        if (width <= 0 || height <= 0 || rgbx.size() != (size_t)width * height * 4)
            throw Error(PZ_ERR_INVALID_ARGUMENT, "setFloorTexture: size mismatch");
        m_floorTexture.upload(rgbx);
        m_floorTextureSize[0] = width;
        m_floorTextureSize[1] = height;
    }
    // Scene from arrays (the reference reads an Alembic frame, pk.h:1246-1366).
    void loadFrame(const std::vector<pz_triangle>& triangles, const std::vector<pz_triangle_attrib>& attribs)
    {
        if (triangles.size() != attribs.size()) throw Error(PZ_ERR_INVALID_ARGUMENT, "loadFrame: size mismatch");
        m_trianglesDevice.upload(triangles);
        m_triangleAttribsDevice.upload(attribs);
        m_gpuBuilder.build(m_trianglesDevice.data(), (int)triangles.size(), 0, m_onesweep, 0);
    }
    void allocate(int imageWidth, int imageHeight)
    {
        m_imageWidth = imageWidth;
        m_imageHeight = imageHeight;
        const size_t n = (size_t)imageWidth * imageHeight;
        if (m_pixels.size() != n) {
            m_pathCache.allocate(pz_path_cache_bytes(kPathCacheCapacity));
            m_specularPathCounter.allocate(1);
            m_specularPaths.allocate(m_maxSpecularPaths);
            m_specularPathsTmp.allocate(m_maxSpecularPaths);
            m_indexedSpecularPaths.allocate(m_maxSpecularPaths);
            m_indexedSpecularPathsTmp.allocate(m_maxSpecularPaths);
            m_pixels.allocate(n);
            m_accumulators.allocate(4 * n);
            m_firstDiffuses.allocate(n);
            m_status.allocate(1);
            check_cuda(cudaMemset(m_accumulators.data(), 0, m_accumulators.bytes()), "allocate");
        }
    }
    // One iteration (pk.h:1393-1627): eye pass, photon pass into the PathCache, then for
    // every event string: lookup / flatten, tuple-coherence sort, reorder, plain solve.
    void step(bool useOptionalPath = true)
    {
        cudaStream_t s = 0;
        const int n = m_gpuBuilder.m_nTriangles;
        m_lightPoint = light_point(m_p_light, m_lightSize[0], m_lightSize[1], m_iteration);
        const pz_texture_rgbx floor = {m_floorTexture.data(), (uint32_t)m_floorTextureSize[0],
                                       (uint32_t)m_floorTextureSize[1]};
        check(pz_solve_primary(m_accumulators.data(), m_firstDiffuses.data(), m_imageWidth, m_imageHeight, &m_camera.g,
                               &m_lensParams, m_gpuBuilder.m_internals, m_gpuBuilder.m_rootNode,
                               m_trianglesDevice.data(), m_triangleAttribsDevice.data(), m_lightPoint, m_lightIntencity,
                               m_radianceClamp, m_cauchyA, m_cauchyB, m_albedo, m_floorTexture.data() ? &floor : nullptr,
                               m_iteration, m_status.data(), (pz_stream_t)s),
              "solvePrimary");
        check(pz_path_cache_clear(m_pathCache.data(), kPathCacheCapacity, (pz_stream_t)s), "PathCache::clear");
        // eta at the two ends of the visible band, 380 and 780 nm (pk.h:1448-1449)
        const float etaMin = m_cauchyA + m_cauchyB / (380.0f * 380.0f);
        const float etaMax = m_cauchyA + m_cauchyB / (780.0f * 780.0f);
        check(pz_photon_trace(m_gpuBuilder.m_internals, m_gpuBuilder.m_rootNode, m_trianglesDevice.data(),
                              m_triangleAttribsDevice.data(), n, m_photonsPerTriangle, m_lightPoint, etaMin, etaMax,
                              m_iteration, m_minThroughput, m_pathCache.data(), kPathCacheCapacity, kCellStep, nullptr,
                              (pz_stream_t)s),
              "photonTrace");
        const char* always[] = {"T", "R", "TT", "TTTT"};
        const char* optional[] = {"TRT", "TTT"};
        for (const char* e : always) solveSpecular(e);
        if (useOptionalPath)
            for (const char* e : optional) solveSpecular(e);
        m_iteration++;
    }
    void clear()
    {
        check_cuda(cudaMemsetAsync(m_accumulators.data(), 0, m_accumulators.bytes(), 0), "clear");
        m_iteration = 0;
    }
    void resolve(std::vector<uint32_t>* imageOut)
    {
        check(pz_resolve(m_pixels.data(), m_accumulators.data(), m_imageWidth * m_imageHeight, 0), "pack");
        m_pixels.download(*imageOut);
    }
    const DeviceBuffer<float>& accumulators() const { return m_accumulators; }
    uint64_t solvedPaths() const { return m_solved; }

private:
    static constexpr uint32_t kPathCacheCapacity = 1u << 22;
    static constexpr float kCellStep = 0.01f;
    pz_float3 m_lightPoint = {0.0f, 0.0f, 0.0f};  // the light's sample for the current step

    void solveSpecular(const char* events)
    {
        cudaStream_t s = 0;
        const uint32_t ev = event_descriptor(events);
        check_cuda(cudaMemsetAsync(m_specularPathCounter.data(), 0, 4, s), "counter");
        check(pz_lookup_flatten(ev, m_specularPaths.data(), m_indexedSpecularPaths.data(), m_specularPathCounter.data(),
                                m_maxSpecularPaths, m_firstDiffuses.data(), m_imageWidth * m_imageHeight,
                                m_pathCache.data(), kPathCacheCapacity, kCellStep, (pz_stream_t)s),
              "lookupFlatten");
        uint32_t nPaths = 0;  // the reference reads the count back here (pk.h:1504)
        check_cuda(cudaMemcpyAsync(&nPaths, m_specularPathCounter.data(), 4, cudaMemcpyDeviceToHost, s), "count");
        check_cuda(cudaStreamSynchronize(s), "count");
        if (nPaths > m_maxSpecularPaths) nPaths = m_maxSpecularPaths;
        if (nPaths == 0) return;
        m_onesweep.sort(KeyValueSoA64{m_indexedSpecularPaths.data(), nullptr},
                        KeyValueSoA64{m_indexedSpecularPathsTmp.data(), nullptr}, nPaths, 0, 32, s);
        check(pz_reorder_specular_paths(m_indexedSpecularPaths.data(), m_specularPathsTmp.data(),
                                        m_specularPaths.data(), nPaths, (pz_stream_t)s),
              "reorderSpecularPath");
        std::swap(m_specularPaths, m_specularPathsTmp);
        pz_solve_desc d{};
        d.K = (int)(ev >> 24);
        d.events = ev;
        d.paths = m_specularPaths.data();
        d.n_paths = nPaths;
        d.first_diffuse = m_firstDiffuses.data();
        d.internals = m_gpuBuilder.m_internals;
        d.root = m_gpuBuilder.m_rootNode;
        d.triangles = m_trianglesDevice.data();
        d.attribs = m_triangleAttribsDevice.data();
        d.cache = m_pathCache.data();
        d.cache_capacity = kPathCacheCapacity;
        d.cell_step = kCellStep;
        d.p_light = m_lightPoint;
        d.light_intensity = m_lightIntencity;
        d.radiance_clamp = m_radianceClamp;
        d.cauchy_a = m_cauchyA;
        d.cauchy_b = m_cauchyB;
        d.accum = m_accumulators.data();
        d.n_bins = 1;
        d.max_iterations = 32;
        d.cost_tolerance = 1.0e-10f;
        d.early_term_warmup = 1;
        check(pz_solve_specular_plain(&d, (pz_stream_t)s), "solveSpecularPath");
        m_solved += nPaths;
    }

    OnesweepSort m_onesweep;
    BVHGPUBuilder m_gpuBuilder;
    DeviceBuffer<uint8_t> m_floorTexture;
    int m_floorTextureSize[2] = {0, 0};
    DeviceBuffer<pz_triangle> m_trianglesDevice;
    DeviceBuffer<pz_triangle_attrib> m_triangleAttribsDevice;
    DeviceBuffer<uint8_t> m_pathCache;
    DeviceBuffer<pz_first_diffuse> m_firstDiffuses;
    DeviceBuffer<pz_specular_path> m_specularPaths, m_specularPathsTmp;
    DeviceBuffer<uint64_t> m_indexedSpecularPaths, m_indexedSpecularPathsTmp;
    DeviceBuffer<uint32_t> m_specularPathCounter, m_pixels, m_status;
    DeviceBuffer<float> m_accumulators;  // float4 per pixel
    int m_imageWidth = 0, m_imageHeight = 0;
    uint64_t m_solved = 0;
};

}  // namespace palzilla_b200
