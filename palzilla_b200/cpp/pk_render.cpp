// pk_render -- renders a scene with the C++ facade (PKRenderer over the C ABI), the way a
// C++ host of the reference drives its renderer: setup, loadFrame, allocate, clear,
// iterations x step, resolve.
//
//   pk_render scene.bin out.bin
//
// scene.bin (little endian): int32 n, width, height, iterations; float eye[3], center[3],
// up[3], fovy, p_light[3], light_size[2] (area light extent along x and z; 0 0 = point
// light), light_intensity, radiance_clamp, min_throughput, cauchy_a, cauchy_b;
// pz_triangle[n]; pz_triangle_attrib[n].
// out.bin: float accum[width * height * 4]; uint32 pixels[width * height]; uint64 paths.
#include <cstdio>
#include <vector>

#include "palzilla_b200.hpp"

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s scene.bin out.bin\n", argv[0]);
        return 2;
    }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[4];
    float cam[10], light[5], params[5];
    bool ok = std::fread(hdr, sizeof(hdr), 1, f) == 1 && std::fread(cam, sizeof(cam), 1, f) == 1 &&
              std::fread(light, sizeof(light), 1, f) == 1 && std::fread(params, sizeof(params), 1, f) == 1;
    const int n = hdr[0], width = hdr[1], height = hdr[2], iterations = hdr[3];
    std::vector<pz_triangle> tris(n);
    std::vector<pz_triangle_attrib> attribs(n);
    ok = ok && std::fread(tris.data(), sizeof(pz_triangle), n, f) == (size_t)n &&
         std::fread(attribs.data(), sizeof(pz_triangle_attrib), n, f) == (size_t)n;
    std::fclose(f);
    if (!ok) {
        std::fprintf(stderr, "bad scene file\n");
        return 2;
    }
    try {
        palzilla_b200::PKRenderer r;
        r.setup(0);
        r.m_camera.lookat({cam[0], cam[1], cam[2]}, {cam[3], cam[4], cam[5]}, {cam[6], cam[7], cam[8]}, cam[9], width,
                          height);
        r.m_p_light = {light[0], light[1], light[2]};
        r.m_lightSize[0] = light[3];
        r.m_lightSize[1] = light[4];
        r.m_lightIntencity = params[0];
        r.m_radianceClamp = params[1];
        r.m_minThroughput = params[2];
        r.m_cauchyA = params[3];
        r.m_cauchyB = params[4];
        r.loadFrame(tris, attribs);
        r.allocate(width, height);
        r.clear();
        for (int i = 0; i < iterations; i++) r.step(true);
        std::vector<uint32_t> image;
        r.resolve(&image);
        std::vector<float> accum;
        r.accumulators().download(accum);
        const uint64_t solved = r.solvedPaths();
        std::FILE* o = std::fopen(argv[2], "wb");
        if (!o) return 2;
        std::fwrite(accum.data(), sizeof(float), accum.size(), o);
        std::fwrite(image.data(), sizeof(uint32_t), image.size(), o);
        std::fwrite(&solved, sizeof(solved), 1, o);
        std::fclose(o);
        std::printf("rendered %d x %d, %d iterations, %llu specular paths\n", width, height, iterations,
                    (unsigned long long)solved);
    } catch (const palzilla_b200::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
        return 1;
    }
    return 0;
}
