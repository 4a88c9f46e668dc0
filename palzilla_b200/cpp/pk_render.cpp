// pk_render -- the C++ facade (PKRenderer over the C ABI) driven as a C++ host of the
// reference drives its renderer.  Three modes:
//
//   pk_render scene.bin out.bin
//     One image of a scene given as arrays: setup, loadFrame, allocate, clear, iterations x
//     step, resolve.  scene.bin (little endian): int32 n, width, height, iterations; float
//     eye[3], center[3], up[3], fovy, p_light[3], light_size[2] (area light extent along x
//     and z; 0 0 = point light), light_intensity, radiance_clamp, min_throughput, cauchy_a,
//     cauchy_b; pz_triangle[n]; pz_triangle_attrib[n].  out.bin: float accum[width * height
//     * 4]; uint32 pixels[width * height]; uint64 paths.
//
//   pk_render --obj PATTERN --frames N [options]
//     The reference's final render (main_gpu.cpp:60-85): for every frame, loadFrame (the
//     frame's OBJ: PATTERN with a printf integer conversion such as frames/%03d.obj, or one
//     file for every frame), clear, --spp steps (32) with the optional event strings on for
//     the frames in --optional A B, resolve, and the frame written as OUT/%03d.png
//     (uncompressed, as the reference writes it) and, with --pfm, the linear image as
//     OUT/%03d.pfm.  Options: --first F, --size W H (1920 1080), --eye x y z, --center x y z,
//     --up x y z, --fovy radians, --light x y z, --light-size sx sz, --intensity I,
//     --lens distance thickness R, --floor texture.ppm, --out DIR.
//
//   pk_render --parse-obj scene.obj out.bin
//     Loads an OBJ (palzilla_b200_scene.hpp) and writes int32 n, pz_triangle[n],
//     pz_triangle_attrib[n]; touches no GPU.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "palzilla_b200.hpp"
#include "palzilla_b200_scene.hpp"

using palzilla_b200::PKRenderer;

static int render_binary_scene(const char* in, const char* out)
{
    std::FILE* f = std::fopen(in, "rb");
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
    PKRenderer r;
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
    std::FILE* o = std::fopen(out, "wb");
    if (!o) return 2;
    std::fwrite(accum.data(), sizeof(float), accum.size(), o);
    std::fwrite(image.data(), sizeof(uint32_t), image.size(), o);
    std::fwrite(&solved, sizeof(solved), 1, o);
    std::fclose(o);
    std::printf("rendered %d x %d, %d iterations, %llu specular paths\n", width, height, iterations,
                (unsigned long long)solved);
    return 0;
}

static int parse_obj(const char* in, const char* out)
{
    std::vector<pz_triangle> tris;
    std::vector<pz_triangle_attrib> attribs;
    palzilla_b200::loadObj(in, tris, attribs);
    std::FILE* o = std::fopen(out, "wb");
    if (!o) return 2;
    const int32_t n = (int32_t)tris.size();
    std::fwrite(&n, sizeof(n), 1, o);
    std::fwrite(tris.data(), sizeof(pz_triangle), tris.size(), o);
    std::fwrite(attribs.data(), sizeof(pz_triangle_attrib), attribs.size(), o);
    std::fclose(o);
    std::printf("%d triangles\n", n);
    return 0;
}

static std::string frame_path(const std::string& pattern, int frame)
{
    if (pattern.find('%') == std::string::npos) return pattern;
    char buf[4096];
    std::snprintf(buf, sizeof(buf), pattern.c_str(), frame);
    return buf;
}

static int final_render(int argc, char** argv)
{
    std::string pattern, out = ".", floor;
    int frames = 1, first = 0, spp = 32, width = 1920, height = 1080, optA = 1, optB = 0;
    bool pfm = false;
    pz_float3 eye = {0.0f, 2.0f, 4.0f}, center = {0.0f, 0.5f, 0.0f}, up = {0.0f, 1.0f, 0.0f};
    float fovy = 0.7f;
    PKRenderer r;
    auto f3 = [&](int& i) {
        if (i + 3 >= argc) throw std::runtime_error(std::string("missing values for ") + argv[i]);
        pz_float3 v = {std::stof(argv[i + 1]), std::stof(argv[i + 2]), std::stof(argv[i + 3])};
        i += 3;
        return v;
    };
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
            return argv[++i];
        };
        if (a == "--obj") pattern = next();
        else if (a == "--frames") frames = std::stoi(next());
        else if (a == "--first") first = std::stoi(next());
        else if (a == "--spp") spp = std::stoi(next());
        else if (a == "--size") { width = std::stoi(next()); height = std::stoi(next()); }
        else if (a == "--eye") eye = f3(i);
        else if (a == "--center") center = f3(i);
        else if (a == "--up") up = f3(i);
        else if (a == "--fovy") fovy = std::stof(next());
        else if (a == "--light") r.m_p_light = f3(i);
        else if (a == "--light-size") { r.m_lightSize[0] = std::stof(next()); r.m_lightSize[1] = std::stof(next()); }
        else if (a == "--intensity") r.m_lightIntencity = std::stof(next());
        else if (a == "--lens") {
            const pz_float3 l = f3(i);
            r.m_lensParams = {l.x, l.y, l.z};
        } else if (a == "--floor") floor = next();
        else if (a == "--optional") { optA = std::stoi(next()); optB = std::stoi(next()); }
        else if (a == "--out") out = next();
        else if (a == "--pfm") pfm = true;
        else throw std::runtime_error("unknown option " + a);
    }
    if (pattern.empty() || frames < 1 || spp < 1 || width < 1 || height < 1)
        throw std::runtime_error("need --obj PATTERN, --frames >= 1, --spp >= 1 and a positive --size");
    r.setup(0);
    r.m_camera.lookat(eye, center, up, fovy, width, height);
    if (!floor.empty()) {
        std::vector<uint8_t> rgbx;
        int tw = 0, th = 0;
        palzilla_b200::readPpm(floor, rgbx, tw, th);
        r.setFloorTexture(rgbx, tw, th);
    }
    r.allocate(width, height);
    for (int fi = first; fi < first + frames; fi++) {
        std::vector<pz_triangle> tris;
        std::vector<pz_triangle_attrib> attribs;
        palzilla_b200::loadObj(frame_path(pattern, fi), tris, attribs);
        r.loadFrame(tris, attribs);
        r.clear();
        const bool useOptionalPath = optA <= fi && fi <= optB;
        for (int j = 0; j < spp; j++) r.step(useOptionalPath);
        std::vector<uint32_t> image;
        r.resolve(&image);
        char name[64];
        std::snprintf(name, sizeof(name), "/%03d.png", fi);
        palzilla_b200::writePng(out + name, image.data(), width, height);
        if (pfm) {
            std::vector<float> accum, rgb((size_t)width * height * 3);
            r.accumulators().download(accum);
            for (size_t p = 0; p < (size_t)width * height; p++)
                for (int c = 0; c < 3; c++) rgb[3 * p + c] = accum[4 * p + 3] > 0.0f ? accum[4 * p + c] / accum[4 * p + 3] : 0.0f;
            std::snprintf(name, sizeof(name), "/%03d.pfm", fi);
            palzilla_b200::writePfm(out + name, rgb.data(), width, height);
        }
        std::printf("frame %03d: %zu triangles, %d steps, %llu specular paths so far\n", fi, tris.size(), spp,
                    (unsigned long long)r.solvedPaths());
        std::fflush(stdout);
    }
    return 0;
}

int main(int argc, char** argv)
{
    try {
        if (argc == 4 && std::strcmp(argv[1], "--parse-obj") == 0) return parse_obj(argv[2], argv[3]);
        if (argc >= 2 && std::strcmp(argv[1], "--obj") == 0) return final_render(argc, argv);
        if (argc == 3) return render_binary_scene(argv[1], argv[2]);
        std::fprintf(stderr,
                     "usage: %s scene.bin out.bin\n"
                     "       %s --obj PATTERN --frames N [--spp 32] [--size W H] [--out DIR] [...]\n"
                     "       %s --parse-obj scene.obj out.bin\n",
                     argv[0], argv[0], argv[0]);
        return 2;
    } catch (const palzilla_b200::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
