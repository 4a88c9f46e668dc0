// palzilla_b200_scene.hpp -- host-side scene and image I/O for hosts of the caustics path.
//
// The reference reads each frame's triangles from an Alembic archive (PKRenderer::loadFrame,
// pk.h:1246-1362): triangles only, per-face-vertex shading normals, and a "material" string
// per mesh, "mirror" or "dielectric" (anything else is diffuse, pk.h:1306-1318).  Alembic is
// not available here; this header reads the same triangle soup from Wavefront OBJ, with the
// material taken from the name given to `usemtl`:
//   loadObj        OBJ -> pz_triangle / pz_triangle_attrib arrays (the reference's layouts);
//   writePng       RGBA8 image -> PNG with stored (uncompressed) deflate blocks, as the
//                  reference's final render writes its frames (main_gpu.cpp:72-84);
//   writePfm       linear RGB floats -> PFM;
//   readPpm        binary PPM (P6) -> RGBX texels, for PKRenderer::setFloorTexture.
// Header only, no dependencies beyond the C++ standard library.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "palzilla_b200.h"

namespace palzilla_b200 {

// Material of a `usemtl` name: the reference's two tags (pk.h:1306-1318); every other name
// is diffuse.  Hosts may map their own names.
struct ObjOptions {
    std::map<std::string, int32_t> materials = {{"mirror", 1}, {"dielectric", 2}};
};

// Reads a Wavefront OBJ triangle soup.  `v x y z`, `vn x y z` and `f` records are read
// (1-based or negative indices; v, v/vt, v//vn and v/vt/vn corners); a polygon with more
// than three corners becomes the fan (0, i, i + 1).  A corner with a normal index takes that
// normal as its shading normal; a triangle whose corners have none takes its unit geometric
// normal, normalize(cross(v1 - v0, v2 - v0)), at all three.  Triangles are appended in file
// order.  Throws std::runtime_error on a malformed file.
inline void loadObj(const std::string& path, std::vector<pz_triangle>& tris, std::vector<pz_triangle_attrib>& attribs,
                    const ObjOptions& opts = ObjOptions())
{
    std::FILE* f = std::fopen(path.c_str(), "r");
    if (!f) throw std::runtime_error("loadObj: cannot open " + path);
    std::vector<pz_float3> pos, nrm;
    int32_t material = 0;
    char line[4096];
    int lineNo = 0;
    auto fail = [&](const char* what) {
        std::fclose(f);
        throw std::runtime_error("loadObj: " + path + ":" + std::to_string(lineNo) + ": " + what);
    };
    auto resolve = [](long idx, size_t n) -> long { return idx > 0 ? idx - 1 : (long)n + idx; };
    while (std::fgets(line, sizeof(line), f)) {
        lineNo++;
        char* s = line;
        while (*s == ' ' || *s == '\t') s++;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            pz_float3 p;
            char* e = s + 2;
            p.x = std::strtof(e, &e);
            p.y = std::strtof(e, &e);
            p.z = std::strtof(e, &e);
            pos.push_back(p);
        } else if (s[0] == 'v' && s[1] == 'n' && (s[2] == ' ' || s[2] == '\t')) {
            pz_float3 n;
            char* e = s + 3;
            n.x = std::strtof(e, &e);
            n.y = std::strtof(e, &e);
            n.z = std::strtof(e, &e);
            nrm.push_back(n);
        } else if (std::strncmp(s, "usemtl", 6) == 0 && (s[6] == ' ' || s[6] == '\t')) {
            std::string name(s + 7);
            while (!name.empty() && (name.back() == '\n' || name.back() == '\r' || name.back() == ' ' ||
                                     name.back() == '\t'))
                name.pop_back();
            size_t b = name.find_first_not_of(" \t");
            name = b == std::string::npos ? std::string() : name.substr(b);
            auto it = opts.materials.find(name);
            material = it == opts.materials.end() ? 0 : it->second;
        } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            std::vector<long> vi, ni;
            std::istringstream in(s + 2);
            std::string tok;
            while (in >> tok) {
                long v = 0, n = 0;
                const char* c = tok.c_str();
                char* e = nullptr;
                v = std::strtol(c, &e, 10);
                if (e == c) fail("bad face corner");
                if (*e == '/') {
                    c = e + 1;
                    if (*c != '/') std::strtol(c, &e, 10);  // texture index: not used
                    else e = const_cast<char*>(c);
                    if (*e == '/') {
                        c = e + 1;
                        n = std::strtol(c, &e, 10);
                        if (e == c) n = 0;
                    }
                }
                const long rv = resolve(v, pos.size());
                if (v == 0 || rv < 0 || rv >= (long)pos.size()) fail("vertex index out of range");
                long rn = -1;
                if (n != 0) {
                    rn = resolve(n, nrm.size());
                    if (rn < 0 || rn >= (long)nrm.size()) fail("normal index out of range");
                }
                vi.push_back(rv);
                ni.push_back(rn);
            }
            if (vi.size() < 3) fail("face with fewer than three corners");
            for (size_t k = 1; k + 1 < vi.size(); k++) {
                const size_t c3[3] = {0, k, k + 1};
                pz_triangle t;
                pz_triangle_attrib a;
                a.material = material;
                for (int j = 0; j < 3; j++) t.vs[j] = pos[vi[c3[j]]];
                bool all = true;
                for (int j = 0; j < 3; j++) all = all && ni[c3[j]] >= 0;
                if (all) {
                    for (int j = 0; j < 3; j++) a.shading_normals[j] = nrm[ni[c3[j]]];
                } else {
                    const pz_float3 e0 = {t.vs[1].x - t.vs[0].x, t.vs[1].y - t.vs[0].y, t.vs[1].z - t.vs[0].z};
                    const pz_float3 e1 = {t.vs[2].x - t.vs[0].x, t.vs[2].y - t.vs[0].y, t.vs[2].z - t.vs[0].z};
                    pz_float3 g = {e0.y * e1.z - e0.z * e1.y, e0.z * e1.x - e0.x * e1.z, e0.x * e1.y - e0.y * e1.x};
                    const float inv = 1.0f / std::sqrt(g.x * g.x + g.y * g.y + g.z * g.z);
                    g = {g.x * inv, g.y * inv, g.z * inv};
                    for (int j = 0; j < 3; j++) a.shading_normals[j] = g;
                }
                tris.push_back(t);
                attribs.push_back(a);
            }
        }
    }
    std::fclose(f);
}

namespace detail {
inline uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xFFFFFFFFu)
{
    for (size_t i = 0; i < n; i++) {
        c ^= p[i];
        for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
    }
    return c;
}
inline void put32(std::vector<uint8_t>& o, uint32_t v)
{
    o.push_back((uint8_t)(v >> 24));
    o.push_back((uint8_t)(v >> 16));
    o.push_back((uint8_t)(v >> 8));
    o.push_back((uint8_t)v);
}
inline void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data)
{
    put32(out, (uint32_t)data.size());
    std::vector<uint8_t> td(type, type + 4);
    td.insert(td.end(), data.begin(), data.end());
    out.insert(out.end(), td.begin(), td.end());
    put32(out, crc32(td.data(), td.size()) ^ 0xFFFFFFFFu);
}
}  // namespace detail

// RGBA8 pixels (byte order R, G, B, A in memory, i.e. 0xAABBGGRR words as pz_resolve writes
// them), rows top to bottom, as an 8-bit RGBA PNG whose zlib stream uses stored blocks.
inline void writePng(const std::string& path, const uint32_t* rgba, int width, int height)
{
    std::vector<uint8_t> raw;
    raw.reserve((size_t)height * (1 + 4 * (size_t)width));
    for (int y = 0; y < height; y++) {
        raw.push_back(0);  // filter: none
        const uint8_t* row = reinterpret_cast<const uint8_t*>(rgba + (size_t)y * width);
        raw.insert(raw.end(), row, row + 4 * (size_t)width);
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;  // Adler-32
    for (uint8_t c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    for (size_t off = 0; off < raw.size(); off += 65535) {  // stored blocks of at most 65535 bytes
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        z.push_back(off + len >= raw.size() ? 1 : 0);
        z.push_back((uint8_t)len);
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)~len);
        z.push_back((uint8_t)(~len >> 8));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
    }
    detail::put32(z, (b << 16) | a);
    std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::vector<uint8_t> ihdr;
    detail::put32(ihdr, (uint32_t)width);
    detail::put32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 6, 0, 0, 0});  // 8 bits, RGBA, deflate, filter 0, no interlace
    detail::chunk(out, "IHDR", ihdr);
    detail::chunk(out, "IDAT", z);
    detail::chunk(out, "IEND", {});
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(out.data(), 1, out.size(), f) != out.size()) {
        if (f) std::fclose(f);
        throw std::runtime_error("writePng: cannot write " + path);
    }
    std::fclose(f);
}

// Linear RGB, 3 floats per pixel, rows top to bottom, as a little-endian PFM (which stores
// rows bottom to top).
inline void writePfm(const std::string& path, const float* rgb, int width, int height)
{
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("writePfm: cannot write " + path);
    std::fprintf(f, "PF\n%d %d\n-1.0\n", width, height);
    for (int y = height - 1; y >= 0; y--) std::fwrite(rgb + (size_t)y * width * 3, sizeof(float), (size_t)width * 3, f);
    std::fclose(f);
}

// Binary PPM (P6, maxval 255) as RGBX texels (X = 255).
inline void readPpm(const std::string& path, std::vector<uint8_t>& rgbx, int& width, int& height)
{
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("readPpm: cannot open " + path);
    char magic[3] = {0, 0, 0};
    int maxval = 0;
    const bool ok = std::fscanf(f, "%2s %d %d %d", magic, &width, &height, &maxval) == 4 &&
                    std::strcmp(magic, "P6") == 0 && maxval == 255 && width > 0 && height > 0;
    if (!ok || std::fgetc(f) == EOF) {
        std::fclose(f);
        throw std::runtime_error("readPpm: " + path + " is not an 8-bit binary PPM");
    }
    std::vector<uint8_t> rgb((size_t)width * height * 3);
    const bool full = std::fread(rgb.data(), 1, rgb.size(), f) == rgb.size();
    std::fclose(f);
    if (!full) throw std::runtime_error("readPpm: " + path + " is truncated");
    rgbx.resize((size_t)width * height * 4);
    for (size_t i = 0; i < (size_t)width * height; i++) {
        rgbx[4 * i + 0] = rgb[3 * i + 0];
        rgbx[4 * i + 1] = rgb[3 * i + 1];
        rgbx[4 * i + 2] = rgb[3 * i + 2];
        rgbx[4 * i + 3] = 255;
    }
}

}  // namespace palzilla_b200
