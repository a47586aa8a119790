// Minimal PNG writer (8-bit RGB, filter 0, one zlib stream) for the CLI,
// standing in for the `image` crate's save_buffer (film.rs:63-67), and the
// 8-bit PNG reader the compare tool uses (image::open(..).to_rgb8()).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <zlib.h>

namespace ifx_cli {

static void put32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 24));
    v.push_back((uint8_t)(x >> 16));
    v.push_back((uint8_t)(x >> 8));
    v.push_back((uint8_t)x);
}

static void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
    put32(out, (uint32_t)data.size());
    size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, out.data() + start, (uInt)(out.size() - start));
    put32(out, (uint32_t)crc);
}

// Returns an empty string on success, else a message.
std::string write_png_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h) {
    std::vector<uint8_t> raw;
    raw.reserve((size_t)h * (1 + (size_t)w * 3));
    for (uint32_t y = 0; y < h; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgb + (size_t)y * w * 3, rgb + (size_t)(y + 1) * w * 3);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return "zlib compression failed";
    z.resize(zlen);
    std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
    std::vector<uint8_t> ihdr;
    put32(ihdr, w);
    put32(ihdr, h);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(2);  // colour type RGB
    ihdr.push_back(0);
    ihdr.push_back(0);
    ihdr.push_back(0);
    chunk(out, "IHDR", ihdr);
    chunk(out, "IDAT", z);
    chunk(out, "IEND", {});
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return "failed to write " + path;
    size_t wrote = fwrite(out.data(), 1, out.size(), f);
    if (fclose(f) != 0 || wrote != out.size()) return "failed to write " + path;
    return "";
}

static uint32_t get32(const uint8_t* p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}

static uint8_t paeth(int a, int b, int c) {
    const int p = a + b - c;
    const int pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return (uint8_t)a;
    return (uint8_t)(pb <= pc ? b : c);
}

// Reads an 8-bit, non-interlaced PNG (grey, grey + alpha, RGB, RGBA or
// palette) as packed RGB, dropping alpha: the conversion the `image` crate's
// to_rgb8 makes for these formats. Returns an empty string on success.
std::string read_png_rgb8(const std::string& path, uint32_t& w, uint32_t& h, std::vector<uint8_t>& rgb) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::vector<uint8_t> d;
    uint8_t buf[65536];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) d.insert(d.end(), buf, buf + k);
    fclose(f);
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
    if (d.size() < 8 || std::memcmp(d.data(), sig, 8) != 0) return path + ": not a PNG file";
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, plte;
    w = h = 0;
    for (size_t pos = 8; pos + 12 <= d.size();) {
        const uint32_t len = get32(&d[pos]);
        if (pos + 12 + (size_t)len > d.size()) return path + ": truncated chunk";
        const uint8_t* type = &d[pos + 4];
        const uint8_t* data = &d[pos + 8];
        if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
            w = get32(data);
            h = get32(data + 4);
            depth = data[8];
            ctype = data[9];
            interlace = data[12];
        } else if (!std::memcmp(type, "PLTE", 4)) {
            plte.assign(data, data + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + (size_t)len;
    }
    int ch = ctype == 0 ? 1 : ctype == 2 ? 3 : ctype == 3 ? 1 : ctype == 4 ? 2 : ctype == 6 ? 4 : 0;
    if (w == 0 || h == 0 || ch == 0) return path + ": unsupported or missing image header";
    if (depth != 8 || interlace != 0) return path + ": only 8-bit non-interlaced PNG is supported";
    if (ctype == 3 && plte.size() < 3) return path + ": palette missing";
    if ((uint64_t)w * h > 400000000ull) return path + ": image too large";
    const size_t stride = (size_t)w * ch;
    std::vector<uint8_t> raw((stride + 1) * h);
    uLongf rlen = (uLongf)raw.size();
    if (uncompress(raw.data(), &rlen, idat.data(), (uLong)idat.size()) != Z_OK || rlen != raw.size())
        return path + ": corrupt image data";
    std::vector<uint8_t> cur(stride), prev(stride, 0);
    rgb.assign((size_t)w * h * 3, 0);
    for (uint32_t y = 0; y < h; ++y) {
        const uint8_t ft = raw[y * (stride + 1)];
        const uint8_t* src = &raw[y * (stride + 1) + 1];
        for (size_t x = 0; x < stride; ++x) {
            const int a = x >= (size_t)ch ? cur[x - ch] : 0, b = prev[x], c = x >= (size_t)ch ? prev[x - ch] : 0;
            int v = src[x];
            switch (ft) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) / 2; break;
                case 4: v += paeth(a, b, c); break;
                default: return path + ": bad filter type";
            }
            cur[x] = (uint8_t)v;
        }
        for (uint32_t x = 0; x < w; ++x) {
            uint8_t* o = &rgb[((size_t)y * w + x) * 3];
            const uint8_t* p = &cur[(size_t)x * ch];
            if (ctype == 0 || ctype == 4) {
                o[0] = o[1] = o[2] = p[0];
            } else if (ctype == 3) {
                const size_t e = (size_t)p[0] * 3;
                if (e + 2 >= plte.size()) return path + ": palette index out of range";
                o[0] = plte[e];
                o[1] = plte[e + 1];
                o[2] = plte[e + 2];
            } else {
                o[0] = p[0];
                o[1] = p[1];
                o[2] = p[2];
            }
        }
        std::swap(cur, prev);
    }
    return "";
}

}  // namespace ifx_cli
