// Image files of Film::savePNG / Film::saveEXR (film.cpp:154-195): an 8-bit RGB PNG and
// a float RGB OpenEXR image, written without the reference's stb / OpenEXR libraries;
// and the OpenEXR reader of the environment map (image2d.h:100-135).
//
// PNG: signature, IHDR (8-bit truecolour), one IDAT holding the zlib stream of the
// filtered scanlines (filter type 0 on every row), IEND; chunk CRCs from zlib's crc32.
// EXR: single-part scanline file, version 2, no compression: the header attributes
// (channels B, G, R as FLOAT, compression, dataWindow, displayWindow, lineOrder,
// pixelAspectRatio, screenWindowCenter, screenWindowWidth), the line offset table, then
// one block per scanline (y, byte count, the three channels' values for that line in
// channel order). All integers little endian.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gnd_gpu.h"
#include "hscene.h"

namespace gnd {
void setLastError(const std::string& msg);   // thread-local message of gnd_last_error
}

namespace {

void put32be(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 24)); v.push_back((uint8_t)(x >> 16)); v.push_back((uint8_t)(x >> 8)); v.push_back((uint8_t)x);
}
template <typename T>
void putLE(std::vector<uint8_t>& v, T x) {
    uint8_t b[sizeof(T)];
    std::memcpy(b, &x, sizeof(T));   // x86: little endian in memory
    v.insert(v.end(), b, b + sizeof(T));
}
void putStr(std::vector<uint8_t>& v, const char* s) { v.insert(v.end(), s, s + std::strlen(s) + 1); }

void pngChunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
    put32be(out, (uint32_t)data.size());
    const size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    const uLong crc = crc32(0L, out.data() + start, (uInt)(out.size() - start));
    put32be(out, (uint32_t)crc);
}

void writeFile(const char* path, const std::vector<uint8_t>& bytes) {
    FILE* f = std::fopen(path, "wb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path + " for writing");
    const size_t n = std::fwrite(bytes.data(), 1, bytes.size(), f);
    const int rc = std::fclose(f);
    if (n != bytes.size() || rc != 0) throw std::runtime_error(std::string("write failed: ") + path);
}

void checkImage(const void* p, int32_t w, int32_t h) {
    if (!p) throw std::runtime_error("null image");
    if (w <= 0 || h <= 0 || (int64_t)w * h > ((int64_t)1 << 28)) throw std::runtime_error("image size out of range");
}

void exrAttr(std::vector<uint8_t>& v, const char* name, const char* type, const std::vector<uint8_t>& value) {
    putStr(v, name);
    putStr(v, type);
    putLE<int32_t>(v, (int32_t)value.size());
    v.insert(v.end(), value.begin(), value.end());
}

// IEEE binary16 -> binary32 (exact)
float halfToFloat(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    const uint32_t e = (h >> 10) & 31u, m = h & 1023u;
    uint32_t bits;
    if (e == 0) {
        if (m == 0) {
            bits = sign;
        } else {   // subnormal: normalise
            int shift = 0;
            uint32_t mm = m;
            while (!(mm & 1024u)) { mm <<= 1; ++shift; }
            bits = sign | ((uint32_t)(127 - 15 + 1 - shift) << 23) | ((mm & 1023u) << 13);
        }
    } else if (e == 31) {
        bits = sign | 0x7f800000u | (m << 13);
    } else {
        bits = sign | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

}  // namespace

namespace gndh {

// Scanline OpenEXR: header attributes, line offset table, blocks of 1 (NO, ZIPS) or 16
// (ZIP) scanlines; a ZIP block is a zlib stream of the block's bytes reordered (the
// first half holds the even bytes, the second the odd ones) and delta coded.
void readEXR(const std::string& path, int& width, int& height, std::vector<float>& rgb) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("EXR: cannot open " + path);
    std::vector<uint8_t> d;
    uint8_t buf[65536];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) d.insert(d.end(), buf, buf + n);
    std::fclose(f);
    auto need = [&](size_t at, size_t len) {
        if (at + len > d.size()) throw std::runtime_error("EXR: truncated file " + path);
    };
    auto rd32 = [&](size_t at) { need(at, 4); int32_t v; std::memcpy(&v, &d[at], 4); return v; };
    auto rd64 = [&](size_t at) { need(at, 8); uint64_t v; std::memcpy(&v, &d[at], 8); return v; };
    auto cstr = [&](size_t& at) {
        std::string s;
        for (;;) { need(at, 1); if (!d[at]) break; s += (char)d[at++]; }
        ++at;
        return s;
    };
    if (rd32(0) != 20000630) throw std::runtime_error("EXR: not an OpenEXR file: " + path);
    const int32_t version = rd32(4);
    if ((version & 0xff) != 2 || (version & 0x1e00)) throw std::runtime_error("EXR: only single-part scanline files are read");
    struct Chan { std::string name; int type; };
    std::vector<Chan> chans;
    int comp = -1, x0 = 0, y0 = 0, x1 = -1, y1 = -1;
    size_t pos = 8;
    for (;;) {
        need(pos, 1);
        if (!d[pos]) break;
        std::string name = cstr(pos), type = cstr(pos);
        const int32_t len = rd32(pos);
        const size_t at = pos + 4;
        need(at, (size_t)std::max(len, 0));
        if (name == "channels") {
            size_t q = at;
            while (q < at + len && d[q]) { std::string c = cstr(q); chans.push_back({c, rd32(q)}); q += 16; }
        } else if (name == "compression") {
            comp = d[at];
        } else if (name == "dataWindow") {
            x0 = rd32(at); y0 = rd32(at + 4); x1 = rd32(at + 8); y1 = rd32(at + 12);
        }
        pos = at + (size_t)len;
    }
    ++pos;
    if (comp != 0 && comp != 2 && comp != 3) throw std::runtime_error("EXR: unsupported compression (only none, ZIPS, ZIP)");
    width = x1 - x0 + 1;
    height = y1 - y0 + 1;
    if (width <= 0 || height <= 0 || (int64_t)width * height > ((int64_t)1 << 28)) throw std::runtime_error("EXR: bad data window");
    for (const Chan& c : chans)
        if (c.type != 1 && c.type != 2) throw std::runtime_error("EXR: channel " + c.name + " is not HALF or FLOAT");
    std::sort(chans.begin(), chans.end(), [](const Chan& a, const Chan& b) { return a.name < b.name; });
    size_t lineBytes = 0;
    for (const Chan& c : chans) lineBytes += (size_t)width * (c.type == 1 ? 2 : 4);
    const int linesPerBlock = comp == 3 ? 16 : 1;
    const int blocks = (height + linesPerBlock - 1) / linesPerBlock;
    rgb.assign((size_t)width * height * 3, 0.0f);
    std::vector<uint8_t> raw, tmp;
    for (int b = 0; b < blocks; ++b) {
        const uint64_t off = rd64(pos + 8 * (size_t)b);
        const int yb = rd32(off) - y0;
        const int32_t size = rd32(off + 4);
        need(off + 8, (size_t)std::max(size, 0));
        const int lines = std::min(linesPerBlock, height - yb);
        if (yb < 0 || lines <= 0) throw std::runtime_error("EXR: block outside the data window");
        const size_t expect = lineBytes * (size_t)lines;
        const uint8_t* src = &d[off + 8];
        if (comp == 0 || (size_t)size == expect) {
            if ((size_t)size != expect) throw std::runtime_error("EXR: bad block size");
            raw.assign(src, src + expect);
        } else {
            tmp.assign(expect, 0);
            uLongf outLen = (uLongf)expect;
            if (uncompress(tmp.data(), &outLen, src, (uLong)size) != Z_OK || outLen != expect)
                throw std::runtime_error("EXR: corrupt ZIP block");
            for (size_t i = 1; i < expect; ++i) tmp[i] = (uint8_t)(tmp[i - 1] + tmp[i] - 128);
            raw.resize(expect);
            const size_t half = (expect + 1) / 2;
            for (size_t i = 0; i < expect; ++i) raw[i] = (i & 1) ? tmp[half + i / 2] : tmp[i / 2];
        }
        size_t at = 0;
        for (int l = 0; l < lines; ++l) {
            const int y = yb + l;
            for (const Chan& c : chans) {
                const int k = c.name == "R" ? 0 : c.name == "G" ? 1 : c.name == "B" ? 2 : -1;
                const size_t sz = c.type == 1 ? 2 : 4;
                for (int x = 0; x < width; ++x, at += sz) {
                    if (k < 0) continue;
                    float v;
                    if (sz == 4) {
                        std::memcpy(&v, &raw[at], 4);
                    } else {
                        uint16_t hv;
                        std::memcpy(&hv, &raw[at], 2);
                        v = halfToFloat(hv);
                    }
                    rgb[3 * ((size_t)y * width + x) + k] = v;
                }
            }
        }
    }
}

namespace {
std::vector<uint8_t> readAll(const std::string& path, const char* what) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error(std::string(what) + ": cannot open " + path);
    std::vector<uint8_t> d;
    uint8_t buf[65536];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) d.insert(d.end(), buf, buf + n);
    std::fclose(f);
    return d;
}

// A float rounded to the nearest binary16 value (ties to even), as Imf::Rgba stores it:
// 11 significant bits in the normal range, multiples of 2^-24 below 2^-14, infinity from
// 65520 on.
float toHalfPrecision(float f) {
    if (!std::isfinite(f) || f == 0.0f) return f;
    const float a = std::fabs(f);
    float r;
    if (a < 6.103515625e-05f) {
        r = std::nearbyint(a * 16777216.0f) / 16777216.0f;
    } else {
        int e;
        const float m = std::frexp(a, &e);   // a = m 2^e, m in [0.5, 1)
        r = std::ldexp(std::nearbyint(std::ldexp(m, 11)), e - 11);
        if (r > 65504.0f) r = INFINITY;
    }
    return f < 0.0f ? -r : r;
}

// PNG (ISO/IEC 15948): 8- or 16-bit grey, grey + alpha, RGB or RGBA, not interlaced;
// the IDAT stream inflated, each row's filter (none, sub, up, average, Paeth) undone.
// 16-bit samples keep their high byte.
void readPNG(const std::string& path, int& w, int& h, int& channels, std::vector<uint8_t>& px) {
    const std::vector<uint8_t> d = readAll(path, "TextureCache");
    const uint8_t magic[8] = {0x89, 0x50, 0x4e, 0x47, 0x0d, 0x0a, 0x1a, 0x0a};
    if (d.size() < 8 || std::memcmp(d.data(), magic, 8) != 0) throw std::runtime_error("TextureCache: Failed to load image " + path);
    auto u32 = [&](size_t at) -> uint32_t {
        if (at + 4 > d.size()) throw std::runtime_error("PNG: truncated file " + path);
        return (uint32_t)d[at] << 24 | (uint32_t)d[at + 1] << 16 | (uint32_t)d[at + 2] << 8 | (uint32_t)d[at + 3];
    };
    int depth = 0, colorType = -1, interlace = 0;
    bool haveHeader = false;
    std::vector<uint8_t> stream;
    for (size_t at = 8;;) {
        const uint32_t len = u32(at);
        if ((uint64_t)at + 12 + len > d.size()) throw std::runtime_error("PNG: truncated file " + path);
        const uint8_t* body = &d[at + 8];
        const std::string type(reinterpret_cast<const char*>(&d[at + 4]), 4);
        if (type == "IHDR" && len >= 13) {
            w = (int)u32(at + 8);
            h = (int)u32(at + 12);
            depth = body[8];
            colorType = body[9];
            interlace = body[12];
            haveHeader = true;
        } else if (type == "IDAT") {
            stream.insert(stream.end(), body, body + len);
        } else if (type == "IEND") {
            break;
        }
        at += 12 + (size_t)len;
    }
    if (!haveHeader || w <= 0 || h <= 0 || (int64_t)w * h > ((int64_t)1 << 28)) throw std::runtime_error("PNG: bad header in " + path);
    channels = colorType == 0 ? 1 : colorType == 4 ? 2 : colorType == 2 ? 3 : colorType == 6 ? 4 : 0;
    if (!channels || interlace || (depth != 8 && depth != 16))
        throw std::runtime_error("PNG: " + path + ": only 8/16-bit, non-interlaced grey, grey+alpha, RGB or RGBA images");
    const size_t sampleBytes = (size_t)depth / 8, pixelBytes = (size_t)channels * sampleBytes;
    const size_t rowBytes = (size_t)w * pixelBytes;
    std::vector<uint8_t> raw((rowBytes + 1) * (size_t)h);
    uLongf rawLen = (uLongf)raw.size();
    if (uncompress(raw.data(), &rawLen, stream.data(), (uLong)stream.size()) != Z_OK || rawLen != raw.size())
        throw std::runtime_error("PNG: corrupt image data in " + path);
    std::vector<uint8_t> rows(rowBytes * (size_t)h);
    for (int y = 0; y < h; ++y) {
        const uint8_t filter = raw[(size_t)y * (rowBytes + 1)];
        const uint8_t* src = &raw[(size_t)y * (rowBytes + 1) + 1];
        uint8_t* dst = &rows[(size_t)y * rowBytes];
        const uint8_t* up = y > 0 ? dst - rowBytes : nullptr;
        if (filter > 4) throw std::runtime_error("PNG: bad row filter in " + path);
        for (size_t i = 0; i < rowBytes; ++i) {
            const int left = i >= pixelBytes ? dst[i - pixelBytes] : 0;
            const int above = up ? up[i] : 0;
            const int corner = (up && i >= pixelBytes) ? up[i - pixelBytes] : 0;
            int pred = 0;
            switch (filter) {
                case 1: pred = left; break;
                case 2: pred = above; break;
                case 3: pred = (left + above) >> 1; break;
                case 4: {
                    const int est = left + above - corner;
                    const int dl = std::abs(est - left), da = std::abs(est - above), dc = std::abs(est - corner);
                    pred = (dl <= da && dl <= dc) ? left : (da <= dc ? above : corner);
                    break;
                }
                default: break;
            }
            dst[i] = (uint8_t)(src[i] + pred);
        }
    }
    px.resize((size_t)w * h * channels);
    for (size_t i = 0; i < px.size(); ++i) px[i] = rows[i * sampleBytes];
}
}  // namespace

void readTextureImage(const std::string& path, bool srgb, int& width, int& height, int& channels, std::vector<float>& rgba) {
    const bool exr = path.size() >= 4 && path.compare(path.size() - 4, 4, ".exr") == 0;
    if (exr) {
        std::vector<float> rgb;
        readEXR(path, width, height, rgb);
        channels = 4;
        rgba.assign((size_t)width * height * 4, 1.0f);
        for (int y = 0; y < height; ++y)
            for (int x = 0; x < width; ++x) {
                const float* s = &rgb[3 * ((size_t)y * width + x)];
                float* o = &rgba[4 * ((size_t)(height - 1 - y) * width + x)];
                for (int k = 0; k < 3; ++k) o[k] = toHalfPrecision(s[k]);
            }
        return;
    }
    std::vector<uint8_t> px;
    readPNG(path, width, height, channels, px);
    const int c = channels;
    auto linearize = [](float v) { return v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f); };
    rgba.assign((size_t)width * height * 4, 1.0f);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const uint8_t* s = &px[((size_t)(height - 1 - y) * width + x) * c];
            float* o = &rgba[4 * ((size_t)y * width + x)];
            for (int k = 0; k < c; ++k) {
                float v = s[k] / 255.0f;
                if (srgb && (c <= 3 || k < 3)) v = linearize(v);
                o[k] = v;
            }
        }
}

}  // namespace gndh

extern "C" {

gnd_status gnd_image_read_exr(const char* path, float* rgb, int64_t capacity, int32_t* width, int32_t* height) {
    try {
        if (!path || !width || !height) throw std::runtime_error("null argument");
        int w = 0, h = 0;
        std::vector<float> px;
        gndh::readEXR(path, w, h, px);
        *width = w;
        *height = h;
        if (rgb) {
            if ((int64_t)(px.size() * sizeof(float)) > capacity) throw std::runtime_error("destination too small");
            std::memcpy(rgb, px.data(), px.size() * sizeof(float));
        }
        return GND_OK;
    } catch (const std::bad_alloc&) {
        gnd::setLastError("host allocation failed");
        return GND_ERR_OOM;
    } catch (const std::exception& e) {
        gnd::setLastError(e.what());
        return GND_ERR_INVALID;
    }
}

gnd_status gnd_image_write_png(const char* path, const uint8_t* rgb8, int32_t w, int32_t h) {
    try {
        if (!path) throw std::runtime_error("null path");
        checkImage(rgb8, w, h);
        std::vector<uint8_t> raw((size_t)h * (3 * (size_t)w + 1));
        for (int32_t y = 0; y < h; ++y) {
            uint8_t* row = raw.data() + (size_t)y * (3 * (size_t)w + 1);
            row[0] = 0;   // filter: none
            std::memcpy(row + 1, rgb8 + (size_t)y * 3 * w, 3 * (size_t)w);
        }
        uLongf zlen = compressBound((uLong)raw.size());
        std::vector<uint8_t> z(zlen);
        if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) throw std::runtime_error("zlib compression failed");
        z.resize(zlen);
        std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
        std::vector<uint8_t> ihdr;
        put32be(ihdr, (uint32_t)w);
        put32be(ihdr, (uint32_t)h);
        ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});   // 8-bit, truecolour, deflate, adaptive filters, no interlace
        pngChunk(out, "IHDR", ihdr);
        pngChunk(out, "IDAT", z);
        pngChunk(out, "IEND", {});
        writeFile(path, out);
        return GND_OK;
    } catch (const std::bad_alloc&) {
        gnd::setLastError("host allocation failed");
        return GND_ERR_OOM;
    } catch (const std::exception& e) {
        gnd::setLastError(e.what());
        return GND_ERR_INVALID;
    }
}

gnd_status gnd_image_write_exr(const char* path, const float* rgb, int32_t w, int32_t h) {
    try {
        if (!path) throw std::runtime_error("null path");
        checkImage(rgb, w, h);
        std::vector<uint8_t> out;
        putLE<uint32_t>(out, 20000630u);   // magic
        putLE<uint32_t>(out, 2u);          // version 2, single-part scanline
        std::vector<uint8_t> ch;
        for (const char* c : {"B", "G", "R"}) {   // channels in alphabetical order
            putStr(ch, c);
            putLE<int32_t>(ch, 2);   // pixel type FLOAT
            ch.insert(ch.end(), {0, 0, 0, 0});   // pLinear, reserved
            putLE<int32_t>(ch, 1);   // xSampling
            putLE<int32_t>(ch, 1);   // ySampling
        }
        ch.push_back(0);
        exrAttr(out, "channels", "chlist", ch);
        exrAttr(out, "compression", "compression", {0});   // NO_COMPRESSION
        std::vector<uint8_t> box;
        putLE<int32_t>(box, 0); putLE<int32_t>(box, 0); putLE<int32_t>(box, w - 1); putLE<int32_t>(box, h - 1);
        exrAttr(out, "dataWindow", "box2i", box);
        exrAttr(out, "displayWindow", "box2i", box);
        exrAttr(out, "lineOrder", "lineOrder", {0});       // INCREASING_Y
        std::vector<uint8_t> one;
        putLE<float>(one, 1.0f);
        exrAttr(out, "pixelAspectRatio", "float", one);
        std::vector<uint8_t> centre;
        putLE<float>(centre, 0.0f); putLE<float>(centre, 0.0f);
        exrAttr(out, "screenWindowCenter", "v2f", centre);
        exrAttr(out, "screenWindowWidth", "float", one);
        out.push_back(0);   // end of header
        const size_t lineBytes = (size_t)w * 3 * sizeof(float);
        const size_t tableAt = out.size();
        uint64_t offset = tableAt + (size_t)h * 8;
        for (int32_t y = 0; y < h; ++y) {
            putLE<uint64_t>(out, offset);
            offset += 8 + lineBytes;
        }
        out.reserve(out.size() + (size_t)h * (8 + lineBytes));
        for (int32_t y = 0; y < h; ++y) {
            putLE<int32_t>(out, y);
            putLE<int32_t>(out, (int32_t)lineBytes);
            const float* row = rgb + (size_t)y * 3 * w;
            for (int c = 2; c >= 0; --c)   // B, G, R
                for (int32_t x = 0; x < w; ++x) putLE<float>(out, row[3 * (size_t)x + c]);
        }
        writeFile(path, out);
        return GND_OK;
    } catch (const std::bad_alloc&) {
        gnd::setLastError("host allocation failed");
        return GND_ERR_OOM;
    } catch (const std::exception& e) {
        gnd::setLastError(e.what());
        return GND_ERR_INVALID;
    }
}

}  // extern "C"
