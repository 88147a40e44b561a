// Image files of Film::savePNG / Film::saveEXR (film.cpp:154-195): an 8-bit RGB PNG and
// a float RGB OpenEXR image, written without the reference's stb / OpenEXR libraries.
//
// PNG: signature, IHDR (8-bit truecolour), one IDAT holding the zlib stream of the
// filtered scanlines (filter type 0 on every row), IEND; chunk CRCs from zlib's crc32.
// EXR: single-part scanline file, version 2, no compression: the header attributes
// (channels B, G, R as FLOAT, compression, dataWindow, displayWindow, lineOrder,
// pixelAspectRatio, screenWindowCenter, screenWindowWidth), the line offset table, then
// one block per scanline (y, byte count, the three channels' values for that line in
// channel order). All integers little endian.
#include <zlib.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gnd_gpu.h"

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

}  // namespace

extern "C" {

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
