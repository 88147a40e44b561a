// The host film (film.h:21-136, film.cpp:50-195): device sums in, resolved radiance and
// the PNG / EXR files out.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "hscene.h"

namespace gndh {

Film::Film(int width, int height) : m_width(width), m_height(height) {
    if (width <= 0 || height <= 0) throw std::runtime_error("Film: the size must be positive");
    m_sums.assign((size_t)width * height * 7, 0.0f);
    m_radiance.assign((size_t)width * height, gnd::v3s(0.0f));
}

void Film::clear() {
    std::fill(m_sums.begin(), m_sums.end(), 0.0f);
    std::fill(m_radiance.begin(), m_radiance.end(), gnd::v3s(0.0f));
}

void Film::setSums(const float* sums) { std::memcpy(m_sums.data(), sums, m_sums.size() * sizeof(float)); }

// film.cpp:50-95 (radiance channel): the weighted mean of each pixel's samples.
void Film::resolve() {
    for (size_t q = 0; q < m_radiance.size(); ++q) {
        const float* a = &m_sums[q * 7];
        const float w = a[3];
        if (w > 0.0f) {
            const float invW = 1.0f / w;
            m_radiance[q] = gnd::v3(a[0] * invW, a[1] * invW, a[2] * invW);
        } else {
            m_radiance[q] = gnd::v3s(0.0f);
        }
    }
}

namespace {
// color.h:84-95
float toSRGB(float x) { return x <= 0.0031308f ? 12.92f * x : 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f; }
}  // namespace

// film.cpp:154-178: sRGB, x 255 + 0.5, clamped to [0, 255], truncated to 8 bits.
void Film::savePNG(const std::string& relativeOutPath) const {
    std::vector<uint8_t> data((size_t)m_width * m_height * 3);
    for (size_t q = 0; q < m_radiance.size(); ++q) {
        const float c[3] = {m_radiance[q].x, m_radiance[q].y, m_radiance[q].z};
        for (int k = 0; k < 3; ++k) {
            const float f = std::clamp(toSRGB(c[k]) * 255.0f + 0.5f, 0.0f, 255.0f);
            data[q * 3 + k] = static_cast<uint8_t>(f);
        }
    }
    const std::string file = outputPath + "/" + relativeOutPath + ".png";
    if (gnd_image_write_png(file.c_str(), data.data(), m_width, m_height) != GND_OK)
        throw std::runtime_error("Film: cannot write " + file + ": " + gnd_last_error());
}

// film.cpp:185-195: the radiance as a float RGB OpenEXR image.
void Film::saveEXR(const std::string& relativeOutPath) const {
    std::vector<float> rgb((size_t)m_width * m_height * 3);
    for (size_t q = 0; q < m_radiance.size(); ++q) {
        rgb[q * 3 + 0] = m_radiance[q].x;
        rgb[q * 3 + 1] = m_radiance[q].y;
        rgb[q * 3 + 2] = m_radiance[q].z;
    }
    const std::string file = outputPath + "/" + relativeOutPath + ".exr";
    if (gnd_image_write_exr(file.c_str(), rgb.data(), m_width, m_height) != GND_OK)
        throw std::runtime_error("Film: cannot write " + file + ": " + gnd_last_error());
}

}  // namespace gndh
