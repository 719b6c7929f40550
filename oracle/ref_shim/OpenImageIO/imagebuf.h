/* Stand-in for OpenImageIO used only to compile the reference's golden
 * generator (tests/fixtures/gen_golden_isp_nodes.cpp) into the oracle's
 * reference build.  ImageBuf::write stores the float pixels as a raw file:
 * 4-byte magic "CPF1", int32 width, height, channels, then float32 data.
 * Test infrastructure only. */
#pragma once
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace OIIO {
struct TypeDesc {
    enum BASETYPE { FLOAT = 11 };
};
struct ImageSpec {
    int width, height, nchannels;
    ImageSpec(int w, int h, int c, int) : width(w), height(h), nchannels(c) {}
};
struct ROI {
    int xbegin, xend, ybegin, yend, zbegin, zend, chbegin, chend;
};
class ImageBuf {
public:
    ImageBuf(const std::string&, const ImageSpec& spec) : spec_(spec) {
        pixels_.resize((size_t)spec.width * spec.height * spec.nchannels);
    }
    bool set_pixels(const ROI&, int, const float* data) {
        std::memcpy(pixels_.data(), data, pixels_.size() * sizeof(float));
        return true;
    }
    std::string geterror() const { return "write failed"; }
    bool write(const std::string& path, int) const {
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return false;
        const int hdr[3] = {spec_.width, spec_.height, spec_.nchannels};
        bool ok = std::fwrite("CPF1", 1, 4, f) == 4 && std::fwrite(hdr, sizeof(int), 3, f) == 3 &&
                  std::fwrite(pixels_.data(), sizeof(float), pixels_.size(), f) == pixels_.size();
        return std::fclose(f) == 0 && ok;
    }
private:
    ImageSpec spec_;
    std::vector<float> pixels_;
};
}  // namespace OIIO
