// Host-side parameter preparation used by the node plugins (host_prep.cpp).
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"

namespace cpb::prep {

using Mat3 = std::array<float, 9>;
using Vec3 = std::array<float, 3>;

float reciprocal_cct_weight(double cct1, double cct2, double cct);
bool invert3(const Mat3& m, Mat3* out);
bool illuminant_cct(uint16_t code, double* cct);
double estimate_scene_cct(const Vec3& neutral, const Mat3& cm1, const Mat3& cm2, double cct1, double cct2);
// Fills the WbParams blob; fm1/fm2 may be null (then the ColorMatrix blend is inverted).
int wb_prepare(const Vec3& neutral, const Mat3* cm1, const Mat3* cm2, const Mat3* fm1, const Mat3* fm2,
               uint16_t illum1, uint16_t illum2, cpipe_WbParams* out, double* scene_cct);

Mat3 mul3(const Mat3& l, const Mat3& r);
Mat3 camera_to_rec2020(const Mat3& camera_to_xyz_d50);

struct GainMap {
    uint32_t top, left, bottom, right, plane, planes, row_pitch, col_pitch, points_v, points_h, map_planes;
    double spacing_v, spacing_h, origin_v, origin_h;
    std::vector<float> gain;
};
int parse_gain_maps(const void* bytes, size_t n, std::vector<GainMap>* maps, std::string* msg);
int validate_and_pack_gain_maps(const std::vector<GainMap>& maps, const uint8_t repeat[2], const uint8_t pattern[16],
                                std::vector<unsigned char>* blob, std::string* msg);
int parse_and_pack_opcode3(const void* bytes, size_t n, std::vector<unsigned char>* blob, uint32_t* count,
                           std::string* msg);
int load_lut(const std::string& path, uint32_t* size, std::vector<float>* values, std::string* msg);

}  // namespace cpb::prep
