// pt_image.h — texture image loading for OBJ import (PNG, PPM) into 8-bit RGB, rows top first.
#pragma once

#include <string>
#include <vector>

namespace ptb {

struct Image {
    int width = 0, height = 0;
    std::vector<unsigned char> rgb;   // width * height * 3
};

// false (and `err`) for a missing file, an unknown or unsupported format, or corrupt data.
bool load_image(const std::string &path, Image &img, std::string &err);
// Baseline JPEG (pt_jpeg.cpp).
bool decode_jpeg(const std::vector<unsigned char> &file, Image &img, std::string &err);

} // namespace ptb
