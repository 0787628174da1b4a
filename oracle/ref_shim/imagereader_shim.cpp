// Test infrastructure (oracle): stand-in for MonkeyGL's ImageReader
// (core/ImageReader.h), whose original needs ITK.  File ingest is not on the
// ray-casting path; both readers report failure, as the original does for an
// unreadable file.
#include <memory>

#include "ImageReader.h"

namespace MonkeyGL {

ImageReader::ImageReader() {}
ImageReader::~ImageReader() {}

bool ImageReader::Read(const char *, std::shared_ptr<short> &, int[], double[], Point3d &,
                       Direction3d &, Direction3d &, Direction3d &) {
    return false;
}

bool ImageReader::ReadMask(const char *, std::shared_ptr<unsigned char> &, int &, int &, int &) {
    return false;
}

}  // namespace MonkeyGL
