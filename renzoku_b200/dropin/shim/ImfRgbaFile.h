/* Build stand-in for OpenEXR, which this image lacks: declarations of the types the
 * reference's image.h names.  Nothing built here writes EXR files. */
#pragma once
namespace Imf {
struct Rgba { Rgba() {} Rgba(float, float, float, float) {} };
namespace RgbaChannels { enum { WRITE_RGBA = 15 }; }
struct RgbaOutputFile {
    RgbaOutputFile(const char *, int, int, int) {}
    void setFrameBuffer(const Rgba *, int, int) {}
    void writePixels(int) {}
};
}
