/* Test-infrastructure shim: declaration-only stand-ins for the OpenEXR types that the
 * reference image header names.  The oracle never writes EXR files. */
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
