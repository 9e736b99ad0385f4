/* Build stand-in for FreeImage, which this image lacks: declarations only, so that the
 * reference's image.h compiles.  Nothing built here loads or writes image files; a build
 * inside the reference's own tree uses the real library instead. */
#pragma once
typedef unsigned char BYTE;
struct FIBITMAP;
struct FIRGBF { float red, green, blue; };
enum FREE_IMAGE_FORMAT { FIF_UNKNOWN = -1 };
enum FREE_IMAGE_TYPE { FIT_BITMAP = 1, FIT_RGBF = 11 };
enum { FI_RGBA_RED = 2, FI_RGBA_GREEN = 1, FI_RGBA_BLUE = 0 };
inline FREE_IMAGE_FORMAT FreeImage_GetFileType(const char *, int) { return FIF_UNKNOWN; }
inline FREE_IMAGE_FORMAT FreeImage_GetFIFFromFilename(const char *) { return FIF_UNKNOWN; }
inline int FreeImage_FIFSupportsReading(FREE_IMAGE_FORMAT) { return 0; }
inline FIBITMAP *FreeImage_Load(FREE_IMAGE_FORMAT, const char *, int) { return 0; }
inline FREE_IMAGE_TYPE FreeImage_GetImageType(FIBITMAP *) { return FIT_BITMAP; }
inline BYTE *FreeImage_GetBits(FIBITMAP *) { return 0; }
inline unsigned FreeImage_GetPitch(FIBITMAP *) { return 0; }
inline unsigned FreeImage_GetLine(FIBITMAP *) { return 0; }
inline unsigned FreeImage_GetWidth(FIBITMAP *) { return 0; }
inline unsigned FreeImage_GetHeight(FIBITMAP *) { return 0; }
inline void FreeImage_Unload(FIBITMAP *) {}
