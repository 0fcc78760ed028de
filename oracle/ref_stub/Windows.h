/* Minimal stand-in for <Windows.h> so that the reference's bmp2texture.c compiles on Linux for the
 * oracle harness.  Only the bitmap header types that file names are declared, with the Win32
 * packing (the 14-byte file header), so that its BMP reader parses real files. */
#ifndef ST_REF_STUB_WINDOWS_H
#define ST_REF_STUB_WINDOWS_H
#include <stdint.h>
typedef uint16_t WORD;
typedef uint32_t DWORD;
typedef int32_t LONG;
#pragma pack(push, 2)
typedef struct BITMAPFILEHEADER { WORD bfType; DWORD bfSize; WORD bfReserved1, bfReserved2; DWORD bfOffBits; } BITMAPFILEHEADER;
#pragma pack(pop)
typedef struct BITMAPINFOHEADER {
    DWORD biSize; LONG biWidth, biHeight; WORD biPlanes, biBitCount; DWORD biCompression, biSizeImage;
    LONG biXPelsPerMeter, biYPelsPerMeter; DWORD biClrUsed, biClrImportant;
} BITMAPINFOHEADER;
#endif
