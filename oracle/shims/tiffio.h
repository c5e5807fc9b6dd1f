/* Minimal stand-in for the libtiff API subset the reference calls (test
 * infrastructure).  Writes uncompressed baseline TIFF with one strip per
 * TIFFTAG_ROWSPERSTRIP rows, little-endian. */
#ifndef MSF_ORACLE_SHIM_TIFFIO_H
#define MSF_ORACLE_SHIM_TIFFIO_H
#include <stddef.h>
#include <stdint.h>

typedef uint32_t uint32;
typedef uint16_t uint16;
typedef ptrdiff_t tsize_t;
typedef void* tdata_t;
typedef struct msf_shim_tiff TIFF;

#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_BITSPERSAMPLE 258
#define TIFFTAG_COMPRESSION 259
#define TIFFTAG_PHOTOMETRIC 262
#define TIFFTAG_STRIPOFFSETS 273
#define TIFFTAG_ORIENTATION 274
#define TIFFTAG_SAMPLESPERPIXEL 277
#define TIFFTAG_ROWSPERSTRIP 278
#define TIFFTAG_STRIPBYTECOUNTS 279
#define TIFFTAG_XRESOLUTION 282
#define TIFFTAG_YRESOLUTION 283
#define TIFFTAG_PLANARCONFIG 284
#define TIFFTAG_RESOLUTIONUNIT 296
#define TIFFTAG_SAMPLEFORMAT 339

#define ORIENTATION_TOPLEFT 1
#define PLANARCONFIG_CONTIG 1
#define PHOTOMETRIC_MINISBLACK 1
#define PHOTOMETRIC_RGB 2
#define SAMPLEFORMAT_UINT 1
#define SAMPLEFORMAT_IEEEFP 3

#ifdef __cplusplus
extern "C" {
#endif
TIFF* TIFFOpen(const char* name, const char* mode);
int TIFFSetField(TIFF* tif, uint32 tag, ...);
uint32 TIFFDefaultStripSize(TIFF* tif, uint32 request);
tsize_t TIFFScanlineSize(TIFF* tif);
int TIFFWriteScanline(TIFF* tif, void* buf, uint32 row, uint16 sample);
void TIFFClose(TIFF* tif);
void* _TIFFmalloc(tsize_t s);
void _TIFFfree(void* p);
#ifdef __cplusplus
}
#endif
#endif
