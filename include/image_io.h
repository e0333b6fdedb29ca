/* PNG file input/output: the API of upstream src/image_io.h:5-8, implemented on
 * zlib by gaseous-gusty-ball_b200/csrc/image_io.c (libggb_image_io.so), for
 * hosts without libpng.  The application driver links it in place of
 * src/image_io.o. */
#ifndef IMAGE_IO_H
#define IMAGE_IO_H

#ifdef __cplusplus
extern "C" {
#endif

/* Returns malloc'd float RGBA [0,1] pixels (row 0 = top, value = byte / 255),
 * or NULL after printing "path: reason" to stderr.  Reads every PNG colour type
 * at every bit depth, interlaced or not, with palette and tRNS transparency;
 * 16-bit samples are rounded to 8 bits and gamma chunks are ignored. */
float *png_load_rgba(const char *path, int *w, int *h);
/* channels = 3 (RGB) or 4 (RGBA); data is 8-bit, row 0 = top.  Returns 0 on
 * success, -1 after printing "path: reason" to stderr (no file is left). */
int png_save(const char *path, int w, int h, int channels, const unsigned char *data);

#ifdef __cplusplus
}
#endif

#endif
