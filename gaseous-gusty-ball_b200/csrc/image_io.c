/* PNG file input/output with the API of upstream src/image_io.h:5-8
 * (png_load_rgba, png_save), written on zlib for hosts without libpng.  Upstream
 * implements both with libpng's simplified API (src/image_io.c:8-52); this file
 * follows the PNG specification (ISO/IEC 15948 / W3C PNG) directly:
 *
 *   file   = 8-byte signature, then chunks {u32 BE length, 4-byte type, data,
 *            u32 BE CRC-32 of type+data}: IHDR first, PLTE, tRNS, IDAT..., IEND
 *   pixels = the IDAT data concatenated is one zlib stream of scanlines, each
 *            preceded by a filter byte (0 None, 1 Sub, 2 Up, 3 Average, 4 Paeth),
 *            for the whole image or, interlaced, for each of the 7 Adam7 passes.
 *
 * Reading returns RGBA bytes / 255 as floats, like upstream.  Gray expands to
 * R=G=B, palette indices through PLTE, tRNS sets alpha (palette entries, or the
 * gray / RGB colour key), samples below 8 bits scale to 0..255, 16-bit samples
 * round to 8 bits.  Gamma / colour-space chunks are ignored: 8-bit files carry
 * sRGB values, as the simplified API assumes when they are absent.
 *
 * Writing emits 8-bit RGB or RGBA, non-interlaced, choosing each row's filter
 * by the minimum sum of absolute filtered bytes (the specification's suggested
 * heuristic), at zlib level 1 (upstream asks libpng for fast writes). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#include "image_io.h"

#define EXPORT __attribute__((visibility("default")))

static const unsigned char kSig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
/* Adam7 passes: x start, y start, x step, y step. */
static const int kAdam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                 {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
/* Largest width / height accepted on read (libpng's default user limit). */
#define MAX_DIM 1000000u

static uint32_t rd32(const unsigned char *p) {
    return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
}
static void wr32(unsigned char *p, uint32_t v) {
    p[0] = (unsigned char)(v >> 24); p[1] = (unsigned char)(v >> 16);
    p[2] = (unsigned char)(v >> 8); p[3] = (unsigned char)v;
}
static int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = abs(p - a), pb = abs(p - b), pc = abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

/* ------------------------------------------------------------------ write */

typedef struct {
    FILE *f;
    int err;
} Out;

static void put_chunk(Out *o, const char *type, const unsigned char *data, uint32_t len) {
    unsigned char hdr[8], crc[4];
    wr32(hdr, len);
    memcpy(hdr + 4, type, 4);
    uLong c = crc32(0L, hdr + 4, 4);
    if (len) c = crc32(c, data, len);
    wr32(crc, (uint32_t)c);
    if (fwrite(hdr, 1, 8, o->f) != 8 || (len && fwrite(data, 1, len, o->f) != len) || fwrite(crc, 1, 4, o->f) != 4)
        o->err = 1;
}

/* Filter one row (bpp bytes per pixel, n bytes) with filter type t into out[0..n]. */
static void filter_row(int t, const unsigned char *cur, const unsigned char *prev, size_t n, int bpp,
                       unsigned char *out) {
    out[0] = (unsigned char)t;
    for (size_t i = 0; i < n; i++) {
        const int a = i >= (size_t)bpp ? cur[i - bpp] : 0, b = prev ? prev[i] : 0;
        const int c = prev && i >= (size_t)bpp ? prev[i - bpp] : 0;
        int p = 0;
        switch (t) {
        case 1: p = a; break;
        case 2: p = b; break;
        case 3: p = (a + b) >> 1; break;
        case 4: p = paeth(a, b, c); break;
        }
        out[1 + i] = (unsigned char)(cur[i] - p);
    }
}

static unsigned long row_cost(const unsigned char *f, size_t n) {
    unsigned long s = 0;
    for (size_t i = 1; i <= n; i++) s += f[i] < 128 ? f[i] : 256 - f[i];
    return s;
}

static const char *encode(Out *o, int w, int h, int channels, const unsigned char *data) {
    const size_t rb = (size_t)w * channels;
    unsigned char ihdr[13];
    wr32(ihdr, (uint32_t)w);
    wr32(ihdr + 4, (uint32_t)h);
    ihdr[8] = 8;
    ihdr[9] = channels == 4 ? 6 : 2;
    ihdr[10] = ihdr[11] = ihdr[12] = 0;
    if (fwrite(kSig, 1, 8, o->f) != 8) o->err = 1;
    put_chunk(o, "IHDR", ihdr, 13);

    enum { kOut = 1 << 18 };
    unsigned char *cand = malloc(5 * (rb + 1)), *zout = malloc(kOut);
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (!cand || !zout || deflateInit(&zs, 1) != Z_OK) {
        free(cand);
        free(zout);
        return "out of memory";
    }
    const char *err = NULL;
    zs.next_out = zout;
    zs.avail_out = kOut;
    for (int y = 0; y <= h && !err && !o->err; y++) {
        const int last = y == h;
        if (!last) {
            const unsigned char *cur = data + (size_t)y * rb, *prev = y ? cur - rb : NULL;
            int best = 0;
            unsigned long best_cost = 0;
            for (int t = 0; t < 5; t++) {
                filter_row(t, cur, prev, rb, channels, cand + t * (rb + 1));
                const unsigned long c = row_cost(cand + t * (rb + 1), rb);
                if (t == 0 || c < best_cost) best = t, best_cost = c;
            }
            zs.next_in = cand + best * (rb + 1);
            zs.avail_in = (uInt)(rb + 1);
        }
        for (;;) {
            const int r = deflate(&zs, last ? Z_FINISH : Z_NO_FLUSH);
            if (r == Z_STREAM_ERROR) {
                err = "zlib deflate failed";
                break;
            }
            if (zs.avail_out == 0) {
                put_chunk(o, "IDAT", zout, kOut);
                zs.next_out = zout;
                zs.avail_out = kOut;
                continue;
            }
            if (last ? r == Z_STREAM_END : zs.avail_in == 0) break;
        }
    }
    if (!err && !o->err && zs.avail_out < kOut) put_chunk(o, "IDAT", zout, kOut - zs.avail_out);
    deflateEnd(&zs);
    free(cand);
    free(zout);
    if (!err && !o->err) put_chunk(o, "IEND", NULL, 0);
    return err ? err : o->err ? "write error" : NULL;
}

EXPORT int png_save(const char *path, int w, int h, int channels, const unsigned char *data) {
    const char *err = NULL;
    if (w <= 0 || h <= 0 || (channels != 3 && channels != 4) || !data)
        err = "invalid image (size, channels 3 or 4, data)";
    else if ((size_t)w * channels + 1 > 0xffffffffu)
        err = "row too long";
    Out o = {NULL, 0};
    if (!err && !(o.f = fopen(path, "wb"))) err = "cannot open for writing";
    if (!err) err = encode(&o, w, h, channels, data);
    if (o.f && fclose(o.f) && !err) err = "write error";
    if (err) {
        if (o.f) remove(path);
        fprintf(stderr, "%s: %s\n", path, err);
        return -1;
    }
    return 0;
}

/* ------------------------------------------------------------------- read */

typedef struct {
    uint32_t w, h;
    int depth, ctype, interlace;
    int channels, bits; /* samples per pixel, bits per pixel */
    unsigned char pal[256][4];
    int npal;
    int has_key;
    unsigned key[3]; /* tRNS colour key at the file's sample depth */
} Head;

static int samples_of(int ctype) {
    switch (ctype) {
    case 0: return 1;
    case 2: return 3;
    case 3: return 1;
    case 4: return 2;
    case 6: return 4;
    }
    return 0;
}

static int valid_depth(int ctype, int d) {
    switch (ctype) {
    case 0: return d == 1 || d == 2 || d == 4 || d == 8 || d == 16;
    case 3: return d == 1 || d == 2 || d == 4 || d == 8;
    case 2: case 4: case 6: return d == 8 || d == 16;
    }
    return 0;
}

static size_t pass_w(const Head *H, int p) {
    const int *a = kAdam7[p];
    return H->w > (uint32_t)a[0] ? (H->w - a[0] + a[2] - 1) / a[2] : 0;
}
static size_t pass_h(const Head *H, int p) {
    const int *a = kAdam7[p];
    return H->h > (uint32_t)a[1] ? (H->h - a[1] + a[3] - 1) / a[3] : 0;
}
static size_t row_bytes(const Head *H, size_t pw) { return (pw * H->bits + 7) / 8; }

/* Sample s of pixel x in an unfiltered row, at the file's depth. */
static unsigned sample(const Head *H, const unsigned char *row, size_t x, int s) {
    if (H->depth == 8) return row[x * H->channels + s];
    if (H->depth == 16) {
        const unsigned char *q = row + 2 * (x * H->channels + s);
        return (unsigned)q[0] << 8 | q[1];
    }
    /* 1, 2, 4 bits: one sample per pixel, packed from the most significant bit */
    const size_t bit = x * H->depth;
    return (row[bit >> 3] >> (8 - H->depth - (bit & 7))) & ((1u << H->depth) - 1);
}

static unsigned char to8(const Head *H, unsigned v) {
    switch (H->depth) {
    case 1: return (unsigned char)(v * 255);
    case 2: return (unsigned char)(v * 85);
    case 4: return (unsigned char)(v * 17);
    case 16: return (unsigned char)((v * 255u + 32767u) / 65535u);
    }
    return (unsigned char)v;
}

static void pixel_rgba(const Head *H, const unsigned char *row, size_t x, unsigned char *o) {
    unsigned v[4] = {0, 0, 0, 0};
    for (int s = 0; s < H->channels; s++) v[s] = sample(H, row, x, s);
    switch (H->ctype) {
    case 0:
        o[0] = o[1] = o[2] = to8(H, v[0]);
        o[3] = H->has_key && v[0] == H->key[0] ? 0 : 255;
        break;
    case 2:
        for (int c = 0; c < 3; c++) o[c] = to8(H, v[c]);
        o[3] = H->has_key && v[0] == H->key[0] && v[1] == H->key[1] && v[2] == H->key[2] ? 0 : 255;
        break;
    case 3: /* indices beyond the palette read as opaque black */
        if ((int)v[0] < H->npal) memcpy(o, H->pal[v[0]], 4);
        else o[0] = o[1] = o[2] = 0, o[3] = 255;
        break;
    case 4:
        o[0] = o[1] = o[2] = to8(H, v[0]);
        o[3] = to8(H, v[1]);
        break;
    case 6:
        for (int c = 0; c < 4; c++) o[c] = to8(H, v[c]);
        break;
    }
}

/* Undo the filters of ph rows of rb bytes (each preceded by its filter byte), in place. */
static const char *unfilter(unsigned char *z, size_t ph, size_t rb, int bpp) {
    unsigned char *prev = NULL;
    for (size_t y = 0; y < ph; y++) {
        unsigned char *f = z + y * (rb + 1), *cur = f + 1;
        const int t = f[0];
        if (t > 4) return "bad filter type";
        for (size_t i = 0; i < rb; i++) {
            const int a = i >= (size_t)bpp ? cur[i - bpp] : 0, b = prev ? prev[i] : 0;
            const int c = prev && i >= (size_t)bpp ? prev[i - bpp] : 0;
            int p = 0;
            switch (t) {
            case 1: p = a; break;
            case 2: p = b; break;
            case 3: p = (a + b) >> 1; break;
            case 4: p = paeth(a, b, c); break;
            }
            cur[i] = (unsigned char)(cur[i] + p);
        }
        prev = cur;
    }
    return NULL;
}

static const char *decode(const unsigned char *f, size_t n, Head *H, unsigned char **rgba) {
    if (n < 8 || memcmp(f, kSig, 8)) return "not a PNG file";
    size_t pos = 8, zsize = 0;
    int seen_ihdr = 0, seen_idat = 0, done = 0, zdone = 0;
    unsigned char *z = NULL;
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    const char *err = NULL;
    while (!err && !done) {
        if (n - pos < 12) { err = "truncated file"; break; }
        const uint32_t len = rd32(f + pos);
        if (len > 0x7fffffffu || len > n - pos - 12) { err = "truncated chunk"; break; }
        const unsigned char *type = f + pos + 4, *d = f + pos + 8;
        const int critical = !(type[0] & 0x20);
        const uint32_t crc = (uint32_t)crc32(crc32(0L, type, 4), d, len);
        pos += 12 + (size_t)len;
        if (crc != rd32(d + len)) {
            if (critical) err = "CRC error";
            continue; /* a damaged ancillary chunk is skipped */
        }
        if (!seen_ihdr && memcmp(type, "IHDR", 4)) { err = "missing IHDR"; break; }
        if (!memcmp(type, "IHDR", 4)) {
            if (seen_ihdr || len != 13) { err = "bad IHDR"; break; }
            seen_ihdr = 1;
            H->w = rd32(d);
            H->h = rd32(d + 4);
            H->depth = d[8];
            H->ctype = d[9];
            H->interlace = d[12];
            if (!H->w || !H->h || H->w > MAX_DIM || H->h > MAX_DIM) { err = "unsupported image size"; break; }
            if (!valid_depth(H->ctype, H->depth) || d[10] || d[11] || H->interlace > 1) {
                err = "bad IHDR";
                break;
            }
            H->channels = samples_of(H->ctype);
            H->bits = H->channels * H->depth;
            for (int p = 0; p < 7; p++) {
                if (!H->interlace && p) break;
                const size_t pw = H->interlace ? pass_w(H, p) : H->w, ph = H->interlace ? pass_h(H, p) : H->h;
                if (pw && ph) zsize += ph * (row_bytes(H, pw) + 1);
            }
            if (!(z = malloc(zsize))) { err = "out of memory"; break; }
            if (inflateInit(&zs) != Z_OK) { err = "zlib init failed"; break; }
            zs.next_out = z;
            zs.avail_out = 0; /* set per IDAT below (zsize can exceed uInt) */
        } else if (!memcmp(type, "PLTE", 4)) {
            if (len % 3 || len / 3 > 256 || len == 0 || seen_idat) { err = "bad PLTE"; break; }
            if (H->ctype == 3 && (int)(len / 3) > (1 << H->depth)) { err = "bad PLTE"; break; }
            H->npal = (int)(len / 3);
            for (int i = 0; i < H->npal; i++) {
                memcpy(H->pal[i], d + 3 * i, 3);
                H->pal[i][3] = 255;
            }
        } else if (!memcmp(type, "tRNS", 4)) {
            if (H->ctype == 3 && len <= (uint32_t)H->npal) {
                for (uint32_t i = 0; i < len; i++) H->pal[i][3] = d[i];
            } else if (H->ctype == 0 && len == 2) {
                H->has_key = 1;
                H->key[0] = (unsigned)d[0] << 8 | d[1];
            } else if (H->ctype == 2 && len == 6) {
                H->has_key = 1;
                for (int c = 0; c < 3; c++) H->key[c] = (unsigned)d[2 * c] << 8 | d[2 * c + 1];
            } /* any other tRNS is invalid and ignored, as an ancillary chunk */
        } else if (!memcmp(type, "IDAT", 4)) {
            if (H->ctype == 3 && !H->npal) { err = "missing PLTE"; break; }
            seen_idat = 1;
            zs.next_in = (unsigned char *)d;
            zs.avail_in = len;
            while (zs.avail_in && !zdone) {
                const size_t left = zsize - (size_t)(zs.next_out - z);
                if (!left) break; /* extra data after the image is ignored */
                zs.avail_out = left > 0x40000000u ? 0x40000000u : (uInt)left;
                const int r = inflate(&zs, Z_NO_FLUSH);
                if (r == Z_STREAM_END) zdone = 1;
                else if (r != Z_OK) { err = "bad compressed data"; break; }
            }
        } else if (!memcmp(type, "IEND", 4)) {
            done = 1;
        } else if (critical) {
            err = "unknown critical chunk";
        }
    }
    if (!err && (size_t)(zs.next_out - z) != zsize) err = "not enough image data";
    if (seen_ihdr && z) inflateEnd(&zs);
    if (!err) {
        const size_t npix = (size_t)H->w * H->h;
        if (!(*rgba = malloc(npix * 4))) err = "out of memory";
    }
    unsigned char *zp = z;
    const int bpp = H->bits >= 8 ? H->bits / 8 : 1;
    for (int p = 0; p < 7 && !err; p++) {
        if (!H->interlace && p) break;
        const size_t pw = H->interlace ? pass_w(H, p) : H->w, ph = H->interlace ? pass_h(H, p) : H->h;
        if (!pw || !ph) continue;
        const size_t rb = row_bytes(H, pw);
        if ((err = unfilter(zp, ph, rb, bpp))) break;
        const int x0 = H->interlace ? kAdam7[p][0] : 0, y0 = H->interlace ? kAdam7[p][1] : 0;
        const int dx = H->interlace ? kAdam7[p][2] : 1, dy = H->interlace ? kAdam7[p][3] : 1;
        for (size_t y = 0; y < ph; y++) {
            const unsigned char *row = zp + y * (rb + 1) + 1;
            unsigned char *o = *rgba + ((size_t)(y0 + y * dy) * H->w + x0) * 4;
            for (size_t x = 0; x < pw; x++) pixel_rgba(H, row, x, o + x * dx * 4);
        }
        zp += ph * (rb + 1);
    }
    free(z);
    if (err) {
        free(*rgba);
        *rgba = NULL;
    }
    return err;
}

EXPORT float *png_load_rgba(const char *path, int *w, int *h) {
    const char *err = NULL;
    unsigned char *file = NULL, *rgba = NULL;
    size_t n = 0;
    FILE *fp = fopen(path, "rb");
    if (!fp) err = "cannot open file";
    if (!err) {
        size_t cap = 1 << 16;
        file = malloc(cap);
        while (file) {
            n += fread(file + n, 1, cap - n, fp);
            if (n < cap) break;
            unsigned char *g = realloc(file, cap *= 2);
            if (!g) free(file);
            file = g;
        }
        if (!file) err = "out of memory";
        else if (ferror(fp)) err = "read error";
        fclose(fp);
    }
    Head H;
    memset(&H, 0, sizeof(H));
    if (!err) err = decode(file, n, &H, &rgba);
    free(file);
    if (err) {
        fprintf(stderr, "%s: %s\n", path, err);
        return NULL;
    }
    const size_t np = (size_t)H.w * H.h * 4;
    float *out = malloc(sizeof(float) * np);
    if (!out) {
        fprintf(stderr, "%s: %s\n", path, "out of memory");
        free(rgba);
        return NULL;
    }
    for (size_t i = 0; i < np; i++) out[i] = rgba[i] / 255.0f;
    free(rgba);
    *w = (int)H.w;
    *h = (int)H.h;
    return out;
}
