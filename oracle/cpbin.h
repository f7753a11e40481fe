/*
 * cpbin.h -- the tiny binary record container shared by the oracle programs
 * (reference harness, C restatement) and the Python test helpers.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the product library includes this file.
 *
 * Layout: 8-byte magic "CPBIN01\n", then records of
 *   name[32] (NUL padded) | type (1 byte: 'd' f64, 'i' i32, 'b' u8) | pad[7] |
 *   count (int64 little endian) | count * sizeof(type) bytes of payload.
 */
#ifndef CPBIN_H
#define CPBIN_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    char name[32];
    char type;
    int64_t count;
    void* data;
} cpbin_rec;

typedef struct {
    int n;
    cpbin_rec* recs;
} cpbin_file;

static inline int cpbin_elsize(char t) { return t == 'd' ? 8 : (t == 'i' ? 4 : 1); }

static inline FILE* cpbin_open_write(const char* path) {
    FILE* f = fopen(path, "wb");
    if (!f) return NULL;
    fwrite("CPBIN01\n", 1, 8, f);
    return f;
}

static inline void cpbin_put(FILE* f, const char* name, char type, int64_t count, const void* data) {
    char hdr[40];
    memset(hdr, 0, sizeof hdr);
    strncpy(hdr, name, 31);
    hdr[32] = type;
    fwrite(hdr, 1, 40, f);
    fwrite(&count, 8, 1, f);
    if (count > 0) fwrite(data, (size_t)cpbin_elsize(type), (size_t)count, f);
}

static inline void cpbin_put_d(FILE* f, const char* name, double v) { cpbin_put(f, name, 'd', 1, &v); }
static inline void cpbin_put_i(FILE* f, const char* name, int v) { cpbin_put(f, name, 'i', 1, &v); }

/* Reads the whole file; returns 0 on success. */
static inline int cpbin_read(const char* path, cpbin_file* out) {
    FILE* f = fopen(path, "rb");
    char magic[8];
    out->n = 0;
    out->recs = NULL;
    if (!f) return -1;
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "CPBIN01\n", 8) != 0) { fclose(f); return -2; }
    for (;;) {
        char hdr[40];
        int64_t count;
        cpbin_rec r;
        size_t bytes;
        if (fread(hdr, 1, 40, f) != 40) break;
        if (fread(&count, 8, 1, f) != 1) { fclose(f); return -3; }
        memcpy(r.name, hdr, 32);
        r.name[31] = 0;
        r.type = hdr[32];
        r.count = count;
        bytes = (size_t)count * (size_t)cpbin_elsize(r.type);
        r.data = malloc(bytes ? bytes : 1);
        if (bytes && fread(r.data, 1, bytes, f) != bytes) { fclose(f); return -4; }
        out->recs = (cpbin_rec*)realloc(out->recs, sizeof(cpbin_rec) * (size_t)(out->n + 1));
        out->recs[out->n++] = r;
    }
    fclose(f);
    return 0;
}

static inline const cpbin_rec* cpbin_get(const cpbin_file* f, const char* name) {
    int i;
    for (i = 0; i < f->n; ++i)
        if (strcmp(f->recs[i].name, name) == 0) return &f->recs[i];
    return NULL;
}

static inline void cpbin_free(cpbin_file* f) {
    int i;
    for (i = 0; i < f->n; ++i) free(f->recs[i].data);
    free(f->recs);
    f->recs = NULL;
    f->n = 0;
}

#endif
