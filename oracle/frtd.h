// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// "FRTD" state-dump container written by the oracle drivers and read by the parity tests
// (oracle/frtd.py). Layout: "FRTD", int32 version, int32 narrays, then per array a 32-byte
// name, int32 dtype code, int32 ndim, int64 dims[4], and the raw little-endian data.
#pragma once
#include <stdint.h>
#include <stdio.h>
#include <string.h>

enum { FRTD_F32 = 0, FRTD_F64 = 1, FRTD_I32 = 2, FRTD_I64 = 3, FRTD_U8 = 4, FRTD_I16 = 5, FRTD_U16 = 6 };

static inline size_t frtd_elem_size(int dtype) {
  switch (dtype) {
    case FRTD_F32: case FRTD_I32: return 4;
    case FRTD_F64: case FRTD_I64: return 8;
    case FRTD_U8: return 1;
    default: return 2;
  }
}

struct frtd_writer {
  FILE* f;
  int32_t count;
};

static inline int frtd_open(struct frtd_writer* w, const char* path) {
  w->f = fopen(path, "wb");
  w->count = 0;
  if (!w->f) return -1;
  const int32_t hdr[2] = {1, 0};
  fwrite("FRTD", 1, 4, w->f);
  fwrite(hdr, sizeof(int32_t), 2, w->f);
  return 0;
}

static inline void frtd_add(struct frtd_writer* w, const char* name, int dtype, int ndim, const int64_t* dims,
                            const void* data) {
  char nm[32];
  memset(nm, 0, sizeof nm);
  strncpy(nm, name, 31);
  int64_t d[4] = {1, 1, 1, 1};
  size_t n = 1;
  for (int i = 0; i < ndim && i < 4; ++i) {
    d[i] = dims[i];
    n *= (size_t)dims[i];
  }
  const int32_t meta[2] = {dtype, ndim};
  fwrite(nm, 1, 32, w->f);
  fwrite(meta, sizeof(int32_t), 2, w->f);
  fwrite(d, sizeof(int64_t), 4, w->f);
  if (n) fwrite(data, frtd_elem_size(dtype), n, w->f);
  w->count++;
}

static inline void frtd_add1(struct frtd_writer* w, const char* name, int dtype, int64_t n, const void* data) {
  frtd_add(w, name, dtype, 1, &n, data);
}

static inline void frtd_close(struct frtd_writer* w) {
  fseek(w->f, 8, SEEK_SET);
  fwrite(&w->count, sizeof(int32_t), 1, w->f);
  fclose(w->f);
}
