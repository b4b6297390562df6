// Binary CCS matrix and vector files: the on-disk format of the reference's
// taucs_ccs_read_binary (src/taucs_ccs_io.c:31-113) and of its MATLAB writer
// (matlab/taucs_ccs_write_binary.m:1-55), native byte order, no padding:
//
//   int nrows, int ncols, int flags,
//   int colptr[ncols + 1], int rowind[colptr[ncols]],
//   values[colptr[ncols]]   (double for TAUCS_DOUBLE, float for TAUCS_SINGLE)
//
// and the vector files of taucs_vec_read_binary / taucs_vec_write_binary
// (src/taucs_ccs_io.c:966-1052): n raw values, no header.
//
// The reference checks nothing (a short file leaves the arrays partly
// uninitialised; a missing file or an unsupported type ends in assert).
// These readers return NULL on an unreadable file, a short read, a negative
// size, a colptr that does not start at 0 or decreases, a row index outside
// [0, nrows), or a value type other than double/single; the reason goes to
// taucs_printf and taucs_b200_last_error.  The reference has no C writer for
// matrices; taucs_b200_ccs_write_binary writes the same format (the flags
// word as stored in the matrix), so a served request can be saved and
// replayed.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "internal.h"

using namespace tb;

namespace {

size_t value_size(int flags) {
  if (flags & TAUCS_DOUBLE) return sizeof(double);
  if (flags & TAUCS_SINGLE) return sizeof(float);
  return 0;
}

bool read_all(FILE* f, void* p, size_t bytes) { return bytes == 0 || fread(p, 1, bytes, f) == bytes; }
bool write_all(FILE* f, const void* p, size_t bytes) { return bytes == 0 || fwrite(p, 1, bytes, f) == bytes; }

taucs_ccs_matrix* fail(FILE* f, taucs_ccs_matrix* A, const std::string& why) {
  if (f) fclose(f);
  taucs_ccs_free(A);
  set_error("taucs_ccs_read_binary: " + why);
  return nullptr;
}

}  // namespace

extern "C" {

taucs_ccs_matrix* taucs_ccs_read_binary(char* filename) {
  if (!filename) return fail(nullptr, nullptr, "no file name");
  tprintf("taucs_ccs_binary: reading binary matrix %s\n", filename);
  FILE* f = fopen(filename, "rb");
  if (!f) return fail(nullptr, nullptr, std::string("cannot open ") + filename);
  int hdr[3];
  if (!read_all(f, hdr, sizeof hdr)) return fail(f, nullptr, "short header");
  const int nrows = hdr[0], ncols = hdr[1], flags = hdr[2];
  tprintf("\t%d-by-%d, flags = %08x\n", nrows, ncols, flags);
  if (nrows < 0 || ncols < 0) return fail(f, nullptr, "negative dimension");
  const size_t esz = value_size(flags);
  if (!esz) return fail(f, nullptr, "only TAUCS_DOUBLE and TAUCS_SINGLE values are supported");
  int* colptr = (int*) malloc(sizeof(int) * ((size_t) ncols + 1));
  if (!colptr) return fail(f, nullptr, "out of memory");
  if (!read_all(f, colptr, sizeof(int) * ((size_t) ncols + 1))) {
    free(colptr);
    return fail(f, nullptr, "short column pointer array");
  }
  bool ok = colptr[0] == 0;
  for (int j = 0; ok && j < ncols; j++) ok = colptr[j + 1] >= colptr[j];
  if (!ok) {
    free(colptr);
    return fail(f, nullptr, "column pointers do not start at 0 or decrease");
  }
  const int nnz = colptr[ncols];
  taucs_ccs_matrix* A = taucs_ccs_create(nrows, ncols, nnz, flags);
  if (!A) {
    free(colptr);
    return fail(f, nullptr, "out of memory");
  }
  memcpy(A->colptr, colptr, sizeof(int) * ((size_t) ncols + 1));
  free(colptr);
  if (!read_all(f, A->rowind, sizeof(int) * (size_t) nnz)) return fail(f, A, "short row index array");
  for (int k = 0; k < nnz; k++)
    if (A->rowind[k] < 0 || A->rowind[k] >= nrows) return fail(f, A, "row index out of range");
  if (!read_all(f, A->values.v, esz * (size_t) nnz)) return fail(f, A, "short value array");
  fclose(f);
  A->flags = flags;
  tprintf("taucs_ccs_read_binary: done reading\n");
  return A;
}

int taucs_b200_ccs_write_binary(taucs_ccs_matrix* A, char* filename) {
  if (!A || !filename || A->n < 0 || A->m < 0 || !A->colptr) {
    set_error("taucs_b200_ccs_write_binary: bad arguments");
    return TAUCS_ERROR_BADARGS;
  }
  const size_t esz = value_size(A->flags);
  if (!esz) {
    set_error("taucs_b200_ccs_write_binary: only TAUCS_DOUBLE and TAUCS_SINGLE values are supported");
    return TAUCS_ERROR_BADARGS;
  }
  FILE* f = fopen(filename, "wb");
  if (!f) {
    set_error(std::string("taucs_b200_ccs_write_binary: cannot create ") + filename);
    return TAUCS_ERROR;
  }
  const int hdr[3] = {A->m, A->n, A->flags};
  const size_t nnz = (size_t) A->colptr[A->n];
  const bool ok = write_all(f, hdr, sizeof hdr) && write_all(f, A->colptr, sizeof(int) * ((size_t) A->n + 1)) &&
                  write_all(f, A->rowind, sizeof(int) * nnz) && write_all(f, A->values.v, esz * nnz);
  if (fclose(f) != 0 || !ok) {
    set_error(std::string("taucs_b200_ccs_write_binary: write failed on ") + filename);
    return TAUCS_ERROR;
  }
  return TAUCS_SUCCESS;
}

void* taucs_vec_read_binary(int n, int flags, char* filename) {
  const size_t esz = value_size(flags);
  if (n < 0 || !esz || !filename) {
    set_error("taucs_vec_read_binary: bad arguments (double or single vectors only)");
    return nullptr;
  }
  tprintf("taucs_vec_read_binary: reading binary vector %s\n", filename);
  FILE* f = fopen(filename, "rb");
  if (!f) {
    set_error(std::string("taucs_vec_read_binary: cannot open ") + filename);
    return nullptr;
  }
  void* v = malloc(esz * (size_t) (n > 0 ? n : 1));
  const bool ok = v && read_all(f, v, esz * (size_t) n);
  fclose(f);
  if (!ok) {
    free(v);
    set_error("taucs_vec_read_binary: short file or out of memory");
    return nullptr;
  }
  return v;
}

int taucs_vec_write_binary(int n, int flags, void* v, char* filename) {
  const size_t esz = value_size(flags);
  if (n < 0 || !esz || (n > 0 && !v) || !filename) {
    set_error("taucs_vec_write_binary: bad arguments (double or single vectors only)");
    return TAUCS_ERROR_BADARGS;
  }
  tprintf("taucs_vec_write_binary: writing binary vector %s\n", filename);
  FILE* f = fopen(filename, "wb");
  if (!f) {
    set_error(std::string("taucs_vec_write_binary: cannot create ") + filename);
    return TAUCS_ERROR;
  }
  const bool ok = write_all(f, v, esz * (size_t) n);
  if (fclose(f) != 0 || !ok) {
    set_error(std::string("taucs_vec_write_binary: write failed on ") + filename);
    return TAUCS_ERROR;
  }
  return 0;
}

}  // extern "C"
