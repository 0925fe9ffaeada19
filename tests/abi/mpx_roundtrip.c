/* A C99 client of the C ABI (no GPU needed): includes the public header,
 * stores a small MPX_matrix (a 2 x 3 matrix with one physical index) with
 * cmps_mpx_store, reads it back with cmps_mpx_stat / cmps_mpx_load and
 * checks every field.  Prints "ok" and exits 0 on success. */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "chainamps_b200.h"

static int fail(const char* what) {
  fprintf(stderr, "%s: %s\n", what, cmps_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const char* path = argv[1];
  /* indices: sigma (physical, in, 2 states), a (out, 3 states) */
  const uint8_t inward[2] = {1, 0}, physical[2] = {1, 0};
  const int64_t sizes[2] = {2, 3};
  const int16_t charges[5] = {1, -1, 0, 2, -2};
  const int64_t colptr[4] = {0, 1, 1, 3};
  const int64_t rowind[3] = {0, 0, 1};
  const double values[6] = {1.0, 0.5, -2.0, 0.0, 0.25, -0.75};
  cmps_mpx_desc d;
  memset(&d, 0, sizeof d);
  d.num_indices = 2;
  d.num_row_indices = 1;
  d.inward = inward;
  d.physical = physical;
  d.sizes = sizes;
  d.charges = charges;
  d.rows = 2;
  d.cols = 3;
  d.colptr = colptr;
  d.rowind = rowind;
  d.values = values;
  if (cmps_mpx_store(&d, 1, path) != CMPS_OK) return fail("store");

  int32_t ni = 0, nr = 0;
  int64_t tot = 0, rows = 0, cols = 0, nnz = 0;
  if (cmps_mpx_stat(path, 1, &ni, &nr, &tot, &rows, &cols, &nnz) != CMPS_OK) return fail("stat");
  if (ni != 2 || nr != 1 || tot != 5 || rows != 2 || cols != 3 || nnz != 3) return fail("stat values");

  uint8_t in2[2], ph2[2];
  int64_t sz2[2], cp2[4], ri2[3];
  int16_t ch2[5];
  double v2[6];
  const int16_t basis[2] = {1, -1};
  if (cmps_mpx_load(path, 1, basis, 2, in2, ph2, sz2, ch2, cp2, ri2, v2) != CMPS_OK) return fail("load");
  for (int i = 0; i < 2; ++i)
    if (in2[i] != inward[i] || ph2[i] != physical[i] || sz2[i] != sizes[i]) return fail("index");
  for (int i = 0; i < 5; ++i)
    if (ch2[i] != charges[i]) return fail("charges");
  for (int i = 0; i < 4; ++i)
    if (cp2[i] != colptr[i]) return fail("colptr");
  for (int i = 0; i < 3; ++i)
    if (ri2[i] != rowind[i]) return fail("rowind");
  for (int i = 0; i < 6; ++i)
    if (v2[i] != values[i]) return fail("values");
  /* a refused call returns its status and leaves a message */
  if (cmps_mpx_load("/nonexistent/x.MPX_matrix", 1, basis, 2, in2, ph2, sz2, ch2, cp2, ri2, v2) == CMPS_OK)
    return fail("missing file accepted");
  if (strlen(cmps_last_error()) == 0) return fail("no message");
  printf("ok %s\n", cmps_version());
  return 0;
}
