// Split-TF32 / split-BF16 tcgen05 grouped GEMM (internal).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "internal.h"

namespace cmps {
namespace tc {

// One output region of up to four column segments: column j belongs to the
// last segment q with seg_n0[q] <= j (seg_n0[0] = 0; unused segments hold
// INT32_MAX), and element (i, j) of C lands at
// seg_off[q] + i*row_stride + (j - seg_n0[q])*col_stride.  out_off repeats
// seg_off[0].
// vstore (mode 3): the output admits 16-byte stores of 8-row runs
// (mark_vector_stores); else the epilogue stores element by element.
struct TcTask {
  int64_t out_off;
  int64_t row_stride, col_stride;
  int32_t m, n;
  int32_t t0, t1;
  int32_t nseg;
  int32_t seg_n0[4];
  int64_t seg_off[4];
  int32_t vstore;
};
// One K-concatenated term: A tile at (a_x0 + k, a_y0 + row) of map a_map, B
// tile at (k, row) of b_map.  a_y0 (a row offset into the A map) applies to A
// tiles loaded by TMA only.
struct TcTerm {
  int32_t a_map, b_map, a_x0, k;
  int32_t a_y0;
};
// A operand read by the converter warps (mode 2): element (i, j) of the block
// at off + i * ld + j in each of two FP32 planes (re, im); rows x cols.
struct TcADesc {
  int64_t off, ld;
  int32_t rows, cols;
};
// b_rows: row count of the B boxes of this tile's task (its N rounded up to
// 16, at most 128); the B tensor maps of that task are encoded with it.
// kiters: k-steps (kstep() columns each) of the task's terms; nmma: the tile's N rounded up
// to 16 (the MMA N) -- so the MMA warp needs no task or term lookups.
// wide: the four-plane MMA form (BF16, N <= 32 with B planes of exactly N
// rows): 4 MMAs of N' = 4N per k-step instead of 12 of N; it rounds
// differently, so a plan opts in (finish_plan).
struct TcTile {
  int32_t task, m0, n0, b_rows, kiters, nmma;
  int32_t wide;
};
// B box rows for a task of N columns.
inline int32_t b_box_rows(int32_t n) { return n >= 128 ? 128 : ((n + 15) & ~15); }

struct TcPlan {
  std::vector<TcTask> tasks;
  std::vector<TcTerm> terms;
  std::vector<TcTile> tiles;
  std::vector<CUtensorMap> amaps, bmaps;
  std::vector<TcADesc> adescs;  // mode 2: A blocks in two FP32 planes
  TcADesc* d_adescs = nullptr;
  TcTask* d_tasks = nullptr;
  TcTerm* d_terms = nullptr;
  TcTile* d_tiles = nullptr;
  CUtensorMap* d_amaps = nullptr;
  CUtensorMap* d_bmaps = nullptr;
  int upload(cudaStream_t st);
  void release();
};

int smem_bytes();
// 3-D tensor map (K, rows, 4 planes) over one operand block of FP32 or BF16
// elements at `base` (plane 0), planes `plane` elements apart, rows `ld`
// elements apart; the block must fit in `room` elements from base.  Box: 64
// bytes of K by box_rows rows by the four planes, 64-byte swizzle.
int encode_map(bool bf16, const void* base, int64_t K, int64_t rows, int64_t ld, int64_t plane, int64_t room,
               int box_rows, CUtensorMap* out);
// Tiles of a task of m x n outputs, 128 x 128 each (row-major over the task).
void add_tiles(TcPlan& p, int32_t task, int32_t m, int32_t n);
// Completes a plan built term by term: k-steps per tile, optionally the
// heaviest tiles first, and checks every term, task, segment list and tile.
// by_tma: the A operands are tensor maps (else converter descriptors);
// b_rows: the row count each B map was encoded with; wide_ok: narrow BF16
// tiles take the four-plane MMA form.
int finish_plan(TcPlan& p, bool bf16, bool by_tma, const std::vector<int32_t>& b_rows, bool heaviest_first,
                bool wide_ok = false);
// Mode 3: marks the tasks whose output takes 16-byte stores of 8-row runs
// (rows contiguous, M a multiple of 8, segment starts and column / plane
// strides multiples of 8 elements) for a BF16 output at `out` (16-byte
// aligned) with plane stride `plane` elements.
void mark_vector_stores(TcPlan& p, const void* out, int64_t plane);
// K columns of one k-step: a 64-byte shared-memory row of 16 TF32 or 32 BF16
inline int32_t kstep(bool bf16) { return bf16 ? 32 : 16; }
// mode 1: A and B by TMA (four TF32 planes each); FP32 output in two planes
//         (re, im; plane stride out32_plane), the raw accumulator.
// mode 2: A read from two FP32 planes (ain, plane stride a_plane; blocks
//         described by p.adescs) and split to TF32 hi/lo in shared memory;
//         B by TMA; FP64 planar output (re, im; plane stride out64_plane).
// mode 3: A and B by TMA (four BF16 planes each: re_hi, re_mid, im_hi,
//         im_mid); output split into four BF16 planes at out32 (read as
//         16-bit elements; plane stride out32_plane elements).
// mode 4: A and B by TMA (four BF16 planes each); FP64 planar output.
int launch(int mode, const TcPlan& p, float* out32, int64_t out32_plane, double* out64, int64_t out64_plane,
           const float* ain, int64_t a_plane, int* d_err, cudaStream_t st);

}  // namespace tc
}  // namespace cmps
