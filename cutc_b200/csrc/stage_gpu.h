// stage_gpu.h -- device-side staging of the mode copies: the records of
// one copy go to the device once, and every other order, the rows' run
// lengths (for the tile plan), the CCD++ slot layout and the per-row
// nonzero counts are made there.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

struct ctc_ctx;

namespace ctc {

// perm[i] = the record at position i of the stable order by the key
// (mode k[0], mode k[1], mode k[2]) with those indices in b[0], b[1], b[2]
// bits (b[2] = 0: two keys).  k = {m, m+1}, b = {bits(m), bits(m+1), 0} is
// the order ctc_tensor_sort gives.
void dev_sort_order(ctc_ctx *ctx, const uint4 *rec, uint32_t n, const int k[3], const int b[3], uint32_t *perm);

// true when the mode-m indices of the records decrease somewhere
bool dev_unsorted(ctc_ctx *ctx, const uint4 *rec, uint32_t n, int m);

// Runs of equal mode-m rows in the order `perm` (null: as stored): run r
// is row rows[r] repeated counts[r] times.  Returns true when the rows
// decrease somewhere (only checked for perm == null).
bool dev_row_runs(ctc_ctx *ctx, const uint4 *rec, const uint32_t *perm, uint32_t n, int m,
                  std::vector<uint32_t> &rows, std::vector<uint32_t> &counts);

// CCD++ slots of the tile plan `tiles` ({start, len, heavy, piece}, slot
// length 32 << eshift): key (row | q1 | q2 packed with shifts s_row, s_q1,
// s_q2; the bits below s_q2 zero) and value of entry lane * E + step of
// each tile, pads kPadKey / 0.
template <typename T>
void dev_fill_slots(ctc_ctx *ctx, const uint4 *rec, const double *v64, const uint32_t *perm, int m,
                    const int4 *tiles, uint64_t nslots, int eshift, uint32_t s_row, uint32_t s_q1, uint32_t s_q2,
                    uint64_t *keys, T *x);

// out[i] = rec[perm[i]] (and the FP64 values when v64 is given)
void dev_gather_records(ctc_ctx *ctx, const uint4 *rec, const double *v64, const uint32_t *perm, uint32_t n,
                        uint4 *out, double *v64_out);

// nonzeros per row of mode m (dim rows), to the host
void dev_row_counts(ctc_ctx *ctx, const uint4 *rec, uint32_t n, int m, uint32_t dim, std::vector<uint32_t> &counts);

}  // namespace ctc
