// book.h — the batched basket book (book.cu).
#pragma once
#include "engine.h"

namespace mcq {

// Argument checks of a book (no device work), so that bad input fails before the GPU is touched.
void book_validate(const mcq_book_option* opts, int n, const mcq_mlmc_cfg& ml, const mcq_qmc_cfg& qc);

// mode 0: batched (one graph replay per adaptive round for all options and levels);
// mode 1: plain (one option at a time, one launch per level on its own stream).
void book_price(const mcq_book_option* opts, int n, const mcq_mlmc_cfg& ml, const mcq_qmc_cfg& qc, int mode,
                mcq_book_result* out, mcq_book_stats* stats);
// Per-replica sums [R][20] of one slice of one option, through the book kernel.
void book_level_sums(const mcq_book_option& opt, const mcq_mlmc_cfg& ml, const mcq_qmc_cfg& qc, int level,
                     uint32_t offset, long long n_points, double* sums_host);

}  // namespace mcq
