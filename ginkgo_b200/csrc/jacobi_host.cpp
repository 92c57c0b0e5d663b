// Host set-up of block Jacobi: the block pointers (no CUDA).  Follows the
// reference's find_natural_blocks and agglomerate_supervariables
// (reference/preconditioner/jacobi_kernels.cpp:28-98) in one pass each.
#include <cstdint>
#include <cstring>

#include "../../include/ginkgo_b200.h"

namespace b2s {
void set_error(const char* fmt, ...);
}

extern "C" int64_t b2s_jacobi_find_blocks(int64_t num_rows, const int32_t* row_ptrs,
                                          const int32_t* col_idxs, int max_block_size,
                                          int32_t* block_ptrs_out)
{
    if (num_rows < 0 || max_block_size < 1 || row_ptrs == nullptr ||
        block_ptrs_out == nullptr || (num_rows > 0 && col_idxs == nullptr)) {
        b2s::set_error("b2s_jacobi_find_blocks: invalid argument");
        return B2S_ERR_INVALID_ARG;
    }
    for (int64_t r = 0; r < num_rows; ++r) {
        if (row_ptrs[r + 1] < row_ptrs[r]) {
            b2s::set_error("b2s_jacobi_find_blocks: row_ptrs decrease at row %lld",
                           (long long)r);
            return B2S_ERR_INVALID_ARG;
        }
    }
    int32_t* p = block_ptrs_out;
    p[0] = 0;
    if (num_rows == 0) return 0;
    // natural blocks: a row joins the current block when it has the previous
    // row's pattern and the block is not full
    int64_t nb = 1;
    int32_t size = 1;
    for (int64_t i = 1; i < num_rows; ++i) {
        const int32_t pb = row_ptrs[i - 1], cb = row_ptrs[i], ce = row_ptrs[i + 1];
        const bool same = ce - cb == cb - pb &&
                          std::memcmp(col_idxs + cb, col_idxs + pb,
                                      sizeof(int32_t) * size_t(ce - cb)) == 0;
        if (size < max_block_size && same) {
            ++size;
        } else {
            p[nb] = p[nb - 1] + size;
            ++nb;
            size = 1;
        }
    }
    p[nb] = p[nb - 1] + size;
    // agglomeration in place: merge neighbours while they fit
    int64_t out = 1;
    int32_t cur = p[1] - p[0];
    for (int64_t i = 1; i < nb; ++i) {
        const int32_t bs = p[i + 1] - p[i];
        if (cur + bs <= max_block_size) {
            cur += bs;
        } else {
            p[out] = p[i];
            ++out;
            cur = bs;
        }
    }
    p[out] = p[nb];
    return out;
}
