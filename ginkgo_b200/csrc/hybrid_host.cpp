// Host set-up of the Hybrid (Ell + Coo) format: the Ell width from the row
// lengths by the reference's strategy classes (include/ginkgo/core/matrix/
// hybrid.hpp:103-360), which run on the host there too.  No CUDA.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <new>
#include <vector>

#include "../../include/ginkgo_b200.h"

namespace b2s {
void set_error(const char* fmt, ...);
}

namespace {

// imbalance_limit::compute_ell_num_stored_elements_per_row: the row length
// at floor(rows * percent) of the sorted lengths (the longest for percent 1)
int64_t imbalance_limit(std::vector<int64_t>& sorted, double percent)
{
    percent = std::min(std::max(percent, 0.0), 1.0);
    const size_t n = sorted.size();
    if (n == 0) return 0;
    if (percent < 1) return sorted[size_t(double(n) * percent)];
    return sorted[n - 1];
}

}  // namespace

extern "C" int b2s_hybrid_config(int64_t num_rows, const int64_t* row_nnz, int strategy,
                                 double param1, double param2, int value_bytes,
                                 int index_bytes, int64_t* config_out)
{
    if (num_rows < 0 || config_out == nullptr || (num_rows > 0 && row_nnz == nullptr)) {
        b2s::set_error("b2s_hybrid_config: invalid argument");
        return B2S_ERR_INVALID_ARG;
    }
    std::vector<int64_t> sorted;
    try {
        sorted.assign(row_nnz, row_nnz + num_rows);
    } catch (const std::bad_alloc&) {
        b2s::set_error("b2s_hybrid_config: out of host memory");
        return B2S_ERR_INVALID_ARG;
    }
    for (int64_t x : sorted) {
        if (x < 0) {
            b2s::set_error("b2s_hybrid_config: negative row length");
            return B2S_ERR_INVALID_ARG;
        }
    }
    std::sort(sorted.begin(), sorted.end());
    const double rows = double(num_rows);
    int64_t width;
    switch (strategy) {
    case B2S_HYBRID_COLUMN_LIMIT:
        // a column limit is a size_type in the reference: finite, >= 0 and
        // representable
        if (!(param1 >= 0 && param1 < 9.2e18)) {
            b2s::set_error("b2s_hybrid_config: column limit must be finite and >= 0");
            return B2S_ERR_INVALID_ARG;
        }
        width = int64_t(param1);
        break;
    case B2S_HYBRID_IMBALANCE_LIMIT:
        if (std::isnan(param1)) {
            b2s::set_error("b2s_hybrid_config: imbalance percent is NaN");
            return B2S_ERR_INVALID_ARG;
        }
        width = imbalance_limit(sorted, param1);
        break;
    case B2S_HYBRID_IMBALANCE_BOUNDED:
        // param2 is the ratio of the Ell width bound to the row count
        if (std::isnan(param1) || !(param2 >= 0 && std::isfinite(param2)) ||
            rows * param2 >= 9.2e18) {
            b2s::set_error("b2s_hybrid_config: imbalance percent must not be NaN "
                           "and the width ratio must be finite and >= 0");
            return B2S_ERR_INVALID_ARG;
        }
        width = std::min(imbalance_limit(sorted, param1), int64_t(rows * param2));
        break;
    case B2S_HYBRID_MINIMAL_STORAGE:
        if (value_bytes <= 0 || index_bytes <= 0) {
            b2s::set_error("b2s_hybrid_config: value and index sizes must be positive");
            return B2S_ERR_INVALID_ARG;
        }
        width = imbalance_limit(sorted, double(index_bytes) /
                                            double(value_bytes + 2 * index_bytes));
        break;
    case B2S_HYBRID_AUTOMATIC:
        width = std::min(imbalance_limit(sorted, 1.0 / 3.0), int64_t(rows * 0.001));
        break;
    default:
        b2s::set_error("b2s_hybrid_config: unknown strategy %d", strategy);
        return B2S_ERR_INVALID_ARG;
    }
    // compute_coo_nnz: every entry past the Ell width goes to Coo
    int64_t coo = 0;
    for (int64_t x : sorted) coo += x > width ? x - width : 0;
    config_out[0] = width;
    config_out[1] = coo;
    return B2S_OK;
}
