// Split-BF16 (Ozaki-style) contraction path on tcgen05 tensor cores.
#include <stdexcept>
#include "kernels.hpp"

namespace ccsd {
namespace kern {

bool split_supported() { return false; }

void slice_rows(const double*, const int64_t*, const int64_t*, int, int, bool, int, SlicedOperand&, cudaStream_t) {
    throw std::runtime_error("split path not built");
}

void gemm_split(const SlicedOperand&, const SlicedOperand&, int, int, int, const GemmArgs&, cudaStream_t) {
    throw std::runtime_error("split path not built");
}

}  // namespace kern
}  // namespace ccsd
