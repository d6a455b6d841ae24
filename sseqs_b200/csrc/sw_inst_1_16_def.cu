// Instantiations of the score kernel for stripe widths 1..16 with msa()'s
// gap parameters as compile-time constants (kDefGap, kDefOpen, kDefExt).
#include "sw_kernel.cuh"

namespace sseqs {
namespace sw {
void register_1_16_def(Tables& t) {
  fill_range<1, true>(t, std::make_integer_sequence<int, 16>{});
}
}  // namespace sw
}  // namespace sseqs
