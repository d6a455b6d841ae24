// Instantiations of the score kernel for stripe widths 17..32 with msa()'s
// gap parameters as compile-time constants (kDefGap, kDefOpen, kDefExt).
#include "sw_kernel.cuh"

namespace sseqs {
namespace sw {
void register_17_32_def(Tables& t) {
  fill_range<17, true>(t, std::make_integer_sequence<int, 16>{});
}
}  // namespace sw
}  // namespace sseqs
