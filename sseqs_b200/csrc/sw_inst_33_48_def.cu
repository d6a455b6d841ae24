// Instantiations of the score kernel for stripe widths 33..48 with msa()'s
// gap parameters as compile-time constants (kDefGap, kDefOpen, kDefExt).
#include "sw_kernel.cuh"

namespace sseqs {
namespace sw {
void register_33_48_def(Tables& t) {
  fill_range<33, true>(t, std::make_integer_sequence<int, 16>{});
}
}  // namespace sw
}  // namespace sseqs
