// Instantiations of the score kernel for stripe widths 33..48 with the gap
// parameters read from the arguments (split across translation units so
// that they compile in parallel).
#include "sw_kernel.cuh"

namespace sseqs {
namespace sw {
void register_33_48(Tables& t) {
  fill_range<33, false>(t, std::make_integer_sequence<int, 16>{});
}
}  // namespace sw
}  // namespace sseqs
