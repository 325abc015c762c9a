// Fast aggregation of a uniform layer: placeholder until the band kernel lands; the emulator covers every layer.
#include "internal.h"
namespace lux {
size_t uniform_supported_planes() { return 0; }
bool uniform_fast_supported(int, int, int, int) { return false; }
}  // namespace lux
