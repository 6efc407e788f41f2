// Combinatorial track finding (clone engine) -- device side and C ABI.
#include "internal.h"

namespace mkfg {
void finder_release(mkfg_context* ctx) { (void)ctx; }
}  // namespace mkfg
