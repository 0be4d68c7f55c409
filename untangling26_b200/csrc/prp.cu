// PRP (penetration-resolving-path) evaluation stages on sm_100a.
#include "u26_internal.h"

void u26_prp_release_ctx(const u26_ctx* ctx) { (void)ctx; }
