// sb_pending.cu — entry points declared by the ABI whose device paths are
// not built yet; each returns SB_ERR_UNSUPPORTED with a message.
#include "sb_kernels.cuh"

extern "C" {
sb_status sb_autotune(sb_ctx*, uint32_t, sb_tuning*) { return SB_ERR_UNSUPPORTED; }
}
