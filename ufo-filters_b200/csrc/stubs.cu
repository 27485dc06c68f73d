// Entry points declared in ufob.h whose kernels are not built yet.
#include "ufob_internal.h"
using namespace ufob;
#define NOTYET(fn) return fail(UFOB_ERR_UNSUPPORTED, #fn " is not implemented yet")
struct ufob_batch {};
extern "C" {
ufob_status ufob_batch_create(const ufob_filter_props *, ufob_dtype, ufob_batch **) { NOTYET(ufob_batch_create); }
ufob_status ufob_batch_run(ufob_batch *, const ufob_job *, uint32_t, void *) { NOTYET(ufob_batch_run); }
void ufob_batch_destroy(ufob_batch *) {}
}
