// Entry points declared in ufob.h whose kernels are not built yet.
#include "ufob_internal.h"
using namespace ufob;
#define NOTYET(fn) return fail(UFOB_ERR_UNSUPPORTED, #fn " is not implemented yet")
struct ufob_gbp {};
struct ufob_batch {};
extern "C" {
ufob_status ufob_gbp_create(ufob_gbp **) { NOTYET(ufob_gbp_create); }
ufob_status ufob_gbp_set_property(ufob_gbp *, const char *, double) { NOTYET(ufob_gbp_set_property); }
ufob_status ufob_gbp_set_property_string(ufob_gbp *, const char *, const char *) { NOTYET(x); }
ufob_status ufob_gbp_set_array(ufob_gbp *, const char *, const double *, uint32_t) { NOTYET(x); }
ufob_status ufob_gbp_setup(ufob_gbp *) { NOTYET(x); }
ufob_status ufob_gbp_get_requisition(ufob_gbp *, uint32_t, uint32_t, uint32_t *, uint32_t *, uint32_t *) { NOTYET(x); }
ufob_status ufob_gbp_run(ufob_gbp *, const float *, uint32_t, uint32_t, void *, void *) { NOTYET(x); }
ufob_status ufob_gbp_process(ufob_gbp *, const float *, uint32_t, uint32_t, void *) { NOTYET(x); }
ufob_status ufob_gbp_generate(ufob_gbp *, void *, uint32_t, void *) { NOTYET(x); }
void ufob_gbp_destroy(ufob_gbp *) {}
ufob_status ufob_batch_create(const ufob_filter_props *, ufob_dtype, ufob_batch **) { NOTYET(x); }
ufob_status ufob_batch_run(ufob_batch *, const ufob_job *, uint32_t, void *) { NOTYET(x); }
void ufob_batch_destroy(ufob_batch *) {}
}
