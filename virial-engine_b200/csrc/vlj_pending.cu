// Entry points whose kernels are not written yet: they report VLJ_NOT_ENABLED.
#include "virial_lj.h"
#include "vlj_common.h"

using vlj::fail;

extern "C" {
vlj_status vlj_batch_create(const vlj_replica_desc*, size_t, double, double, double, int32_t, void*, vlj_batch**) { return fail(VLJ_NOT_ENABLED, "batches are not available yet"); }
vlj_status vlj_batch_destroy(vlj_batch*) { return VLJ_OK; }
vlj_status vlj_batch_step(vlj_batch*, uint32_t) { return fail(VLJ_NOT_ENABLED, "batches are not available yet"); }
vlj_status vlj_batch_measure(vlj_batch*, vlj_measurement*) { return fail(VLJ_NOT_ENABLED, "batches are not available yet"); }
vlj_status vlj_batch_read_particles(vlj_batch*, size_t, vlj_particle*) { return fail(VLJ_NOT_ENABLED, "batches are not available yet"); }
vlj_status vlj_batch_count(const vlj_batch*, size_t*, uint64_t*) { return fail(VLJ_NOT_ENABLED, "batches are not available yet"); }
}
