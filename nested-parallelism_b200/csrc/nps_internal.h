// Internal helpers shared by the host translation units of libnps.
#ifndef NPS_INTERNAL_H_
#define NPS_INTERNAL_H_

#include <string>

#include "nps.h"

// Records `msg` as this thread's last error (nps_last_error_string) and
// returns `code`, so call sites read `return nps_fail(NPS_ERR_..., "...")`.
nps_status nps_fail(nps_status code, const std::string& msg);
void nps_clear_error();

nps_status nps_build_csr(int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                         const uint32_t* w, bool dedupe, bool drop_self, nps_graph* out);

// Device copy of the learned-policy weights of `device` (null if none loaded).
const void* nps_policy_device_weights(int device);

#endif  // NPS_INTERNAL_H_
