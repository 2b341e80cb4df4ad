// cohort.h -- (internal, C++) many FP32 simulations stepped through one
// launch per phase (multi.h).  Used by the batches and the request server
// of batch.cu; the C ABI exposes it through irbc_schedule.fused.
#pragma once
#include <cstdint>
#include <vector>

struct irbc_handle;

namespace irbc {

struct Cohort;
Cohort* cohort_create(int device);
void cohort_destroy(Cohort* c);

// Members that can share a cohort have equal keys: the same device, the
// FP32 solvent, a mesh, the same collision interval and phase, the same
// step parity and the same snapshot state.  A key of -1 means the handle
// cannot join a cohort (FP64, no mesh): it is stepped on its own.
int64_t cohort_key(const irbc_handle* h);

// Advances every member (equal keys, one device, each at most once) by n
// steps through the cohort's fused launches and returns without waiting
// for the device.  A member whose health word already shows a problem is
// left out with IRBC_ERR_HEALTH in status[i]; status[i] is 0 for the
// others, which end exactly as irbc_step(h, n) would have left them.
// Returns 0, or the error of a launch or a list update (the members are
// then in an undefined state).  The kernels launched are counted in the
// process-wide launch count that irbc_launch_count reads.
int cohort_step(Cohort* c, const std::vector<irbc_handle*>& members, int64_t n, std::vector<int>& status);

}  // namespace irbc
