// ib_time.cu -- the main loop's time bookkeeping on the device, for loops that replay a captured
// CUDA graph without reading the timestep back every iteration.
//
// Restated from time/TimeManager.m:
//   update (:124-186): dt = CFL * min over fluids of tau; if t + 2 dt > TIMEMAX, dt = (TIMEMAX - t)/2
//   step   (:270-277): iteration += 1; t += 2 dt with Kahan compensation
// and the loop condition of imogen.m:115 (t < TIMEMAX within 1e-14 relative).  Once the end time
// is reached dt is set to 0; every kernel that reads the device timestep then returns at once, so
// iterations replayed past the end leave the state and the clock unchanged.
#include <cmath>

#include "ib_internal.cuh"

namespace ib {

__global__ void time_update_kernel(ib_time_state *ts)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nf = (ts->nfluids < 1) ? 1 : (ts->nfluids > 4 ? 4 : ts->nfluids);
    double tau = 1e38;
    bool finite = true;
    for (int k = 0; k < nf; k++) {
        const double t = ts->tau[k];
        finite = finite && isfinite(t);
        tau = (t < tau) ? t : tau;
    }
    const double tmax = ts->tmax;
    const bool running = isfinite(tmax) ? (ts->time < tmax * (1 - 1e-14)) : true;
    double dt = 0.0;
    if (!finite) {
        ts->status = 1;  // the reference stops on a non-finite timestep (flux_multi.cu:295-298)
    } else if (running && ts->status == 0) {
        dt = ts->cfl * tau;
        if (ts->time + 2 * dt > tmax) dt = .5 * (tmax - ts->time);
    }
    ts->dt = dt;
}

__global__ void time_advance_kernel(ib_time_state *ts)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = ts->dt;
    if (!(dt > 0)) return;
    ts->iteration += 1;
    const double y = (2 * dt) - ts->kahan;
    const double t = ts->time + y;
    ts->kahan = (t - ts->time) - y;
    ts->time = t;
}

}  // namespace ib

using namespace ib;

extern "C" {

int ib_timeUpdate(ib_time_state *ts, void *stream)
{
    if (!ts) return IB_ERROR_NULL_POINTER;
    time_update_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(ts);
    return check_launch();
}

int ib_timeAdvance(ib_time_state *ts, void *stream)
{
    if (!ts) return IB_ERROR_NULL_POINTER;
    time_advance_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(ts);
    return check_launch();
}

}  // extern "C"
