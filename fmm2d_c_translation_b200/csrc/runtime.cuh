// runtime.cuh -- per-call execution context of the C-ABI entry points.
//
// Every entry point runs on its own non-blocking stream of the calling
// thread's current device, so concurrent calls from several host threads
// are independent (the reference's routines are reentrant too).  Device
// workspace comes from the device's default memory pool, whose release
// threshold is raised once per device so that repeated calls reuse blocks
// instead of returning them to the driver.
#pragma once

#include "common.cuh"

#include <exception>

namespace fmm2d {

std::string get_last_error();
std::string prof_report();
unsigned long long launch_count();
void set_profiling(int on);
void set_user_stream(cudaStream_t s, bool on);

class CallCtx {
  public:
    CallCtx();
    ~CallCtx();
    CallCtx(const CallCtx &) = delete;
    CallCtx &operator=(const CallCtx &) = delete;
    cudaStream_t stream() const { return s_; }
    int device() const { return dev_; }
    // A second non-blocking stream of the calling thread and device, for
    // host<->device copies that overlap the work on stream().
    cudaStream_t copy_stream() const;

  private:
    int dev_;
    cudaStream_t s_;
};

// Runs f(); maps exceptions to the reference's error code (4) and records
// the message for fmm2d_b200_last_error().
template <class F>
inline int guarded(F &&f) {
    try {
        f();
        return 0;
    } catch (const FmmError &e) {
        set_last_error(e.what());
        return e.ier;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return 4;
    }
}

}  // namespace fmm2d

#define FMM_EXPORT extern "C" __attribute__((visibility("default")))
