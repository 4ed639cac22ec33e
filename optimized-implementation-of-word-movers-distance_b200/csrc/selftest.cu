// Self-test of the bounded device-side wait that every mbarrier wait of the
// tensor-core kernels uses (tcgen05.cuh mbar_wait_ns): one thread waits on a
// freshly initialised mbarrier that nothing ever arrives on, with a short
// limit.  The wait must give up after the limit, set ERR_TIMEOUT in the
// error word and let the kernel return, so that the host sees a status and
// the CUDA context stays usable.  No tensor memory, no bulk copies, no
// other thread: the only thing exercised is the give-up path itself.
#include "tcgen05.cuh"

namespace wmd {
namespace {

__global__ void wait_selftest_kernel(unsigned* err, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  tc::mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  // Phase 0 of a new barrier completes only when one arrival lands; none
  // does, so this wait can end only through its time limit.
  tc::mbar_wait_ns(&bar, 0u, err, limit_ns);
}

}  // namespace

int launch_wait_selftest(unsigned* err, unsigned long long limit_ns, cudaStream_t st) {
  wait_selftest_kernel<<<1, 32, 0, st>>>(err, limit_ns);
  return 1;
}

}  // namespace wmd
